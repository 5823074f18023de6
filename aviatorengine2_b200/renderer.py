"""Host-side mirror of the reference's Renderer (renderer/renderer.h:325-411)
over the C ABI.

`Context` is the thin handle on ae_ctx; `Renderer` keeps the reference's
per-frame entry points and state machine (accumulation frame count, camera
moves, convergence at maxSamples) so code written against the reference reads
the same:

    r = Renderer()
    r.Initialize(RendererSettings(width=320, height=240, hybrid=False))
    r.LoadScene(packed_scene)
    r.SyncCamera(source, target, fov)
    while not r.Converged():
        r.RenderFrame()
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, lib, ptr


class Context:
    """One device context: scene buffers, images, a stream."""

    def __init__(self, width, height, samples=1, hybrid=False, trace_scale=1.0, device=0, hybrid_max_depth=3,
                 history_while_moving=32, max_samples=0):
        s = np.zeros(1, _lib.SETTINGS)
        s["width"], s["height"], s["samples"] = width, height, samples
        s["max_samples"], s["hybrid"], s["hybrid_max_depth"] = max_samples, int(hybrid), hybrid_max_depth
        s["trace_scale"], s["history_while_moving"], s["device"] = trace_scale, history_while_moving, device
        self._h = lib().ae_create(ptr(s))
        if not self._h:
            raise _lib.AeError(lib().ae_create_status(), "ae_create failed (see stderr)")
        self.width, self.height = width, height
        self.scene = None

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            lib().ae_destroy(h)

    def __del__(self):
        # At interpreter exit the ctypes module state may already be gone;
        # the process is ending and the driver releases the device anyway.
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def _chk(self, code):
        return check(code, self._h)

    # --- uploads -----------------------------------------------------------
    def upload_geometry(self, vertices, indices, blas):
        self._keep_geo = (np.ascontiguousarray(vertices), np.ascontiguousarray(indices, np.uint32),
                          np.ascontiguousarray(blas))
        v, i, b = self._keep_geo
        self._chk(lib().ae_upload_geometry(self._h, ptr(v), len(v), ptr(i), len(i), ptr(b), len(b)))

    def reserve_scene(self, max_objects, max_lights):
        self._chk(lib().ae_reserve_scene(self._h, max_objects, max_lights))

    def upload_scene(self, objects, tlas, lights, instances):
        o, t = np.ascontiguousarray(objects), np.ascontiguousarray(tlas)
        lt, ins = np.ascontiguousarray(lights, np.uint32), np.ascontiguousarray(instances)
        self._chk(lib().ae_upload_scene(self._h, ptr(o), len(o), ptr(t), len(t), ptr(lt), len(lt), ptr(ins), len(ins)))

    def upload_textures(self, textures):
        """The material texture array: (layers, height, width, 4) RGBA8 sRGB."""
        t = np.ascontiguousarray(textures, np.uint8)
        self._keep_tex = t
        layers, h, w, _ = t.shape
        self._chk(lib().ae_upload_textures(self._h, ptr(t), w, h, layers))

    def upload(self, scene):
        """Geometry once, then the per-frame arrays, then the scene's config
        (and its texture array when it has one)."""
        if getattr(scene, "textures", None) is not None:
            self.upload_textures(scene.textures)
        self.upload_geometry(scene.vertices, scene.indices, scene.blas)
        self.upload_scene(scene.objects, scene.tlas, scene.lights, scene.instances)
        cfg = scene.config.copy()
        cfg["width"], cfg["height"] = self.width, self.height
        self.set_config(cfg)
        self.scene = scene

    def set_config(self, cfg):
        c = np.ascontiguousarray(np.array(cfg, dtype=_lib.CONFIG).reshape(1))
        self._chk(lib().ae_set_config(self._h, ptr(c)))

    def get_config(self):
        c = np.zeros(1, _lib.CONFIG)
        self._chk(lib().ae_get_config(self._h, ptr(c)))
        return c[0]

    # --- frames ------------------------------------------------------------
    def render_frame(self, mode=_lib.MODE_COMPUTE_ONLY, gbuffer=None):
        self._chk(lib().ae_render_frame(self._h, mode, None if gbuffer is None else ctypes.byref(gbuffer)))

    def read_image(self, which=_lib.IMAGE_ACCUM):
        if which == _lib.IMAGE_DISPLAY:
            out = np.zeros((self.height, self.width, 4), np.uint8)
        elif which == _lib.IMAGE_REDUCED:
            cfg = self.get_config()
            s = float(cfg["traceScale"])
            w = int(np.ceil(np.float32(self.width) * np.float32(s)))
            h = int(np.ceil(np.float32(self.height) * np.float32(s)))
            out = np.zeros((h, w, 4), np.float32)
        else:
            out = np.zeros((self.height, self.width, 4), np.float32)
        self._chk(lib().ae_read_image(self._h, which, ptr(out), out.nbytes))
        return out

    def read_planes(self):
        """The deferred path's G-buffer planes (position, normal, albedo bytes,
        depth) as the last ae_build_gbuffer / G-buffer upload left them."""
        h, w = self.height, self.width
        out = (np.zeros((h, w, 4), np.float32), np.zeros((h, w, 4), np.float32), np.zeros((h, w, 4), np.uint8),
               np.zeros((h, w), np.float32))
        for k, a in enumerate(out):
            self._chk(lib().ae_read_image(self._h, 101 + k, ptr(a), a.nbytes))
        return out

    def read_deferred_accum(self):
        out = np.zeros((self.height, self.width, 4), np.float32)
        self._chk(lib().ae_read_image(self._h, 100, ptr(out), out.nbytes))
        return out

    def build_gbuffer(self):
        self._chk(lib().ae_build_gbuffer(self._h))

    # --- rays --------------------------------------------------------------
    def closest_hit(self, rays, variant=_lib.VARIANT_PLAIN):
        r = np.ascontiguousarray(rays, dtype=_lib.RAY)
        hits = np.zeros(len(r), _lib.HIT)
        self._chk(lib().ae_closest_hit(self._h, ptr(r), len(r), ptr(hits), variant))
        return hits

    def closest_hit_device(self, d_rays, n, d_hits, variant=_lib.VARIANT_PLAIN):
        self._chk(lib().ae_closest_hit_device(self._h, ctypes.c_void_p(d_rays), n, ctypes.c_void_p(d_hits), variant))

    def any_hit(self, rays, tmax):
        r = np.ascontiguousarray(rays, dtype=_lib.RAY)
        t = np.ascontiguousarray(tmax, dtype=np.float32)
        out = np.zeros(len(r), np.uint8)
        self._chk(lib().ae_any_hit(self._h, ptr(r), ptr(t), len(r), ptr(out)))
        return out

    def camera_rays(self):
        out = np.zeros(self.width * self.height, _lib.RAY)
        self._chk(lib().ae_camera_rays(self._h, ptr(out)))
        return out

    def bounce_rays(self, primary, hits):
        p = np.ascontiguousarray(primary, dtype=_lib.RAY)
        h = np.ascontiguousarray(hits, dtype=_lib.HIT)
        out = np.zeros(len(p), _lib.RAY)
        valid = np.zeros(len(p), np.uint8)
        self._chk(lib().ae_bounce_rays(self._h, ptr(p), ptr(h), len(p), ptr(out), ptr(valid)))
        return out, valid.astype(bool)

    def rebuild_scene(self, entities, meshes):
        """RebuildAcceleration + UploadScene on the GPU (ae_rebuild_scene): the
        scene becomes exactly what scenes.pack(entities, meshes) uploads."""
        ents = np.ascontiguousarray(np.array(entities, dtype=_lib.ENTITY))
        self._chk(lib().ae_rebuild_scene(self._h, ptr(ents), len(ents), meshes.handle if meshes else None))

    def refit_instances(self, instances):
        ins = np.ascontiguousarray(instances, dtype=_lib.INSTANCE)
        self._chk(lib().ae_refit_instances(self._h, ptr(ins), len(ins)))

    def scene_sizes(self):
        """(objects, TLAS nodes, lights, instances) of the scene on the device."""
        v = [ctypes.c_uint32() for _ in range(4)]
        self._chk(lib().ae_scene_sizes(self._h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def download_scene(self):
        n_obj, n_nodes, _, n_inst = self.scene_sizes()
        o = np.zeros(n_obj, _lib.OBJECT)
        t = np.zeros(n_nodes, _lib.NODE)
        i = np.zeros(n_inst, _lib.INSTANCE)
        self._chk(lib().ae_download_scene(self._h, ptr(o), ptr(t), ptr(i)))
        return o, t, i

    def wavefront_info(self):
        th, st, err = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_uint32()
        ms = np.zeros(9, np.float32)
        self._chk(lib().ae_wavefront_info(self._h, ctypes.byref(th), ctypes.byref(st), ptr(ms), ctypes.byref(err)))
        return {"threads": th.value, "stack": st.value, "tune_ms": ms.tolist(), "errors": err.value}

    def wavefront_walk_info(self, precision=False):
        """The walker stages' autotuned launch for one form: run lengths (0 =
        static) and resident blocks per SM of the shadow stage and the bounce
        extend, and the timings behind them (static, 32, 64, 256 at 6 blocks,
        then at 7, for each stage)."""
        sh, ex, shb, exb = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        ms = np.zeros(16, np.float32)
        self._chk(lib().ae_wavefront_walk_info(self._h, 1 if precision else 0, ctypes.byref(sh), ctypes.byref(ex),
                                               ctypes.byref(shb), ctypes.byref(exb), ptr(ms)))
        return {"shadow_run": sh.value, "extend_run": ex.value, "shadow_blocks": shb.value,
                "extend_blocks": exb.value, "shadow_ms": ms[:8].tolist(), "extend_ms": ms[8:].tolist()}

    def set_wavefront_walk_runs(self, shadow_run, extend_run, precision=False, shadow_blocks=0, extend_blocks=0):
        """Pin the walker stages' launch of one form (runs: 0 = static;
        blocks: 6 or 7, 0 = 7)."""
        self._chk(lib().ae_wavefront_set_walk_runs(self._h, 1 if precision else 0, shadow_run, extend_run,
                                                   shadow_blocks, extend_blocks))

    def image_error(self, reference, which=_lib.IMAGE_ACCUM, eps=1e-3):
        """FP64 error of an image against a reference (H, W, 4) float64 image,
        reduced on the GPU: (mean relative, mean absolute, max absolute, rms)."""
        ref = np.ascontiguousarray(reference, dtype=np.float64)
        assert ref.shape == (self.height, self.width, 4), ref.shape
        out = np.zeros(4, np.float64)
        self._chk(lib().ae_image_error(self._h, which, ptr(ref), eps, ptr(out)))
        return {"mre": out[0], "mae": out[1], "max": out[2], "rmse": out[3]}

    def image_error_pixels(self, pixels, reference, which=_lib.IMAGE_ACCUM, eps=1e-3):
        """image_error over a pixel subset: `pixels` (n, 2) as (x, y),
        `reference` (n, 4) float64 in the same order."""
        xy = np.ascontiguousarray(pixels, dtype=np.uint32).reshape(-1, 2)
        ref = np.ascontiguousarray(reference, dtype=np.float64).reshape(-1, 4)
        assert len(ref) == len(xy), (ref.shape, xy.shape)
        out = np.zeros(4, np.float64)
        self._chk(lib().ae_image_error_pixels(self._h, which, ptr(xy), len(xy), ptr(ref), eps, ptr(out)))
        return {"mre": out[0], "mae": out[1], "max": out[2], "rmse": out[3]}

    def debug_flags(self):
        """AE_CHECK_* bits the debug walk (VARIANT_PLAIN_CHECKED) set since the
        last read (ae_debug_flags); reading clears them."""
        f = ctypes.c_uint32()
        self._chk(lib().ae_debug_flags(self._h, ctypes.byref(f)))
        return f.value

    def debug_inject(self, fault, on=True):
        """Test hook (ae_debug_inject): e.g. _lib.FAULT_TILE_WAIT."""
        self._chk(lib().ae_debug_inject(self._h, fault, 1 if on else 0))

    def prepare_fast(self):
        self._chk(lib().ae_prepare_fast(self._h))

    def synchronize(self):
        self._chk(lib().ae_synchronize(self._h))

    def last_kernel_ms(self):
        ms = ctypes.c_float()
        self._chk(lib().ae_last_kernel_ms(self._h, ctypes.byref(ms)))
        return ms.value

    @property
    def stream(self):
        return lib().ae_stream(self._h)

    @property
    def launch_count(self):
        return int(lib().ae_launch_count(self._h))


@dataclass
class RendererSettings:
    """RendererSettings, renderer/renderer.h:225-274 (no window or shader name)."""
    width: int = 1920
    height: int = 1080
    samples: int = 1
    maxSamples: int = 0
    hybrid: bool = True
    hybridMaxDepth: int = 3
    traceScale: float = 1.0
    historyWhileMoving: int = 32
    device: int = 0


class Renderer:
    """Renderer, renderer/renderer.h:325-411, over a device Context."""

    def __init__(self):
        self.ctx = None
        self.accumulationFrame = 0
        self.frameIndex = 0
        self.historyResetPending = True
        self.cameraMovedPending = False
        self.sceneMaxDepth = 1
        self.hybrid = False
        self.maxSamples = 0
        self.config = None

    def Initialize(self, settings):
        s = settings
        self.ctx = Context(s.width, s.height, s.samples, s.hybrid, s.traceScale, s.device, s.hybridMaxDepth,
                           s.historyWhileMoving, s.maxSamples)
        self.settings = s
        self.hybrid = s.hybrid
        self.maxSamples = s.maxSamples
        self.config = self.ctx.get_config()
        return True

    def LoadScene(self, scene):
        self.ctx.upload(scene)
        self.config = self.ctx.get_config()
        self.sceneMaxDepth = max(int(self.config["depth"]), 1)
        self.ApplyDepthCap()
        return True

    def SyncCamera(self, source, target, fov=None, focus_dist=None, defocus_angle=None):
        c = self.config
        c["source_x"], c["source_y"], c["source_z"] = source
        c["target_x"], c["target_y"], c["target_z"] = target
        if fov is not None:
            c["fov"] = fov
        if focus_dist is not None:
            c["focus_dist"] = focus_dist
        if defocus_angle is not None:
            c["defocus_angle"] = defocus_angle

    def SyncSceneSettings(self, sky=(0, 0, 0), horizon=(0, 0, 0), max_depth=8):
        c = self.config
        c["sky_r"], c["sky_g"], c["sky_b"] = sky
        c["horizon_r"], c["horizon_g"], c["horizon_b"] = horizon
        self.sceneMaxDepth = max(int(max_depth), 1)
        self.ApplyDepthCap()

    def ApplyDepthCap(self):
        hd = self.settings.hybridMaxDepth
        self.config["depth"] = min(self.sceneMaxDepth, hd) if self.hybrid else self.sceneMaxDepth

    def MarkSceneDirty(self):
        pass  # uploads are explicit: call LoadScene/upload_scene with the rebuilt arrays

    def ResetAccumulation(self):
        self.accumulationFrame = 0
        self.historyResetPending = True

    def CameraMoved(self):
        if not self.hybrid:
            self.ResetAccumulation()
            return
        self.accumulationFrame = 0
        self.cameraMovedPending = True

    def SetExposure(self, value):
        self.config["exposure"] = max(float(value), 0.01)

    def Exposure(self):
        return float(self.config["exposure"])

    def AccumulatedSamples(self):
        return self.accumulationFrame * int(self.config["samples"])

    def Converged(self):
        return self.maxSamples > 0 and int(self.config["debugView"]) == 0 and self.AccumulatedSamples() >= self.maxSamples

    def SetHybrid(self, enabled):
        self.hybrid = bool(enabled)
        self.ApplyDepthCap()
        self.ResetAccumulation()

    def RenderFrame(self):
        """renderer/renderer.cpp:1332-1588 minus raster and blit."""
        c = self.config
        converged = self.Converged()
        c["batch"] = self.accumulationFrame
        c["displayOnly"] = 1 if converged else 0
        c["frameIndex"] = self.frameIndex
        c["historyReset"] = 1 if self.historyResetPending else 0
        c["cameraMoved"] = 1 if self.cameraMovedPending else 0
        self.ctx.set_config(c)
        if self.hybrid:
            self.ctx.render_frame(_lib.MODE_DEFERRED)
        else:
            self.ctx.render_frame(_lib.MODE_COMPUTE_ONLY)
        if not converged:
            self.accumulationFrame += 1
            self.frameIndex += 1
            self.historyResetPending = False
            self.cameraMovedPending = False
        return True

    def Shutdown(self):
        if self.ctx:
            self.ctx.close()
            self.ctx = None
