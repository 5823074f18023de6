"""Test-side bindings of the oracle (oracle/liboracle.so) and of the
reference's own code compiled for the CPU pin (oracle/_ref/*.so).

Only tests/, bench.py's CPU baseline and reference arm, and
__graft_entry__.smoke() use this.  It imports nothing from the library under
test: the byte layouts come from oracle/layouts.py.
"""
import ctypes
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load_module(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


_lib = _load_module("ae_oracle_layouts", os.path.join(ROOT, "oracle", "layouts.py"))
ORACLE = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SCENE = os.path.join(ROOT, "oracle", "_ref", "libaeref_scene.so")
REF_SHADER = os.path.join(ROOT, "oracle", "_ref", "libaeref_shader.so")

_P = ctypes.c_void_p


class OScene(ctypes.Structure):
    _fields_ = [("objects", _P), ("n_objects", ctypes.c_uint32), ("tlas", _P), ("n_nodes", ctypes.c_uint32),
                ("lights", _P), ("n_lights", ctypes.c_uint32), ("vertices", _P), ("indices", _P), ("blas", _P),
                ("instances", _P), ("tex", _P), ("tex_w", ctypes.c_uint32), ("tex_h", ctypes.c_uint32),
                ("tex_layers", ctypes.c_uint32)]


def texture_words(scene):
    """(words, width, height, layers) of a scene's texture array: RGBA8 as
    little-endian uint32 words, layer-major; (None, 0, 0, 0) without one."""
    t = getattr(scene, "textures", None)
    if t is None or len(t) == 0:
        return None, 0, 0, 0
    t = np.ascontiguousarray(t, np.uint8)
    layers, h, w, _ = t.shape
    return t.view(np.uint32).reshape(-1), w, h, layers


def ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


_cache = {}


def _load(path):
    if path not in _cache:
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        _cache[path] = ctypes.CDLL(path)
    return _cache[path]


def oracle():
    return _load(ORACLE)


def ref_available():
    return os.path.exists(REF_SCENE) and os.path.exists(REF_SHADER)


def ref_scene():
    return _load(REF_SCENE)


def ref_shader():
    return _load(REF_SHADER)


def oscene(scene):
    """An oracle Scene view; keeps the arrays alive on the returned object."""
    keep = [np.ascontiguousarray(a) for a in (scene.objects, scene.tlas, scene.lights, scene.vertices, scene.indices,
                                              scene.blas, scene.instances)]
    o, t, l, v, i, b, ins = keep
    tw, w, h, layers = texture_words(scene)
    s = OScene(ptr(o), len(o), ptr(t), len(t), ptr(l), len(l), ptr(v), ptr(i), ptr(b), ptr(ins), ptr(tw), w, h, layers)
    s._keep = keep + [tw]
    return s


def closest_hit(scene, rays, threads=0, counters=False):
    s = oscene(scene)
    r = np.ascontiguousarray(rays, dtype=_lib.RAY)
    hits = np.zeros(len(r), _lib.HIT)
    cnt = np.zeros(6, np.uint64)
    f = oracle().oracle_closest_hit
    f.restype = ctypes.c_int
    f(ctypes.byref(s), ptr(r), ctypes.c_uint32(len(r)), ptr(hits), ptr(cnt) if counters else None, ctypes.c_int(threads))
    return (hits, cnt) if counters else hits


def camera_rays(config):
    c = np.ascontiguousarray(np.array(config, dtype=_lib.CONFIG).reshape(1))
    out = np.zeros(int(c["width"][0]) * int(c["height"][0]), _lib.RAY)
    oracle().oracle_camera_rays(ptr(c), ptr(out))
    return out


def render_frame(scene, config, accum=None, precision=32, pixels=None, threads=0):
    """One frame; returns (accum, display, frame) as (H, W, 4) arrays."""
    s = oscene(scene)
    c = np.ascontiguousarray(np.array(config, dtype=_lib.CONFIG).reshape(1))
    w, h = int(c["width"][0]), int(c["height"][0])
    dt = np.float32 if precision == 32 else np.float64
    acc = np.zeros((h, w, 4), dt) if accum is None else np.ascontiguousarray(accum, dtype=dt).copy()
    disp = np.zeros((h, w, 4), dt)
    frame = np.zeros((h, w, 4), dt)
    xy = None if pixels is None else np.ascontiguousarray(pixels, dtype=np.uint32).reshape(-1, 2)
    fn = oracle().oracle_render_frame_f32 if precision == 32 else oracle().oracle_render_frame_f64
    fn(ctypes.byref(s), ptr(c), ptr(acc), ptr(disp), ptr(frame), ptr(xy), ctypes.c_uint32(0 if xy is None else len(xy)),
       ctypes.c_int(threads))
    return acc, disp, frame


def pixel_rays(scene, config, x, y, cap=8192):
    """Every closest-hit query the float oracle makes for pixel (x, y) in one
    frame (camera, shadow and bounce rays, in order)."""
    s = oscene(scene)
    c = np.ascontiguousarray(np.array(config, dtype=_lib.CONFIG).reshape(1))
    out = np.zeros(cap, _lib.RAY)
    f = oracle().oracle_pixel_rays
    f.restype = ctypes.c_uint32
    n = f(ctypes.byref(s), ptr(c), ctypes.c_uint32(x), ctypes.c_uint32(y), ptr(out), ctypes.c_uint32(cap))
    return out[:min(n, cap)].copy()


def counters_bytes(cnt):
    """Algorithmic bytes of the counted touches (the roofline's formula)."""
    t, o, i, b, tri, win = (int(x) for x in cnt)
    return 48 * t + 128 * o + 48 * i + 48 * b + 48 * tri + 60 * win


# --- the reference's own code ------------------------------------------------
def ref_bind(scene):
    L = ref_shader()
    keep = [np.ascontiguousarray(a) for a in (scene.objects, scene.tlas, scene.lights, scene.vertices, scene.indices,
                                              scene.blas, scene.instances)]
    o, t, l, v, i, b, ins = keep
    u32 = ctypes.c_uint32
    L.aeref_bind(ptr(o), u32(len(o)), ptr(t), u32(len(t)), ptr(l), u32(len(l)), ptr(v), u32(len(v)), ptr(i),
                 u32(len(i)), ptr(b), u32(len(b)), ptr(ins), u32(len(ins)))
    tw, w, h, layers = texture_words(scene)
    L.aeref_bind_textures(ptr(tw), u32(w), u32(h), u32(layers))
    _cache["_ref_keep"] = keep + [tw]


def ref_set_config(config):
    c = np.ascontiguousarray(np.array(config, dtype=_lib.CONFIG).reshape(1))
    ref_shader().aeref_set_config(ptr(c))


def ref_closest_hit(scene, rays, threads=0):
    ref_bind(scene)
    r = np.ascontiguousarray(rays, dtype=_lib.RAY)
    hits = np.zeros(len(r), _lib.HIT)
    ref_shader().aeref_closest_hit(ptr(r), ctypes.c_uint32(len(r)), ptr(hits), ctypes.c_int(threads))
    return hits


def ref_render(scene, config, accum=None, threads=0, pixels=None):
    ref_bind(scene)
    ref_set_config(config)
    w, h = int(config["width"]), int(config["height"])
    acc = np.zeros((h, w, 4), np.float32) if accum is None else np.ascontiguousarray(accum, np.float32).copy()
    disp = np.zeros((h, w, 4), np.float32)
    if pixels is None:
        ref_shader().aeref_render(ptr(acc), ptr(disp), ctypes.c_int(threads))
    else:
        xy = np.ascontiguousarray(pixels, dtype=np.uint32).reshape(-1, 2)
        ref_shader().aeref_render_pixels(ptr(xy), ctypes.c_uint32(len(xy)), ptr(acc), ptr(disp), ctypes.c_int(threads))
    return acc, disp


def ref_build_bvh(bounds):
    b = np.ascontiguousarray(bounds, dtype=np.float32).reshape(-1, 6)
    n = len(b)
    nodes = np.zeros(max(2 * n, 1), _lib.NODE)
    order = np.zeros(max(n, 1), np.uint32)
    cnt = ctypes.c_uint32()
    ref_scene().aeref_build_bvh(ptr(b), ctypes.c_uint32(n), ptr(nodes), ctypes.byref(cnt), ptr(order))
    return nodes[:cnt.value].copy(), order[:n].copy()


def ref_mesh_add(vertices, indices16):
    v = np.ascontiguousarray(np.stack([vertices[k] for k in ("px", "py", "pz", "nx", "ny", "nz", "u", "v")], 1),
                             np.float32)
    i = np.ascontiguousarray(indices16, np.uint16)
    ov = np.zeros(len(v), _lib.VERTEX)
    oi = np.zeros(len(i), np.uint32)
    ob = np.zeros(max(2 * (len(i) // 3), 1), _lib.NODE)
    nb = ctypes.c_uint32()
    ref_scene().aeref_mesh_add(ptr(v), ctypes.c_uint32(len(v)), ptr(i), ctypes.c_uint32(len(i)), ptr(ov), ptr(oi),
                               ptr(ob), ctypes.byref(nb))
    return ov, oi, ob[:nb.value].copy()


def ref_bounds(kind, position, rotation, a, b=None):
    p = np.asarray(position, np.float32)
    q = np.asarray(rotation, np.float32)
    a = np.asarray(a, np.float32)
    b = None if b is None else np.asarray(b, np.float32)
    out = np.zeros(6, np.float32)
    L = ref_scene()
    if kind == "mesh":
        L.aeref_mesh_bounds(ptr(p), ptr(q), ptr(a), ptr(out))
    elif kind == "quad":
        L.aeref_quad_bounds(ptr(p), ptr(q), ptr(a), ptr(b), ptr(out))
    elif kind == "box":
        L.aeref_box_bounds(ptr(p), ptr(q), ptr(a), ptr(out))
    return out


def bounce_rays(scene, config, primary, hits):
    s = oscene(scene)
    c = np.ascontiguousarray(np.array(config, dtype=_lib.CONFIG).reshape(1))
    p = np.ascontiguousarray(primary, dtype=_lib.RAY)
    h = np.ascontiguousarray(hits, dtype=_lib.HIT)
    out = np.zeros(len(p), _lib.RAY)
    valid = np.zeros(len(p), np.uint8)
    oracle().oracle_bounce_rays(ctypes.byref(s), ptr(c), ptr(p), ptr(h), ctypes.c_uint32(len(p)), ptr(out), ptr(valid))
    return out, valid.astype(bool)


class Planes(ctypes.Structure):
    _fields_ = [("gpos", _P), ("gnrm", _P), ("galb", _P), ("gdepth", _P), ("prev_img", _P), ("prev_geo", _P),
                ("img", _P), ("display", _P), ("reduced", _P), ("cur_geo", _P), ("red_w", ctypes.c_uint32),
                ("red_h", ctypes.c_uint32)]


def gbuffer(scene, config, threads=0):
    """The oracle's ray-cast G-buffer: (pos, nrm, alb_bytes, depth)."""
    s = oscene(scene)
    c = np.ascontiguousarray(np.array(config, dtype=_lib.CONFIG).reshape(1))
    w, h = int(c["width"][0]), int(c["height"][0])
    pos = np.zeros((h, w, 4), np.float32)
    nrm = np.zeros((h, w, 4), np.float32)
    alb = np.zeros((h, w, 4), np.uint8)
    dep = np.zeros((h, w), np.float32)
    oracle().oracle_gbuffer(ctypes.byref(s), ptr(c), ptr(pos), ptr(nrm), ptr(alb), ptr(dep), ctypes.c_int(threads))
    return pos, nrm, alb, dep


def albedo_float(alb):
    """RGBA8 UNORM as the shader reads it: byte / 255."""
    return (alb.astype(np.float32) / np.float32(255.0)).astype(np.float32)


def reduced_extent(config):
    s = np.float32(config["traceScale"])
    if s >= 1.0:
        return int(config["width"]), int(config["height"])
    return int(np.ceil(np.float32(config["width"]) * s)), int(np.ceil(np.float32(config["height"]) * s))


class HybridState:
    """Ping-pong history of the hybrid renderer for the CPU implementations."""

    def __init__(self, w, h):
        self.img = [np.zeros((h, w, 4), np.float32) for _ in range(2)]
        self.geo = [np.zeros((h, w, 4), np.float32) for _ in range(2)]
        self.display = np.zeros((h, w, 4), np.float32)
        self.history = 0
        self.reduced = None


def hybrid_frame(scene, config, gb, state, impl="oracle", threads=0):
    """One hybrid frame (deferred, then upsample when reduced) on the CPU by the
    oracle or by the reference's own shaders; mutates `state`."""
    pos, nrm, alb, dep = gb
    albf = albedo_float(alb)
    c = np.ascontiguousarray(np.array(config, dtype=_lib.CONFIG).reshape(1))
    w, h = int(c["width"][0]), int(c["height"][0])
    rw, rh = reduced_extent(c[0])
    reduced = np.zeros((rh, rw, 4), np.float32) if state.reduced is None or state.reduced.shape[:2] != (rh, rw) \
        else state.reduced
    writes = int(c["debugView"][0]) == 0 and int(c["displayOnly"][0]) == 0
    ws = 1 - state.history if writes else state.history
    rs = 1 - ws
    red = float(c["traceScale"][0]) < 1.0
    if impl == "oracle":
        s = oscene(scene)
        P = Planes(ptr(pos), ptr(nrm), ptr(albf), ptr(dep), ptr(state.img[rs]), ptr(state.geo[rs]), ptr(state.img[ws]),
                   ptr(state.display), ptr(reduced), ptr(state.geo[ws]), rw, rh)
        if not (red and int(c["displayOnly"][0])):
            oracle().oracle_deferred(ctypes.byref(s), ptr(c), ctypes.byref(P), ctypes.c_int(threads))
        if red:
            oracle().oracle_upsample(ctypes.byref(s), ptr(c), ctypes.byref(P), ctypes.c_int(threads))
    else:
        L = _load(os.path.join(ROOT, "oracle", "_ref", "libaeref_deferred.so"))
        keep = [np.ascontiguousarray(a) for a in (scene.objects, scene.tlas, scene.lights, scene.vertices,
                                                  scene.indices, scene.blas, scene.instances)]
        o, t, l, v, i, b, ins = keep
        u32 = ctypes.c_uint32
        L.aeref_d_bind(ptr(o), u32(len(o)), ptr(t), u32(len(t)), ptr(l), u32(len(l)), ptr(v), u32(len(v)), ptr(i),
                       u32(len(i)), ptr(b), u32(len(b)), ptr(ins), u32(len(ins)))
        tw, tw_w, tw_h, tw_l = texture_words(scene)
        L.aeref_d_bind_textures(ptr(tw), u32(tw_w), u32(tw_h), u32(tw_l))
        keep.append(tw)
        L.aeref_d_set_config(ptr(c))
        if not (red and int(c["displayOnly"][0])):
            L.aeref_deferred(ptr(pos), ptr(nrm), ptr(albf), ptr(dep), ptr(state.img[rs]), ptr(state.geo[rs]),
                             ptr(state.img[ws]), ptr(state.display), ptr(reduced), u32(rw), u32(rh), ptr(state.geo[ws]),
                             ctypes.c_int(threads))
        if red:
            L.aeref_upsample(ptr(pos), ptr(nrm), ptr(albf), ptr(reduced), u32(rw), u32(rh), ptr(state.img[rs]),
                             ptr(state.geo[rs]), ptr(state.img[ws]), ptr(state.display), ptr(state.geo[ws]),
                             ctypes.c_int(threads))
    state.reduced = reduced
    if writes:
        state.history = ws
    return state


def any_hit(scene, rays, tmax, threads=0):
    s = oscene(scene)
    r = np.ascontiguousarray(rays, dtype=_lib.RAY)
    t = np.ascontiguousarray(tmax, dtype=np.float32)
    out = np.zeros(len(r), np.uint8)
    oracle().oracle_any_hit(ctypes.byref(s), ptr(r), ptr(t), ctypes.c_uint32(len(r)), ptr(out), ctypes.c_int(threads))
    return out


def ggx_samples(d, n, albedo, alpha, seed, count):
    """`count` GGX metal samples of the FP64 oracle: (directions (count, 3),
    weights (count, 3), continues (count,) bool)."""
    out = np.zeros((count, 7), np.float64)
    a = [np.ascontiguousarray(x, np.float64) for x in (d, n, albedo)]
    oracle().oracle_ggx_samples(ptr(a[0]), ptr(a[1]), ptr(a[2]), ctypes.c_double(alpha), ctypes.c_uint32(seed),
                                ctypes.c_uint32(count), ptr(out))
    return out[:, 0:3], out[:, 3:6], out[:, 6] > 0.5
