"""ctypes binding of libae_b200.so and numpy dtypes of its byte contract.

Loading fails loudly when the library is missing: there is no fallback path.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libae_b200.so")

# --- byte contract (include/ae_b200.h) --------------------------------------
VERTEX = np.dtype([("px", "<f4"), ("py", "<f4"), ("pz", "<f4"), ("nx", "<f4"), ("ny", "<f4"), ("nz", "<f4"),
                   ("u", "<f4"), ("v", "<f4")])
NODE = np.dtype([("min_x", "<f4"), ("min_y", "<f4"), ("min_z", "<f4"), ("pad0", "<f4"), ("max_x", "<f4"),
                 ("max_y", "<f4"), ("max_z", "<f4"), ("left", "<i4"), ("right", "<i4"), ("count", "<i4"),
                 ("padding", "<i4"), ("pad_trailing", "<i4")])
OBJECT = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("prevRotX", "<f4"), ("x2", "<f4"), ("y2", "<f4"),
                   ("z2", "<f4"), ("radius", "<f4"), ("u_x", "<f4"), ("u_y", "<f4"), ("u_z", "<f4"),
                   ("prevRotY", "<f4"), ("v_x", "<f4"), ("v_y", "<f4"), ("v_z", "<f4"), ("prevRotZ", "<f4"),
                   ("half_x", "<f4"), ("half_y", "<f4"), ("half_z", "<f4"), ("rotation", "<f4"),
                   ("density", "<f4"), ("emission", "<f4"), ("instanceIndex", "<u4"), ("textureTint", "<f4"),
                   ("r", "<f4"), ("g", "<f4"), ("b", "<f4"), ("fuzz", "<f4"), ("refraction", "<f4"),
                   ("shapeType", "<u4"), ("colorType", "<u4"), ("textureID", "<u4")])
INSTANCE = np.dtype([("px", "<f4"), ("py", "<f4"), ("pz", "<f4"), ("scale", "<f4"), ("qx", "<f4"), ("qy", "<f4"),
                     ("qz", "<f4"), ("qw", "<f4"), ("vertexBase", "<u4"), ("indexBase", "<u4"),
                     ("triangleCount", "<u4"), ("blasBase", "<u4")])
AABB = np.dtype([("min_x", "<f4"), ("min_y", "<f4"), ("min_z", "<f4"), ("max_x", "<f4"), ("max_y", "<f4"),
                 ("max_z", "<f4")])
RAY = np.dtype([("ox", "<f4"), ("oy", "<f4"), ("oz", "<f4"), ("tnear", "<f4"), ("dx", "<f4"), ("dy", "<f4"),
                ("dz", "<f4"), ("time", "<f4")])
HIT = np.dtype([("t", "<f4"), ("alpha", "<f4"), ("beta", "<f4"), ("object", "<u4"), ("prim", "<u4")])
CONFIG = np.dtype([("source_x", "<f4"), ("source_y", "<f4"), ("source_z", "<f4"), ("fov", "<f4"),
                   ("target_x", "<f4"), ("target_y", "<f4"), ("target_z", "<f4"), ("focus_dist", "<f4"),
                   ("defocus_angle", "<f4"), ("padding", "<f4", 3), ("up_x", "<f4"), ("up_y", "<f4"),
                   ("up_z", "<f4"), ("oof", "<f4"), ("sky_r", "<f4"), ("sky_g", "<f4"), ("sky_b", "<f4"),
                   ("width", "<u4"), ("horizon_r", "<f4"), ("horizon_g", "<f4"), ("horizon_b", "<f4"),
                   ("height", "<u4"), ("samples", "<u4"), ("batches", "<u4"), ("batch", "<u4"), ("depth", "<u4"),
                   ("num_spheres", "<u4"), ("renderType", "<u4"), ("num_lights", "<u4"), ("exposure", "<f4"),
                   ("debugView", "<u4"), ("zNear", "<f4"), ("zFar", "<f4"), ("jitter_x", "<f4"),
                   ("jitter_y", "<f4"), ("displayOnly", "<u4"), ("traceScale", "<f4"), ("frameIndex", "<u4"),
                   ("historyReset", "<u4"), ("cameraMoved", "<u4"), ("historyCap", "<f4"), ("padding3", "<f4"),
                   ("prevViewProj", "<f4", 16)])
ENTITY = np.dtype([("shape", "<u4"), ("material", "<u4"), ("position", "<f4", 3), ("rotation", "<f4", 4),
                   ("scale", "<f4"), ("albedo", "<f4", 3), ("fuzz", "<f4"), ("ior", "<f4"), ("emission", "<f4"),
                   ("density", "<f4"), ("texture_tint", "<f4"), ("texture_id", "<u4"), ("radius", "<f4"),
                   ("u", "<f4", 3), ("v", "<f4", 3), ("half_extent", "<f4", 3), ("mesh", "<u4"),
                   ("prev_position", "<f4", 3), ("prev_rotation", "<f4", 4)])
SETTINGS = np.dtype([("width", "<u4"), ("height", "<u4"), ("samples", "<u4"), ("max_samples", "<u4"),
                     ("hybrid", "<u4"), ("hybrid_max_depth", "<u4"), ("trace_scale", "<f4"),
                     ("history_while_moving", "<u4"), ("device", "<i4"), ("reserved", "<u4", 7)])
QNODE = np.dtype([("origin", "<f4", 3), ("exp", "i1", 3), ("nchild", "u1"), ("lo", "u1", (3, 4)),
                  ("hi", "u1", (3, 4)), ("child", "<u4", 4), ("pad", "<u4", 2)])
MESH_RANGE = np.dtype([("vertexBase", "<u4"), ("indexBase", "<u4"), ("triangleCount", "<u4"), ("blasBase", "<u4"),
                       ("localBounds", AABB), ("doubleSided", "<u4")])

SERVE_SETTINGS = np.dtype([("device", "<i4"), ("slots", "<u4"), ("max_lights", "<u4"), ("max_requests", "<u4"),
                           ("arena_bytes", "<u8"), ("ticks_per_launch", "<u4"), ("extend_threads", "<u4"),
                           ("max_scenes", "<u4"), ("claim_policy", "<u4"), ("queue_run", "<u4"),
                           ("reserved", "<u4", 3)])
SERVE_REQUEST = np.dtype([("scene", "<u4"), ("width", "<u4"), ("height", "<u4"), ("frames", "<u4"),
                          ("config", CONFIG), ("accum", "<u8"), ("display", "<u8"), ("user", "<u8")])
SERVE_RESULT = np.dtype([("id", "<u8"), ("user", "<u8"), ("status", "<i4"), ("scene_version", "<u4"),
                         ("submit_ms", "<f8"), ("admit_ms", "<f8"), ("done_ms", "<f8"), ("paths", "<u8"),
                         ("footprint", "<u8")])
SERVE_STATS = np.dtype([("submitted", "<u8"), ("completed", "<u8"), ("rejected", "<u8"), ("failed", "<u8"),
                        ("paths", "<u8"), ("rays", "<u8"), ("first_submit_ms", "<f8"), ("last_done_ms", "<f8"),
                        ("p50_ms", "<f8"), ("p99_ms", "<f8"), ("mean_ms", "<f8"), ("max_ms", "<f8"),
                        ("launches", "<u8"), ("peak_arena_bytes", "<u8"), ("peak_resident", "<u4"),
                        ("moves_applied", "<u4"), ("errors", "<u4"), ("cancelled", "<u4"),
                        ("moves_coalesced", "<u4"), ("pad", "<u4")])
POLICY_EVENT = np.dtype([("kind", "<u4"), ("scene", "<u4"), ("tick", "<u4"), ("service_ticks", "<u4"),
                         ("footprint", "<u8")])
POLICY_OUTCOME = np.dtype([("admit_tick", "<i4"), ("done_tick", "<i4"), ("version", "<u4"), ("status", "<i4"),
                           ("offset", "<u8")])

for _dt, _size in ((VERTEX, 32), (NODE, 48), (OBJECT, 128), (INSTANCE, 48), (RAY, 32), (HIT, 20), (CONFIG, 240),
                   (AABB, 24), (SETTINGS, 64), (QNODE, 64), (SERVE_SETTINGS, 56), (SERVE_REQUEST, 280),
                   (SERVE_RESULT, 64), (SERVE_STATS, 136), (POLICY_EVENT, 24), (POLICY_OUTCOME, 24)):
    assert _dt.itemsize == _size, (_dt, _size)

# Enumerations (include/ae_b200.h)
SHAPE_SPHERE, SHAPE_QUAD, SHAPE_BOX, SHAPE_TRIANGLE, SHAPE_MESH = range(5)
MAT_LAMBERTIAN, MAT_METAL, MAT_DIELECTRIC, MAT_DIFFUSE_LIGHT, MAT_ISOTROPIC, MAT_GGX_METAL = range(6)
NO_TEXTURE = 0xFFFFFFFF
MISS = 0xFFFFFFFF
VARIANT_PLAIN, VARIANT_FAST, VARIANT_QUANT, VARIANT_FAST_WALK, VARIANT_PLAIN_WT, VARIANT_PLAIN_CHECKED = 0, 1, 2, 3, 4, 5
MODE_COMPUTE_ONLY, MODE_DEFERRED, MODE_WAVEFRONT, MODE_WAVEFRONT_PRECISION = 0, 1, 2, 3
IMAGE_ACCUM, IMAGE_DISPLAY, IMAGE_FRAME, IMAGE_REDUCED, IMAGE_HISTORY_GEOMETRY = range(5)
POLICY_REQUEST, POLICY_MOVE, POLICY_CANCEL = 0, 1, 2
CLAIM_OLDEST_FIRST, CLAIM_SHARED = 0, 1
STATUS = {0: "AE_OK", -1: "AE_ERR_INVALID", -2: "AE_ERR_OOM", -3: "AE_ERR_OVERSIZE", -4: "AE_ERR_LAYOUT",
          -5: "AE_ERR_CUDA", -6: "AE_ERR_TIMEOUT", -7: "AE_ERR_STATE", -8: "AE_ERR_REJECTED", -9: "AE_ERR_CANCELLED"}
FAULT_TILE_WAIT = 1
FAULT_CHECK_LIMITS = 2
CHECK_STACK, CHECK_INDEX = 1, 2

# Every symbol include/ae_b200.h declares, with (restype, argtypes).
_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_I = ctypes.c_int
SIGNATURES = {
    "ae_build_bvh": (_I, [_P, _U32, _P, _P, _P]),
    "ae_build_bvh_gpu": (_I, [_P, _U32, _P, _P, _P]),
    "ae_build_bvh_gpu_ex": (_I, [_P, _U32, _U32, _P, _P, _P]),
    "ae_build_bvh_device": (_I, [_P, _U32, _U32, _P, _P, _P, _P]),
    "ae_mesh_blas_device": (_I, [_P, _U32, _P, _U32, _P, _P, _P, _P]),
    "ae_mesh_blas_device_many": (_I, [_U32, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ae_bvh_builder_release": (None, []),
    "ae_mesh_library_create": (_P, []),
    "ae_mesh_library_destroy": (None, [_P]),
    "ae_mesh_library_add": (_I, [_P, _P, _U32, _P, _U32, _I]),
    "ae_mesh_library_add_gpu": (_I, [_P, _P, _U32, _P, _U32, _I]),
    "ae_mesh_library_add_many_gpu": (_I, [_P, _U32, _P, _P, _P, _P, _P, _P]),
    "ae_mesh_library_range": (_I, [_P, _U32, _P]),
    "ae_mesh_library_sizes": (None, [_P, _P, _P, _P]),
    "ae_mesh_library_vertices": (_P, [_P]),
    "ae_mesh_library_indices": (_P, [_P]),
    "ae_mesh_library_blas": (_P, [_P]),
    "ae_pack_scene": (_I, [_P, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ae_pack_scene_gpu": (_I, [_P, _U32, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ae_entity_bounds": (_I, [_P, _P, _P]),
    "ae_create": (_P, [_P]),
    "ae_destroy": (None, [_P]),
    "ae_last_error": (ctypes.c_char_p, [_P]),
    "ae_upload_geometry": (_I, [_P, _P, _U32, _P, _U32, _P, _U32]),
    "ae_reserve_scene": (_I, [_P, _U32, _U32]),
    "ae_upload_textures": (_I, [_P, _P, _U32, _U32, _U32]),
    "ae_upload_scene": (_I, [_P, _P, _U32, _P, _U32, _P, _U32, _P, _U32]),
    "ae_set_config": (_I, [_P, _P]),
    "ae_get_config": (_I, [_P, _P]),
    "ae_reset_accumulation": (_I, [_P]),
    "ae_render_frame": (_I, [_P, _I, _P]),
    "ae_build_gbuffer": (_I, [_P]),
    "ae_read_image": (_I, [_P, _I, _P, ctypes.c_size_t]),
    "ae_image_error": (_I, [_P, _I, _P, ctypes.c_double, _P]),
    "ae_image_error_pixels": (_I, [_P, _I, _P, _U32, _P, ctypes.c_double, _P]),
    "ae_closest_hit": (_I, [_P, _P, _U32, _P, _I]),
    "ae_closest_hit_device": (_I, [_P, _P, _U32, _P, _I]),
    "ae_closest_hit_noalloc": (_I, [_P, _P, _U32, _P, _I]),
    "ae_any_hit": (_I, [_P, _P, _P, _U32, _P]),
    "ae_camera_rays": (_I, [_P, _P]),
    "ae_bounce_rays": (_I, [_P, _P, _P, _U32, _P, _P]),
    "ae_trace_counters": (_I, [_P, _P, _U32, _P]),
    "ae_trace_counters_variant": (_I, [_P, _P, _U32, _I, _P]),
    "ae_path_counters": (_I, [_P, _P]),
    "ae_wavefront_info": (_I, [_P, _P, _P, _P, _P]),
    "ae_wavefront_walk_info": (_I, [_P, ctypes.c_int, _P, _P, _P, _P, _P]),
    "ae_wavefront_set_walk_runs": (_I, [_P, ctypes.c_int, _U32, _U32, _U32, _U32]),
    "ae_synchronize": (_I, [_P]),
    "ae_last_kernel_ms": (_I, [_P, _P]),
    "ae_stream": (_P, [_P]),
    "ae_launch_count": (ctypes.c_uint64, [_P]),
    "ae_prepare_fast": (_I, [_P]),
    "ae_refit_instances": (_I, [_P, _P, _U32]),
    "ae_rebuild_scene": (_I, [_P, _P, _U32, _P]),
    "ae_scene_sizes": (_I, [_P, _P, _P, _P, _P]),
    "ae_download_scene": (_I, [_P, _P, _P, _P]),
    "ae_build_wide_bvh": (_I, [_P, _U32, _U32, _P, _U32, _P, _P, _P]),
    "ae_serve_create": (_P, [_P]),
    "ae_serve_destroy": (None, [_P]),
    "ae_serve_last_error": (ctypes.c_char_p, [_P]),
    "ae_serve_add_scene": (_I, [_P, _P, _P]),
    "ae_serve_submit": (_I, [_P, _P, _P]),
    "ae_serve_move_instances": (_I, [_P, _U32, _P, _U32]),
    "ae_serve_cancel": (_I, [_P, ctypes.c_uint64]),
    "ae_serve_wait": (_I, [_P, ctypes.c_uint64, ctypes.c_int32, _P]),
    "ae_serve_drain": (_I, [_P, ctypes.c_int32]),
    "ae_serve_get_stats": (_I, [_P, _P]),
    "ae_serve_reset_stats": (_I, [_P]),
    "ae_serve_policy_simulate": (_I, [_P, _U32, ctypes.c_uint64, _U32, _U32, _U32, _U32, _P]),
    "ae_debug_fail_alloc_after": (_I, [ctypes.c_int64]),
    "ae_debug_live_allocations": (ctypes.c_int64, []),
    "ae_create_status": (_I, []),
    "ae_debug_inject": (_I, [_P, _I, _U32]),
    "ae_debug_flags": (_I, [_P, _P]),
    "ae_serve_debug_inject": (_I, [_P, _I, _U32]),
}

_lib = None


def lib():
    """The loaded library (built by aviatorengine2_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m aviatorengine2_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a):
    """Address of a numpy array's data (None for None)."""
    if a is None:
        return None
    return ctypes.c_void_p(a.ctypes.data)


class AeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def check(code, ctx=None, what=""):
    if code != 0:
        msg = lib().ae_last_error(ctx).decode() if ctx else what
        raise AeError(code, msg or what)
    return code
