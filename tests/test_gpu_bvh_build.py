"""The device SAH builder (ae_build_bvh_gpu) against the host builder and
the reference's own BuildBVH compiled for the CPU (oracle/_ref): the same
nodes and the same leaf-slot order, byte for byte, whichever of its two
phases (one tree level per round over blocks of boxes, or one warp per
subtree) builds each node.  Also the mesh library's device path
(ae_mesh_library_add_gpu) and whole scenes built with it."""
import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import AeError, scenes

pytestmark = pytest.mark.gpu

# warp_subtree: None = the default (256); 0 = every node in the level
# rounds; 1 << 30 = the whole tree in one warp.
PHASES = [None, 0, 4, 37, 1024, 1 << 30]


def boxes(n, seed, flat=0.0, dup=0.0, zeros=0.0, spread=50.0):
    rng = np.random.default_rng(seed)
    c = rng.normal(0, spread, (n, 3)).astype(np.float32)
    e = rng.uniform(0, 3, (n, 3)).astype(np.float32)
    e[rng.random((n, 3)) < flat] = 0
    c[: int(n * dup)] = c[0]
    b = np.concatenate([c - e, c + e], 1)
    if zeros:
        # Coordinates of both zero signs in random order: the node box must
        # carry the sign of the first zero in each node's range.
        z = rng.random(b.shape) < zeros
        b[z] = np.where(rng.random(int(z.sum())) < 0.5, np.float32(0.0), np.float32(-0.0))
        b[:, :3] = np.minimum(b[:, :3], b[:, 3:])
    return b


def check_same(b, warp_subtree=None, with_reference=True):
    g_nodes, g_order = scenes.build_bvh(b, gpu=True, warp_subtree=warp_subtree)
    h_nodes, h_order = scenes.build_bvh(b)
    assert len(g_nodes) == len(h_nodes)
    assert np.array_equal(g_nodes.view(np.uint8), h_nodes.view(np.uint8))
    assert np.array_equal(g_order, h_order)
    if with_reference and O.ref_available():
        r_nodes, r_order = O.ref_build_bvh(b)
        assert np.array_equal(g_nodes.view(np.uint8), r_nodes.view(np.uint8))
        assert np.array_equal(g_order, r_order)
    return g_nodes


@pytest.mark.parametrize("warp_subtree", PHASES)
@pytest.mark.parametrize("n,seed,flat,dup,zeros", [
    (1, 0, 0, 0, 0), (2, 1, 0, 0, 0), (5, 2, 0.5, 0, 0), (64, 3, 1.0, 1.0, 0), (100, 4, 0.3, 0.5, 0),
    (1023, 5, 0, 0, 0), (1025, 6, 0.1, 0, 0), (3000, 7, 0.3, 0.2, 0.3), (5000, 8, 0, 0.5, 0),
    (40000, 9, 0.05, 0.01, 0.02)])
def test_random_boxes(n, seed, flat, dup, zeros, warp_subtree):
    check_same(boxes(n, seed, flat, dup, zeros), warp_subtree)


@pytest.mark.parametrize("warp_subtree", [None, 0])
def test_large(warp_subtree):
    check_same(boxes(400_000, 11, flat=0.1, dup=0.001, zeros=0.001, spread=300.0), warp_subtree,
               with_reference=False)


def test_signed_zeros_everywhere():
    # Every box touches the planes x = 0, y = 0 or z = 0 with either zero.
    rng = np.random.default_rng(12)
    n = 6000
    b = np.abs(rng.normal(0, 5, (n, 6))).astype(np.float32)
    b[:, :3] = -b[:, :3]
    z = rng.random((n, 6)) < 0.5
    b[z] = np.where(rng.random(int(z.sum())) < 0.5, np.float32(0.0), np.float32(-0.0))
    for ws in PHASES:
        check_same(b, ws)


def test_depth_cap_leaves():
    # Centroids in a geometric progression: the SAH peels a few boxes off per
    # level and the depth-20 cap ends the left spine in a leaf of > 4 boxes.
    c = np.array([[1.7 ** (i % 80), 0.0, 0.0] for i in range(5000)], np.float32)
    b = np.concatenate([c - 0.25, c + 0.25], 1)
    for ws in PHASES:
        nodes = check_same(b, ws)
        assert nodes["count"].max() > 4


def test_identical_boxes_median_splits():
    b = np.tile(np.array([[1, 2, 3, 4, 5, 6]], np.float32), (3000, 1))
    for ws in (None, 0, 1 << 30):
        nodes = check_same(b, ws)
        assert nodes["count"].max() <= 4


def test_empty_and_non_finite():
    nodes, order = scenes.build_bvh(np.zeros((0, 6), np.float32), gpu=True)
    assert len(nodes) == 0 and len(order) == 0
    for bad in (np.nan, np.inf, -np.inf):
        b = boxes(100, 13)
        b[37, 4] = bad
        with pytest.raises(AeError) as e:
            scenes.build_bvh(b, gpu=True)
        assert e.value.code == -1  # AE_ERR_INVALID


def _library(gpu, rng_seed=14):
    rng = np.random.default_rng(rng_seed)
    lib = scenes.MeshLibrary(gpu=gpu)
    handles = [lib.add(*scenes.heightfield(300, 20.0, 2.5, rng)), lib.add(*scenes.icosphere(6, 5.0)),
               lib.add(*scenes.box_mesh((1.0, 2.0, 0.5))),
               lib.add(*scenes.quad_mesh((2.0, 0.0, 0.0), (0.0, 0.0, 3.0)), double_sided=True),
               lib.add(*scenes.icosphere(2, 1.0))]
    return lib, handles


def test_mesh_library_gpu_equals_host():
    g, gh = _library(True)
    h, hh = _library(False)
    for a, b in zip(g.arrays(), h.arrays()):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    for x, y in zip(gh, hh):
        assert g.range(x).tobytes() == h.range(y).tobytes()


def test_scene_built_on_gpu_equals_host():
    kw = dict(seed=15, width=64, height=48, depth=4, n_meshes=6, n_instances=40, n_lights=4, target_tris=400_000)
    a = scenes.wavefront_scene(gpu_build=True, **kw)
    b = scenes.wavefront_scene(gpu_build=False, **kw)
    for name in ("objects", "tlas", "lights", "vertices", "indices", "blas", "instances"):
        assert np.array_equal(getattr(a, name).view(np.uint8), getattr(b, name).view(np.uint8)), name


def test_device_pointer_entry_points():
    import ctypes

    import torch
    from aviatorengine2_b200 import _lib
    from aviatorengine2_b200._lib import lib
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    b = boxes(20000, 16, flat=0.2, zeros=0.05)
    d_b = torch.from_numpy(b.view(np.uint8)).to(dev)
    d_n = torch.empty(2 * len(b) * 48, dtype=torch.uint8, device=dev)
    d_o = torch.empty(len(b), dtype=torch.int32, device=dev)
    cnt = ctypes.c_uint32()
    assert lib().ae_build_bvh_device(d_b.data_ptr(), len(b), 64, d_n.data_ptr(), ctypes.byref(cnt), d_o.data_ptr(),
                                     ctypes.c_void_p(stream.cuda_stream)) == 0
    h_nodes, h_order = scenes.build_bvh(b)
    assert cnt.value == len(h_nodes)
    assert np.array_equal(d_n[: cnt.value * 48].cpu().numpy(), h_nodes.view(np.uint8).ravel())
    assert np.array_equal(d_o.cpu().numpy().view(np.uint32), h_order)

    v, i = scenes.icosphere(5, 2.0)
    d_v = torch.from_numpy(np.ascontiguousarray(v, _lib.VERTEX).view(np.uint8)).to(dev)
    d_i = torch.from_numpy(np.ascontiguousarray(i, np.uint32).view(np.int32)).to(dev)
    d_n = torch.empty(2 * (len(i) // 3) * 48, dtype=torch.uint8, device=dev)
    d_o = torch.empty(len(i), dtype=torch.int32, device=dev)
    assert lib().ae_mesh_blas_device(d_v.data_ptr(), len(v), d_i.data_ptr(), len(i), d_n.data_ptr(),
                                     ctypes.byref(cnt), d_o.data_ptr(), ctypes.c_void_p(stream.cuda_stream)) == 0
    host = scenes.MeshLibrary()
    host.add(v, i)
    _, h_idx, h_blas = host.arrays()
    assert np.array_equal(d_n[: cnt.value * 48].cpu().numpy(), h_blas.view(np.uint8).ravel())
    assert np.array_equal(d_o.cpu().numpy().view(np.uint32), h_idx)
    # An index past the vertex count is refused before any vertex is read.
    d_i[7] = len(v)
    assert lib().ae_mesh_blas_device(d_v.data_ptr(), len(v), d_i.data_ptr(), len(i), d_n.data_ptr(),
                                     ctypes.byref(cnt), d_o.data_ptr(), ctypes.c_void_p(stream.cuda_stream)) == -4
    lib().ae_bvh_builder_release()


def _entities(n, seed, meshes, handles):
    """n entities of every shape and material, meshes instanced from
    `handles`, about 2 % emissive."""
    from aviatorengine2_b200 import _lib
    rng = np.random.default_rng(seed)
    shapes = [_lib.SHAPE_SPHERE, _lib.SHAPE_QUAD, _lib.SHAPE_TRIANGLE, _lib.SHAPE_BOX, _lib.SHAPE_MESH]
    mats = [_lib.MAT_LAMBERTIAN, _lib.MAT_METAL, _lib.MAT_DIELECTRIC]
    out = []
    for k in range(n):
        shape = shapes[int(rng.integers(0, 5))]
        mat = _lib.MAT_DIFFUSE_LIGHT if rng.random() < 0.02 else mats[int(rng.integers(0, 3))]
        pos = tuple(float(x) for x in rng.uniform(-200, 200, 3))
        kw = dict(albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)), emission=4.0, fuzz=0.1)
        if shape == _lib.SHAPE_SPHERE:
            kw["radius"] = float(rng.uniform(0.2, 3))
        elif shape in (_lib.SHAPE_QUAD, _lib.SHAPE_TRIANGLE):
            kw["u"], kw["v"] = (float(rng.uniform(0.5, 4)), 0.0, 0.0), (0.0, 0.0, float(rng.uniform(0.5, 4)))
        elif shape == _lib.SHAPE_BOX:
            kw["half_extent"] = tuple(float(x) for x in rng.uniform(0.2, 2, 3))
        else:
            kw["mesh"] = handles[int(rng.integers(0, len(handles)))]
            kw["scale"] = float(rng.uniform(0.5, 2.0))
        rot = scenes.random_quat(rng) if shape != _lib.SHAPE_SPHERE else scenes.yaw_quat(float(rng.uniform(0, 6)))
        out.append(scenes.entity(shape, mat, pos, rotation=rot, **kw))
    return out


@pytest.mark.parametrize("n", [1, 7, 900, 5000, 70000])
def test_pack_scene_gpu_equals_host(n):
    meshes, handles = _library(False)
    ents = _entities(n, 17 + n, meshes, handles)
    g = scenes.pack(ents, meshes, gpu=True)
    h = scenes.pack(ents, meshes)
    for a, b in zip(g, h):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_rebuild_scene_equals_reference_rebuild():
    # A moved scene rebuilt on the device renders the frames of the same scene
    # packed on the host and uploaded: the reference's rebuild, exactly.
    from aviatorengine2_b200 import Context, _lib
    meshes, handles = _library(False)
    ents = _entities(600, 18, meshes, handles)
    cfg = scenes.make_config(64, 48, (0.0, 60.0, 420.0), (0.0, 0.0, 0.0), fov=60.0, depth=4, sky=(0.3, 0.4, 0.5))
    first = scenes._finish(ents, meshes, cfg, "entities")
    rng = np.random.default_rng(19)
    moved = []
    for e in ents:
        m = e.copy()
        m["prev_position"], m["prev_rotation"] = e["position"], e["rotation"]
        m["position"] = e["position"] + rng.normal(0, 3.0, 3).astype(np.float32)
        moved.append(m)
    twin_scene = scenes._finish(moved, meshes, cfg, "entities moved")
    with Context(64, 48) as ctx, Context(64, 48) as twin:
        ctx.upload(first)
        ctx.rebuild_scene(moved, meshes)
        twin.upload(twin_scene)
        for a, b in zip(ctx.download_scene(), twin.download_scene()):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
        c = twin_scene.config.copy()
        for b in range(2):
            c["batch"] = b
            for x in (ctx, twin):
                x.set_config(c)
                x.render_frame(_lib.MODE_COMPUTE_ONLY)
        assert np.array_equal(ctx.read_image(_lib.IMAGE_ACCUM).view(np.uint32),
                              twin.read_image(_lib.IMAGE_ACCUM).view(np.uint32))


def _forest_meshes():
    rng = np.random.default_rng(21)
    return [scenes.heightfield(200, 20.0, 2.5, rng), scenes.box_mesh((1.0, 2.0, 0.5)),
            (np.zeros(0, dtype=scenes._lib.VERTEX), np.zeros(0, np.uint32)), scenes.icosphere(5, 3.0),
            scenes.quad_mesh((2.0, 0.0, 0.0), (0.0, 0.0, 3.0)), scenes.icosphere(1, 1.0),
            scenes.heightfield(64, 10.0, 1.0, rng)]


def test_library_add_many_equals_separate_adds():
    meshes = _forest_meshes()
    ds = [False, False, False, False, True, False, False]
    g = scenes.MeshLibrary(gpu=True)
    gh = g.add_many(meshes, ds)
    h = scenes.MeshLibrary()
    hh = [h.add(v, i, d) for (v, i), d in zip(meshes, ds)]
    assert gh == hh
    for a, b in zip(g.arrays(), h.arrays()):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    for x, y in zip(gh, hh):
        assert g.range(x).tobytes() == h.range(y).tobytes()


def test_device_many_equals_per_mesh():
    import ctypes

    import torch
    from aviatorengine2_b200 import _lib
    from aviatorengine2_b200._lib import lib
    meshes = [m for m in _forest_meshes() if len(m[1])]
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    k = len(meshes)
    d_v = [torch.from_numpy(np.ascontiguousarray(v, _lib.VERTEX).view(np.uint8)).to(dev) for v, _ in meshes]
    d_i = [torch.from_numpy(np.ascontiguousarray(i, np.uint32).view(np.int32)).to(dev) for _, i in meshes]
    d_n = [torch.empty(2 * (len(i) // 3) * 48, dtype=torch.uint8, device=dev) for _, i in meshes]
    d_o = [torch.empty(len(i), dtype=torch.int32, device=dev) for _, i in meshes]
    P = ctypes.c_void_p
    nv = np.array([len(v) for v, _ in meshes], np.uint32)
    ni = np.array([len(i) for _, i in meshes], np.uint32)
    counts = np.zeros(k, np.uint32)
    for _ in range(2):  # twice: the builder's scratch is reused
        rc = lib().ae_mesh_blas_device_many(k, (P * k)(*[t.data_ptr() for t in d_v]), _lib.ptr(nv),
                                            (P * k)(*[t.data_ptr() for t in d_i]), _lib.ptr(ni),
                                            (P * k)(*[t.data_ptr() for t in d_n]), _lib.ptr(counts),
                                            (P * k)(*[t.data_ptr() for t in d_o]), P(stream.cuda_stream))
        assert rc == 0
        for m, (v, i) in enumerate(meshes):
            host = scenes.MeshLibrary()
            host.add(v, i)
            _, h_idx, h_blas = host.arrays()
            assert counts[m] == len(h_blas)
            assert np.array_equal(d_n[m][: int(counts[m]) * 48].cpu().numpy(), h_blas.view(np.uint8).ravel())
            assert np.array_equal(d_o[m].cpu().numpy().view(np.uint32), h_idx)
