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

# warp_subtree: None = the default (1024); 0 = every node in the level
# rounds; 1 << 30 = the whole tree in one warp.
PHASES = [None, 0, 4, 37, 1 << 30]


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
