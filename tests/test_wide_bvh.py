"""The 4-wide quantised BVH built for the optimised kernels (host side, no
GPU): every binary leaf appears exactly once, every decoded child box
contains the exact binary box (outward rounding: no hit can be lost), links
stay in range and the traversal stack bound holds."""
import ctypes

import numpy as np
import pytest

from aviatorengine2_b200 import _lib, scenes

LEAF = 0x80000000


def build(blas, tri_count):
    out = np.zeros(max(len(blas), 1), _lib.QNODE)
    cnt, root, stack = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_int32()
    rc = _lib.lib().ae_build_wide_bvh(_lib.ptr(blas), len(blas), tri_count, _lib.ptr(out), len(out),
                                      ctypes.byref(cnt), ctypes.byref(root), ctypes.byref(stack))
    assert rc == 0, rc
    return out[:cnt.value], root.value, stack.value


def binary_leaves(blas):
    return sorted((int(n["left"]), int(n["count"])) for n in blas if n["count"] > 0)


def decoded(q, k):
    s = np.ldexp(np.float32(1.0), q["exp"].astype(np.int32)).astype(np.float32)
    lo = np.array([np.fma(np.float32(q["lo"][a][k]), s[a], q["origin"][a]) if hasattr(np, "fma") else
                   np.float32(q["lo"][a][k]) * s[a] + q["origin"][a] for a in range(3)], np.float64)
    hi = np.array([np.float32(q["hi"][a][k]) * s[a] + q["origin"][a] for a in range(3)], np.float64)
    return lo, hi


@pytest.mark.parametrize("mesh", ["sphere5", "grid128", "box"])
def test_wide_bvh_structure(mesh):
    rng = np.random.default_rng(4)
    lib = scenes.MeshLibrary()
    if mesh == "sphere5":
        h = lib.add(*scenes.icosphere(5, 3.0))
    elif mesh == "grid128":
        h = lib.add(*scenes.heightfield(128, 40.0, 3.0, rng))
    else:
        h = lib.add(*scenes.box_mesh((1, 2, 3)))
    v, i, blas = lib.arrays()
    tri = len(i) // 3
    nodes, root, stack = build(blas, tri)
    assert stack + 1 <= 64
    leaves = []
    # Walk from the root: every link in range, every box conservative.
    bin_boxes = {}
    for n in blas:
        if n["count"] > 0:
            bin_boxes[("L", int(n["left"]))] = n
    todo = [root]
    seen = set()
    while todo:
        r = todo.pop()
        if r & LEAF:
            leaves.append((r & 0xFFFFFF, (r >> 24) & 0x7F))
            continue
        assert r < len(nodes) and r not in seen
        seen.add(r)
        q = nodes[r]
        assert 2 <= q["nchild"] <= 4
        for k in range(q["nchild"]):
            todo.append(int(q["child"][k]))
    assert sorted(leaves) == binary_leaves(blas)
    assert len(seen) == len(nodes)
    # Conservative boxes: each leaf child's decoded box contains its binary box.
    leaf_box = {(int(n["left"]), int(n["count"])): n for n in blas if n["count"] > 0}
    for q in nodes:
        s = np.ldexp(1.0, q["exp"].astype(np.int64))
        for k in range(q["nchild"]):
            c = int(q["child"][k])
            if not c & LEAF:
                continue
            b = leaf_box[(c & 0xFFFFFF, (c >> 24) & 0x7F)]
            lo = [float(np.float32(q["origin"][a]) + np.float32(q["lo"][a][k]) * np.float32(s[a])) for a in range(3)]
            hi = [float(np.float32(q["origin"][a]) + np.float32(q["hi"][a][k]) * np.float32(s[a])) for a in range(3)]
            assert lo[0] <= b["min_x"] and lo[1] <= b["min_y"] and lo[2] <= b["min_z"]
            assert hi[0] >= b["max_x"] and hi[1] >= b["max_y"] and hi[2] >= b["max_z"]


def test_wide_bvh_rejects_bad_links():
    lib = scenes.MeshLibrary()
    lib.add(*scenes.icosphere(2, 1.0))
    v, i, blas = lib.arrays()
    bad = blas.copy()
    bad["left"][0] = len(bad) + 5
    out = np.zeros(len(bad), _lib.QNODE)
    cnt, root, stack = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_int32()
    rc = _lib.lib().ae_build_wide_bvh(_lib.ptr(bad), len(bad), len(i) // 3, _lib.ptr(out), len(out),
                                      ctypes.byref(cnt), ctypes.byref(root), ctypes.byref(stack))
    assert rc == -4
