"""The host builders (BuildBVH, MeshLibrary::Add, world bounds, TLAS packing)
against the reference's own headers compiled here (oracle/_ref) and against
golden fixtures made from them (tests/golden/bvh_build.npz).  Bit-exact."""
import os

import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import _lib, scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")


def test_bvh_golden():
    g = np.load(os.path.join(GOLD, "bvh_build.npz"))
    for k in range(4):
        nodes, order = scenes.build_bvh(g[f"bvh{k}_boxes"])
        assert np.array_equal(nodes.view(np.uint8).ravel(), g[f"bvh{k}_nodes"].ravel())
        assert np.array_equal(order, g[f"bvh{k}_order"])


def test_bvh_empty_and_single():
    nodes, order = scenes.build_bvh(np.zeros((0, 6), np.float32))
    assert len(nodes) == 0 and len(order) == 0
    nodes, order = scenes.build_bvh(np.array([[0, 0, 0, 0, 0, 0]], np.float32))
    assert len(nodes) == 1 and nodes[0]["count"] == 1
    # A flat box is inflated by bounds_minimum on every thin axis (scene/bvh.h:69-83).
    assert nodes[0]["max_x"] - nodes[0]["min_x"] > 0


@needs_ref
@pytest.mark.parametrize("n,seed,flat,dup", [(2, 0, 0, 0), (7, 1, 0.5, 0), (100, 2, 0.3, 0.5), (5000, 3, 0.1, 0.1),
                                             (40000, 4, 0, 0), (64, 5, 1.0, 1.0)])
def test_bvh_matches_reference(n, seed, flat, dup):
    rng = np.random.default_rng(seed)
    c = rng.normal(0, 50, (n, 3)).astype(np.float32)
    e = rng.uniform(0, 3, (n, 3)).astype(np.float32)
    e[rng.random((n, 3)) < flat] = 0
    c[: int(n * dup)] = c[0]
    boxes = np.concatenate([c - e, c + e], 1)
    a_nodes, a_order = scenes.build_bvh(boxes)
    r_nodes, r_order = O.ref_build_bvh(boxes)
    assert np.array_equal(a_nodes.view(np.uint8), r_nodes.view(np.uint8))
    assert np.array_equal(a_order, r_order)


@needs_ref
@pytest.mark.parametrize("gen", ["box", "sphere4", "grid"])
def test_mesh_library_matches_reference(gen):
    rng = np.random.default_rng(9)
    if gen == "box":
        v, i = scenes.box_mesh((1.0, 2.0, 0.5))
    elif gen == "sphere4":
        v, i = scenes.icosphere(4, 3.0)
    else:
        v, i = scenes.heightfield(100, 10.0, 1.0, rng)
    lib = scenes.MeshLibrary()
    lib.add(v, i)
    av, ai, ab = lib.arrays()
    rv, ri, rb = O.ref_mesh_add(v, i.astype(np.uint16))
    assert np.array_equal(av.view(np.uint8), rv.view(np.uint8))
    assert np.array_equal(ai, ri)
    assert np.array_equal(ab.view(np.uint8), rb.view(np.uint8))


@needs_ref
def test_world_bounds_match_reference():
    rng = np.random.default_rng(3)
    lib = scenes.MeshLibrary()
    h = lib.add(*scenes.icosphere(2, 2.0))
    local = lib.range(h)["localBounds"]
    for _ in range(200):
        p = tuple(float(x) for x in rng.uniform(-50, 50, 3))
        q = scenes.random_quat(rng)
        e = np.array([scenes.entity(_lib.SHAPE_MESH, 0, p, rotation=q, mesh=h)])
        ours = np.zeros(1, _lib.AABB)
        _lib.check(_lib.lib().ae_entity_bounds(_lib.ptr(e), lib.handle, _lib.ptr(ours)))
        ref = O.ref_bounds("mesh", p, q, [local[k] for k in local.dtype.names])
        assert np.array_equal(ours.view(np.float32).ravel(), ref)
        u, v = rng.normal(0, 3, 3), rng.normal(0, 3, 3)
        e = np.array([scenes.entity(_lib.SHAPE_QUAD, 0, p, rotation=q, u=u, v=v)])
        _lib.check(_lib.lib().ae_entity_bounds(_lib.ptr(e), None, _lib.ptr(ours)))
        assert np.array_equal(ours.view(np.float32).ravel(), O.ref_bounds("quad", p, q, u, v))
        yq = scenes.yaw_quat(float(rng.uniform(-3, 3)))
        half = rng.uniform(0.1, 4, 3)
        e = np.array([scenes.entity(_lib.SHAPE_BOX, 0, p, rotation=yq, half_extent=half)])
        _lib.check(_lib.lib().ae_entity_bounds(_lib.ptr(e), None, _lib.ptr(ours)))
        assert np.array_equal(ours.view(np.float32).ravel(), O.ref_bounds("box", p, yq, half))


def test_pack_scene_layout():
    s = scenes.cornell_box()
    assert len(s.objects) == 8 and s.triangles == 34
    # Light IDs are slots of emissive objects (renderer/renderer.cpp:803-813).
    assert all(s.objects[k]["colorType"] == _lib.MAT_DIFFUSE_LIGHT for k in s.lights)
    # Instance indices follow slot order (renderer/renderer.cpp:838-864).
    mesh_slots = [k for k in range(len(s.objects)) if s.objects[k]["shapeType"] == _lib.SHAPE_MESH]
    assert [int(s.objects[k]["instanceIndex"]) for k in mesh_slots] == list(range(len(mesh_slots)))
    # Rigid instances keep pad0 = 0, byte-identical to the reference packer.
    assert np.all(s.instances["scale"] == 0)


def test_pack_rejects_unknown_mesh():
    e = scenes.entity(_lib.SHAPE_MESH, 0, (0, 0, 0), mesh=7)
    with pytest.raises(_lib.AeError):
        scenes.pack([e], scenes.MeshLibrary())
