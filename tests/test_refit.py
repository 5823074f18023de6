"""GPU refit of the TLAS after instances move: the device's object boxes and
node boxes equal the host computation (MeshBounds of scene/shapes.h:124-145,
pinned against the reference in test_host_scene, unioned bottom-up and widened
as MakeNode does), and closest hits against the refit scene equal the oracle's
on the same arrays."""
import copy

import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import Context, _lib, scenes


def host_refit(scene, new_inst, lib_bounds):
    """The refit in numpy, op for op: per-object boxes from ae_entity_bounds
    (host C), union per leaf, union per interior node, MakeNode widening."""
    objs = scene.objects
    boxes = np.zeros((len(objs), 6), np.float32)
    for s, o in enumerate(objs):
        if o["shapeType"] == _lib.SHAPE_MESH:
            I = new_inst[o["instanceIndex"]]
            boxes[s] = lib_bounds(I)
    tl = scene.tlas.copy()
    raw = np.zeros((len(tl), 6), np.float32)
    depth = np.zeros(len(tl), int)
    for i in range(len(tl)):
        if tl[i]["count"] <= 0:
            depth[tl[i]["left"]] = depth[i] + 1
            depth[tl[i]["right"]] = depth[i] + 1
    for d in range(depth.max(), -1, -1):
        for i in np.where(depth == d)[0]:
            n = tl[i]
            if n["count"] > 0:
                b = boxes[n["left"]:n["left"] + n["count"]]
                raw[i, :3] = b[:, :3].min(0)
                raw[i, 3:] = b[:, 3:].max(0)
            else:
                raw[i, :3] = np.minimum(raw[n["left"], :3], raw[n["right"], :3])
                raw[i, 3:] = np.maximum(raw[n["left"], 3:], raw[n["right"], 3:])
            lo, hi = raw[i, :3].copy(), raw[i, 3:].copy()
            half = np.float32(0.0001) * np.float32(0.5)
            thin = (hi - lo) < np.float32(0.0001)
            lo[thin] -= half
            hi[thin] += half
            tl[i]["min_x"], tl[i]["min_y"], tl[i]["min_z"] = lo
            tl[i]["max_x"], tl[i]["max_y"], tl[i]["max_z"] = hi
    return tl


@pytest.mark.gpu
def test_refit_matches_host_and_oracle():
    s = scenes.instanced_meshes(width=320, height=180, levels=(4, 3, 3, 2, 2), grid=64)
    rng = np.random.default_rng(5)
    new = s.instances.copy()
    new["px"] += rng.normal(0, 3, len(new)).astype(np.float32)
    new["pz"] += rng.normal(0, 3, len(new)).astype(np.float32)
    q = np.array([scenes.random_quat(rng) for _ in range(len(new))], np.float32)
    new["qx"], new["qy"], new["qz"], new["qw"] = q.T
    # Mesh local boxes: a library with the same meshes gives them by handle.
    lib = scenes.MeshLibrary()
    ranges = {}

    def bounds_of(I):
        key = (int(I["vertexBase"]), int(I["indexBase"]), int(I["triangleCount"]))
        if key not in ranges:
            idx = s.indices[I["indexBase"]:I["indexBase"] + 3 * I["triangleCount"]]
            v = s.vertices[I["vertexBase"] + idx]
            ranges[key] = np.array([v["px"].min(), v["py"].min(), v["pz"].min(), v["px"].max(), v["py"].max(),
                                    v["pz"].max()], np.float32)
        lb = ranges[key]
        # MeshBounds through the host C library (entity with that local box).
        vv, ii = scenes.box_mesh((1, 1, 1))
        e = np.array([scenes.entity(_lib.SHAPE_MESH, 0, (float(I["px"]), float(I["py"]), float(I["pz"])),
                                    rotation=(float(I["qx"]), float(I["qy"]), float(I["qz"]), float(I["qw"])),
                                    scale=float(I["scale"]) if I["scale"] != 0 else 1.0, mesh=0)])
        ml = scenes.MeshLibrary()
        corners = np.array([[lb[0], lb[1], lb[2]], [lb[3], lb[4], lb[5]]], np.float32)
        verts = np.zeros(2, _lib.VERTEX)
        verts["px"], verts["py"], verts["pz"] = corners.T
        ml.add(verts, np.array([0, 1, 0], np.uint32))
        out = np.zeros(1, _lib.AABB)
        _lib.check(_lib.lib().ae_entity_bounds(_lib.ptr(e), ml.handle, _lib.ptr(out)))
        return out.view(np.float32)

    want_tlas = host_refit(s, new, bounds_of)
    with Context(320, 180) as ctx:
        ctx.upload(s)
        ctx.refit_instances(new)
        objs, tlas, inst = ctx.download_scene()
        assert np.array_equal(inst.view(np.uint8), new.view(np.uint8))
        assert np.array_equal(tlas.view(np.uint8), want_tlas.view(np.uint8))
        moved = copy.copy(s)
        moved.objects, moved.tlas, moved.instances = objs, tlas, inst
        rays = ctx.camera_rays()
        got = ctx.closest_hit(rays)
        got_fast = ctx.closest_hit(rays, _lib.VARIANT_FAST)
    want = O.closest_hit(moved, rays)
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
    assert np.array_equal(got_fast.view(np.uint8), want.view(np.uint8))
    # Previous transforms follow the replaced instance records.
    m = objs["shapeType"] == _lib.SHAPE_MESH
    assert np.array_equal(objs["x2"][m], s.objects["x"][m])
