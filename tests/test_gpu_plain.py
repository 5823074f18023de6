"""Parity of the plain CUDA kernels with the oracle, through the C ABI.

Bit-exact: closest-hit IDs, t and barycentrics; camera rays; accumulated
radiance of RGB-driven frames (every arithmetic step is a correctly rounded
binary32 operation on both sides).  The display image is 8-bit: within one
code of the oracle's float value quantised.
"""
import os

import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import AeError, Context, _lib, scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def ctx_for(scene, w=None, h=None):
    c = Context(w or int(scene.config["width"]), h or int(scene.config["height"]))
    c.upload(scene)
    return c


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


@pytest.fixture(scope="module")
def cornell():
    return scenes.cornell_box()


@pytest.fixture(scope="module")
def instanced():
    return scenes.instanced_meshes(width=480, height=270)


def test_camera_rays_bit_exact(cornell, instanced):
    for s in (cornell, instanced):
        with ctx_for(s) as c:
            assert same(c.camera_rays(), O.camera_rays(s.config))


def test_closest_hit_golden(cornell):
    g = np.load(os.path.join(GOLD, "cornell_box.npz"))
    with ctx_for(cornell) as c:
        hits = c.closest_hit(g["rays"].view(_lib.RAY).ravel())
    assert same(hits, g["hits"].view(_lib.HIT).ravel())


def test_closest_hit_golden_instanced():
    g = np.load(os.path.join(GOLD, "instanced_small.npz"))
    s = scenes.instanced_meshes(width=240, height=135, levels=(4, 3, 3, 2, 2), grid=64)
    s.instances["scale"] = 0.0
    with ctx_for(s) as c:
        hits = c.closest_hit(g["rays"].view(_lib.RAY).ravel())
    assert same(hits, g["hits"].view(_lib.HIT).ravel())


def test_closest_hit_camera_and_bounce(instanced):
    s = instanced
    with ctx_for(s) as c:
        prim = c.camera_rays()
        hits = c.closest_hit(prim)
        assert same(hits, O.closest_hit(s, prim))
        assert (hits["object"] != _lib.MISS).mean() > 0.3
        bounce, valid = c.bounce_rays(prim, hits)
        ob, ov = O.bounce_rays(s, s.config, prim, hits)
        assert np.array_equal(valid, ov) and same(bounce[valid], ob[ov])
        b = bounce[valid]
        bh = c.closest_hit(b)
        assert same(bh, O.closest_hit(s, b))


def test_closest_hit_random_rays(cornell):
    rng = np.random.default_rng(11)
    n = 100000
    r = np.zeros(n, _lib.RAY)
    o = rng.uniform(-2, 12, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r["ox"], r["oy"], r["oz"] = o.T
    r["dx"], r["dy"], r["dz"] = d.T
    r["tnear"] = 0.001
    # Axis-parallel directions exercise the infinite inverse direction.
    r["dx"][:1000], r["dy"][:1000], r["dz"][:1000] = 0.0, -1.0, 0.0
    with ctx_for(cornell) as c:
        assert same(c.closest_hit(r), O.closest_hit(cornell, r))


def test_empty_batch_and_device_counters(cornell):
    with ctx_for(cornell) as c:
        assert len(c.closest_hit(np.zeros(0, _lib.RAY))) == 0


def test_render_frames_bit_exact(cornell):
    s = cornell
    cfg = s.config.copy()
    with ctx_for(s) as c:
        acc_o = None
        for b in range(4):
            cfg["batch"] = b
            c.set_config(cfg)
            c.render_frame(_lib.MODE_COMPUTE_ONLY)
            acc_o, disp_o, frame_o = O.render_frame(s, cfg, acc_o)
            acc = c.read_image(_lib.IMAGE_ACCUM)
            assert same(acc, acc_o), f"frame {b}"
            assert same(c.read_image(_lib.IMAGE_FRAME), frame_o)
            disp = c.read_image(_lib.IMAGE_DISPLAY)
            want = np.rint(np.clip(disp_o[..., :3], 0, 1) * 255).astype(np.int32)
            assert np.abs(disp[..., :3].astype(np.int32) - want).max() <= 1


def test_render_materials_bit_exact():
    s = scenes.cornell_box(seed=5, width=160, height=120)
    meshes = np.where(s.objects["shapeType"] == _lib.SHAPE_MESH)[0]
    s.objects["colorType"][meshes[-2:]] = [_lib.MAT_METAL, _lib.MAT_DIELECTRIC]
    s.objects["fuzz"] = 0.2
    s.objects["refraction"] = 1.5
    cfg = s.config.copy()
    with ctx_for(s) as c:
        for b in range(2):
            cfg["batch"] = b
            c.set_config(cfg)
            c.render_frame(_lib.MODE_COMPUTE_ONLY)
            assert same(c.read_image(_lib.IMAGE_FRAME), O.render_frame(s, cfg)[2])


def test_scaled_instances_bit_exact(instanced):
    # Non-rigid instances (pad0 scale) against the oracle's restatement.
    assert np.any(instanced.instances["scale"] != 0)
    with ctx_for(instanced) as c:
        rays = c.camera_rays()
        assert same(c.closest_hit(rays), O.closest_hit(instanced, rays))


def test_traffic_counters_match_oracle(instanced):
    import torch
    s = instanced
    with ctx_for(s) as c:
        rays = c.camera_rays()
        d = torch.from_numpy(rays.view(np.uint8)).cuda()
        cnt = np.zeros(6, np.uint64)
        torch.cuda.synchronize()
        _lib.check(_lib.lib().ae_trace_counters(c.handle, d.data_ptr(), len(rays), _lib.ptr(cnt)), c.handle)
    _, ocnt = O.closest_hit(s, rays, counters=True)
    assert np.array_equal(cnt, ocnt)


def test_upload_validation(cornell):
    s = cornell
    with Context(64, 48) as c:
        c.upload_geometry(s.vertices, s.indices, s.blas)
        bad = s.tlas.copy()
        bad["left"][bad["count"] == 0] = 999
        with pytest.raises(AeError) as e:
            c.upload_scene(s.objects, bad, s.lights, s.instances)
        assert e.value.code == -4
        c.reserve_scene(4, 1)
        with pytest.raises(AeError) as e:
            c.upload_scene(s.objects, s.tlas, s.lights, s.instances)
        assert e.value.code == -3
        with pytest.raises(AeError) as e:
            c.closest_hit(np.zeros(4, _lib.RAY))
        assert e.value.code == -7
