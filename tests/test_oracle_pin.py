"""The oracle restatement pinned against the reference: its closest hits and
rendered frames must equal, bit for bit, the reference's own compute-only
shader run on the CPU (oracle/_ref, live where the reference tree exists) and
the golden fixtures made from it (tests/golden/)."""
import os

import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import _lib, scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")


def as_hits(b):
    return np.ascontiguousarray(b).view(_lib.HIT).ravel()


def as_rays(b):
    return np.ascontiguousarray(b).view(_lib.RAY).ravel()


def test_oracle_cornell_golden_hits():
    g = np.load(os.path.join(GOLD, "cornell_box.npz"))
    s = scenes.cornell_box()
    hits = O.closest_hit(s, as_rays(g["rays"]))
    assert np.array_equal(hits.view(np.uint8), as_hits(g["hits"]).view(np.uint8))


def test_oracle_cornell_golden_frames():
    g = np.load(os.path.join(GOLD, "cornell_box.npz"))
    s = scenes.cornell_box()
    cfg = s.config.copy()
    px = g["pixels"]
    acc = None
    for b in range(4):
        cfg["batch"] = b
        acc, _, _ = O.render_frame(s, cfg, acc, pixels=px)
        assert np.array_equal(acc[px[:, 1], px[:, 0]], g["accum"][b])


def test_oracle_camera_rays_golden():
    g = np.load(os.path.join(GOLD, "cornell_box.npz"))
    s = scenes.cornell_box()
    rays = O.camera_rays(s.config)
    pick = g["pixels"][:, 1] * s.config["width"] + g["pixels"][:, 0]
    assert np.array_equal(rays[pick].view(np.uint8), as_rays(g["rays"])[:1024].view(np.uint8))


def test_oracle_instanced_golden():
    g = np.load(os.path.join(GOLD, "instanced_small.npz"))
    s = scenes.instanced_meshes(width=240, height=135, levels=(4, 3, 3, 2, 2), grid=64)
    s.instances["scale"] = 0.0
    hits = O.closest_hit(s, as_rays(g["rays"]))
    assert np.array_equal(hits.view(np.uint8), as_hits(g["hits"]).view(np.uint8))


@needs_ref
def test_oracle_equals_reference_cornell_full_frames():
    s = scenes.cornell_box()
    cfg = s.config.copy()
    acc_o = acc_r = None
    for b in range(3):
        cfg["batch"] = b
        acc_o, disp_o, _ = O.render_frame(s, cfg, acc_o)
        acc_r, disp_r = O.ref_render(s, cfg, acc_r)
        assert np.array_equal(acc_o, acc_r)
        assert np.array_equal(disp_o, disp_r)


@needs_ref
def test_oracle_equals_reference_materials():
    """Metal, glass and a second light: every branch of GetBounce and the
    glass-stepping shadow loop (hybrid:965-1033, 1167-1191)."""
    s = scenes.cornell_box(seed=5)
    s.objects["colorType"][np.where(s.objects["shapeType"] == _lib.SHAPE_MESH)[0][-2:]] = [_lib.MAT_METAL,
                                                                                         _lib.MAT_DIELECTRIC]
    s.objects["fuzz"] = 0.2
    s.objects["refraction"] = 1.5
    cfg = s.config.copy()
    cfg["width"], cfg["height"] = 160, 120
    for b in range(2):
        cfg["batch"] = b
        acc_o, _, _ = O.render_frame(s, cfg)
        acc_r, _ = O.ref_render(s, cfg)
        assert np.array_equal(acc_o, acc_r)


@needs_ref
def test_oracle_equals_reference_instanced_full():
    s = scenes.instanced_meshes(width=320, height=180)
    s.instances["scale"] = 0.0
    rays = O.camera_rays(s.config)
    a = O.closest_hit(s, rays)
    b = O.ref_closest_hit(s, rays)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    assert (a["object"] != _lib.MISS).mean() > 0.2
