"""Materials beyond flat albedo, pinned against the reference's own shaders
run on the CPU.  Textures (SurfaceAlbedo with textureColor, hybrid:919-949,
deferred:1173-1203) over a scene where every intersector supplies UVs (mesh
vertex UVs, quad alpha/beta, sphere get_sphere_uv, box BoxFaceUV) with tints
0, 0.25, 1; the texture sampler itself (one definition shared by the kernels,
the oracle and the reference harness) against an independent numpy
restatement of bilinear, REPEAT, sRGB-decoded sampling; and participating
media with the remaining analytic shapes (HitVolume, ISOTROPIC, analytic
triangle, a sphere moving over the shutter)."""
import ctypes

import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import _lib, scenes

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")


def numpy_sample(tex, layer, u, v):
    """Bilinear, REPEAT, sRGB-decoded sample in float64."""
    L, h, w, _ = tex.shape
    layer = min(layer, L - 1)
    c = tex[layer, ..., :3].astype(np.float64) / 255.0
    lin = np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)
    x, y = u * w - 0.5, v * h - 0.5
    fx, fy = np.floor(x), np.floor(y)
    ax, ay = x - fx, y - fy
    x0, x1 = int(fx) % w, int(fx + 1) % w
    y0, y1 = int(fy) % h, int(fy + 1) % h
    top = lin[y0, x0] + (lin[y0, x1] - lin[y0, x0]) * ax
    bot = lin[y1, x0] + (lin[y1, x1] - lin[y1, x0]) * ax
    return top + (bot - top) * ay


def test_sampler_matches_numpy_restatement():
    """The shared float sampler (through the reference harness's
    Texture2DArray) within float rounding of a float64 restatement, at texel
    centres, between texels, across the REPEAT seams and out of range."""
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    tex = scenes.procedural_textures(layers=3, width=7, height=5, seed=3)
    L = O.ref_shader()
    words = np.ascontiguousarray(tex).view(np.uint32).reshape(-1)
    L.aeref_bind_textures(O.ptr(words), 7, 5, 3)
    f = L.aeref_sample_texture
    f.restype = None
    rng = np.random.default_rng(0)
    pts = [(0.5 / 7, 0.5 / 5), (0.0, 0.0), (1.0, 1.0), (-0.3, 1.7), (2.25, -3.5), (0.999, 0.001)]
    pts += [tuple(rng.uniform(-2, 3, 2)) for _ in range(200)]
    out = np.zeros(3, np.float32)
    for layer in (0, 2, 5):
        for u, v in pts:
            f(ctypes.c_float(u), ctypes.c_float(v), ctypes.c_uint32(layer), O.ptr(out))
            want = numpy_sample(tex, layer, np.float32(u), np.float32(v))
            assert np.allclose(out, want, rtol=2e-6, atol=2e-7), (layer, u, v, out, want)


@needs_ref
def test_textured_frames_equal_reference():
    s = scenes.textured_box()
    cfg = s.config.copy()
    acc_o = acc_r = None
    for b in range(3):
        cfg["batch"] = b
        acc_o, disp_o, _ = O.render_frame(s, cfg, acc_o)
        acc_r, disp_r = O.ref_render(s, cfg, acc_r)
        assert np.array_equal(acc_o.view(np.uint32), acc_r.view(np.uint32)), f"frame {b}"
        assert np.array_equal(disp_o, disp_r)
    # The textures show: the frame differs from the same scene untextured.
    plain = scenes.textured_box()
    plain.objects["textureID"] = _lib.NO_TEXTURE
    plain.textures = None
    c0 = s.config.copy()
    a_tex, _, _ = O.render_frame(s, c0)
    a_flat, _, _ = O.render_frame(plain, c0)
    assert np.abs(a_tex - a_flat).mean() > 1e-3


@needs_ref
def test_textured_hybrid_frames_equal_reference():
    s = scenes.textured_box(width=96, height=72, depth=4)
    c = s.config.copy()
    c["traceScale"] = 1.0
    c["historyCap"] = 32.0
    c["historyReset"] = 1
    w, h = int(c["width"]), int(c["height"])
    so, sr = O.HybridState(w, h), O.HybridState(w, h)
    for f in range(2):
        c["frameIndex"] = f
        c["historyReset"] = 1 if f == 0 else 0
        gb = O.gbuffer(s, c)
        O.hybrid_frame(s, c, gb, so, "oracle")
        O.hybrid_frame(s, c, gb, sr, "reference")
        for a, b, what in ((so.img[so.history], sr.img[sr.history], "image"),
                           (so.display, sr.display, "display")):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"frame {f}: {what} differs"


@needs_ref
def test_media_and_analytic_frames_equal_reference():
    """Participating media (HitVolume and ISOTROPIC scattering, with their RNG
    draws inside the walk), an analytic triangle, a moving sphere and a glass
    box: oracle equals the reference's compute-only shader bit for bit."""
    s = scenes.media_box()
    cfg = s.config.copy()
    acc_o = acc_r = None
    for b in range(3):
        cfg["batch"] = b
        acc_o, disp_o, _ = O.render_frame(s, cfg, acc_o)
        acc_r, disp_r = O.ref_render(s, cfg, acc_r)
        assert np.array_equal(acc_o.view(np.uint32), acc_r.view(np.uint32)), f"frame {b}"
        assert np.array_equal(disp_o, disp_r)


@needs_ref
def test_media_hybrid_frames_equal_reference():
    s = scenes.media_box(width=96, height=72, depth=4)
    c = s.config.copy()
    c["traceScale"], c["historyCap"] = 1.0, 32.0
    w, h = int(c["width"]), int(c["height"])
    so, sr = O.HybridState(w, h), O.HybridState(w, h)
    for f in range(2):
        c["frameIndex"] = f
        c["historyReset"] = 1 if f == 0 else 0
        gb = O.gbuffer(s, c)
        O.hybrid_frame(s, c, gb, so, "oracle")
        O.hybrid_frame(s, c, gb, sr, "reference")
        assert np.array_equal(so.img[so.history].view(np.uint32), sr.img[sr.history].view(np.uint32)), f"frame {f}"
        assert np.array_equal(so.display.view(np.uint32), sr.display.view(np.uint32))
