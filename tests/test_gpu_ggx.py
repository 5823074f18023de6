"""GGX rough metal (AE_MAT_GGX_METAL, the library's extension: Walter et al.
2007 microfacet reflection with roughness alpha in Object_GPU::fuzz) on the
GPU against the oracle's restatement of the same published model, through
the C ABI: the plain megakernel bit for bit against the float oracle, the
wavefront form and a served request bit for bit against the megakernel, the
precision form scored against the FP64 oracle, and the hybrid passes
refusing such scenes."""
import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import AeError, Context, Server, _lib, scenes

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


def ggx_box(width=96, height=72, depth=6):
    """The Cornell box with its two cubes and two walls turned into GGX rough
    metal of roughness 0.08, 0.25, 0.45 and 0.6."""
    s = scenes.cornell_box(width=width, height=height, depth=depth)
    lit = s.objects["colorType"] == _lib.MAT_DIFFUSE_LIGHT
    idx = np.flatnonzero(~lit)[:4]
    for k, a in zip(idx, (0.08, 0.25, 0.45, 0.6)):
        s.objects["colorType"][k] = _lib.MAT_GGX_METAL
        s.objects["fuzz"][k] = a
    return s


def render(s, mode, frames):
    c = s.config.copy()
    out = []
    with Context(int(c["width"]), int(c["height"])) as ctx:
        ctx.upload(s)
        for b in range(frames):
            c["batch"] = b
            ctx.set_config(c)
            ctx.render_frame(mode)
            out.append((ctx.read_image(_lib.IMAGE_ACCUM), ctx.read_image(_lib.IMAGE_DISPLAY),
                        ctx.read_image(_lib.IMAGE_FRAME)))
    return out


def test_ggx_frames_equal_oracle():
    s = ggx_box()
    gpu = render(s, _lib.MODE_COMPUTE_ONLY, 3)
    cfg = s.config.copy()
    acc = None
    for b in range(3):
        cfg["batch"] = b
        acc, _, frame = O.render_frame(s, cfg, acc)
        assert same(gpu[b][2], frame), f"frame {b}"
        assert same(gpu[b][0], acc)
    # The GGX surfaces are seen and shaded: the image is not black.
    assert gpu[-1][0][..., :3].mean() > 0.01


def test_ggx_wavefront_and_precision():
    s = ggx_box()
    plain = render(s, _lib.MODE_COMPUTE_ONLY, 4)
    wave = render(s, _lib.MODE_WAVEFRONT, 4)
    for k in range(4):
        assert same(wave[k][0], plain[k][0]), f"frame {k}"
    # Precision form (watertight test, FP16 normals, Kahan sum) against the
    # FP64 oracle: within one percentage point of the plain form's MRE.
    cfg = s.config.copy()
    ref = None
    for b in range(4):
        cfg["batch"] = b
        ref, _, _ = O.render_frame(s, cfg, ref, precision=64)
    errs = {}
    for label, mode in (("plain", _lib.MODE_COMPUTE_ONLY), ("precision", _lib.MODE_WAVEFRONT_PRECISION)):
        with Context(96, 72) as ctx:
            ctx.upload(s)
            c = s.config.copy()
            for b in range(4):
                c["batch"] = b
                ctx.set_config(c)
                ctx.render_frame(mode)
            errs[label] = ctx.image_error(ref)["mre"]
    print(f"GGX box MRE vs FP64 oracle: plain {errs['plain']:.3e} precision {errs['precision']:.3e}")
    assert errs["precision"] <= errs["plain"] + 0.01


def test_ggx_served_request_equals_frames():
    s = ggx_box(width=64, height=48)
    ref = render(s, _lib.MODE_COMPUTE_ONLY, 2)[-1]
    with Context(64, 48) as ctx:
        ctx.upload(s)
        with Server(slots=2048, max_requests=4, arena_bytes=1 << 24) as srv:
            sid = srv.add_scene(ctx)
            res, acc, dsp = srv.wait(srv.submit(sid, 64, 48, 2, s.config), 60000)
    assert res["status"] == 0
    assert same(acc, ref[0]) and np.array_equal(dsp, ref[1])


def test_ggx_refused_by_hybrid_passes():
    s = ggx_box(width=32, height=24)
    with Context(32, 24, hybrid=True) as ctx:
        ctx.upload(s)
        with pytest.raises(AeError) as e:
            ctx.build_gbuffer()
        assert e.value.code == -7
        with pytest.raises(AeError) as e:
            ctx.render_frame(_lib.MODE_DEFERRED)
        assert e.value.code == -7


def test_ggx_wavefront_scene_mix_renders_on_both_forms():
    """The wavefront workload's material mix with GGX for its metals, at a
    small size: wavefront frames equal the megakernel's."""
    s = scenes.wavefront_scene(seed=21, width=96, height=64, depth=6, n_meshes=8, n_instances=48, n_lights=4,
                               target_tris=60_000, ggx=True)
    assert (s.objects["colorType"] == _lib.MAT_GGX_METAL).any()
    a = render(s, _lib.MODE_COMPUTE_ONLY, 2)
    b = render(s, _lib.MODE_WAVEFRONT, 2)
    for k in range(2):
        assert same(a[k][0], b[k][0]), f"frame {k}"
