"""The hybrid renderer's kernels (ray-cast G-buffer, deferred resolve,
temporal upsample) against the oracle through the C ABI: G-buffer planes and
accumulated radiance bit for bit, the 8-bit display within one code, across
still frames, a camera move, reduced trace grids and display-only frames."""
import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import Context, _lib, scenes
from test_oracle_hybrid import frames

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


def test_gbuffer_planes_bit_exact():
    s = scenes.hybrid_box()
    c = s.config.copy()
    c["jitter_x"], c["jitter_y"] = 0.25, -0.125
    with Context(int(c["width"]), int(c["height"])) as ctx:
        ctx.upload(s)
        ctx.set_config(c)
        ctx.build_gbuffer()
        pos, nrm, alb, dep = ctx.read_planes()
    opos, onrm, oalb, odep = O.gbuffer(s, c)
    assert same(pos, opos) and same(nrm, onrm) and np.array_equal(alb, oalb) and same(dep, odep)


@pytest.mark.parametrize("scale", [1.0, 0.5, 0.75])
def test_hybrid_frames_bit_exact(scale):
    s, cfgs = frames(scale)
    w, h = int(cfgs[0]["width"]), int(cfgs[0]["height"])
    st = O.HybridState(w, h)
    with Context(w, h, hybrid=True, trace_scale=scale) as ctx:
        ctx.upload(s)
        for k, c in enumerate(cfgs):
            ctx.set_config(c)
            ctx.build_gbuffer()
            gb = ctx.read_planes()
            ctx.render_frame(_lib.MODE_DEFERRED)
            O.hybrid_frame(s, c, gb, st, "oracle")
            assert same(ctx.read_deferred_accum(), st.img[st.history]), f"frame {k} accumulation"
            assert same(ctx.read_image(_lib.IMAGE_HISTORY_GEOMETRY), st.geo[st.history]), f"frame {k} geometry"
            if scale < 1.0:
                assert same(ctx.read_image(_lib.IMAGE_REDUCED), st.reduced), f"frame {k} reduced grid"
            disp = ctx.read_image(_lib.IMAGE_DISPLAY)[..., :3].astype(np.int32)
            want = np.rint(np.clip(st.display[..., :3], 0, 1) * 255).astype(np.int32)
            assert np.abs(disp - want).max() <= 1, f"frame {k} display"


def test_hybrid_debug_views():
    s, cfgs = frames(1.0)
    w, h = int(cfgs[0]["width"]), int(cfgs[0]["height"])
    with Context(w, h, hybrid=True) as ctx:
        ctx.upload(s)
        for view in (1, 2, 3, 4, 5, 6):
            c = cfgs[0].copy()
            c["debugView"] = view
            ctx.set_config(c)
            ctx.build_gbuffer()
            gb = ctx.read_planes()
            ctx.render_frame(_lib.MODE_DEFERRED)
            st = O.HybridState(w, h)
            O.hybrid_frame(s, c, gb, st, "oracle")
            disp = ctx.read_image(_lib.IMAGE_DISPLAY)[..., :3].astype(np.int32)
            want = np.rint(np.clip(st.display[..., :3], 0, 1) * 255).astype(np.int32)
            assert np.abs(disp - want).max() <= 1, f"debug view {view}"


def test_deferred_without_gbuffer_is_an_error():
    s = scenes.hybrid_box()
    with Context(64, 48, hybrid=True) as ctx:
        ctx.upload(s)
        with pytest.raises(_lib.AeError):
            ctx.render_frame(_lib.MODE_DEFERRED)


def test_any_hit_matches_oracle():
    """ae_any_hit: the deferred shader's shadow-ray rules (glass and lights do
    not block) over random segments in the hybrid box."""
    s = scenes.hybrid_box()
    rng = np.random.default_rng(21)
    n = 100000
    r = np.zeros(n, _lib.RAY)
    o = rng.uniform(0.1, 9.9, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r["ox"], r["oy"], r["oz"] = o.T
    r["dx"], r["dy"], r["dz"] = d.T
    r["tnear"] = 0.001
    tmax = rng.uniform(0.5, 12.0, n).astype(np.float32)
    with Context(64, 48) as ctx:
        ctx.upload(s)
        got = ctx.any_hit(r, tmax)
    want = O.any_hit(s, r, tmax)
    assert np.array_equal(got, want)
    assert 0.1 < want.mean() < 0.95
