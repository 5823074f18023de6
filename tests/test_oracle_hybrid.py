"""The oracle's restatement of the hybrid renderer's compute passes
(deferred.comp.hlsl, upsample.comp.hlsl) against the reference's own shaders
run on the CPU (oracle/_ref), over the same G-buffer: every output plane bit
for bit, across frames that exercise history, reprojection after a camera
move, the reduced trace grid and display-only re-grading."""
import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import scenes

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")


def frames(scale):
    """A sequence of configs: still frames, a camera move, still again."""
    s = scenes.hybrid_box()
    base = s.config.copy()
    base["traceScale"] = scale
    base["historyCap"] = 32.0
    out = []
    for f in range(5):
        c = base.copy()
        c["frameIndex"] = f
        c["jitter_x"] = [0.0, 0.25, -0.25, 0.125, -0.375][f]
        c["jitter_y"] = [0.0, -0.333, 0.333, 0.111, 0.222][f]
        c["historyReset"] = 1 if f == 0 else 0
        if f == 3:  # the camera moved: reproject through last frame's matrix
            c["cameraMoved"] = 1
            c["source_x"] += 0.3
            vp = np.eye(4, dtype=np.float32)
            vp[0, 0] = vp[1, 1] = 0.12
            vp[3, 2] = -0.05
            vp[3, 3] = 0.9
            c["prevViewProj"] = vp.ravel()
        out.append(c)
    disp = out[-1].copy()
    disp["displayOnly"] = 1
    disp["exposure"] = 0.5
    out.append(disp)
    return s, out


@needs_ref
@pytest.mark.parametrize("scale", [1.0, 0.5, 0.75])
def test_hybrid_frames_equal_reference(scale):
    s, cfgs = frames(scale)
    w, h = int(cfgs[0]["width"]), int(cfgs[0]["height"])
    so, sr = O.HybridState(w, h), O.HybridState(w, h)
    for k, c in enumerate(cfgs):
        gb = O.gbuffer(s, c)
        O.hybrid_frame(s, c, gb, so, "oracle")
        O.hybrid_frame(s, c, gb, sr, "reference")
        assert so.history == sr.history
        for a, b, what in ((so.img[so.history], sr.img[sr.history], "image"),
                           (so.geo[so.history], sr.geo[sr.history], "geometry"),
                           (so.display, sr.display, "display"), (so.reduced, sr.reduced, "reduced")):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"frame {k}: {what} differs"
    assert np.isfinite(so.img[so.history]).all()
    assert so.img[so.history][..., :3].mean() > 0.01


@needs_ref
def test_hybrid_debug_views_equal_reference():
    s, cfgs = frames(1.0)
    w, h = int(cfgs[0]["width"]), int(cfgs[0]["height"])
    for view in (1, 2, 3, 4, 5, 6):
        c = cfgs[0].copy()
        c["debugView"] = view
        gb = O.gbuffer(s, c)
        so, sr = O.HybridState(w, h), O.HybridState(w, h)
        O.hybrid_frame(s, c, gb, so, "oracle")
        O.hybrid_frame(s, c, gb, sr, "reference")
        assert np.array_equal(so.display, sr.display)


def test_gbuffer_covers_rasterized_objects():
    s = scenes.hybrid_box()
    pos, nrm, alb, dep = O.gbuffer(s, s.config)
    cov = nrm[..., 3] > 0.5
    assert 0.3 < cov.mean() < 1.0
    slots = pos[..., 3][cov].astype(int)
    shapes = s.objects["shapeType"][slots]
    assert set(np.unique(shapes)) <= {2, 4}   # boxes (raster proxies) and meshes only
    assert np.all((dep[cov] > 0) & (dep[cov] < 1))
