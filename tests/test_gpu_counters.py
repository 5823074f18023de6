"""Measurement entry points on the GPU: the FP64 image-error reduction over a
pixel subset against numpy, the device path counters against the ray
counters of the same traversals, and the optimised walk's fetch counters."""
import numpy as np
import pytest

from aviatorengine2_b200 import Context, _lib, scenes

pytestmark = pytest.mark.gpu


def test_image_error_pixels_matches_numpy():
    s = scenes.cornell_box(width=80, height=60, depth=4)
    with Context(80, 60) as ctx:
        ctx.upload(s)
        ctx.render_frame(_lib.MODE_COMPUTE_ONLY)
        acc = ctx.read_image(_lib.IMAGE_ACCUM)
        rng = np.random.default_rng(5)
        pick = np.sort(rng.choice(80 * 60, 500, replace=False))
        xy = np.stack([pick % 80, pick // 80], 1).astype(np.uint32)
        x = acc[xy[:, 1], xy[:, 0]].astype(np.float64)
        ref = x * (1.0 + rng.normal(0.0, 0.01, x.shape))
        got = ctx.image_error_pixels(xy, ref, eps=1e-3)
        d = np.abs(x[:, :3] - ref[:, :3])
        want = {"mre": (d / (np.abs(ref[:, :3]) + 1e-3)).mean(), "mae": d.mean(), "max": d.max(),
                "rmse": np.sqrt((d * d).mean())}
        for k in want:
            assert got[k] == pytest.approx(want[k], rel=1e-12), k
        with pytest.raises(_lib.AeError) as e:
            ctx.image_error_pixels(np.array([[80, 0]], np.uint32), np.zeros((1, 4)))
        assert e.value.code == -1


def test_path_counters_equal_ray_counters_without_lights():
    """With depth 1 and no lights a path is its camera ray: the frame's path
    counters equal the reference walk's counters over the camera rays."""
    import torch
    s = scenes.instanced_meshes(width=128, height=96, levels=(4, 3, 3, 2, 2), grid=64)
    with Context(128, 96) as ctx:
        ctx.upload(s)
        c = s.config.copy()
        c["depth"] = 1
        ctx.set_config(c)
        pc = np.zeros(7, np.uint64)
        _lib.check(_lib.lib().ae_path_counters(ctx.handle, _lib.ptr(pc)), ctx.handle)
        rays = ctx.camera_rays()
        d = torch.from_numpy(rays.view(np.uint8)).cuda()
        rc6 = np.zeros(6, np.uint64)
        _lib.check(_lib.lib().ae_trace_counters(ctx.handle, d.data_ptr(), len(rays), _lib.ptr(rc6)), ctx.handle)
    assert int(pc[6]) == 128 * 96
    assert np.array_equal(pc[:6], rc6)


def test_quant_counters():
    import torch
    s = scenes.instanced_meshes(width=128, height=96, levels=(4, 3, 3, 2, 2), grid=64)
    with Context(128, 96) as ctx:
        ctx.upload(s)
        ctx.prepare_fast()
        rays = ctx.camera_rays()
        hits = ctx.closest_hit(rays, _lib.VARIANT_QUANT)
        d = torch.from_numpy(rays.view(np.uint8)).cuda()
        out = {}
        for name, v in (("plain", _lib.VARIANT_PLAIN), ("quant", _lib.VARIANT_QUANT)):
            c6 = np.zeros(6, np.uint64)
            _lib.check(_lib.lib().ae_trace_counters_variant(ctx.handle, d.data_ptr(), len(rays), v, _lib.ptr(c6)),
                       ctx.handle)
            out[name] = c6
    assert int(out["quant"][5]) == int((hits["object"] != _lib.MISS).sum())
    # The 4-wide tree visits fewer BLAS nodes than the binary one.
    assert 0 < out["quant"][3] < out["plain"][3]
    assert out["quant"][4] > 0
