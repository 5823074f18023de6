"""ae_closest_hit_noalloc, the entry point for callers that cannot let the
library allocate device memory: its hits must equal ae_closest_hit's (bit for
bit, the tolerance of every closest-hit test here) on two calls in a row that
reuse its fixed staging array, and batches beyond its fixed size are refused.

Kept in a file collected last so a run that stops at the first failure has
run every other test; it creates its own context, so it passes alone in a
fresh process too."""
import ctypes

import numpy as np
import pytest

from aviatorengine2_b200 import Context, _lib, scenes

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536


def noalloc(ctx, rays, variant):
    r = np.ascontiguousarray(rays, dtype=_lib.RAY)
    hits = np.zeros(len(r), _lib.HIT)
    rc = _lib.lib().ae_closest_hit_noalloc(ctx.handle, _lib.ptr(r), len(r), _lib.ptr(hits), variant)
    return rc, hits


def random_rays(n, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, _lib.RAY)
    o = rng.uniform(0, 100, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r["ox"], r["oy"], r["oz"] = o.T
    r["dx"], r["dy"], r["dz"] = d.T
    r["tnear"] = 0.001
    return r


@pytest.mark.parametrize("variant", [_lib.VARIANT_PLAIN, _lib.VARIANT_FAST, _lib.VARIANT_QUANT])
def test_noalloc_matches_closest_hit_twice(variant):
    s = scenes.instanced_meshes(width=256, height=256, levels=(4, 3, 3, 2, 2), grid=64)
    with Context(256, 256) as ctx:
        ctx.upload(s)
        if variant != _lib.VARIANT_PLAIN:
            ctx.prepare_fast()
        first = ctx.camera_rays()            # 65,536 rays: the full staging array
        second = random_rays(3001, 9)        # a shorter second call over the same array
        for rays in (first, second):
            rc, got = noalloc(ctx, rays, variant)
            assert rc == 0, _lib.lib().ae_last_error(ctx.handle)
            want = ctx.closest_hit(rays, variant)
            assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
        assert (got["object"] != _lib.MISS).any()


def test_noalloc_refuses_oversize_batches():
    s = scenes.cornell_box(width=64, height=48)
    with Context(64, 48) as ctx:
        ctx.upload(s)
        rc, _ = noalloc(ctx, np.zeros(MAX_RAYS + 1, _lib.RAY), _lib.VARIANT_PLAIN)
        assert rc == -3
        assert b"at most 65536" in _lib.lib().ae_last_error(ctx.handle)


def test_noalloc_refuses_stale_or_unprepared_structures():
    """The optimised variants need ae_prepare_fast to have accepted the scene
    now uploaded: before it, after a new scene upload, and after a prepare that
    refused a scene with participating media, the call returns AE_ERR_STATE
    (as ae_closest_hit refuses the media scene) instead of tracing with
    structures of another scene."""
    box = scenes.cornell_box(width=64, height=48)
    rays = random_rays(512, 3)
    with Context(64, 48) as ctx:
        ctx.reserve_scene(64, 16)  # room for the media scene uploaded later
        ctx.upload(box)
        for v in (_lib.VARIANT_FAST, _lib.VARIANT_QUANT):
            assert noalloc(ctx, rays, v)[0] == -7          # before ae_prepare_fast
        ctx.prepare_fast()
        rc, got = noalloc(ctx, rays, _lib.VARIANT_FAST)
        assert rc == 0 and np.array_equal(got.view(np.uint8), ctx.closest_hit(rays, _lib.VARIANT_FAST).view(np.uint8))
        ctx.upload_scene(box.objects, box.tlas, box.lights, box.instances)
        assert noalloc(ctx, rays, _lib.VARIANT_FAST)[0] == -7  # a new scene version, not prepared yet
        media = scenes.media_box(width=64, height=48)
        ctx.upload(media)
        with pytest.raises(_lib.AeError):
            ctx.prepare_fast()                               # media are refused by the optimised forms
        for v in (_lib.VARIANT_FAST, _lib.VARIANT_QUANT):
            assert noalloc(ctx, rays, v)[0] == -7
        assert noalloc(ctx, rays, _lib.VARIANT_PLAIN)[0] == 0


def test_noalloc_refuses_walk_variant_with_its_reason():
    s = scenes.cornell_box(width=64, height=48)
    with Context(64, 48) as ctx:
        ctx.upload(s)
        ctx.prepare_fast()
        rc, _ = noalloc(ctx, random_rays(64, 4), _lib.VARIANT_FAST_WALK)
        assert rc == -1
        assert b"FAST_WALK" in _lib.lib().ae_last_error(ctx.handle)
