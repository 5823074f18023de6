"""The debug walk (AE_VARIANT_PLAIN_CHECKED): the reference walk with every
stack push checked against the stack's capacity and every buffer index
against its array's length.

On valid scenes its hits equal the plain walk's bit for bit and it raises no
check.  With AE_FAULT_CHECK_LIMITS it checks against smaller capacities and
lengths than the real ones (stacks of 2, half of every array), so both kinds
of check fire on a valid scene while every access it still makes stays inside
the real arrays: the call succeeds, the check word carries both bits, and
reading it clears it."""
import numpy as np
import pytest

from aviatorengine2_b200 import Context, _lib, scenes

pytestmark = pytest.mark.gpu


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


@pytest.mark.parametrize("make", [lambda: scenes.cornell_box(width=96, height=64),
                                  lambda: scenes.instanced_meshes(width=160, height=96, levels=(4, 3, 3, 2, 2),
                                                                  grid=64)])
def test_checked_walk_equals_plain_and_raises_nothing(make):
    s = make()
    w, h = int(s.config["width"]), int(s.config["height"])
    with Context(w, h) as ctx:
        ctx.upload(s)
        rays = np.concatenate([ctx.camera_rays(), random_rays(4000, 5)])
        want = ctx.closest_hit(rays, _lib.VARIANT_PLAIN)
        got = ctx.closest_hit(rays, _lib.VARIANT_PLAIN_CHECKED)
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
        assert ctx.debug_flags() == 0


def test_checks_fire_under_reduced_limits_and_clear_on_read():
    s = scenes.instanced_meshes(width=160, height=96, levels=(4, 3, 3, 2, 2), grid=64)
    with Context(160, 96) as ctx:
        ctx.upload(s)
        rays = np.concatenate([ctx.camera_rays(), random_rays(4000, 6)])
        want = ctx.closest_hit(rays, _lib.VARIANT_PLAIN)
        ctx.debug_inject(_lib.FAULT_CHECK_LIMITS)
        try:
            ctx.closest_hit(rays, _lib.VARIANT_PLAIN_CHECKED)
            flags = ctx.debug_flags()
            assert flags & _lib.CHECK_STACK and flags & _lib.CHECK_INDEX, flags
            assert ctx.debug_flags() == 0      # reading cleared the word
        finally:
            ctx.debug_inject(_lib.FAULT_CHECK_LIMITS, False)
        got = ctx.closest_hit(rays, _lib.VARIANT_PLAIN_CHECKED)
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
        assert ctx.debug_flags() == 0
