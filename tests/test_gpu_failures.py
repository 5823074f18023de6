"""Failure detection without faulting a GPU: the failures are made on the
host (an injected allocation failure, a cancelled request) or are a bounded
device-side wait that is made to run out with nothing in flight
(AE_FAULT_TILE_WAIT: the tile-staged extend issues no bulk copy and its
mbarrier wait on the unarmed phase gives up after a few polls).  Each test
checks the error code that comes back through the C ABI, that nothing leaks
(live device allocations return to their count before the call) and that the
context or server stays usable where the contract says so."""
import numpy as np
import pytest

from aviatorengine2_b200 import AeError, Context, Server, _lib, scenes

pytestmark = pytest.mark.gpu

L = _lib.lib


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


@pytest.fixture(autouse=True)
def _no_pending_failure():
    L().ae_debug_fail_alloc_after(-1)
    yield
    L().ae_debug_fail_alloc_after(-1)


def plain_frame(s, batch=0):
    c = s.config.copy()
    c["batch"] = batch
    with Context(int(c["width"]), int(c["height"])) as ctx:
        ctx.upload(s)
        ctx.set_config(c)
        ctx.render_frame(_lib.MODE_COMPUTE_ONLY)
        return ctx.read_image(_lib.IMAGE_FRAME)


def test_wavefront_tile_wait_timeout_is_reported_and_recoverable():
    s = scenes.cornell_box(width=96, height=64)
    with Context(96, 64) as ctx:
        ctx.upload(s)
        ctx.render_frame(_lib.MODE_WAVEFRONT)          # tunes the extend stage; a clean frame
        ctx.debug_inject(_lib.FAULT_TILE_WAIT)
        for mode in (_lib.MODE_WAVEFRONT, _lib.MODE_WAVEFRONT_PRECISION):
            with pytest.raises(AeError) as e:
                ctx.render_frame(mode)
            assert e.value.code == -6                   # AE_ERR_TIMEOUT
            assert ctx.wavefront_info()["errors"] != 0
        ctx.debug_inject(_lib.FAULT_TILE_WAIT, False)
        ctx.render_frame(_lib.MODE_WAVEFRONT)          # the context is still usable
        assert ctx.wavefront_info()["errors"] == 0
        got = ctx.read_image(_lib.IMAGE_FRAME)
    assert same(got, plain_frame(s))


def test_serving_tile_wait_timeout_fails_every_unfinished_request():
    s = scenes.cornell_box(width=64, height=48)
    with Context(64, 48) as ctx:
        ctx.upload(s)
        with Server(slots=4096, max_requests=4, arena_bytes=1 << 24, extend_threads=128) as srv:
            sid = srv.add_scene(ctx)
            srv.debug_inject(_lib.FAULT_TILE_WAIT)
            ids = [srv.submit(sid, 64, 48, 4, s.config) for _ in range(3)]
            for r in ids:
                with pytest.raises(AeError) as e:
                    srv.wait(r, 60000)
                assert e.value.code == -6
            assert srv.stats()["errors"] != 0
            with pytest.raises(AeError) as e:               # a failed server refuses new work
                srv.submit(sid, 64, 48, 1, s.config)
            assert e.value.code == -7


def test_allocation_failure_in_create_leaks_nothing():
    base = L().ae_debug_live_allocations()
    failures = 0
    for n in range(4):
        L().ae_debug_fail_alloc_after(n)
        try:
            ctx = Context(64, 48)
        except AeError as e:
            assert e.code == -2                              # AE_ERR_OOM
            assert L().ae_create_status() == -2
            failures += 1
        else:
            ctx.close()
        L().ae_debug_fail_alloc_after(-1)
        assert L().ae_debug_live_allocations() == base, n
    assert failures == 3  # accumulation, frame and display images


def test_allocation_failure_in_prepare_fast_leaks_nothing_and_recovers():
    s = scenes.instanced_meshes(width=64, height=48, levels=(3, 2, 2, 1, 1), grid=32)
    base = L().ae_debug_live_allocations()
    with Context(64, 48) as ctx:
        ctx.upload(s)
        rays = ctx.camera_rays()
        want = ctx.closest_hit(rays, _lib.VARIANT_PLAIN)
        failures = 0
        for n in range(6):
            L().ae_debug_fail_alloc_after(n)
            rc = L().ae_prepare_fast(ctx.handle)
            L().ae_debug_fail_alloc_after(-1)
            if rc == 0:
                break
            assert rc == -2, rc
            failures += 1
        assert failures >= 2
        ctx.prepare_fast()
        got = ctx.closest_hit(rays, _lib.VARIANT_FAST)
        assert np.array_equal(got["object"], want["object"]) and np.array_equal(got["prim"], want["prim"])
    assert L().ae_debug_live_allocations() == base


def test_allocation_failure_in_serve_create_leaks_nothing():
    base = L().ae_debug_live_allocations()
    failures = 0
    for n in range(0, 24, 3):
        L().ae_debug_fail_alloc_after(n)
        try:
            srv = Server(slots=4096, max_requests=4, arena_bytes=1 << 22)
        except AeError as e:
            assert e.code == -2, e
            failures += 1
        else:
            srv.close()
        L().ae_debug_fail_alloc_after(-1)
        assert L().ae_debug_live_allocations() == base, n
    assert failures >= 5


def test_cancel_reclaims_slots_and_arena_others_identical():
    """A large request is withdrawn while on the GPU; the small ones beside
    it finish with the images they have alone, and the arena block and the
    slots of the cancelled request are reused by a request that needs them."""
    s = scenes.cornell_box(width=160, height=120)
    small = [(64, 48, 2), (80, 60, 3)]
    with Context(160, 120) as ctx:
        ctx.upload(s)
        alone = []
        # 1.2 MB of arena: the 160x120 request (384 KB of images) and the two
        # small ones fit together; the 256x200 request after them (1.02 MB)
        # fits only once the cancelled request's block is back.
        arena = 1_200_000
        with Server(slots=8192, max_requests=4, arena_bytes=arena) as srv:
            sid = srv.add_scene(ctx)
            for w, h, f in small:
                res, acc, dsp = srv.wait(srv.submit(sid, w, h, f, s.config), 60000)
                alone.append((acc, dsp))
        with Server(slots=8192, max_requests=4, arena_bytes=arena) as srv:
            sid = srv.add_scene(ctx)
            big = srv.submit(sid, 160, 120, 400, s.config)
            mixed = [srv.submit(sid, w, h, f, s.config) for w, h, f in small]
            srv.cancel(big)
            with pytest.raises(AeError) as e:
                srv.wait(big, 120000)
            assert e.value.code == -9                       # AE_ERR_CANCELLED
            for (acc0, dsp0), r in zip(alone, mixed):
                res, acc, dsp = srv.wait(r, 120000)
                assert res["status"] == 0
                assert same(acc, acc0) and np.array_equal(dsp, dsp0)
            res, acc, _ = srv.wait(srv.submit(sid, 256, 200, 1, s.config), 120000)
            assert res["status"] == 0
            st = srv.stats()
            assert st["cancelled"] == 1 and st["failed"] == 0


def test_cancel_queued_request():
    s = scenes.cornell_box(width=64, height=48)
    with Context(64, 48) as ctx:
        ctx.upload(s)
        # The arena holds one 64x48 request at a time: the second queues.
        with Server(slots=2048, max_requests=4, arena_bytes=64 * 48 * 20 + 512) as srv:
            sid = srv.add_scene(ctx)
            first = srv.submit(sid, 64, 48, 1000, s.config)
            second = srv.submit(sid, 64, 48, 1, s.config)
            srv.cancel(second)
            with pytest.raises(AeError) as e:
                srv.wait(second, 1000)
            assert e.value.code == -9
            res, _, _ = srv.wait(first, 120000)
            assert res["status"] == 0
            with pytest.raises(AeError) as e:
                srv.cancel(first)                           # finished and returned: unknown now
            assert e.value.code == -1
