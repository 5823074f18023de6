"""The render server on the GPU: every request's images equal those of
`frames` compute-only frames rendered alone, bit for bit - when served alone,
when mixed with requests of other scenes, resolutions and sample counts that
overlap it on the device, and across instance moves (GPU refit) queued
between requests.  Also admission by image footprint and rejection."""
import numpy as np
import pytest

from aviatorengine2_b200 import AeError, Context, Server, _lib, scenes

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


def config_for(scene, width, height, samples=1, depth=None, source=None):
    c = scene.config.copy()
    c["width"], c["height"], c["samples"], c["batches"] = width, height, samples, 1
    if depth is not None:
        c["depth"] = depth
    if source is not None:
        c["source_x"], c["source_y"], c["source_z"] = source
    return c


def frames_alone(scene, cfg, frames, mode=_lib.MODE_COMPUTE_ONLY, instances=None):
    """accum and display after `frames` frames (Batch = 0..frames-1) on a
    fresh context, optionally after a refit to `instances`."""
    w, h = int(cfg["width"]), int(cfg["height"])
    with Context(w, h, samples=int(cfg["samples"])) as ctx:
        ctx.upload(scene)
        if instances is not None:
            ctx.refit_instances(instances)
        c = cfg.copy()
        for b in range(frames):
            c["batch"] = b
            ctx.set_config(c)
            ctx.render_frame(mode)
        return ctx.read_image(_lib.IMAGE_ACCUM), ctx.read_image(_lib.IMAGE_DISPLAY)


def resident(scene):
    ctx = Context(int(scene.config["width"]), int(scene.config["height"]))
    ctx.upload(scene)
    return ctx


def test_single_request_equals_plain_frames():
    s = scenes.cornell_box(width=96, height=64, depth=6)
    cfg = config_for(s, 96, 64, samples=2)
    ref_acc, ref_dsp = frames_alone(s, cfg, 3)
    ctx = resident(s)
    # Fewer slots than pixels: slots move on to new pixels many times.
    with Server(slots=2048, max_requests=4, arena_bytes=1 << 24) as srv:
        sid = srv.add_scene(ctx)
        for _ in range(2):
            rid = srv.submit(sid, 96, 64, 3, cfg)
            res, acc, dsp = srv.wait(rid, 60000)
            assert res["status"] == 0
            assert same(acc, ref_acc)
            assert np.array_equal(dsp, ref_dsp)
        st = srv.stats()
        assert st["completed"] == 2 and st["errors"] == 0
        assert st["paths"] == 2 * 96 * 64 * 3 * 2
    ctx.close()


def _mixed_requests(s_a, s_b):
    return [
        (0, 96, 64, 2, config_for(s_a, 96, 64, samples=1)),
        (1, 80, 60, 1, config_for(s_b, 80, 60, samples=3)),
        (0, 128, 96, 1, config_for(s_a, 128, 96, samples=1, source=(4.0, 5.0, 24.0))),
        (1, 64, 48, 3, config_for(s_b, 64, 48, samples=1)),
        (0, 32, 32, 4, config_for(s_a, 32, 32, samples=2, depth=3)),
    ]


def test_mixed_requests_equal_alone():
    s_a = scenes.cornell_box(depth=6)
    s_b = scenes.hybrid_box(depth=5)
    reqs = _mixed_requests(s_a, s_b)
    ctx_a, ctx_b = resident(s_a), resident(s_b)
    with Server(slots=8192, max_requests=8, arena_bytes=1 << 26) as srv:
        ids = [srv.add_scene(ctx_a), srv.add_scene(ctx_b)]
        alone = []
        for sc, w, h, f, cfg in reqs:
            res, acc, dsp = srv.wait(srv.submit(ids[sc], w, h, f, cfg), 60000)
            assert res["status"] == 0
            alone.append((acc, dsp))
        srv.reset_stats()
        mixed = [srv.submit(ids[sc], w, h, f, cfg) for sc, w, h, f, cfg in reqs]
        for k, rid in enumerate(mixed):
            res, acc, dsp = srv.wait(rid, 60000)
            assert res["status"] == 0
            assert same(acc, alone[k][0]), f"request {k} differs when mixed"
            assert np.array_equal(dsp, alone[k][1])
        st = srv.stats()
        assert st["peak_resident"] >= 2, "requests did not overlap on the device"
        assert st["p99_ms"] >= st["p50_ms"] > 0
    # And alone equals the plain megakernel's frames.
    for k, (sc, w, h, f, cfg) in enumerate(reqs):
        ref_acc, ref_dsp = frames_alone((s_a, s_b)[sc], cfg, f)
        assert same(alone[k][0], ref_acc), f"request {k} differs from plain frames"
        assert np.array_equal(alone[k][1], ref_dsp)
    ctx_a.close()
    ctx_b.close()


def test_moves_between_requests():
    s = scenes.wavefront_scene(seed=11, width=64, height=48, depth=4, n_meshes=4, n_instances=48,
                               n_lights=4, target_tris=30_000)
    cfg = config_for(s, 64, 48, samples=1)
    rng = np.random.default_rng(3)
    moved1 = scenes.random_walk(s.instances, rng, step=2.0, angle=0.2)
    moved2 = scenes.random_walk(moved1, rng, step=2.0, angle=0.2)
    ctx = resident(s)
    with Server(slots=4096, max_requests=8, arena_bytes=1 << 24) as srv:
        sid = srv.add_scene(ctx)
        r0 = srv.submit(sid, 64, 48, 2, cfg)
        srv.move_instances(sid, moved1)
        r1 = srv.submit(sid, 64, 48, 2, cfg)
        srv.move_instances(sid, moved2)
        r2 = srv.submit(sid, 64, 48, 1, cfg)
        out = [srv.wait(r, 60000) for r in (r0, r1, r2)]
        assert [int(o[0]["scene_version"]) for o in out] == [0, 1, 2]
        assert srv.stats()["moves_applied"] == 2
    ctx.close()
    # References on a twin context refit the same way, through the wavefront
    # renderer (same optimised traversal as the server).
    with Context(64, 48) as twin:
        twin.upload(s)
        for k, (inst, frames) in enumerate(((None, 2), (moved1, 2), (moved2, 1))):
            if inst is not None:
                twin.refit_instances(inst)
            c = cfg.copy()
            for b in range(frames):
                c["batch"] = b
                twin.set_config(c)
                twin.render_frame(_lib.MODE_WAVEFRONT)
            assert same(out[k][1], twin.read_image(_lib.IMAGE_ACCUM)), f"request {k}"
            assert np.array_equal(out[k][2], twin.read_image(_lib.IMAGE_DISPLAY))


def test_frame_rate_moves_coalesce_and_requests_see_their_version():
    """Moves submitted faster than requests (several per request, as a world
    moving every frame): a request renders the transforms of the last move
    submitted before it, bit for bit, while moves no request sees are
    coalesced or refit eagerly; every move is accounted for."""
    s = scenes.wavefront_scene(seed=12, width=64, height=48, depth=4, n_meshes=4, n_instances=48,
                               n_lights=4, target_tris=30_000)
    cfg = config_for(s, 64, 48, samples=1)
    rng = np.random.default_rng(9)
    walk = [s.instances]
    for _ in range(15):
        walk.append(scenes.random_walk(walk[-1], rng, step=1.0, angle=0.1))
    ctx = resident(s)
    with Server(slots=4096, max_requests=8, arena_bytes=1 << 24) as srv:
        sid = srv.add_scene(ctx)
        r0 = srv.submit(sid, 64, 48, 3, cfg)
        for k in range(1, 11):
            srv.move_instances(sid, walk[k])
        r1 = srv.submit(sid, 64, 48, 2, cfg)
        for k in range(11, 16):
            srv.move_instances(sid, walk[k])
        r2 = srv.submit(sid, 64, 48, 1, cfg)
        out = [srv.wait(r, 60000) for r in (r0, r1, r2)]
        srv.drain(60000)
        st = srv.stats()
    ctx.close()
    assert [int(o[0]["scene_version"]) for o in out] == [0, 10, 15]
    assert st["moves_applied"] + st["moves_coalesced"] == 15 and st["moves_applied"] >= 2
    with Context(64, 48) as twin:
        twin.upload(s)
        for k, (inst, frames) in enumerate(((None, 3), (walk[10], 2), (walk[15], 1))):
            if inst is not None:
                twin.refit_instances(inst)
            c = cfg.copy()
            for b in range(frames):
                c["batch"] = b
                twin.set_config(c)
                twin.render_frame(_lib.MODE_WAVEFRONT)
            assert same(out[k][1], twin.read_image(_lib.IMAGE_ACCUM)), f"request {k}"


def test_admission_by_footprint_and_rejection():
    s = scenes.cornell_box(depth=3)
    ctx = resident(s)
    arena = 1 << 20  # 64x64 needs 80 KiB: at most 12 resident
    with Server(slots=4096, max_requests=16, arena_bytes=arena) as srv:
        sid = srv.add_scene(ctx)
        with pytest.raises(AeError) as e:
            srv.submit(sid, 256, 256, 1, config_for(s, 256, 256))
        assert e.value.code == -8
        cfg = config_for(s, 64, 64)
        ids = [srv.submit(sid, 64, 64, 2, cfg) for _ in range(40)]
        first = None
        for rid in ids:
            res, acc, dsp = srv.wait(rid, 120000)
            assert res["status"] == 0
            if first is None:
                first = acc
            assert same(acc, first)
        st = srv.stats()
        assert st["completed"] == 40 and st["rejected"] == 1
        assert 0 < st["peak_arena_bytes"] <= arena
        assert st["peak_resident"] <= 12
    ctx.close()
