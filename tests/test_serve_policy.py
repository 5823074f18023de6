"""Admission policy of the render server, run on the host through
ae_serve_policy_simulate (the same C++ Policy and Arena the server's scheduler
thread uses; no GPU)."""
import numpy as np
import pytest

from aviatorengine2_b200 import _lib
from aviatorengine2_b200.serving import simulate_policy

MB = 1 << 20


def _req(tick, fp, service, scene=0):
    return dict(kind=_lib.POLICY_REQUEST, tick=tick, footprint=fp, service_ticks=service, scene=scene)


def _move(tick, scene=0):
    return dict(kind=_lib.POLICY_MOVE, tick=tick, scene=scene)


def _align(x):
    return (x + 255) // 256 * 256


def _check_invariants(events, out, arena, max_resident):
    reqs = [i for i, e in enumerate(events) if e["kind"] == _lib.POLICY_REQUEST and out[i]["status"] == 0]
    last = max([int(out[i]["done_tick"]) for i in range(len(events))] + [0])
    for t in range(last + 1):
        live = [i for i in reqs if out[i]["admit_tick"] <= t <= out[i]["done_tick"]]
        assert len(live) <= max_resident
        spans = sorted((int(out[i]["offset"]), int(out[i]["offset"]) + _align(events[i]["footprint"])) for i in live)
        assert all(a[1] <= b[0] for a, b in zip(spans, spans[1:])), f"overlapping blocks at tick {t}"
        assert all(hi <= arena for _, hi in spans)
    for i in reqs:
        assert out[i]["admit_tick"] >= events[i]["tick"]
        assert out[i]["done_tick"] - out[i]["admit_tick"] + 1 == max(events[i]["service_ticks"], 1)


def test_fifo_by_footprint():
    ev = [_req(0, 40 * MB, 3) for _ in range(5)]
    code, out = simulate_policy(ev, 100 * MB, 16, 1)
    assert code == 0
    admits = [int(o["admit_tick"]) for o in out]
    assert admits == sorted(admits)            # arrival order
    assert admits[:2] == [0, 0] and admits[2] == 3  # two fit, the third waits for a release
    _check_invariants(ev, out, 100 * MB, 16)


def test_large_request_is_not_starved():
    # A large request at the head blocks later small ones until it fits.
    ev = [_req(0, 60 * MB, 4), _req(1, 60 * MB, 2), _req(1, 1 * MB, 1), _req(1, 1 * MB, 1)]
    code, out = simulate_policy(ev, 100 * MB, 16, 1)
    assert code == 0
    assert out[1]["admit_tick"] == 4
    assert out[2]["admit_tick"] >= out[1]["admit_tick"]
    _check_invariants(ev, out, 100 * MB, 16)


def test_resident_limit():
    ev = [_req(0, 1 * MB, 2) for _ in range(7)]
    code, out = simulate_policy(ev, 100 * MB, 3, 1)
    assert code == 0
    _check_invariants(ev, out, 100 * MB, 3)
    assert sorted(int(o["admit_tick"]) for o in out) == [0, 0, 0, 2, 2, 2, 4]


def test_oversize_rejected():
    ev = [_req(0, 200 * MB, 1), _req(0, 1 * MB, 1)]
    code, out = simulate_policy(ev, 100 * MB, 4, 1)
    assert code == 0
    assert out[0]["status"] == -8  # AE_ERR_REJECTED
    assert out[0]["admit_tick"] == -1
    assert out[1]["admit_tick"] == 0


NONE = (1 << 64) - 1  # outcome offset of a coalesced move


def test_move_waits_for_earlier_requests_one_frame_set():
    # With a single copy of the per-frame arrays a move waits for every
    # earlier request of its scene.
    ev = [_req(0, 1 * MB, 5, scene=0), _req(0, 1 * MB, 2, scene=0), _move(1, scene=0),
          _req(1, 1 * MB, 1, scene=0), _req(1, 1 * MB, 1, scene=1), _req(2, 1 * MB, 1, scene=0)]
    code, out = simulate_policy(ev, 100 * MB, 16, 2, frame_sets=1)
    assert code == 0
    assert out[2]["admit_tick"] > max(out[0]["done_tick"], out[1]["done_tick"])
    assert out[2]["version"] == 1 and out[2]["offset"] == 0
    for i in (3, 5):  # later scene-0 requests see the move
        assert out[i]["version"] == 1 and out[i]["admit_tick"] >= out[2]["admit_tick"]
    assert out[4]["version"] == 0 and out[4]["admit_tick"] == 1  # scene 1 is not held up
    _check_invariants(ev, out, 100 * MB, 16)


def test_two_frame_sets_overlap_versions():
    # With two copies a move is refit into the copy no request renders while
    # the older version still runs; the next move takes whichever copy frees
    # first - here the one of version 1, long before version 0's request ends.
    ev = [_req(0, 1 * MB, 6), _move(1), _req(1, 1 * MB, 2), _move(2), _req(2, 1 * MB, 1)]
    code, out = simulate_policy(ev, 100 * MB, 16, 1, frame_sets=2)
    assert code == 0
    assert out[1]["admit_tick"] == 1 and out[1]["version"] == 1 and out[1]["offset"] == 1
    assert out[2]["version"] == 1 and out[2]["admit_tick"] == 1  # overlaps request 0
    assert out[3]["admit_tick"] == out[2]["done_tick"] + 1 and out[3]["offset"] == 1
    assert out[3]["admit_tick"] < out[0]["done_tick"]
    assert out[4]["version"] == 2 and out[4]["admit_tick"] == out[3]["admit_tick"]
    _check_invariants(ev, out, 100 * MB, 16)


def test_pending_request_of_previous_version_still_admitted():
    # A request queued for memory when the next move lands keeps its version
    # and is admitted from the copy that still holds it.
    ev = [_req(0, 80 * MB, 3), _req(0, 80 * MB, 1), _move(1), _req(1, 1 * MB, 1)]
    code, out = simulate_policy(ev, 100 * MB, 16, 1, frame_sets=2)
    assert code == 0
    assert out[2]["admit_tick"] == 1               # move applied while request 1 waits for memory
    assert out[1]["version"] == 0 and out[1]["admit_tick"] == 3
    assert out[3]["version"] == 1


def test_back_to_back_moves_coalesce():
    # Two moves before any request: the first is superseded (moves carry
    # absolute transforms) and only version 2 is refit.
    ev = [_move(0), _move(0), _req(0, 1 * MB, 1), _move(1), _req(1, 1 * MB, 1)]
    code, out = simulate_policy(ev, 100 * MB, 16, 1, frame_sets=1)
    assert code == 0
    assert out[0]["version"] == 1 and out[0]["offset"] == NONE and out[0]["admit_tick"] == 0
    assert out[1]["version"] == 2 and out[1]["offset"] == 0
    assert out[2]["version"] == 2 and out[4]["version"] == 3
    assert out[3]["admit_tick"] > out[2]["done_tick"]
    assert out[4]["admit_tick"] >= out[3]["admit_tick"]


def test_moves_every_tick_are_refit_every_tick():
    # A move per tick and no requests: each is refit at its tick (the newest
    # state is materialized eagerly whenever a copy is free).
    ev = [_move(t) for t in range(10)]
    code, out = simulate_policy(ev, 100 * MB, 16, 1, frame_sets=2)
    assert code == 0
    assert [int(o["admit_tick"]) for o in out] == list(range(10))
    assert all(o["offset"] != NONE for o in out)


def test_frame_rate_moves_do_not_hold_up_requests():
    # A move every tick while requests of 20 ticks arrive every 4 ticks:
    # with 8 copies every request is admitted when it arrives, and the moves
    # keep being refit (or coalesced when every copy is pinned).
    ev = []
    for t in range(60):
        ev.append(_move(t))
        if t % 4 == 0:
            ev.append(_req(t, 1 * MB, 20))
    code, out = simulate_policy(ev, 100 * MB, 64, 1, frame_sets=8)
    assert code == 0
    for i, e in enumerate(ev):
        if e["kind"] == _lib.POLICY_REQUEST:
            assert out[i]["admit_tick"] == e["tick"], (i, out[i])
    applied = [o for o, e in zip(out, ev) if e["kind"] == _lib.POLICY_MOVE and o["offset"] != NONE]
    assert len(applied) >= 45
    _check_invariants(ev, out, 100 * MB, 64)


@pytest.mark.parametrize("frame_sets", [1, 2, 8])
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_random_streams_keep_invariants(seed, frame_sets):
    rng = np.random.default_rng(seed)
    ev, t = [], 0
    for _ in range(300):
        t += int(rng.poisson(1.0))
        if rng.random() < 0.3:
            ev.append(_move(t, scene=int(rng.integers(0, 4))))
        else:
            ev.append(_req(t, int(rng.choice([1, 4, 16, 33]) * MB), int(rng.integers(1, 8)), scene=int(rng.integers(0, 4))))
    code, out = simulate_policy(ev, 64 * MB, 8, 4, frame_sets=frame_sets)
    assert code == 0
    _check_invariants(ev, out, 64 * MB, 8)
    moves_before = {s: 0 for s in range(4)}
    made = {(s, 0): (0, 0) for s in range(4)}  # (scene, version) -> (tick, copy) it was materialized
    for i, e in enumerate(ev):
        s = e["scene"]
        if e["kind"] == _lib.POLICY_MOVE:
            moves_before[s] += 1
            assert int(out[i]["version"]) == moves_before[s]
            if out[i]["offset"] != NONE:
                made[(s, moves_before[s])] = (int(out[i]["admit_tick"]), int(out[i]["offset"]))
        else:
            # every request renders the version of its scene current at its arrival
            assert out[i]["version"] == moves_before[s]
    reqs = [i for i, e in enumerate(ev) if e["kind"] == _lib.POLICY_REQUEST and out[i]["status"] == 0]
    for i in reqs:
        key = (ev[i]["scene"], int(out[i]["version"]))
        assert key in made, f"request {i} renders version {key} that was coalesced"
        assert out[i]["admit_tick"] >= made[key][0]
    # A copy is overwritten only after every request of the version it held is done.
    for s in range(4):
        timeline = sorted((tick, copy, v) for (ss, v), (tick, copy) in made.items() if ss == s)
        held = {}
        for tick, copy, v in timeline:
            if copy in held:
                old = held[copy]
                for i in reqs:
                    if ev[i]["scene"] == s and int(out[i]["version"]) == old:
                        assert out[i]["done_tick"] < tick, (s, copy, old, v, i)
            held[copy] = v


def _cancel(tick, target):
    return dict(kind=_lib.POLICY_CANCEL, tick=tick, footprint=target)


def test_cancel_queued_request_frees_its_turn():
    # Request 1 waits behind request 0; withdrawn while queued, it never runs
    # and request 3 takes the arena after request 0.
    ev = [_req(0, 60 * MB, 5), _req(1, 60 * MB, 5), _cancel(2, 1), _req(3, 60 * MB, 1)]
    code, out = simulate_policy(ev, 100 * MB, 16, 1)
    assert code == 0
    assert out[1]["status"] == -9 and out[1]["admit_tick"] == -1 and out[1]["done_tick"] == 2
    assert out[3]["admit_tick"] == 5


def test_cancel_admitted_request_releases_arena_and_slot():
    # Request 0 holds most of the arena for 50 ticks; withdrawn at tick 3,
    # its block is released and request 1 is admitted that tick.
    ev = [_req(0, 90 * MB, 50), _req(1, 90 * MB, 2), _cancel(3, 0)]
    code, out = simulate_policy(ev, 100 * MB, 1, 1)
    assert code == 0
    assert out[0]["status"] == -9 and out[0]["done_tick"] == 3
    assert out[1]["status"] == 0 and out[1]["admit_tick"] == 3


def test_cancel_of_finished_request_changes_nothing():
    ev = [_req(0, 10 * MB, 1), _cancel(5, 0)]
    code, out = simulate_policy(ev, 100 * MB, 4, 1)
    assert code == 0 and out[0]["status"] == 0 and out[0]["done_tick"] == 0


def test_cancel_unblocks_move_waiting_for_its_version():
    # With one frame set a move waits for every request of the old version;
    # withdrawing the long one lets the move apply at the cancel tick.
    ev = [_req(0, 1 * MB, 100), _move(1), _cancel(4, 0)]
    code, out = simulate_policy(ev, 100 * MB, 4, 1, frame_sets=1)
    assert code == 0
    assert out[0]["status"] == -9
    assert out[1]["admit_tick"] == 4
