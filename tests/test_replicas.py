"""bench.py's multi-GPU path on the CPU: world size 2 over gloo.  The path
does not shard (each rank is an independent replica on its own GPU), so the
only cross-rank steps are the barrier and the max of the step time over
ranks; the reference arm runs on rank 0 alone."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        step_ms = 10.0 + 5.0 * rank  # rank 1 is the slow replica
        ms = bench.max_over_ranks(step_ms, dist)
        out[rank] = (ms, bench.replica_value(1_000_000, world, ms / 1e3))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_replicas():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        ps = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    # Every rank sees the slowest replica's time; the job's value is both
    # replicas' units over that time.
    assert res[0][0] == res[1][0] == 15.0
    assert res[0][1] == pytest.approx(2 * 1_000_000 / 0.015 / 1e6)


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.replica_value(10, 1, 2.0) == pytest.approx(5e-6)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
