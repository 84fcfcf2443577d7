"""The multi-GPU path of bench.py on CPU: replicas only, so the only
cross-rank steps are the barrier and the max-over-ranks timing.  Two gloo
ranks check that every rank sees the slowest rank's time and that the
whole-job rate counts all replicas; the reference arm does no work on
ranks other than 0."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        own_ms = 10.0 + 5.0 * rank                 # rank 1 is the slow one
        t_ms = bench.max_over_ranks(own_ms, dist, device="cpu")
        rate = bench.replica_rate(world, 1000, 64, 4, t_ms / 1e3)
        out.put((rank, t_ms, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_rate_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t_ms, rate in res:
        assert t_ms == 15.0, (rank, t_ms)
        assert rate == pytest.approx(2 * 1000 * 64 * 4 / 0.015)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_rate(1, 10, 10, 1, 0.5) == 200.0


def test_reference_arm_does_nothing_off_rank_zero():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
