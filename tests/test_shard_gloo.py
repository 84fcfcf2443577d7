"""Velocity-space sharding, host side, on CPU: the row partition, the NCCL
id exchange over a gloo group, and the phase protocol of a host-reduced
sharded step with two gloo ranks (a stand-in solver computes known partial
sums, so the test checks what each phase sees after the reduction)."""
import os
import socket
import sys

import numpy as np
import pytest

from dugks_b200 import lib as dl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("rows,world", [(8, 1), (8, 2), (8, 3), (256, 7), (28, 28), (5, 4)])
def test_dv_rows_partition(rows, world):
    spans = [dl.dv_rows(rows, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == rows
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 == b0
    sizes = [b - a for a, b in spans]
    assert min(sizes) >= 1 and max(sizes) - min(sizes) <= 1


def test_shard_descriptor():
    s = dl.shard(1, 4)
    assert (s.rank, s.world, s.use_nccl) == (1, 4, 0)
    s = dl.shard(2, 4, bytes(range(128)))
    assert s.use_nccl == 1 and bytes(s.nccl_id) == bytes(range(128))
    with pytest.raises(ValueError):
        dl.shard(0, 2, b"short")


class _Shard:
    """Stands in for a sharded Solver: phase 0 yields this rank's face
    partials (rank + 1) * [1, 2, ...], phase 1 records the reduced face
    buffer and yields cell partials; phase 2 records the reduced cell
    buffer."""

    def __init__(self, rank, n_face=6, n_cell=4):
        import torch
        self.rank = rank
        self.bufs = {1: torch.zeros(n_face, dtype=torch.float64), 2: torch.zeros(n_cell, dtype=torch.float64)}
        self.seen = []
        self.expected = 0

    def shard_phase(self, phase, dt=0.0):
        import torch
        assert phase == self.expected, (phase, self.expected)
        self.expected = (phase + 1) % 3
        if phase == 0:
            assert dt == 0.25
            b = self.bufs[1]
            b.copy_(torch.from_numpy((self.rank + 1) * (1.0 + np.arange(b.numel()))))
            return 1, b.numel()
        if phase == 1:
            self.seen.append(("faces", self.bufs[1].tolist()))
            b = self.bufs[2]
            b.copy_(torch.from_numpy(10.0 * (self.rank + 1) * (1.0 + np.arange(b.numel()))))
            return 2, b.numel()
        self.seen.append(("cells", self.bufs[2].tolist()))
        return 0, 0


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "psp-vst_b200", "python"))
    from dugks_b200 import shard as sh
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s = sh.init_nccl_shard(rank, world)
        fake = _Shard(rank)
        sh.step_allreduce(fake, 2, 0.25, view=lambda addr, n: fake.bufs[addr])
        out.put((rank, bytes(s.nccl_id), s.rank, s.world, s.use_nccl, fake.seen))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_nccl_id_and_reduce_between_phases():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, id0, r0, w0, n0, seen0), (_, id1, r1, w1, n1, seen1) = res
    assert id0 == id1 and len(id0) == 128 and any(id0)
    assert (r0, w0, n0, r1, w1, n1) == (0, 2, 1, 1, 2, 1)
    faces = (3.0 * (1.0 + np.arange(6))).tolist()        # (1 + 2) * [1..6]
    cells = (30.0 * (1.0 + np.arange(4))).tolist()       # 10 (1 + 2) * [1..4]
    expect = [("faces", faces), ("cells", cells)] * 2     # two steps
    assert seen0 == expect and seen1 == expect
