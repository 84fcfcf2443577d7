"""Velocity-space sharding on the host side.

A sharded solver (``lib.Solver(case, shard=lib.shard(rank, world, ...))``)
holds one contiguous block of DV rows.  Each step needs two sums over all
shards: the raw face moments after the face reconstruction and the raw cell
moments after the update (the reductions of fieldMPIreducer in the
reference's velocity-space decomposition, src/fvDVM/fvDVM/fvDVM.C:1241-1245,
:1547-1552, :1738-1740).

* With NCCL (one process per GPU): ``init_nccl_shard`` makes the NCCL id on
  rank 0, sends it to the other ranks over an existing process group, and
  the library reduces inside ``Solver.step``.
* Host-reduced: ``step_local`` sums the shards of one process (several
  shards on one device, e.g. to check a decomposition on one GPU), and
  ``step_allreduce`` sums across processes with ``torch.distributed``
  between the phases of ``dugks_shard_phase``.
"""
from __future__ import annotations

from typing import Callable, Sequence

from . import lib as dl


def device_view(addr: int, n: int):
    """A torch tensor over n doubles at a device address of the current
    device (no copy)."""
    import torch

    class _Buf:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (addr, False), "version": 3}

    return torch.as_tensor(_Buf(), device="cuda")


def init_nccl_shard(rank: int, world: int, group=None) -> dl.Shard:
    """The shard descriptor of this rank with a common NCCL id: rank 0 makes
    the id, torch.distributed broadcasts it (any backend)."""
    import torch.distributed as dist

    box = [dl.nccl_unique_id() if rank == 0 else None]
    dist.broadcast_object_list(box, src=0, group=group)
    return dl.shard(rank, world, box[0])


def _phases(solvers: Sequence, dt: float, reduce: Callable[[list], None]) -> None:
    for phase in (0, 1):
        reduce([s.shard_phase(phase, dt) for s in solvers])
    for s in solvers:
        s.shard_phase(2)


def step_local(solvers: Sequence, n_steps: int, dt: float, view: Callable = device_view) -> None:
    """n steps of all shards of one process: the partial moments of every
    shard are summed (in shard order) and the sum written back to each."""
    def reduce(parts):
        bufs = [view(a, n) for a, n in parts]
        total = bufs[0].clone()
        for b in bufs[1:]:
            total += b
        for b in bufs:
            b.copy_(total)
        _sync(bufs[0])

    for _ in range(n_steps):
        _phases(solvers, dt, reduce)


def step_allreduce(solver, n_steps: int, dt: float, view: Callable = device_view,
                   all_reduce: Callable | None = None, group=None) -> None:
    """n steps of this process's shard, summing the partial moments over the
    ranks of a torch.distributed group between the phases.  Every rank
    makes the same calls."""
    if all_reduce is None:
        import torch.distributed as dist

        def all_reduce(t):
            dist.all_reduce(t, group=group)

    def reduce(parts):
        (a, n), = parts
        t = view(a, n)
        all_reduce(t)
        _sync(t)

    for _ in range(n_steps):
        _phases([solver], dt, reduce)


def _sync(t) -> None:
    # the library's stream runs the next phase: the reduction has to be done
    if getattr(t, "is_cuda", False):
        import torch

        torch.cuda.synchronize(t.device)
