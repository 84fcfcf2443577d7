"""Velocity-space sharding on one GPU.

Host-reduced shards are separate handles in one process; between the phases
of a step the host sums their partial moments (dugks_b200.shard.step_local),
so no kernel waits on another.  The NCCL path is checked with a one-rank
communicator: the same sequence of chunk sums and all-reduces as on many
GPUs, which must leave the result bitwise equal to the unsharded step."""
import numpy as np
import pytest

import oracle_bind as ob
from dugks_b200 import case as cs
from dugks_b200 import lib as dl
from dugks_b200 import shard as sh

pytestmark = pytest.mark.gpu


def _shards(case, world, **kw):
    return [dl.Solver(case, shard=dl.shard(r, world), **kw) for r in range(world)]


def _stacked_state(solvers):
    gs, hs = zip(*(s.state() for s in solvers))
    return np.concatenate(gs), np.concatenate(hs)


@pytest.mark.parametrize("world", [2, 3])
def test_host_reduced_shards_match_the_unsharded_step_and_the_oracle(world):
    c = cs.cavity_case(8, 8)
    shards = _shards(c, world, dv_chunks=2)
    rows = len(c.xis) ** (c.D - 1)
    for r, s in enumerate(shards):
        r0, r1 = dl.dv_rows(rows, r, world)
        assert (s.dv_first, s.n_dv_local) == (r0 * len(c.xis), (r1 - r0) * len(c.xis))
    sh.step_local(shards, 6, c.dt)
    plain = dl.Solver(c)
    plain.step(6, c.dt)
    orc = ob.Oracle(c)
    for _ in range(6):
        orc.evolution(c.dt)
    for s in shards:
        e_plain = ob.macro_errors(s.macros(), plain.macros(), c.gas["R"])
        assert max(e_plain.values()) <= 1e-12, e_plain
        e_orc = ob.macro_errors(s.macros(), orc.macros(), c.gas["R"])
        assert max(e_orc.values()) <= 1e-10, e_orc
    g, h = _stacked_state(shards)
    gp, hp = plain.state()
    assert ob.rel_l2(g, gp) <= 1e-12 and ob.rel_l2(h, hp) <= 1e-12


def test_uneven_shards_on_a_far_field_ball():
    # 64 DV rows over 3 shards: 21, 21, 22 rows; wall and far-field faces
    c = cs.ball_case(4, 4, 1.12, 8, kn=0.1, mach=0.5)
    shards = _shards(c, 3)
    assert [s.n_dv_local for s in shards] == [21 * 8, 21 * 8, 22 * 8]
    sh.step_local(shards, 5, c.dt)
    orc = ob.Oracle(c)
    for _ in range(5):
        orc.evolution(c.dt)
    errs = ob.macro_errors(shards[2].macros(), orc.macros(), c.gas["R"])
    assert max(errs.values()) <= 1e-10, errs
    ferrs = ob.macro_errors(shards[0].face_macros(), orc.face_macros(), c.gas["R"])
    assert max(ferrs.values()) <= 1e-10, ferrs
    assert ob.rel_l2(shards[1].boundary_rho(), orc.boundary_rho()) <= 1e-10


def test_fp32c_shards():
    c = cs.cavity_case(8, 8)
    shards = _shards(c, 2, precision=dl.FP32C)
    sh.step_local(shards, 6, c.dt)
    plain = dl.Solver(c, precision=dl.FP32C)
    plain.step(6, c.dt)
    errs = ob.macro_errors(shards[0].macros(), plain.macros(), c.gas["R"], floor=1e-2)
    assert max(errs.values()) <= 1e-6, errs


def test_nccl_one_rank_is_bitwise_the_unsharded_step():
    c = cs.cavity_case(8, 8)
    a = dl.Solver(c, shard=dl.shard(0, 1, dl.nccl_unique_id()), dv_chunks=3)
    b = dl.Solver(c, dv_chunks=3)
    a.step(4, c.dt)
    b.step(4, c.dt)
    da, ha = a.step_adaptive(3, c.dt, 0.5)
    db, hb = b.step_adaptive(3, c.dt, 0.5)
    assert da == db and np.array_equal(ha, hb)
    ga, ha_ = a.state()
    gb, hb_ = b.state()
    assert np.array_equal(ga, gb) and np.array_equal(ha_, hb_)
    for k in ("rho", "U", "T", "q"):
        assert np.array_equal(a.macros()[k], b.macros()[k]), k
    # set_state reduces the recomputed cell moments over the shards too
    a.set_state(ga, ha_, c.dt)
    b.set_state(gb, hb_, c.dt)
    assert np.array_equal(a.macros()["rho"], b.macros()["rho"])


def test_host_reduced_shard_refuses_internal_steps_and_bad_phases():
    c = cs.cavity_case(4, 6)
    s = dl.Solver(c, shard=dl.shard(0, 2))
    with pytest.raises(dl.DugksError) as e:
        s.step(1, c.dt)
    assert e.value.code == 6
    with pytest.raises(dl.DugksError):
        s.shard_phase(1)
    s.shard_phase(0, c.dt)
    with pytest.raises(dl.DugksError):
        s.shard_phase(0, c.dt)


def test_more_shards_than_rows_is_an_error():
    c = cs.cavity_case(4, 6)   # 6 DV rows
    with pytest.raises(dl.DugksError) as e:
        dl.Solver(c, shard=dl.shard(0, 7))
    assert e.value.code == 1
