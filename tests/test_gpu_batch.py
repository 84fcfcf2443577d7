"""Batched stepping (dugks_batch_*): independent cases of different sizes,
Knudsen numbers, lid speeds and wall temperatures advance through one CUDA
graph with a branch per case; each must equal the same case stepped alone,
bit for bit, for even and odd step counts, FP64 and FP32c."""
import numpy as np
import pytest

from dugks_b200 import case as cs
from dugks_b200 import lib as dl

pytestmark = pytest.mark.gpu


def _cases():
    specs = [(8, 0.1, 50.0, 273.0), (12, 1.0, 30.0, 300.0), (6, 0.03, 80.0, 260.0), (10, 5.0, 20.0, 330.0)]
    return [cs.cavity_case(n, 6, kn=kn, u_lid=u, T_wall=tw) for n, kn, u, tw in specs]


@pytest.mark.parametrize("precision", [dl.FP64, dl.FP32C])
def test_batch_equals_each_case_alone(precision):
    cases = _cases()
    batched = [dl.Solver(c, precision=precision) for c in cases]
    alone = [dl.Solver(c, precision=precision) for c in cases]
    batch = dl.Batch(batched, [c.dt for c in cases])
    assert batch.graph_kernels() >= 2 * 5 * len(cases)
    batch.step(4)
    batch.step(3)           # odd: one ordinary step per case at the end
    for s, c in zip(alone, cases):
        s.step(7, c.dt)
    for a, b in zip(batched, alone):
        ga, ha = a.state()
        gb, hb = b.state()
        assert np.array_equal(ga, gb) and np.array_equal(ha, hb)
        for k in ("rho", "U", "T", "q"):
            assert np.array_equal(a.macros()[k], b.macros()[k]), k
    # a batched solver keeps working on its own afterwards
    batched[0].step(2, cases[0].dt)
    alone[0].step(2, cases[0].dt)
    assert np.array_equal(batched[0].state()[0], alone[0].state()[0])
    batch.step(2)
    batch.close()


def test_batch_rejects_bad_input():
    c = cs.cavity_case(6, 6)
    s = dl.Solver(c)
    with pytest.raises(dl.DugksError):
        dl.Batch([s, s], [c.dt, c.dt])          # the same handle twice
    with pytest.raises(dl.DugksError):
        dl.Batch([s], [-1.0])
    sh = dl.Solver(c, shard=dl.shard(0, 2))
    with pytest.raises(dl.DugksError):
        dl.Batch([sh], [c.dt])


def test_autotuner_picks_a_measured_candidate_and_keeps_the_result():
    """tune_batch measures every (tile, chunk scale) candidate on the whole
    batch and returns the fastest; solvers built with its choice give the
    oracle-parity result of the default layout (FP64, to 1e-12)."""
    cases = _cases()
    dts = [c.dt for c in cases]
    best, table = dl.tune_batch(cases, dts, precision=dl.FP64, tiles=(0, 16), chunk_scales=(0.5, 1.0),
                                steps=2, warmup=2)
    assert len(table) == 4
    assert best["ms_per_step"] == min(t["ms_per_step"] for t in table)
    tuned = [dl.Solver(c, precision=dl.FP64, **kw) for c, kw in zip(cases, best["solver_kwargs"])]
    for s, kw in zip(tuned, best["solver_kwargs"]):
        assert s.layout()["dv_chunks"] == kw["dv_chunks"]
    default = [dl.Solver(c, precision=dl.FP64) for c in cases]
    b = dl.Batch(tuned, dts)
    b.step(4)
    b.close()
    for s, c in zip(default, cases):
        s.step(4, c.dt)
    for a, d in zip(tuned, default):
        ma, md = a.macros(), d.macros()
        for k in ("rho", "T"):
            assert np.linalg.norm(ma[k] - md[k]) <= 1e-12 * np.linalg.norm(md[k]), k
