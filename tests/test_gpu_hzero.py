"""h identically zero in 3-D with KInner = 0.

With D = 3 and KInner = 0 the factor K + 3 - D is zero in every formula
that feeds h: the initial state h = (K+3-D) RT g (fvDVM.C:414-426), the
Shakhov h equilibrium (fvDVM.C:673-679, discreteVelocity.C:997-1007) and the
incoming boundary DFs (fvDVM.C:926-938, :1079-1092).  h then stays exactly
zero, and the tensor-DV passes carry g alone.  These tests check, against
the oracle (which carries h in full):
* the g-only passes keep h exactly zero and match the oracle to 1e-10;
* the full passes in 3-D (KInner = 2, so h is not zero) match it too;
* a state with a nonzero h loaded into a KInner = 0 handle leaves the
  g-only passes, and the run again matches the oracle."""
import numpy as np
import pytest

import oracle_bind as ob
from dugks_b200 import case as cs
from dugks_b200 import lib as dl

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _check(gpu, orc, R):
    errs = ob.macro_errors(gpu.macros(), orc.macros(), R)
    assert max(errs.values()) <= TOL, errs
    ferrs = ob.macro_errors(gpu.face_macros(), orc.face_macros(), R)
    assert max(ferrs.values()) <= TOL, ferrs
    gs, hs = gpu.state()
    go, ho = orc.state()
    assert ob.rel_l2(gs, go) <= TOL
    return hs, ho


def test_g_only_passes_keep_h_zero():
    c = cs.cube_case(6, 6, kn=0.1)
    gpu, orc = dl.Solver(c), ob.Oracle(c)
    gpu.step(8, c.dt)
    orc.step(8, c.dt)
    hs, ho = _check(gpu, orc, c.gas["R"])
    assert not np.any(hs) and not np.any(ho)


def test_internal_dof_3d_full_passes():
    c = cs.cube_case(6, 6, kn=0.1, flatten=False)
    c.gas = dict(c.gas, K=2)
    c.flatten()
    gpu, orc = dl.Solver(c), ob.Oracle(c)
    gpu.step(8, c.dt)
    orc.step(8, c.dt)
    hs, ho = _check(gpu, orc, c.gas["R"])
    assert np.any(hs) and ob.rel_l2(hs, ho) <= TOL


def test_nonzero_h_state_leaves_g_only_passes():
    c = cs.ball_case(4, 4, 1.12, 8, kn=0.1, mach=0.5)
    a, orc = dl.Solver(c), ob.Oracle(c)
    a.step(3, c.dt)
    orc.step(3, c.dt)
    g, h = a.state()
    rec = a.step_record()
    assert not np.any(h)
    h2 = 0.01 * c.gas["R"] * 273.0 * g
    b = dl.Solver(c)
    b.set_state(g, h2, c.dt, rec)
    go, _ = orc.state()
    orc.set_state(go, h2)
    b.step(6, c.dt)
    orc.step(6, c.dt)
    hs, ho = _check(b, orc, c.gas["R"])
    assert np.any(hs) and ob.rel_l2(hs, ho) <= TOL


@pytest.mark.parametrize("precision", [dl.FP64, dl.FP32C])
def test_g_only_passes_twenty_nodes(precision):
    # 20 nodes per dimension (the mixed-precision configuration's DV set):
    # the g-only passes in batches of 10 DVs (FP64) or of a whole row (FP32
    # storage)
    c = cs.cube_case(4, 20, kn=0.1)
    gpu, orc = dl.Solver(c, precision=precision), ob.Oracle(c)
    gpu.step(4, c.dt)
    orc.step(4, c.dt)
    if precision == dl.FP64:
        _check(gpu, orc, c.gas["R"])
    else:
        errs = ob.macro_errors(gpu.macros(), orc.macros(), c.gas["R"], floor=1e-2)
        assert max(errs.values()) <= 5e-6, errs
