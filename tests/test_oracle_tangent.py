"""The dual-number tangent of the oracle (oracle/dugks_tangent.cpp), the CPU
reference the GPU adjoint is checked against: its value part reproduces
the oracle's trajectory and objective, and its derivative matches central
finite differences of the oracle itself."""
import numpy as np
import pytest

import adjoint_cases as ac
import oracle_bind as ob
from dugks_b200 import case as cs

N_STEPS = 6


_objective_weights = ac.objective_weights
_perturbed = ac.perturbed
_cases = ac.cases


def _oracle_J(c, hw, fw, steps=N_STEPS):
    xi, w = c.dv_set()
    o = ob.Oracle(c)
    J = 0.0
    for _ in range(steps):
        o.evolution(c.dt)
        _, _, gb, hb = o.face_values()
        J += ob.boundary_flux_objective(c, xi, w, gb, hb, hw, fw)
    return J / steps, o


@pytest.mark.parametrize("which", ["cavity", "farfield"])
def test_tangent_value_is_the_oracle_trajectory(which):
    c = _cases()[which]
    hw, fw, _ = _objective_weights(c)
    J, o = _oracle_J(c, hw, fw)
    Jt, _, g, h = ob.Oracle(c).tangent(N_STEPS, c.dt, hw, fw)
    assert abs(Jt - J) <= 1e-12 * abs(J)
    gs, hs = o.state()
    assert ob.rel_l2(g, gs) <= 1e-13 and ob.rel_l2(h, hs) <= 1e-13


@pytest.mark.parametrize("which", ["cavity", "farfield"])
def test_tangent_matches_central_differences(which):
    c = _cases()[which]
    hw, fw, first = _objective_weights(c)
    nb = c.flat["n_boundary"]
    rng = np.random.default_rng(7)
    dirs = [{"dT_b": rng.uniform(-1.0, 1.0, nb)},
            {"dU_b": np.where(first[:, None], [1.0, 0.0, 0.0], 0.0)},
            {"d_mu": c.gas["muRef"]}]
    o = ob.Oracle(c)
    for d in dirs:
        _, dJ, _, _ = o.tangent(N_STEPS, c.dt, hw, fw, **d)
        eps = 1e-4
        fd = (_oracle_J(_perturbed(c, eps, **d), hw, fw)[0] - _oracle_J(_perturbed(c, -eps, **d), hw, fw)[0]) / (2 * eps)
        assert abs(fd - dJ) <= 1e-6 * abs(dJ), (d.keys(), fd, dJ)


def test_tangent_refuses_other_patch_types():
    c = cs.channel_case(6, 3, 6, sides={"outlet": {"kind": "zeroGradient"}})
    with pytest.raises(ValueError):
        ob.Oracle(c).tangent(2, c.dt, np.ones(c.flat["n_boundary"]))
