"""The dual-number tangent of the oracle (oracle/dugks_tangent.cpp), the CPU
reference the GPU adjoint is checked against: its value part reproduces
the oracle's trajectory and objective, and its derivative matches central
finite differences of the oracle itself."""
import copy

import numpy as np
import pytest

import oracle_bind as ob
from dugks_b200 import case as cs

N_STEPS = 6


def _objective_weights(c):
    """Energy flux through every wall face, x-momentum flux through the
    first patch (the lid of the cavity)."""
    fl = c.flat
    nb = fl["n_boundary"]
    first = np.zeros(nb, bool)
    first[fl["patch_start"][0]:fl["patch_start"][1]] = True
    fw = np.zeros((nb, 3))
    fw[first, 0] = 1.0
    return np.ones(nb), fw, first


def _oracle_J(c, hw, fw, steps=N_STEPS):
    xi, w = c.dv_set()
    o = ob.Oracle(c)
    J = 0.0
    for _ in range(steps):
        o.evolution(c.dt)
        _, _, gb, hb = o.face_values()
        J += ob.boundary_flux_objective(c, xi, w, gb, hb, hw, fw)
    return J / steps, o


def _perturbed(c, eps, dT_b=None, dU_b=None, d_mu=0.0):
    cc = copy.copy(c)
    cc.flat = dict(c.flat)
    cc.gas = dict(c.gas)
    if dT_b is not None:
        cc.flat["T_b"] = c.flat["T_b"] + eps * dT_b
    if dU_b is not None:
        cc.flat["U_b"] = c.flat["U_b"] + eps * np.reshape(dU_b, (-1, 3))
    cc.gas["muRef"] = c.gas["muRef"] + eps * d_mu
    return cc


def _cases():
    ff = {"inlet": {"kind": "farField", "T": 300.0}, "outlet": {"kind": "farField", "T": 273.0}}
    ch = cs.channel_case(8, 4, 8, sides=ff, U0=(40.0, 0.0, 0.0), flatten=False)
    rho = float(ch.rho0[0])
    for p in ch.patches:
        if p.kind == "farField":
            p.rho = rho
    return {"cavity": cs.cavity_case(8, 8, kn=0.1), "farfield": ch.flatten()}


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
