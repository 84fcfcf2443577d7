"""Known answers for the oracle's boundary types (zeroGradient, mixed,
symmetryPlane, DVMsymmetry, pressureIn/Out; discreteVelocity::setBCtype,
discreteVelocity.C:188-195, fvDVM.C:866-1027, :1100-1179, :1429-1453,
:1745-1821): a uniform gas at rest in a channel closed by each type stays
uniform and at rest to round-off; a pressure difference drives a flow
along the channel."""
import numpy as np
import pytest

import oracle_bind as ob
from dugks_b200 import case as cs

SIDES = ("inlet", "outlet", "bottom", "top")


def _run(sides, steps=5, rho=None):
    c = cs.channel_case(8, 4, 8, sides=sides, flatten=False)
    if rho is not None:
        c.rho0 = np.full(c.n_cells, rho)
    c.flatten()
    o = ob.Oracle(c, threads=2)
    m0 = o.macros()
    for _ in range(steps):
        o.evolution(c.dt)
    return c, m0, o.macros(), o


def _assert_uniform_rest(m0, m, c_scale=300.0):
    for k in ("rho", "T"):
        assert np.max(np.abs(m[k] - m0[k])) <= 1e-12 * np.max(np.abs(m0[k])), k
    assert np.max(np.abs(m["U"])) <= 1e-12 * c_scale


@pytest.mark.parametrize("kind", ["symmetryPlane", "DVMsymmetry", "zeroGradient"])
def test_closed_channel_keeps_uniform_rest(kind):
    _, m0, m, _ = _run({s: {"kind": kind} for s in SIDES})
    _assert_uniform_rest(m0, m)


def test_mixed_patches_at_the_interior_state_keep_it():
    rho = float(cs.channel_case(8, 4, 8).rho0[0])
    _, m0, m, _ = _run({s: {"kind": "mixed", "rho": rho, "T": 273.0} for s in SIDES})
    _assert_uniform_rest(m0, m)


def test_pressure_patches_at_the_interior_pressure_keep_it():
    # the pressure patches' rho starts at one (pressureInFvPatchField.C:72-75),
    # so the interior density is one as well
    p = 1.0 * cs.R_DEMO * 273.0
    sides = {"inlet": {"kind": "pressureIn", "p": p, "T": 273.0}, "outlet": {"kind": "pressureOut", "p": p, "T": 273.0}}
    _, m0, m, o = _run(sides, rho=1.0)
    _assert_uniform_rest(m0, m)
    rho_b = o.boundary_rho()
    c = cs.channel_case(8, 4, 8)
    fl = c.flat
    inlet = slice(fl["patch_start"][0], fl["patch_start"][1])
    assert np.allclose(rho_b[inlet], p / cs.R_DEMO / 273.0, rtol=1e-14)


def test_pressure_difference_drives_the_flow_downstream():
    p = 1.0 * cs.R_DEMO * 273.0
    sides = {"inlet": {"kind": "pressureIn", "p": 1.2 * p, "T": 273.0},
             "outlet": {"kind": "pressureOut", "p": p, "T": 273.0}}
    c, _, m, _ = _run(sides, steps=20, rho=1.0)
    assert np.all(np.isfinite(m["rho"])) and np.mean(m["U"][:, 0]) > 1.0
    # more gas near the inlet than near the outlet
    x = c.flat["C"][:, 0]
    assert np.mean(m["rho"][x < 0.5]) > np.mean(m["rho"][x > 1.5])


def test_macro_flux_conserves_mass_in_a_closed_cavity():
    # macroFlux yes: rho advances by face fluxes that cancel between
    # neighbours and vanish through the walls (rho_f U_f . S = 0 there only in
    # the sum over the wall's DVs, which the diffuse wall makes zero)
    c = cs.cavity_case(8, 8)
    o = ob.Oracle(c, threads=2, macro_flux=True)
    V = c.flat["V"]
    m0 = float(np.sum(c.rho0 * V))
    for _ in range(10):
        o.evolution(c.dt)
    m = o.macros()
    assert abs(float(np.sum(m["rho"] * V)) - m0) <= 1e-13 * m0


def test_velocity_mesh_macro_flux_keeps_a_gas_at_rest():
    # the DF-flux branch (fvDVM.C:1562-1611) on a fine velocity mesh
    # symmetric about zero (spacing 150 m/s, +-2400 m/s: its midpoint sums
    # integrate the Maxwellian to round-off): between walls at rest and at
    # the gas temperature, the uniform gas at rest stays put.  (Coarse or
    # jittered velocity meshes do not integrate it exactly, so their rest
    # state is no fixed point.)
    from dugks_b200 import meshgen
    c = cs.channel_case(6, 4, 6, flatten=False)
    c.use_velocity_mesh(meshgen.velocity_box(32, 2400.0, 2))
    c.flatten()
    o = ob.Oracle(c, threads=2, macro_flux=True)
    m0 = o.macros()
    for _ in range(5):
        o.evolution(c.dt)
    m = o.macros()
    assert np.max(np.abs(m["rho"] - m0["rho"])) <= 1e-12 * np.max(m0["rho"])
    assert np.max(np.abs(m["U"])) <= 1e-9
