"""GPU parity of the boundary types beyond maxwellWall and farField
(discreteVelocity::setBCtype, discreteVelocity.C:188-195): zeroGradient,
mixed (rho fixedValue), symmetryPlane, DVMsymmetry, pressureIn and
pressureOut, each against the oracle on a 2-D channel whose other sides
are diffuse walls.  FP64 to 1e-10 (cell and face macros, boundary rho,
state), as the plain path."""
import numpy as np
import pytest

import oracle_bind as ob
from dugks_b200 import case as cs
from dugks_b200 import lib as dl
from dugks_b200 import shard as sh

pytestmark = pytest.mark.gpu

TOL = 1e-10
P1 = 1.0 * cs.R_DEMO * 273.0        # pressure of argon at rho 1, T 273


def _case(sides, rho=None, nx=12, ny=6, n_dv=8, U0=(0.0, 0.0, 0.0)):
    c = cs.channel_case(nx, ny, n_dv, sides=sides, U0=U0, flatten=False)
    if rho is not None:
        c.rho0 = np.full(c.n_cells, rho)
    return c.flatten()


def _parity(c, steps, tol=TOL, **kw):
    gpu, orc = dl.Solver(c, **kw), ob.Oracle(c)
    for _ in range(steps):
        gpu.evolution(c.dt)
        orc.evolution(c.dt)
    R = c.gas["R"]
    errs = ob.macro_errors(gpu.macros(), orc.macros(), R)
    assert max(errs.values()) <= tol, errs
    ferrs = ob.macro_errors(gpu.face_macros(), orc.face_macros(), R)
    assert max(ferrs.values()) <= tol, ferrs
    assert ob.rel_l2(gpu.boundary_rho(), orc.boundary_rho()) <= tol
    gs, hs = gpu.state()
    go, ho = orc.state()
    assert ob.rel_l2(gs, go) <= tol and ob.rel_l2(hs, ho) <= tol
    return gpu, orc


def test_pressure_driven_channel():
    sides = {"inlet": {"kind": "pressureIn", "p": 1.2 * P1, "T": 273.0},
             "outlet": {"kind": "pressureOut", "p": P1, "T": 273.0}}
    gpu, _ = _parity(_case(sides, rho=1.0), 12)
    assert np.mean(gpu.macros()["U"][:, 0]) > 0


def test_mixed_inlet_zero_gradient_outlet():
    rho = float(cs.channel_case(4, 2, 6).rho0[0])
    sides = {"inlet": {"kind": "mixed", "rho": rho, "U": (60.0, 0.0, 0.0), "T": 300.0},
             "outlet": {"kind": "zeroGradient"}}
    _parity(_case(sides), 12)


def test_symmetry_plane_over_a_sheared_layer():
    sides = {"bottom": {"kind": "maxwellWall", "U": (80.0, 0.0, 0.0), "T": 273.0},
             "top": {"kind": "symmetryPlane"}, "inlet": {"kind": "zeroGradient"}, "outlet": {"kind": "zeroGradient"}}
    _parity(_case(sides), 10)


def test_dvm_symmetry_with_far_field_ends():
    rho = float(cs.channel_case(4, 2, 6).rho0[0])
    sides = {"top": {"kind": "DVMsymmetry"},
             "inlet": {"kind": "farField", "rho": rho, "T": 273.0}, "outlet": {"kind": "farField", "rho": rho, "T": 273.0}}
    _parity(_case(sides, U0=(40.0, 0.0, 0.0)), 10)


def test_odd_newton_cotes_set_on_symmetry_planes():
    # a zero node: DVs tangential to the planes mirror into themselves
    from dugks_b200 import quadrature
    c = cs.channel_case(10, 5, 8, sides={"top": {"kind": "symmetryPlane"}, "outlet": {"kind": "DVMsymmetry"},
                                         "bottom": {"kind": "maxwellWall", "U": (50.0, 0.0, 0.0)}},
                        flatten=False)
    c.xis, c.weights = quadrature.newton_cotes(1600.0, 9)
    c.xi_max = 1600.0
    c.flatten()
    _parity(c, 8)


def test_fp32c_boundary_types():
    sides = {"inlet": {"kind": "pressureIn", "p": 1.1 * P1, "T": 273.0},
             "outlet": {"kind": "pressureOut", "p": P1, "T": 273.0}, "top": {"kind": "symmetryPlane"}}
    c = _case(sides, rho=1.0)
    gpu, orc = dl.Solver(c, precision=dl.FP32C), ob.Oracle(c)
    for _ in range(8):
        gpu.evolution(c.dt)
        orc.evolution(c.dt)
    errs = ob.macro_errors(gpu.macros(), orc.macros(), c.gas["R"], floor=1e-2)
    assert max(errs.values()) <= 5e-6, errs


def test_fp32c_mirror_across_the_reference_velocity():
    """FP32 storage holds deviations from the reference Maxwellian of the
    mean state; with the gas moving along x, a DVMsymmetry outlet mirrors x
    and the mirror DV has another reference value, which k_symmetry_in must
    carry over.  FP32c = oracle to 5e-6 after 8 steps."""
    c = cs.channel_case(10, 5, 8, sides={"top": {"kind": "symmetryPlane"}, "outlet": {"kind": "DVMsymmetry"},
                                         "bottom": {"kind": "maxwellWall", "U": (50.0, 0.0, 0.0)}},
                        U0=(60.0, 0.0, 0.0))
    gpu, orc = dl.Solver(c, precision=dl.FP32C), ob.Oracle(c)
    for _ in range(8):
        gpu.evolution(c.dt)
        orc.evolution(c.dt)
    errs = ob.macro_errors(gpu.macros(), orc.macros(), c.gas["R"], floor=1e-2)
    assert max(errs.values()) <= 5e-6, errs


def test_restart_with_pressure_patches_is_exact():
    sides = {"inlet": {"kind": "pressureIn", "p": 1.2 * P1, "T": 273.0},
             "outlet": {"kind": "pressureOut", "p": P1, "T": 273.0}}
    c = _case(sides, rho=1.0)
    a = dl.Solver(c)
    a.step(4, c.dt)
    g, h = a.state()
    rec = a.step_record()
    assert rec.size == 9 * c.n_cells + 2 + 2 * c.flat["n_boundary"]
    b = dl.Solver(c)
    b.set_state(g, h, c.dt, rec)
    a.step(3, c.dt)
    b.step(3, c.dt)
    assert np.array_equal(a.state()[0], b.state()[0])
    assert np.array_equal(a.boundary_rho(), b.boundary_rho())


def test_host_reduced_shards_with_pressure_and_mixed_patches():
    rho = float(cs.channel_case(4, 2, 6).rho0[0])
    sides = {"inlet": {"kind": "mixed", "rho": rho, "U": (60.0, 0.0, 0.0), "T": 300.0},
             "outlet": {"kind": "zeroGradient"}}
    c = _case(sides)
    shards = [dl.Solver(c, shard=dl.shard(r, 2)) for r in range(2)]
    sh.step_local(shards, 6, c.dt)
    orc = ob.Oracle(c)
    for _ in range(6):
        orc.evolution(c.dt)
    errs = ob.macro_errors(shards[1].macros(), orc.macros(), c.gas["R"])
    assert max(errs.values()) <= TOL, errs


def test_symmetry_needs_the_whole_dv_set_and_an_axis_plane():
    c = _case({"top": {"kind": "symmetryPlane"}})
    with pytest.raises(dl.DugksError) as e:
        dl.Solver(c, shard=dl.shard(0, 2))
    assert e.value.code == 7
    # the same channel turned by 30 degrees: its planes are oblique
    t = np.radians(30.0)
    rot = np.array([[np.cos(t), -np.sin(t), 0.0], [np.sin(t), np.cos(t), 0.0], [0.0, 0.0, 1.0]])
    c2 = cs.channel_case(12, 6, 8, sides={"top": {"kind": "symmetryPlane"}}, flatten=False)
    c2.mesh.points = c2.mesh.points @ rot.T
    c2.flatten()
    with pytest.raises(dl.DugksError) as e:
        dl.Solver(c2)
    assert e.value.code == 7


# macroFlux yes (fvDVM.C:1613-1679): cell rho, rho U, rho E from the face
# macro fluxes; the oracle restates the same branch
@pytest.mark.parametrize("which", ["cavity", "ball", "pressure"])
def test_macro_flux_matches_oracle(which):
    if which == "cavity":
        c, steps = cs.cavity_case(8, 8), 10
    elif which == "ball":
        c, steps = cs.ball_case(4, 4, 1.12, 8, kn=0.1, mach=0.5), 8
    else:
        c = _case({"inlet": {"kind": "pressureIn", "p": 1.2 * P1, "T": 273.0},
                   "outlet": {"kind": "pressureOut", "p": P1, "T": 273.0}, "top": {"kind": "symmetryPlane"}}, rho=1.0)
        steps = 10
    gpu, orc = dl.Solver(c, macro_flux=True), ob.Oracle(c, macro_flux=True)
    for _ in range(steps):
        gpu.evolution(c.dt)
        orc.evolution(c.dt)
    errs = ob.macro_errors(gpu.macros(), orc.macros(), c.gas["R"])
    assert max(errs.values()) <= TOL, errs
    gs, _ = gpu.state()
    go, _ = orc.state()
    assert ob.rel_l2(gs, go) <= TOL
    # the flux update differs from the moments of the DFs
    plain = dl.Solver(c)
    plain.step(steps, c.dt)
    assert not np.array_equal(plain.macros()["rho"], gpu.macros()["rho"])
