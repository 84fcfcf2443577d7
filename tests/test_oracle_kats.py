"""Known-answer tests of the CPU oracle (the reference ships none for this
path, so these pin the restatement's physics and algebra)."""
import math

import numpy as np

import golden_cases
import oracle_bind as ob
from dugks_b200 import case as cs


def _oracle_case(c):
    c.flatten(ob.geometry(c.mesh))
    return c


def test_rest_equilibrium_is_a_fixed_point():
    c = _oracle_case(cs.cavity_case(8, 8, u_lid=0.0, flatten=False))
    o = ob.Oracle(c, threads=2)
    g0, h0 = o.state()
    o.step(10, c.dt)
    g1, h1 = o.state()
    assert np.max(np.abs(g1 - g0)) <= 1e-13 * np.max(g0)
    assert np.max(np.abs(h1 - h0)) <= 1e-13 * np.max(h0)
    m = o.macros()
    assert np.max(np.abs(m["U"])) < 1e-9 and np.max(np.abs(m["T"] - 273.0)) < 1e-9


def test_initial_moments_reproduce_macros():
    # discrete moments of the Maxwellian at the quadrature (fvDVM.C:414-426)
    c = _oracle_case(cs.cavity_case(4, 28, flatten=False))
    rng = np.random.default_rng(20261203)
    rho = c.rho0 * (1 + 0.1 * rng.random(c.n_cells))
    U = np.zeros((c.n_cells, 3))
    U[:, :2] = 60 * (rng.random((c.n_cells, 2)) - 0.5)
    T = 273 + 20 * rng.random(c.n_cells)
    c.rho0, c.U0, c.T0 = rho, U, T
    o = ob.Oracle(c, threads=2)
    g, h = o.state()
    xi, w = c.dv_set()
    r = (w[:, None] * g).sum(0)
    ru = (w[:, None, None] * g[:, :, None] * xi[:, None, :]).sum(0)
    e = 0.5 * (w[:, None] * (g * (xi ** 2).sum(1)[:, None] + h)).sum(0)
    Um = ru / r[:, None]
    Tm = (e - 0.5 * r * (Um ** 2).sum(1)) / (1.5 * c.gas["R"] * r)
    assert np.max(np.abs(r / rho - 1)) < 1e-13
    assert np.max(np.abs(Um - U)) < 1e-10
    assert np.max(np.abs(Tm / T - 1)) < 1e-12


def test_least_squares_gradient_exact_for_linear_fields():
    # stock leastSquares reproduces a linear field exactly where every
    # neighbour difference is a true difference; at boundary cells the
    # zero patch difference (fixedGradient, zero gradient) enters the fit
    c = _oracle_case(cs.cube_case(5, 6, flatten=False))
    o = ob.Oracle(c, threads=1)
    p, n, b = o.ls_vectors()
    fl = c.flat
    C = fl["C"]
    a = np.array([0.3, -1.7, 2.2])
    phi = C @ a
    nIF = fl["n_internal"]
    own, nei = fl["owner"][:nIF], fl["neighbour"]
    G = np.zeros((c.n_cells, 3))
    dphi = phi[nei] - phi[own]
    np.add.at(G, own, p * dphi[:, None])
    np.add.at(G, nei, -n * dphi[:, None])
    interior = np.ones(c.n_cells, bool)
    interior[fl["owner"][nIF:]] = False
    assert np.max(np.abs(G[interior] - a)) < 1e-10
    # with the boundary faces' own difference (phi(Cf) - phi(C)) the fit is exact everywhere
    d = np.zeros(fl["n_boundary"])
    nrm = fl["Sf"][nIF:] / np.linalg.norm(fl["Sf"][nIF:], axis=1)[:, None]
    delta = nrm * np.einsum("ij,ij->i", nrm, fl["Cf"][nIF:] - C[fl["owner"][nIF:]])[:, None]
    d = delta @ a
    np.add.at(G, fl["owner"][nIF:], b * d[:, None])
    assert np.max(np.abs(G - a)) < 1e-10


def test_least_squares_2d_zero_z_gradient():
    c = _oracle_case(cs.cavity_case(5, 6, flatten=False))
    o = ob.Oracle(c, threads=1)
    p, n, b = o.ls_vectors()
    # cell-centre z from the pyramid sums differs between cells by rounding
    # only, so the z components are round-off against the in-plane ones
    for v in (p, n, b):
        assert np.max(np.abs(v[:, 2])) < 1e-12 * np.max(np.abs(v[:, :2]))


def test_wall_density_balances_outgoing_flux_first_step():
    # at rest, rho_w reproduces the cell density at the wall to quadrature accuracy
    c = _oracle_case(cs.cavity_case(6, 16, u_lid=0.0, flatten=False))
    o = ob.Oracle(c, threads=2)
    o.evolution(c.dt)
    rw = o.boundary_rho()
    assert np.max(np.abs(rw / c.rho0[0] - 1)) < 1e-12
    # inComingByRho = sqrt(R T / (2 pi)) |S| for a Maxwellian at rest
    ib = o.in_coming_by_rho()
    magS = np.linalg.norm(c.flat["Sf"][c.flat["n_internal"]:], axis=1)
    expect = math.sqrt(c.gas["R"] * 273.0 / (2 * math.pi)) * magS
    assert np.max(np.abs(ib / expect - 1)) < 1e-10


def test_lid_driven_flow_direction():
    c = _oracle_case(cs.cavity_case(8, 8, flatten=False))
    o = ob.Oracle(c, threads=2)
    o.step(30, c.dt)
    m = o.macros()
    C = c.flat["C"]
    top = C[:, 1] > 0.85
    assert m["U"][top, 0].mean() > 1.0        # dragged by the lid
    assert np.all(np.isfinite(m["q"])) and np.all(m["T"] > 200)


def test_demo_cavity_runs_in_oracle():
    c = golden_cases.demo_cavity(flatten=False)
    c.flatten(ob.geometry(c.mesh))
    o = ob.Oracle(c)
    o.evolution(c.dt)
    m = o.macros()
    assert np.all(np.isfinite(m["rho"])) and abs(np.mean(m["rho"]) / 1.14423514927e-06 - 1) < 1e-3
