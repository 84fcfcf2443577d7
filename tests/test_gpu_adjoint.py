"""The GPU adjoint (dugks_adjoint_run) against the oracle's dual-number
tangent and against central finite differences of the GPU's own objective:
the gradient with respect to the boundary-face T and U patch values and
muRef of the time-averaged wall heat flux + lid shear objective."""
import numpy as np
import pytest

import adjoint_cases as ac
import oracle_bind as ob
from dugks_b200 import case as cs
from dugks_b200 import lib as dl
from dugks_b200 import meshgen

pytestmark = pytest.mark.gpu

N_STEPS = 6


def _directions(c, first, seed=7):
    nb = c.flat["n_boundary"]
    rng = np.random.default_rng(seed)
    return [{"dT_b": rng.uniform(-1.0, 1.0, nb)},
            {"dU_b": np.where(first[:, None], [1.0, 0.0, 0.0], 0.0)},
            {"d_mu": c.gas["muRef"]},
            {"dU_b": rng.uniform(-1.0, 1.0, (nb, 3)), "dT_b": rng.uniform(-1.0, 1.0, nb)}]


def _project(r, d):
    a = 0.0
    if "dT_b" in d:
        a += float(r["dT_b"] @ d["dT_b"])
    if "dU_b" in d:
        a += float(np.sum(r["dU_b"] * d["dU_b"]))
    if "d_mu" in d:
        a += r["dmu"] * d["d_mu"]
    return a


@pytest.mark.parametrize("which", ["cavity", "farfield"])
@pytest.mark.parametrize("snapshots", [64, 2])
def test_adjoint_matches_oracle_tangent(which, snapshots):
    """Every directional derivative of the tangent equals the adjoint
    gradient projected on that direction (FP64, 1e-9 relative), with and
    without recomputation between checkpoints."""
    c = ac.cases()[which]
    hw, fw, first = ac.objective_weights(c)
    s = dl.Solver(c)
    r = s.adjoint(N_STEPS, c.dt, hw, fw, max_snapshots=snapshots)
    Jt, _, _, _ = ob.Oracle(c).tangent(N_STEPS, c.dt, hw, fw)
    assert abs(r["J"] - Jt) <= 1e-10 * abs(Jt)
    assert r["stats"]["reverse_steps"] == N_STEPS
    if snapshots >= N_STEPS:
        assert r["stats"]["forward_steps"] == N_STEPS - 1
    else:
        assert r["stats"]["forward_steps"] > N_STEPS - 1
    for d in _directions(c, first):
        _, dJ, _, _ = ob.Oracle(c).tangent(N_STEPS, c.dt, hw, fw, **d)
        if dJ == 0.0:
            assert abs(_project(r, d)) <= 1e-14
            continue
        assert abs(_project(r, d) - dJ) <= 1e-9 * abs(dJ), (which, d.keys(), _project(r, d), dJ)


def _vmesh_cavity():
    c = cs.cavity_case(8, 8, flatten=False)
    c.use_velocity_mesh(meshgen.velocity_box(10, 1600.0, 2, jitter=0.2))
    return c.flatten()


@pytest.mark.parametrize("which", ["ball3d", "vmesh", "refined"])
def test_adjoint_matches_tangent_in_3d_and_on_a_velocity_mesh(which):
    """The 3-D far-field ball (cubed sphere 6x4x4x4, 6^3 DVs; objective: energy
    flux through every face, drag through the sphere), a cavity on a
    jittered unstructured velocity mesh (100 DVs) and a 2:1 refined cavity
    whose octagon cells have eight internal faces (more than the reverse
    keeps in registers): tangent = projected adjoint to 1e-9."""
    if which == "ball3d":
        c = cs.ball_case(4, 4, 1.12, 6, kn=0.1, mach=0.5)
    elif which == "vmesh":
        c = _vmesh_cavity()
    else:
        c = cs.refined_cavity_case(6, 8, kn=0.1)
    hw, fw, _ = ac.objective_weights(c)
    r = dl.Solver(c, tile_cells=32).adjoint(4, c.dt, hw, fw, max_snapshots=2)
    Jt, _, _, _ = ob.Oracle(c).tangent(4, c.dt, hw, fw)
    assert abs(r["J"] - Jt) <= 1e-10 * abs(Jt)
    nb = c.flat["n_boundary"]
    rng = np.random.default_rng(3)
    for d in ({"dT_b": rng.uniform(-1.0, 1.0, nb)}, {"dU_b": rng.uniform(-1.0, 1.0, (nb, 3))},
              {"d_mu": c.gas["muRef"]}):
        _, dJ, _, _ = ob.Oracle(c).tangent(4, c.dt, hw, fw, **d)
        assert abs(_project(r, d) - dJ) <= 1e-9 * abs(dJ), (which, d.keys(), _project(r, d), dJ)


def test_adjoint_leaves_the_state_and_repeats_bitwise():
    c = ac.cases()["cavity"]
    hw, fw, _ = ac.objective_weights(c)
    s = dl.Solver(c)
    s.step(3, c.dt)
    g0, h0 = s.state()
    r1 = s.adjoint(5, c.dt, hw, fw, max_snapshots=2)
    g1, h1 = s.state()
    assert np.array_equal(g0, g1) and np.array_equal(h0, h1)
    r2 = s.adjoint(5, c.dt, hw, fw, max_snapshots=2)
    assert r1["J"] == r2["J"] and r1["dmu"] == r2["dmu"]
    assert np.array_equal(r1["dT_b"], r2["dT_b"]) and np.array_equal(r1["dU_b"], r2["dU_b"])
    # the solver steps on from its state as if no adjoint had run
    ref = dl.Solver(c)
    ref.step(4, c.dt)
    s.step(1, c.dt)
    gr, hr = ref.state()
    gs, hs = s.state()
    assert np.array_equal(gr, gs) and np.array_equal(hr, hs)


def _gpu_J(c, hw, fw, n, window):
    return dl.Solver(c).objective(n, c.dt, hw, fw, window_start=window)[0]


def test_objective_run_is_the_adjoint_objective():
    """dugks_objective_run (forward only) gives the adjoint run's J and
    advances the solver as dugks_step does."""
    c = ac.cases()["farfield"]
    hw, fw, _ = ac.objective_weights(c)
    s = dl.Solver(c)
    r = s.adjoint(7, c.dt, hw, fw, window_start=3, max_snapshots=3)
    J, _ = s.objective(7, c.dt, hw, fw, window_start=3)
    assert abs(J - r["J"]) <= 1e-12 * abs(J)
    ref = dl.Solver(c)
    ref.step(7, c.dt)
    g1, _ = s.state()
    g2, _ = ref.state()
    assert np.array_equal(g1, g2)


def test_adjoint_matches_central_differences_with_window():
    """A 16x16 cavity with 8x8 DVs, 40 steps, the objective averaged over
    the last 10, 3 checkpoints: the adjoint gradient against central
    differences (h = 1e-6 relative) of the GPU objective along the lid speed,
    Kn (muRef) and a random wall-temperature direction, within 1e-5."""
    c = cs.cavity_case(16, 8, kn=0.1)
    hw, fw, first = ac.objective_weights(c)
    n, window = 40, 30
    r = dl.Solver(c).adjoint(n, c.dt, hw, fw, window_start=window, max_snapshots=3)
    assert r["stats"]["snapshots"] == 3
    rng = np.random.default_rng(11)
    nb = c.flat["n_boundary"]
    dirs = [({"dU_b": np.where(first[:, None], [50.0, 0.0, 0.0], 0.0)}),
            ({"d_mu": c.gas["muRef"]}),
            ({"dT_b": 273.0 * rng.uniform(-1.0, 1.0, nb)})]
    for d in dirs:
        eps = 1e-6
        fd = (_gpu_J(ac.perturbed(c, eps, **d), hw, fw, n, window) -
              _gpu_J(ac.perturbed(c, -eps, **d), hw, fw, n, window)) / (2 * eps)
        a = _project(r, d)
        assert abs(a - fd) <= 1e-5 * abs(a), (d.keys(), a, fd)


@pytest.mark.parametrize("which", ["cavity", "farfield"])
def test_boundary_fluxes_match_the_oracle_step(which):
    """dugks_boundary_fluxes after 3 steps gives the 4th step's per-face
    fluxes: their energy and momentum sums equal the oracle's boundary-flux
    objective of its 4th step's relaxed DFs (1e-10), and the state does not
    advance."""
    c = ac.cases()[which]
    hw, fw, first = ac.objective_weights(c)
    s = dl.Solver(c)
    s.step(3, c.dt)
    g0, _ = s.state()
    F = s.boundary_fluxes(c.dt)
    g1, _ = s.state()
    assert np.array_equal(g0, g1)
    o = ob.Oracle(c)
    o.step(4, c.dt)
    xi, w = c.dv_set()
    _, _, gb, hb = o.face_values()
    nb = c.flat["n_boundary"]
    e_ref = ob.boundary_flux_objective(c, xi, w, gb, hb, np.ones(nb), np.zeros((nb, 3)))
    m_ref = ob.boundary_flux_objective(c, xi, w, gb, hb, np.zeros(nb), fw)
    assert abs(F[:, 4].sum() - e_ref) <= 1e-10 * abs(e_ref)
    assert abs(F[first, 1].sum() - m_ref) <= 1e-10 * abs(m_ref)
    # the same step through dugks_objective_run
    J, _ = s.objective(1, c.dt, np.ones(nb), None)
    assert abs(J - F[:, 4].sum()) <= 1e-12 * abs(J)


def test_adjoint_refuses_unsupported_cases():
    c = cs.cavity_case(6, 6)
    s = dl.Solver(c, precision=dl.FP32C)
    with pytest.raises(dl.DugksError) as e:
        s.adjoint(2, c.dt, np.ones(c.flat["n_boundary"]))
    assert e.value.code == 7
    ch = cs.channel_case(6, 3, 6, sides={"outlet": {"kind": "zeroGradient"}})
    s = dl.Solver(ch)
    with pytest.raises(dl.DugksError) as e:
        s.adjoint(2, ch.dt, np.ones(ch.flat["n_boundary"]))
    assert e.value.code == 7
    s = dl.Solver(c)
    for bad in ({"n_steps": 0}, {"window_start": 2}, {"max_snapshots": 0}):
        kw = {"n_steps": 2, "window_start": 0, "max_snapshots": 4}
        kw.update(bad)
        with pytest.raises(dl.DugksError) as e:
            s.adjoint(kw["n_steps"], c.dt, None, None, window_start=kw["window_start"],
                      max_snapshots=kw["max_snapshots"])
        assert e.value.code == 1
