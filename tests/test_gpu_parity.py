"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on
the same seeded inputs.

Tolerances: the FP64 path must match the oracle to <= 1e-10 relative L2 in
rho, U, T and q (cell and face macros), the boundary rho and the whole
state -- the bar the reference sets for the plain path.  U and q errors are
taken against max(|field|, 1e-4 x its natural scale) (oracle_bind.
macro_errors): both paths sum DVs in different orders, and where a moment
cancels to near zero the results are rounding noise of the sum.  The FP32c
path is compared with the FP64 oracle at <= 5e-6 over these short runs
(its q sits at the FP32 noise floor of the floored scale there); its
long-run error is measured on the full workload by bench.py."""
import numpy as np
import pytest

import golden_cases
import oracle_bind as ob
from dugks_b200 import case as cs
from dugks_b200 import lib as dl
from dugks_b200 import quadrature

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 5e-6


def _pair(case, **kw):
    return dl.Solver(case, **kw), ob.Oracle(case)


def _run(case, steps, tol=TOL64, check_faces=True, floor=1e-4, **kw):
    gpu, orc = _pair(case, **kw)
    for _ in range(steps):
        gpu.evolution(case.dt)
        orc.evolution(case.dt)
    R = case.gas["R"]
    errs = ob.macro_errors(gpu.macros(), orc.macros(), R, floor)
    assert max(errs.values()) <= tol, f"{case.name}: cell macros {errs}"
    if check_faces:
        ferrs = ob.macro_errors(gpu.face_macros(), orc.face_macros(), R)
        assert max(ferrs.values()) <= tol, f"{case.name}: face macros {ferrs}"
        assert ob.rel_l2(gpu.boundary_rho(), orc.boundary_rho()) <= tol, f"{case.name}: boundary rho"
        gs, hs = gpu.state()
        go, ho = orc.state()
        assert ob.rel_l2(gs, go) <= tol and ob.rel_l2(hs, ho) <= tol, f"{case.name}: state"
    return gpu, orc


def test_cavity_one_step_face_and_cell_macros():
    c = cs.cavity_case(8, 8)
    _run(c, 1)


def test_cavity_fp64_20_steps():
    c = cs.cavity_case(8, 8)
    gpu, orc = _run(c, 20)
    co_g, co_o = gpu.get_co_num(c.dt), orc.get_co_num(c.dt)
    assert abs(co_g[0] - co_o[0]) <= 1e-12 * co_o[0]
    assert abs(co_g[1] - co_o[1]) <= 1e-10 * co_o[1]


def test_cavity_small_tiles_many_chunks():
    # tile-boundary faces (XB hand-over) and DV-chunk partial sums everywhere
    c = cs.cavity_case(12, 10)
    _run(c, 8, tile_cells=7, dv_chunks=9)


def test_cavity_newton_cotes_parallel_faces():
    # odd Newton-Cotes rule: xi components of exactly zero make xi.S == 0 on
    # Cartesian faces, exercising the averaged reconstruction (fvDVM.C:847-863)
    c = cs.cavity_case(9, 8, flatten=False)
    xis, w = quadrature.newton_cotes(1600.0, 9)
    c.xis, c.weights, c.xi_max = xis, w, 1600.0
    c.flatten()
    _run(c, 6, tile_cells=11, dv_chunks=3)


@pytest.mark.parametrize("tile_cells,dv_chunks", [(0, 0), (16, 3)])
def test_refined_cavity_octagon_cells(tile_cells, dv_chunks):
    # 2:1 refined squares beside octagons with eight internal faces (ten in
    # all): more neighbours than the gradient stencil and more faces than the
    # flux list hold in registers, so the passes take their general paths
    c = cs.refined_cavity_case(8, 8)
    _run(c, 20, tile_cells=tile_cells, dv_chunks=dv_chunks)
    _run(c, 8, tol=TOL32, check_faces=False, floor=1e-2, precision=dl.FP32C, tile_cells=tile_cells,
         dv_chunks=dv_chunks)


def _uniform_dvs(c, n, xi_max):
    """n uniform nodes per dimension on [-xi_max, xi_max], trapezoid weights."""
    x = np.linspace(-xi_max, xi_max, n)
    w = np.full(n, x[1] - x[0])
    w[0] = w[-1] = 0.5 * w[0]
    c.xis, c.weights, c.xi_max = x, w, xi_max
    return c.flatten()


@pytest.mark.parametrize("which", ["cavity", "cube"])
def test_largest_dv_rows(which):
    # 64 nodes per dimension, the most the passes' DV tables hold: 4,096 DVs
    # on a 4 x 4 cavity, 262,144 on a 3^3 cube (g only there)
    if which == "cavity":
        c = _uniform_dvs(cs.cavity_case(4, 8, flatten=False), 64, 2400.0)
        _run(c, 6)
        _run(c, 6, tol=TOL32, check_faces=False, floor=1e-2, precision=dl.FP32C)
    else:
        _run(_uniform_dvs(cs.cube_case(3, 8, flatten=False), 64, 2400.0), 3)


def test_cube_fp64_multi_tile():
    c = cs.cube_case(6, 6, kn=0.1)
    _run(c, 6, tile_cells=16, dv_chunks=2)


def test_ball_far_field_fp64():
    # cubed sphere: non-orthogonal faces, far field + wall, faces on the cube
    # diagonals where xi.S is tangential up to rounding
    c = cs.ball_case(4, 4, 1.12, 8, kn=0.1, mach=0.5)
    _run(c, 10)


def test_ball_far_field_small_tiles():
    c = cs.ball_case(4, 4, 1.12, 8, kn=0.1, mach=0.5)
    _run(c, 6, tile_cells=32, dv_chunks=3)


def test_demo_cavity_mesh_fp64():
    # the reference demo's own polyMesh (blockMesh face order, which the
    # boundary h relaxation's internal-face index depends on), quadrature and fields
    c = golden_cases.demo_cavity()
    _run(c, 3)


# FP32 storage: the noise floor of the U and q sums is FP32 rounding, so
# their denominators are floored at 1e-2 of the natural scale (~1e-8 of it
# in absolute terms, a fraction of an FP32 ulp of the sums)
def test_fp32c_cavity():
    c = cs.cavity_case(8, 8)
    _run(c, 20, tol=TOL32, check_faces=False, floor=1e-2, precision=dl.FP32C)


def test_fp32c_ball():
    c = cs.ball_case(4, 4, 1.12, 8, kn=0.1, mach=0.5)
    _run(c, 6, tol=TOL32, check_faces=False, floor=1e-2, precision=dl.FP32C)


@pytest.mark.parametrize("steps", [200])
def test_fp32c_long_run_within_1e6_of_fp64(steps):
    # FP32 storage with the equilibrium and the relaxation in FP64: after
    # hundreds of steps rho, U and T stay within 1e-6 (plain relative L2)
    # of the FP64 path on a far-field flow past a sphere.  q is a small
    # difference of large velocity moments of the FP32 state; on this
    # coarse mesh it is compared against max(|q|, 1e-2 rho (RT)^1.5)
    c = cs.ball_case(6, 6, 1.12, 8, kn=0.1, mach=0.5)
    f64, f32 = dl.Solver(c), dl.Solver(c, precision=dl.FP32C)
    f64.step(steps, c.dt)
    f32.step(steps, c.dt)
    a, b = f32.macros(), f64.macros()
    for k in ("rho", "U", "T"):
        err = float(np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k]))
        assert err <= 1e-6, (k, err)
    errs = ob.macro_errors(a, b, c.gas["R"], floor=1e-2)
    assert errs["q"] <= 1e-6, errs


def test_fp32c_cube_thousand_steps_within_1e6_of_fp64():
    """The FP32 state is stored as deviations from a per-DV reference
    Maxwellian, so rounding does not accumulate into the small moments: on
    a lid-driven cube (8^3 cells, 8^3 DVs, Kn 0.1) after 1000 steps rho, U,
    T and q all stay within 1e-6 (plain relative L2) of the FP64 path."""
    c = cs.cube_case(8, 8, kn=0.1)
    f64, f32 = dl.Solver(c), dl.Solver(c, precision=dl.FP32C)
    f64.step(1000, c.dt)
    f32.step(1000, c.dt)
    a, b = f32.macros(), f64.macros()
    for k in ("rho", "U", "T", "q"):
        err = float(np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k]))
        assert err <= 1e-6, (k, err)
    # the state read back through the C ABI carries the reference: g = stored + ref
    ga, _ = f32.state()
    gb, _ = f64.state()
    assert float(np.linalg.norm(ga - gb) / np.linalg.norm(gb)) <= 1e-6


def test_state_restart_is_exact():
    # the DFs alone give the macros to rounding (another summation order);
    # with the step record the run continues bit for bit, adaptive steps too
    c = cs.cavity_case(8, 8)
    a = dl.Solver(c)
    a.step(5, c.dt)
    g, h = a.state()
    rec = a.step_record()
    b = dl.Solver(c)
    b.set_state(g, h, c.dt)
    errs = ob.macro_errors(b.macros(), a.macros(), c.gas["R"])
    assert max(errs.values()) <= 1e-13, errs
    b.set_state(g, h, c.dt, rec)
    assert np.array_equal(b.step_record(), rec)
    a.step(3, c.dt)
    b.step(3, c.dt)
    da, ha = a.step_adaptive(3, c.dt, 0.5)
    db, hb = b.step_adaptive(3, c.dt, 0.5)
    assert da == db and np.array_equal(ha, hb)
    ga, _ = a.state()
    gb, _ = b.state()
    assert np.array_equal(ga, gb)
    bad = rec.copy()
    bad[0] = -1.0
    with pytest.raises(dl.DugksError):
        b.set_state(g, h, c.dt, bad)


def test_df_output_matches_state():
    c = cs.cavity_case(6, 6)
    s = dl.Solver(c)
    s.step(2, c.dt)
    g, h = s.state()
    cells = np.array([0, 7, 35], dtype=np.int32)
    gd, hd = s.df(cells)
    assert np.array_equal(gd, g[:, cells].T) and np.array_equal(hd, h[:, cells].T)


def test_multi_step_call_equals_single_steps():
    # dugks_step(n) precomputes the next step's relax factors; the result
    # must equal n separate calls
    c = cs.cavity_case(8, 8)
    a, b = dl.Solver(c), dl.Solver(c)
    a.step(7, c.dt)
    for _ in range(7):
        b.step(1, c.dt)
    ga, _ = a.state()
    gb, _ = b.state()
    assert np.array_equal(ga, gb)


def _oracle_adaptive(orc, n, dt, max_co, max_dt):
    """The reference's time loop with adjustTimeStep on (src/dugksFoam.C:63-75:
    CourantNo.H, setDeltaTvar.H:34-48 with SMALL = 1e-15, then evolution)."""
    hist = []
    for _ in range(n):
        co = orc.get_co_num(dt)[0]
        F = max_co / (co + 1e-15)
        f = min(min(F, 1.0 + 0.1 * F), 1.2)
        dt = min(f * dt, max_dt)
        hist.append(dt)
        orc.evolution(dt)
    return dt, np.array(hist)


@pytest.mark.parametrize("max_dt", [1e300, None])
def test_adaptive_time_step_matches_oracle(max_dt):
    # the case's dt sits at Co 0.5; starting from a quarter of it, the step
    # grows by 1.2 per step until the Courant limit (or maxDeltaT) holds it
    c = cs.cavity_case(8, 8)
    dt0 = 0.25 * c.dt
    if max_dt is None:
        max_dt = 0.5 * c.dt
    gpu, orc = _pair(c)
    dg, hg = gpu.step_adaptive(16, dt0, 0.5, max_dt)
    do, ho = _oracle_adaptive(orc, 16, dt0, 0.5, max_dt)
    assert np.max(np.abs(hg - ho) / ho) <= 1e-12, (hg, ho)
    assert dg == hg[-1]
    errs = ob.macro_errors(gpu.macros(), orc.macros(), c.gas["R"])
    assert max(errs.values()) <= TOL64, errs
    if max_dt < 1e300:
        assert np.max(hg) == max_dt


def test_adaptive_time_step_ball_far_field():
    c = cs.ball_case(6, 6, 1.12, 8)
    gpu, orc = _pair(c)
    _, hg = gpu.step_adaptive(8, c.dt, 0.4)
    _, ho = _oracle_adaptive(orc, 8, c.dt, 0.4, 1e300)
    assert np.max(np.abs(hg - ho) / ho) <= 1e-12, (hg, ho)
    errs = ob.macro_errors(gpu.macros(), orc.macros(), c.gas["R"])
    assert max(errs.values()) <= TOL64, errs


def test_adaptive_calls_chain_exactly():
    # one call of n adaptive steps equals n calls of one step, and a fixed
    # step after an adaptive call rebuilds its relax factors
    c = cs.cavity_case(8, 8)
    a, b = dl.Solver(c), dl.Solver(c)
    da, ha = a.step_adaptive(6, c.dt, 0.5)
    db, hb = c.dt, []
    for _ in range(6):
        db, h1 = b.step_adaptive(1, db, 0.5)
        hb.append(h1[0])
    assert da == db and np.array_equal(ha, np.array(hb))
    ga, _ = a.state()
    gb, _ = b.state()
    assert np.array_equal(ga, gb)
    orc = ob.Oracle(c)
    _oracle_adaptive(orc, 6, c.dt, 0.5, 1e300)
    a.step(2, 0.7 * da)
    orc.evolution(0.7 * da)
    orc.evolution(0.7 * da)
    errs = ob.macro_errors(a.macros(), orc.macros(), c.gas["R"])
    assert max(errs.values()) <= TOL64, errs


def test_errors_are_reported_not_fatal():
    c = cs.cavity_case(4, 6)
    s = dl.Solver(c)
    with pytest.raises(dl.DugksError):
        s.step(1, -1.0)
    with pytest.raises(dl.DugksError):
        s.df(np.array([10 ** 6], dtype=np.int32))
    s.step(1, c.dt)  # still usable


def test_fp32c_rows_not_whole_batches():
    # 6 nodes per dimension: DV rows do not split into whole 8-DV batches
    # (the guarded passes; with FP32 storage pass A double-buffers gbar+)
    c = cs.cube_case(6, 6, kn=0.1)
    f64, f32 = dl.Solver(c), dl.Solver(c, precision=dl.FP32C)
    f64.step(30, c.dt)
    f32.step(30, c.dt)
    a, b = f32.macros(), f64.macros()
    for k in ("rho", "U", "T"):
        err = float(np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k]))
        assert err <= 1e-6, (k, err)
    errs = ob.macro_errors(a, b, c.gas["R"], floor=1e-2)
    assert errs["q"] <= 5e-6, errs
