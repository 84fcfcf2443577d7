"""GPU parity at the benchmark shapes and at the reference's run lengths.

The CUDA path (through the C ABI) and the CPU oracle advance the same case
from the same start for hundreds to a thousand steps; then rho, U, T and q
of the cells and of the faces, the boundary rho and the whole state are
compared by PLAIN relative L2 (no floored denominators: after these runs
every compared field is far from zero), at <= 1e-10.

Cases:
* the 61 x 61 lid-driven cavity with the 28 x 28 Gauss-Hermite set
  (Kn 0.075, lid 50 m/s) for 1000 steps -- the plain-FP64 benchmark
  configuration at its full length;
* the reference's own demo cavity (demo/cavity: its polyMesh face order,
  Xis, weights and 0/ fields) for 250 steps; its controlDict runs 500,000
  steps of deltaT 4e-4 (demo/cavity/system/controlDict:24-26), the
  oracle's cost bounds the length here;
* flow past the sphere on a 6 x 6 x 6 x 6 cubed sphere with the full
  16^3 = 4096-DV Gauss-Hermite set of the ball benchmark, for 24 steps;
* a 32 x 32 cavity with the 32 x 32 DV set of the adjoint configuration
  (Kn 0.1), for 120 steps.

The step is fvDVM::evolution (src/fvDVM/fvDVM/fvDVM.C:2128-2174); the
oracle follows it sub-step by sub-step."""
import numpy as np
import pytest

import golden_cases
import oracle_bind as ob
from dugks_b200 import case as cs
from dugks_b200 import lib as dl

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def _plain(a: dict, b: dict) -> dict:
    return {k: ob.rel_l2(a[k], b[k]) for k in ("rho", "U", "T", "q")}


def _run_long(case, steps, chunk=50):
    gpu = dl.Solver(case)
    orc = ob.Oracle(case)
    done = 0
    while done < steps:
        n = min(chunk, steps - done)
        gpu.step(n, case.dt)
        orc.step(n, case.dt)
        done += n
    cell = _plain(gpu.macros(), orc.macros())
    face = _plain(gpu.face_macros(), orc.face_macros())
    assert max(cell.values()) <= TOL64, f"{case.name} after {steps} steps: cell macros {cell}"
    assert max(face.values()) <= TOL64, f"{case.name} after {steps} steps: face macros {face}"
    assert ob.rel_l2(gpu.boundary_rho(), orc.boundary_rho()) <= TOL64, f"{case.name}: boundary rho"
    gs, hs = gpu.state()
    go, ho = orc.state()
    assert ob.rel_l2(gs, go) <= TOL64 and ob.rel_l2(hs, ho) <= TOL64, f"{case.name}: state"
    # the flow has developed: no compared field is near zero
    m = orc.macros()
    assert np.linalg.norm(m["U"]) > 0 and np.linalg.norm(m["q"]) > 0
    return cell, face


def test_cavity61_dv28_thousand_steps():
    c = cs.cavity_case(61, 28, kn=0.075, u_lid=50.0)
    assert c.n_cells == 3721 and c.n_dv == 784
    _run_long(c, 1000, chunk=100)


def test_demo_cavity_250_steps():
    c = golden_cases.demo_cavity()
    assert c.n_cells == 3600
    _run_long(c, 250)


def test_ball_full_16cubed_dv_set():
    c = cs.ball_case(6, 6, 1.12, 16, kn=0.1, mach=0.5)
    assert c.n_dv == 4096
    _run_long(c, 24, chunk=8)


def test_cavity32_adjoint_dv_set_120_steps():
    c = cs.cavity_case(32, 32, kn=0.1)
    assert c.n_dv == 1024
    _run_long(c, 120, chunk=40)
