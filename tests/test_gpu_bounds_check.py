"""The bounds-checked build (libdugks_b200_check.so, -DDUGKS_CHECK) on small
cases.

Every index the kernels read from a device table (tile cells, gradient
stencils, item sides, flux lists, boundary owners, the items of a face) is
range-checked there; one out of range would set an error flag, be replaced
by a safe index and make the call return DUGKS_ERR_ARG.  On these cases no
check may fire, and the checked build must give what the normal build gives
(the checks only read; the results agree to an ulp, as the compiler may
contract multiply-adds differently around the checks).  Nothing here plants a bad index on the
device: the host validates the mesh before building the tables
(tests/test_failures.py)."""
import os

import numpy as np
import pytest

import golden_cases
from dugks_b200 import case as cs
from dugks_b200 import lib as dl
from dugks_b200 import meshgen

pytestmark = pytest.mark.gpu


def _same(case, steps, **kw):
    assert os.path.exists(dl.CHECK_LIB_PATH), "build the checked library (make -C psp-vst_b200/csrc)"
    a = dl.Solver(case, **kw)
    b = dl.Solver(case, lib_path=dl.CHECK_LIB_PATH, **kw)
    a.step(steps, case.dt)
    b.step(steps, case.dt)   # raises DugksError if a check fired
    # The checks change the compiled code around them, so the compiler may
    # contract a multiply-add differently in the two builds: equal to an ulp
    # or so of the largest entry, not bit for bit.
    ma, mb = a.macros(), b.macros()
    for k in ("rho", "U", "T", "q"):
        np.testing.assert_allclose(mb[k], ma[k], rtol=1e-13, atol=1e-15 * max(np.abs(ma[k]).max(), 1e-300),
                                   err_msg=k)
    for xa, xb in zip(a.state(), b.state()):
        np.testing.assert_allclose(xb, xa, rtol=1e-13, atol=1e-15 * max(np.abs(xa).max(), 1e-300))


def test_checked_cavity8():
    _same(cs.cavity_case(8, 8), 5)


def test_checked_cavity_small_tiles_many_chunks():
    _same(cs.cavity_case(12, 10), 4, tile_cells=7, dv_chunks=9)


def test_checked_ball_far_field():
    _same(cs.ball_case(4, 4, 1.12, 8, kn=0.1, mach=0.5), 3)


def test_checked_refined_cavity():
    # octagon cells: the general stencil and flux-list paths, of the factored
    # passes and of the DV-list passes
    _same(cs.refined_cavity_case(6, 8), 3, tile_cells=12, dv_chunks=2)
    c = cs.refined_cavity_case(6, 8, flatten=False)
    c.use_velocity_mesh(meshgen.velocity_box(8, 1600.0, 2, jitter=0.2))
    _same(c.flatten(), 3, tile_cells=12, dv_chunks=2)


def test_checked_largest_dv_rows():
    # 64 nodes per dimension (2-D and 3-D)
    for c in (cs.cavity_case(4, 8, flatten=False), cs.cube_case(3, 8, flatten=False)):
        x = np.linspace(-2400.0, 2400.0, 64)
        w = np.full(64, x[1] - x[0])
        w[0] = w[-1] = 0.5 * w[0]
        c.xis, c.weights, c.xi_max = x, w, 2400.0
        _same(c.flatten(), 2)


def test_checked_demo_cavity():
    _same(golden_cases.demo_cavity(), 2)


def test_checked_boundary_types_and_fp32c():
    P1 = cs.R_DEMO * 273.0    # pressure of argon at rho 1, T 273
    sides = {"inlet": {"kind": "pressureIn", "p": 1.2 * P1, "T": 273.0},
             "outlet": {"kind": "pressureOut", "p": P1, "T": 273.0},
             "bottom": {"kind": "symmetryPlane"}, "top": {"kind": "zeroGradient"}}
    c = cs.channel_case(12, 6, 8, sides=sides, flatten=False)
    c.rho0 = np.full(c.n_cells, 1.0)
    c.flatten()
    _same(c, 3)
    _same(c, 3, precision=dl.FP32C)


@pytest.mark.parametrize("precision", [dl.FP64, dl.FP32C])
def test_checked_wide_batches(precision):
    # the g-only passes in 16-DV (16 nodes per dimension) and 10-DV (20
    # nodes) batches
    _same(cs.ball_case(2, 3, 1.12, 16, kn=0.1, mach=0.5), 2, precision=precision)
    _same(cs.cube_case(4, 20, kn=0.1), 2, precision=precision)
