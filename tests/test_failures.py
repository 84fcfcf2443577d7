"""Failures are reported, not fatal.

The reference stops on OpenFOAM FatalError or runs on into NaNs
(fieldMPIreducer.C:39-46; fvDVM.C has no state checks).  This library
returns a status instead:
* a bad mesh (CSR addressing out of range, a cell without faces, patch
  starts that do not span the boundary faces, non-positive volumes,
  non-finite geometry) -> DUGKS_ERR_ARG from dugks_create, checked on the
  host before any device work (no GPU needed);
* a non-finite or non-positive rho/T given to dugks_set_macros, or DFs
  given to dugks_set_state whose moments are -> DUGKS_ERR_NAN, and the
  handle stays usable.
Every failure here is made on the host; none faults, traps or hangs a GPU."""
import ctypes as C

import numpy as np
import pytest

from dugks_b200 import case as cs
from dugks_b200 import lib as dl

ERR_ARG, ERR_NAN = 1, 5


def _create(fl, n_cells, dvs=None, **over):
    """dugks_create on the flattened arrays of a case, with some replaced
    (dvs: a 1-D DV set (xis, weights, xi_max) instead of the case's)."""
    lib = dl.load()
    a = {k: np.ascontiguousarray(v) for k, v in fl.items() if isinstance(v, np.ndarray)}
    a.update({k: np.ascontiguousarray(v) for k, v in over.items()})
    mesh = dl.Mesh(n_cells, fl["n_internal"], fl["n_boundary"], 2, dl.ptr(a["owner"], C.c_int64),
                   dl.ptr(a["neighbour"], C.c_int64), dl.ptr(a["C"]), dl.ptr(a["V"]), dl.ptr(a["Cf"]),
                   dl.ptr(a["Sf"]), len(a["patch_type"]), dl.ptr(a["patch_start"], C.c_int32))
    c = cs.cavity_case(4, 6)
    x, w, xmax = dvs if dvs is not None else (c.xis, c.weights, c.xi_max)
    xis, ws = np.ascontiguousarray(x, dtype=np.float64), np.ascontiguousarray(w, dtype=np.float64)
    dv = dl.DVSet(len(xis), dl.ptr(xis), dl.ptr(ws), xmax)
    gas = dl.Gas(c.gas["R"], c.gas["omega"], c.gas["Tref"], c.gas["muRef"], c.gas["Pr"], 0)
    bc = dl.BC(dl.ptr(a["patch_type"], C.c_int32), dl.ptr(a["rho_b"]), dl.ptr(a["U_b"]), dl.ptr(a["T_b"]))
    h = C.c_void_p()
    st = lib.dugks_create(C.byref(mesh), C.byref(dv), C.byref(gas), C.byref(bc), None, C.byref(h))
    msg = lib.dugks_last_error(h).decode() if h.value else ""
    lib.dugks_destroy(h)
    return st, msg


def _flat():
    c = cs.cavity_case(4, 6)
    return c.flat, c.n_cells


def test_more_than_64_nodes_per_dimension_is_refused():
    fl, n = _flat()
    x = np.linspace(-2400.0, 2400.0, 65)
    st, msg = _create(fl, n, dvs=(x, np.full(65, x[1] - x[0]), 2400.0))
    assert (st, msg) == (7, "dugks_create: more than 64 DV nodes per dimension")


@pytest.mark.parametrize("n", [1, 2])
def test_patch_larger_than_the_internal_faces_is_refused(n):
    # the boundary relaxation reads the internal-face T at each face's
    # patch-local index (fvDVM.C:1367): a 1 x 1 cavity has no internal face, a
    # 2 x 2 one 4 internal faces and 6 fixed-wall faces
    c = cs.cavity_case(n, 6, flatten=False)
    c.dt = 1e-5
    c.flatten()
    st, msg = _create(c.flat, c.n_cells)
    assert st == 7 and "more than the" in msg, (st, msg)


def test_neighbour_out_of_range_is_refused():
    fl, n = _flat()
    nei = fl["neighbour"].copy()
    nei[3] = n
    assert _create(fl, n, neighbour=nei) == (ERR_ARG, "dugks_create: neighbour out of range")


def test_face_with_owner_as_neighbour_is_refused():
    fl, n = _flat()
    nei = fl["neighbour"].copy()
    nei[2] = fl["owner"][2]
    assert _create(fl, n, neighbour=nei)[0] == ERR_ARG


def test_negative_owner_is_refused():
    fl, n = _flat()
    own = fl["owner"].copy()
    own[-1] = -1
    assert _create(fl, n, owner=own) == (ERR_ARG, "dugks_create: owner out of range")


def test_cell_without_faces_is_refused():
    # one more cell than the faces address
    fl, n = _flat()
    Cc = np.vstack([fl["C"], [[9.0, 9.0, 0.0]]])
    V = np.append(fl["V"], 1.0)
    st, msg = _create(fl, n + 1, C=Cc, V=V)
    assert st == ERR_ARG and "has no faces" in msg


def test_patch_starts_must_span_the_boundary():
    fl, n = _flat()
    ps = fl["patch_start"].copy()
    ps[-1] -= 1
    assert _create(fl, n, patch_start=ps)[0] == ERR_ARG


def test_non_positive_volume_is_refused():
    fl, n = _flat()
    V = fl["V"].copy()
    V[5] = 0.0
    assert _create(fl, n, V=V) == (ERR_ARG, "dugks_create: non-positive cell volume")


def test_non_finite_geometry_is_refused():
    fl, n = _flat()
    Sf = fl["Sf"].copy()
    Sf[7, 1] = np.nan
    assert _create(fl, n, Sf=Sf)[0] == ERR_ARG
    Cc = fl["C"].copy()
    Cc[1, 0] = np.inf
    assert _create(fl, n, C=Cc)[0] == ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("field,index,value", [("rho", 3, np.nan), ("rho", 0, 0.0), ("T", 7, -5.0),
                                               ("T", 2, np.inf), ("U", 4, np.nan)])
def test_bad_macros_return_err_nan(field, index, value):
    c = cs.cavity_case(8, 8)
    s = dl.Solver(c)
    s.step(2, c.dt)
    before = s.macros()
    rho, U, T = c.rho0.copy(), c.U0.copy(), c.T0.copy()
    {"rho": rho, "U": U.reshape(-1), "T": T}[field][index] = value
    with pytest.raises(dl.DugksError) as e:
        s.set_macros(rho, U, T)
    assert e.value.code == ERR_NAN
    # the handle is untouched and still steps
    after = s.macros()
    assert all(np.array_equal(before[k], after[k]) for k in ("rho", "U", "T", "q"))
    s.step(1, c.dt)
    assert np.all(np.isfinite(s.macros()["rho"]))


@pytest.mark.gpu
def test_bad_state_returns_err_nan():
    c = cs.cavity_case(8, 8)
    s = dl.Solver(c)
    s.step(2, c.dt)
    g, h = s.state()
    bad = g.copy()
    bad[5, 9] = np.nan
    with pytest.raises(dl.DugksError) as e:
        s.set_state(bad, h, c.dt)
    assert e.value.code == ERR_NAN
    # h far below zero in one cell: negative energy, T < 0
    hb = h.copy()
    hb[:, 11] = -50.0 * np.abs(h[:, 11]) - 1.0
    with pytest.raises(dl.DugksError) as e:
        s.set_state(g, hb, c.dt)
    assert e.value.code == ERR_NAN
    # a good state loads again
    s.set_state(g, h, c.dt)
    s.step(1, c.dt)
    assert np.all(np.isfinite(s.macros()["T"]))
