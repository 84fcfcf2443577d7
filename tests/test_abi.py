"""The C-ABI library loads and exports every symbol include/dugks.h
declares; host-side argument checking works without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from dugks_b200 import case as cs
from dugks_b200 import lib as dl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    txt = open(os.path.join(ROOT, "include", "dugks.h")).read()
    txt = re.sub(r"/\*.*?\*/", " ", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dugks_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = dl.load()
    names = _declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
        assert n in dl.SIGNATURES, n
    assert lib.dugks_abi_version() == 2


def test_default_options():
    lib = dl.load()
    o = dl.Options()
    lib.dugks_default_options(C.byref(o))
    assert o.precision == dl.FP64 and o.ls_weighting == dl.LS_MAGSF and o.tile_cells == 0


def test_create_rejects_bad_arguments_on_host():
    lib = dl.load()
    h = C.c_void_p()
    assert lib.dugks_create(None, None, None, None, None, C.byref(h)) == 1
    c = cs.cavity_case(4, 6)
    fl = c.flat
    own = np.ascontiguousarray(fl["owner"])
    own_bad = own.copy()
    own_bad[0] = 10 ** 6
    nei = np.ascontiguousarray(fl["neighbour"])
    arrs = [np.ascontiguousarray(fl[k]) for k in ("C", "V", "Cf", "Sf")]
    ps = np.ascontiguousarray(fl["patch_start"])
    mesh = dl.Mesh(c.n_cells, fl["n_internal"], fl["n_boundary"], 2, dl.ptr(own_bad, C.c_int64),
                   dl.ptr(nei, C.c_int64), *[dl.ptr(a) for a in arrs], len(fl["patch_type"]), dl.ptr(ps, C.c_int32))
    xis = np.ascontiguousarray(c.xis)
    ws = np.ascontiguousarray(c.weights)
    dv = dl.DVSet(len(xis), dl.ptr(xis), dl.ptr(ws), c.xi_max)
    gas = dl.Gas(c.gas["R"], c.gas["omega"], c.gas["Tref"], c.gas["muRef"], c.gas["Pr"], 0)
    pt = np.ascontiguousarray(fl["patch_type"])
    rb, ub, tb = (np.ascontiguousarray(fl[k]) for k in ("rho_b", "U_b", "T_b"))
    bc = dl.BC(dl.ptr(pt, C.c_int32), dl.ptr(rb), dl.ptr(ub), dl.ptr(tb))
    st = lib.dugks_create(C.byref(mesh), C.byref(dv), C.byref(gas), C.byref(bc), None, C.byref(h))
    assert st == 1
    assert b"owner out of range" in lib.dugks_last_error(h)
    lib.dugks_destroy(h)


def test_geometry_rejects_bad_face():
    lib = dl.load()
    pts = np.zeros((3, 3))
    fo = np.array([0, 2], dtype=np.int64)   # a face with 2 points
    fp = np.array([0, 1], dtype=np.int64)
    own = np.array([0], dtype=np.int64)
    out = [np.zeros(3) for _ in range(4)]
    st = lib.dugks_mesh_geometry(3, dl.ptr(pts), 1, dl.ptr(fo, C.c_int64), dl.ptr(fp, C.c_int64),
                                 dl.ptr(own, C.c_int64), 0, None, 1, *[dl.ptr(o) for o in out])
    assert st == 1


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(FileNotFoundError):
        dl.load(str(tmp_path / "nope.so"))


def test_adjoint_rejects_null_arguments_on_host():
    lib = dl.load()
    obj = dl.Objective(None, None, 4, 0, 1e-6, 4)
    assert lib.dugks_adjoint_run(None, C.byref(obj), None, None, None, None, None) == 1
