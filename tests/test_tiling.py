"""Host-side tile layout (no GPU needed).

dugks_create builds the tiles on the host before it looks for a device, and
returns the handle even when it then fails; dugks_layout reads the layout.
The default greedy tiles respect the per-tile limits (128 L0 cells) and are
no more numerous than the uniform tiles the same limits allow."""
import ctypes as C

import numpy as np
import pytest

from dugks_b200 import case as cs
from dugks_b200 import lib as dl


def _layout(case, tile_cells):
    lib = dl.load()
    fl = case.flat
    keep = {k: np.ascontiguousarray(v) for k, v in fl.items() if isinstance(v, np.ndarray)}
    mesh = dl.Mesh(case.n_cells, fl["n_internal"], fl["n_boundary"], case.D, dl.ptr(keep["owner"], C.c_int64),
                   dl.ptr(keep["neighbour"], C.c_int64), dl.ptr(keep["C"]), dl.ptr(keep["V"]), dl.ptr(keep["Cf"]),
                   dl.ptr(keep["Sf"]), len(keep["patch_type"]), dl.ptr(keep["patch_start"], C.c_int32))
    xis, ws = np.ascontiguousarray(case.xis), np.ascontiguousarray(case.weights)
    dv = dl.DVSet(len(xis), dl.ptr(xis), dl.ptr(ws), case.xi_max)
    g = case.gas
    gas = dl.Gas(g["R"], g["omega"], g["Tref"], g["muRef"], g["Pr"], 0)
    bc = dl.BC(dl.ptr(keep["patch_type"], C.c_int32), dl.ptr(keep["rho_b"]), dl.ptr(keep["U_b"]),
               dl.ptr(keep["T_b"]), dl.ptr(keep["p_b"]))
    opt = dl.Options()
    lib.dugks_default_options(C.byref(opt))
    opt.tile_cells = tile_cells
    h = C.c_void_p()
    st = lib.dugks_create(C.byref(mesh), C.byref(dv), C.byref(gas), C.byref(bc), C.byref(opt), C.byref(h))
    assert st in (0, 2), (st, lib.dugks_last_error(h))   # 2: no CUDA device here
    t, n, ch = C.c_int32(), C.c_int32(), C.c_int32()
    assert lib.dugks_layout(h, C.byref(t), C.byref(n), C.byref(ch)) == 0
    lib.dugks_destroy(h)
    return t.value, n.value


@pytest.mark.parametrize("which", ["ball", "cube"])
def test_greedy_tiles_fit_and_are_fewer(which):
    c = cs.ball_case(8, 8, 1.12, 6) if which == "ball" else cs.cube_case(16, 6)
    tg, ng = _layout(c, 0)
    tu, nu = _layout(c, 128)
    assert 0 < tg <= 128 and 0 < tu <= 128
    assert ng * 128 >= c.n_cells and ng <= nu


@pytest.mark.parametrize("tile_cells", [0, 16])
def test_octagon_cells_tile(tile_cells):
    # cells with ten faces (a 2:1 refined cavity): the stencil and flux lists
    # outgrow the passes' register copies; the tiles still fit their limits
    c = cs.refined_cavity_case(10, 6)
    t, n = _layout(c, tile_cells)
    assert 0 < t <= (tile_cells or 128) and n * t >= c.n_cells
