"""dugks_cell_macros_noalloc (the allocation-free cell-macro reduction)
against the existing entry points, through the C ABI.

It must give the cell macros dugks_get_macros reports after a step, from
the state dugks_get_state returns, on two calls in a row (FP64, same
<= 1e-10 relative-L2 bar as the parity tests, taken with the same floors:
both paths sum the DVs in different orders), and the two calls must agree
bitwise.  At its largest size it is checked against a plain torch FP64
restatement of the moments.  This file is collected last so that it also
runs after the other GPU tests in one process."""
import ctypes as C

import numpy as np
import pytest

import oracle_bind as ob
from dugks_b200 import case as cs
from dugks_b200 import lib as dl
from dugks_b200 import quadrature

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
MAX_CELLS = 131072


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _call(lib, torch, D, xi, w, g, hh, gas, dt):
    """One call on torch's current stream; returns host macros."""
    n = g.shape[1]
    dev = torch.device("cuda:0")
    rho = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
    T = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
    U = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
    q = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
    msg = C.create_string_buffer(256)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = lib.dugks_cell_macros_noalloc(D, xi.shape[0], xi.data_ptr(), w.data_ptr(), n, g.data_ptr(), hh.data_ptr(),
                                       C.byref(gas), dt, rho.data_ptr(), U.data_ptr(), T.data_ptr(), q.data_ptr(),
                                       stream, msg, len(msg))
    assert st == 0, msg.value.decode()
    torch.cuda.synchronize()
    return {"rho": rho.cpu().numpy(), "U": U.cpu().numpy(), "T": T.cpu().numpy(), "q": q.cpu().numpy()}


def _gas(case):
    g = case.gas
    return dl.Gas(g["R"], g["omega"], g["Tref"], g["muRef"], g["Pr"], int(g.get("K", 0)))


@pytest.mark.parametrize("which", ["cavity", "cube"])
def test_noalloc_matches_step_macros_twice(which):
    torch = _torch()
    case = cs.cavity_case(12, 8) if which == "cavity" else cs.cube_case(6, 6, kn=0.1)
    solver = dl.Solver(case)
    for _ in range(3):
        solver.evolution(case.dt)
    ref = solver.macros()
    g, hh = solver.state()
    solver.close()
    xi, w = quadrature.tensor_product(case.xis, case.weights, case.D)
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    xi_d, w_d, g_d, h_d = t(xi), t(w), t(g), t(hh)
    lib = dl.load()
    gas = _gas(case)
    first = _call(lib, torch, case.D, xi_d, w_d, g_d, h_d, gas, case.dt)
    second = _call(lib, torch, case.D, xi_d, w_d, g_d, h_d, gas, case.dt)
    R = case.gas["R"]
    for out in (first, second):
        errs = ob.macro_errors(out, ref, R)
        assert max(errs.values()) <= TOL64, errs
    for k in first:
        assert np.array_equal(first[k], second[k]), k


def test_noalloc_largest_size_against_torch():
    torch = _torch()
    dev = torch.device("cuda:0")
    D, n1, n = 3, 4, MAX_CELLS
    X =np.linspace(-3.0, 3.0, n1) * np.sqrt(cs.R_DEMO * 273.0)
    W = np.full(n1, X[1] - X[0])
    xi, w = quadrature.tensor_product(X, W, D)
    gen = torch.Generator(device="cpu").manual_seed(7)
    RT0 = cs.R_DEMO * 273.0
    rho0 = 1e-6 * (1.0 + 0.1 * torch.rand(n, generator=gen, dtype=torch.float64))
    U0 = 30.0 * (torch.rand(n, 3, generator=gen, dtype=torch.float64) - 0.5)
    RT = RT0 * (1.0 + 0.2 * torch.rand(n, generator=gen, dtype=torch.float64))
    xt = torch.from_numpy(xi)
    c2 = ((xt[:, None, :] - U0[None, :, :]) ** 2).sum(-1)                  # [nv, n]
    g = rho0 * (2 * np.pi * RT) ** -1.5 * torch.exp(-0.5 * c2 / RT)
    g = g * (1.0 + 0.05 * torch.rand(g.shape, generator=gen, dtype=torch.float64))
    K = 2
    hh = g * RT * (K + 3 - D) * (1.0 + 0.05 * torch.rand(g.shape, generator=gen, dtype=torch.float64))
    gas = dl.Gas(cs.R_DEMO, 0.81, 273.0, 2.117e-5, 2.0 / 3.0, K)
    dt = 1e-6
    lib = dl.load()
    args = [torch.from_numpy(a).to(dev) for a in (xi, w)] + [g.contiguous().to(dev), hh.contiguous().to(dev)]
    first = _call(lib, torch, D, *args, gas, dt)
    second = _call(lib, torch, D, *args, gas, dt)
    # torch FP64 restatement: raw moments, then the macros as updateMacroVol forms them
    wt = torch.from_numpy(w)[:, None]
    a, b = wt * g, wt * hh
    rho = a.sum(0)
    U = (a[:, :, None] * xt[:, None, :]).sum(0) / rho[:, None]
    E = (a * (xt ** 2).sum(-1)[:, None] + b).sum(0)
    T = (0.5 * E - 0.5 * rho * (U ** 2).sum(-1)) / ((K + 3.0) / 2.0 * gas.R * rho)
    c = xt[:, None, :] - U[None, :, :]
    qv = 0.5 * ((a * (c ** 2).sum(-1) + b)[:, :, None] * c).sum(0)
    tau = gas.mu_ref * torch.exp(gas.omega * torch.log(T / gas.Tref)) / rho / T / gas.R
    qv = qv * (2 * tau / (2 * tau + dt * gas.Pr))[:, None]
    ref = {"rho": rho.numpy(), "U": U.numpy(), "T": T.numpy(), "q": qv.numpy()}
    for out in (first, second):
        errs = ob.macro_errors(out, ref, gas.R)
        assert max(errs.values()) <= TOL64, errs
    for k in first:
        assert np.array_equal(first[k], second[k]), k


def test_noalloc_rejects_oversize_and_host_buffers():
    torch = _torch()
    lib = dl.load()
    dev = torch.device("cuda:0")
    gas = dl.Gas(cs.R_DEMO, 0.81, 273.0, 2.117e-5, 2.0 / 3.0, 0)
    xi = torch.zeros(4, 3, dtype=torch.float64, device=dev)
    w = torch.ones(4, dtype=torch.float64, device=dev)
    g = torch.ones(4, 8, dtype=torch.float64, device=dev)
    msg = C.create_string_buffer(256)
    st = lib.dugks_cell_macros_noalloc(2, 4, xi.data_ptr(), w.data_ptr(), MAX_CELLS + 1, g.data_ptr(), g.data_ptr(),
                                       C.byref(gas), 1e-6, None, None, None, None, None, msg, len(msg))
    assert st == 1 and b"at most 131072" in msg.value
    host = np.ones(32)
    st = lib.dugks_cell_macros_noalloc(2, 4, xi.data_ptr(), w.data_ptr(), 8, host.ctypes.data, g.data_ptr(),
                                       C.byref(gas), 1e-6, None, None, None, None, None, msg, len(msg))
    assert st == 1 and b"not device memory" in msg.value


def _rt():
    """The CUDA runtime the library itself links (already loaded by dl.load)."""
    dl.load()
    return C.CDLL("libcudart.so.12")


def test_noalloc_rejects_short_device_buffers():
    # a buffer from plain cudaMalloc holding far fewer doubles than n_dv x
    # n_cells: the allocation range check refuses it before any launch
    _torch()
    lib = dl.load()
    rt = _rt()
    n_dv, n = 64, 1024
    ptrs = []

    def dmalloc(nbytes):
        p = C.c_void_p()
        assert rt.cudaMalloc(C.byref(p), C.c_size_t(nbytes)) == 0
        ptrs.append(p)
        return p

    try:
        xi, w = dmalloc(3 * n_dv * 8), dmalloc(n_dv * 8)
        g_ok, g_short = dmalloc(n_dv * n * 8), dmalloc(4096)
        rho = dmalloc(n * 8)
        gas = dl.Gas(cs.R_DEMO, 0.81, 273.0, 2.117e-5, 2.0 / 3.0, 0)
        msg = C.create_string_buffer(256)
        st = lib.dugks_cell_macros_noalloc(3, n_dv, xi, w, n, g_short, g_ok, C.byref(gas), 1e-6, rho, None, None,
                                           None, None, msg, len(msg))
        assert st == 1 and b"argument 2 is too small" in msg.value, msg.value
        for p, nbytes in zip(ptrs, (3 * n_dv * 8, n_dv * 8, n_dv * n * 8, 4096, n * 8)):
            assert rt.cudaMemset(p, 0, C.c_size_t(nbytes)) == 0
        st = lib.dugks_cell_macros_noalloc(3, n_dv, xi, w, n, g_ok, g_ok, C.byref(gas), 1e-6, rho, None, None,
                                           None, None, msg, len(msg))
        assert st == 0, msg.value
        st = lib.dugks_cell_macros_noalloc(3, n_dv, xi, w, n, g_ok, g_ok, C.byref(gas), 1e-6, g_short, None, None,
                                           None, None, msg, len(msg))
        assert st == 1 and b"argument 4 is too small" in msg.value, msg.value
        st = lib.dugks_cell_macros_noalloc(3, n_dv, xi, w, n, g_ok, g_ok, C.byref(gas), 1e-6, rho, rho, None,
                                           None, None, msg, len(msg))
        assert st == 1 and b"argument 5 is too small" in msg.value, msg.value
        assert rt.cudaDeviceSynchronize() == 0
    finally:
        for p in ptrs:
            rt.cudaFree(p)


_RESET_SCRIPT = r'''
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from dugks_b200 import case as cs
from dugks_b200 import lib as dl
from dugks_b200 import quadrature
lib = dl.load()
rt = C.CDLL("libcudart.so.12")
c = cs.cavity_case(10, 8)
xi, w = quadrature.tensor_product(c.xis, c.weights, 2)
rng = np.random.default_rng(3)
RT = c.gas["R"] * 273.0
c2 = ((xi[:, None, :2] - 20.0 * rng.random((1, c.n_cells, 2))) ** 2).sum(-1)
g = np.ascontiguousarray(1e-6 / (2 * np.pi * RT) * np.exp(-0.5 * c2 / RT) * (1 + 0.01 * rng.random(c2.shape)))
hh = np.ascontiguousarray(g * RT)
gas = dl.Gas(c.gas["R"], c.gas["omega"], c.gas["Tref"], c.gas["muRef"], c.gas["Pr"], 0)

def run():
    bufs = []
    def put(a):
        p = C.c_void_p()
        assert rt.cudaMalloc(C.byref(p), C.c_size_t(a.nbytes)) == 0
        assert rt.cudaMemcpy(p, a.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes), 1) == 0
        bufs.append(p)
        return p
    n = c.n_cells
    outs = [np.zeros(n), np.zeros(3 * n), np.zeros(n), np.zeros(3 * n)]
    d_in = [put(np.ascontiguousarray(a)) for a in (xi, w, g, hh)]
    d_out = [put(o) for o in outs]
    msg = C.create_string_buffer(256)
    st = lib.dugks_cell_macros_noalloc(2, len(w), d_in[0], d_in[1], n, d_in[2], d_in[3], C.byref(gas), c.dt,
                                       d_out[0], d_out[1], d_out[2], d_out[3], None, msg, len(msg))
    assert st == 0, msg.value
    assert rt.cudaDeviceSynchronize() == 0
    for o, p in zip(outs, d_out):
        assert rt.cudaMemcpy(o.ctypes.data_as(C.c_void_p), p, C.c_size_t(o.nbytes), 2) == 0
    for p in bufs:
        rt.cudaFree(p)
    return outs

first = run()
assert rt.cudaDeviceReset() == 0
second = run()
assert all(np.array_equal(a, b) for a, b in zip(first, second))
assert np.all(first[0] > 0) and np.all(first[2] > 0)
print("reset ok")
'''


def test_noalloc_after_device_reset(tmp_path):
    # the scratch address is cached per context: after cudaDeviceReset the
    # next call looks it up again and gives the same macros (a fresh process
    # without torch, which does not survive a device reset)
    _torch()
    import os
    import subprocess
    import sys
    script = tmp_path / "reset.py"
    script.write_text(_RESET_SCRIPT)
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "psp-vst_b200", "python")
    r = subprocess.run([sys.executable, str(script), pkg], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "reset ok" in r.stdout, r.stdout + r.stderr
