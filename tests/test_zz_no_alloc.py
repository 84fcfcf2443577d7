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
