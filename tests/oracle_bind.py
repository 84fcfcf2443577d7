"""ctypes binding of the CPU oracle (oracle/dugks_oracle.c) -- test
infrastructure: the tests, the smoke check and the benchmark's CPU-baseline
leg use it as the checker; the product never does."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "build", "liboracle_dugks.so")

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_ip = C.POINTER(C.c_int)
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_LIB):
        build()
    lib = C.CDLL(ORACLE_LIB)
    lib.oracle_geometry.argtypes = [C.c_int, _dp, C.c_int, _i64p, _i64p, _i64p, C.c_int, _i64p, C.c_int, _dp, _dp,
                                    _dp, _dp]
    lib.oracle_geometry.restype = None
    lib.oracle_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                  C.c_int, C.c_int, C.c_int, _i64p, _i64p, _dp, _dp, _dp, _dp, C.c_int, _ip, _ip, _dp,
                                  _dp, _dp, C.c_int, _dp, _dp, C.c_double, C.c_int, C.c_int]
    lib.oracle_create.restype = C.c_void_p
    lib.oracle_destroy.argtypes = [C.c_void_p]
    lib.oracle_set_macros.argtypes = [C.c_void_p, _dp, _dp, _dp]
    lib.oracle_set_patch_extra.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.oracle_set_macro_flux.argtypes = [C.c_void_p, C.c_int]
    lib.oracle_evolve.argtypes = [C.c_void_p, C.c_double]
    lib.oracle_co_num.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
    for name in ("oracle_get_macros", "oracle_get_face_macros"):
        getattr(lib, name).argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
    lib.oracle_get_wall.argtypes = [C.c_void_p, _dp, _dp]
    lib.oracle_get_state.argtypes = [C.c_void_p, _dp, _dp]
    lib.oracle_set_state.argtypes = [C.c_void_p, _dp, _dp]
    lib.oracle_get_ghbar.argtypes = [C.c_void_p, _dp, _dp]
    lib.oracle_get_face_values.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
    lib.oracle_get_ls.argtypes = [C.c_void_p, _dp, _dp, _dp]
    lib.oracle_get_weights.argtypes = [C.c_void_p, _dp, _dp]
    lib.oracle_tangent.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp, _dp, _dp, C.c_double, _dp, _dp, _dp,
                                   _dp]
    lib.oracle_tangent.restype = C.c_int
    _lib = lib
    return lib


def _p(a, t=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def geometry(pm) -> dict:
    lib = load()
    nF = pm.n_faces
    out = {"Cf": np.zeros((nF, 3)), "Sf": np.zeros((nF, 3)), "C": np.zeros((pm.n_cells, 3)), "V": np.zeros(pm.n_cells)}
    pts = np.ascontiguousarray(pm.points, dtype=np.float64)
    fo = np.ascontiguousarray(pm.face_offsets, dtype=np.int64)
    fp = np.ascontiguousarray(pm.face_points, dtype=np.int64)
    own = np.ascontiguousarray(pm.owner, dtype=np.int64)
    nei = np.ascontiguousarray(pm.neighbour, dtype=np.int64)
    lib.oracle_geometry(len(pts), _p(pts), nF, _p(fo, C.c_int64), _p(fp, C.c_int64), _p(own, C.c_int64),
                        pm.n_internal_faces, _p(nei, C.c_int64), pm.n_cells, _p(out["Cf"]), _p(out["Sf"]),
                        _p(out["C"]), _p(out["V"]))
    return out


class Oracle:
    """Same interface as dugks_b200.lib.Solver, on the CPU restatement."""

    def __init__(self, case, ls_weighting: int = 0, threads: int = 0, xi=None, w=None, macro_flux: bool | None = None):
        self.lib = load()
        self.case = case
        fl = case.flat
        if xi is None:
            xi, w = case.dv_set()
        self._keep = [np.ascontiguousarray(a) for a in (
            fl["owner"].astype(np.int64), fl["neighbour"].astype(np.int64), fl["C"], fl["V"], fl["Cf"], fl["Sf"],
            fl["patch_type"].astype(np.int32), fl["patch_start"].astype(np.int32), fl["rho_b"], fl["U_b"], fl["T_b"],
            np.ascontiguousarray(xi, dtype=np.float64), np.ascontiguousarray(w, dtype=np.float64))]
        own, nei, Cc, V, Cf, Sf, pt, ps, rb, ub, tb, xa, wa = self._keep
        g = case.gas
        self.n_dv = len(wa)
        threads = threads or (os.cpu_count() or 1)
        self.s = self.lib.oracle_create(case.D, int(g.get("K", 0)), g["R"], g["omega"], g["Tref"], g["muRef"], g["Pr"],
                                        case.n_cells, fl["n_internal"], fl["n_boundary"], _p(own, C.c_int64),
                                        _p(nei, C.c_int64), _p(Cc), _p(V), _p(Cf), _p(Sf), len(pt), _p(pt, C.c_int),
                                        _p(ps, C.c_int), _p(rb), _p(ub), _p(tb), self.n_dv, _p(xa), _p(wa),
                                        case.xi_max, ls_weighting, threads)
        self._p_b = np.ascontiguousarray(fl.get("p_b", np.zeros(fl["n_boundary"])), dtype=np.float64)
        self.lib.oracle_set_patch_extra(self.s, len(case.xis), _p(self._p_b))
        if macro_flux is None:
            macro_flux = getattr(case, "macro_flux", False)
        # the velocity-mesh build takes the DF-flux branch of macroFlux yes
        mode = (2 if getattr(case, "dv_w", None) is not None else 1) if macro_flux else 0
        self.lib.oracle_set_macro_flux(self.s, mode)
        self.set_macros(case.rho0, case.U0, case.T0)

    def set_macros(self, rho, U, T):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        U = np.ascontiguousarray(U, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        self.lib.oracle_set_macros(self.s, _p(rho), _p(U), _p(T))

    def evolution(self, dt):
        self.lib.oracle_evolve(self.s, dt)

    def step(self, n, dt):
        for _ in range(n):
            self.evolution(dt)

    def get_co_num(self, dt):
        a, b = C.c_double(), C.c_double()
        self.lib.oracle_co_num(self.s, dt, C.byref(a), C.byref(b))
        return a.value, b.value

    def macros(self):
        n = self.case.n_cells
        out = {"rho": np.zeros(n), "U": np.zeros((n, 3)), "T": np.zeros(n), "q": np.zeros((n, 3)), "tau": np.zeros(n)}
        self.lib.oracle_get_macros(self.s, _p(out["rho"]), _p(out["U"]), _p(out["T"]), _p(out["q"]), _p(out["tau"]))
        return out

    def face_macros(self):
        nF = self.case.flat["n_internal"] + self.case.flat["n_boundary"]
        out = {"rho": np.zeros(nF), "U": np.zeros((nF, 3)), "T": np.zeros(nF), "q": np.zeros((nF, 3)),
               "tau": np.zeros(nF)}
        self.lib.oracle_get_face_macros(self.s, _p(out["rho"]), _p(out["U"]), _p(out["T"]), _p(out["q"]),
                                        _p(out["tau"]))
        return out

    def boundary_rho(self):
        out = np.zeros(self.case.flat["n_boundary"])
        self.lib.oracle_get_wall(self.s, _p(out), None)
        return out

    def in_coming_by_rho(self):
        out = np.zeros(self.case.flat["n_boundary"])
        self.lib.oracle_get_wall(self.s, None, _p(out))
        return out

    def state(self):
        g = np.zeros((self.n_dv, self.case.n_cells))
        h = np.zeros((self.n_dv, self.case.n_cells))
        self.lib.oracle_get_state(self.s, _p(g), _p(h))
        return g, h

    def set_state(self, g, h):
        g = np.ascontiguousarray(g, dtype=np.float64)
        h = np.ascontiguousarray(h, dtype=np.float64)
        self.lib.oracle_set_state(self.s, _p(g), _p(h))

    def ghbar(self):
        g = np.zeros((self.n_dv, self.case.n_cells))
        h = np.zeros((self.n_dv, self.case.n_cells))
        self.lib.oracle_get_ghbar(self.s, _p(g), _p(h))
        return g, h

    def ls_vectors(self):
        fl = self.case.flat
        p = np.zeros((fl["n_internal"], 3))
        n = np.zeros((fl["n_internal"], 3))
        b = np.zeros((fl["n_boundary"], 3))
        self.lib.oracle_get_ls(self.s, _p(p), _p(n), _p(b))
        return p, n, b

    def face_values(self):
        """Relaxed face DFs of the last step, DV-major: internal g, h and
        boundary g, h."""
        fl = self.case.flat
        out = [np.zeros((self.n_dv, fl[k])) for k in ("n_internal", "n_internal", "n_boundary", "n_boundary")]
        self.lib.oracle_get_face_values(self.s, *[_p(a) for a in out])
        return out

    def tangent(self, n_steps, dt, heat_w=None, force_w=None, dT_b=None, dU_b=None, d_mu=0.0):
        """Objective J of n_steps from the current state and its derivative
        along (dT_b, dU_b, d_mu), on the dual-number restatement; the state is
        left unchanged.  Returns (J, dJ, g, h) with the final g~, h~."""
        nb = self.case.flat["n_boundary"]
        arr = lambda a, n: None if a is None else np.ascontiguousarray(np.reshape(a, n), dtype=np.float64)  # noqa: E731
        hw, fw, dT, dU = arr(heat_w, nb), arr(force_w, 3 * nb), arr(dT_b, nb), arr(dU_b, 3 * nb)
        J, dJ = C.c_double(), C.c_double()
        g = np.zeros((self.n_dv, self.case.n_cells))
        h = np.zeros((self.n_dv, self.case.n_cells))
        rc = self.lib.oracle_tangent(self.s, int(n_steps), float(dt), _p(hw), _p(fw), _p(dT), _p(dU), float(d_mu),
                                     C.byref(J), C.byref(dJ), _p(g), _p(h))
        if rc != 0:
            raise ValueError("oracle_tangent: maxwellWall and farField patches only, macroFlux no")
        return J.value, dJ.value, g, h

    def close(self):
        if getattr(self, "s", None):
            self.lib.oracle_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def boundary_flux_objective(case, xi, w, g_b, h_b, heat_w, force_w) -> float:
    """One step's term of the boundary-flux objective from relaxed boundary
    face DFs g_b, h_b [dv][boundary face]: sum over faces b and DVs i of
    w_i (xi_i . S_b) [heat_w_b (|xi_i|^2 g + h)/2 + (force_w_b . xi_i) g]."""
    fl = case.flat
    Sb = np.asarray(fl["Sf"])[fl["n_internal"]:]
    xs = np.asarray(xi) @ Sb.T                                   # [dv, b]
    wx = np.asarray(w)[:, None] * xs
    x2 = np.sum(np.asarray(xi) ** 2, axis=1)[:, None]
    cg = np.asarray(xi) @ np.reshape(force_w, (-1, 3)).T          # [dv, b]
    return float(np.sum(wx * (np.asarray(heat_w)[None, :] * 0.5 * (x2 * g_b + h_b) + cg * g_b)))


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def macro_errors(a: dict, b: dict, R: float, floor: float = 1e-4) -> dict:
    """Relative L2 errors of macro fields a against reference b.

    rho and T: plain relative L2.  U and q are sums over DVs that cancel to
    (nearly) zero in quiescent regions, where both results are rounding noise
    of size ~1e-16 of the sums' natural scale; their denominators are floored
    at `floor` times that scale (thermal speed sqrt(RT) for U, rho (RT)^1.5
    for q), i.e. about 100 ulps of the sums."""
    rt = R * np.asarray(b["T"], dtype=np.float64)
    out = {"rho": rel_l2(a["rho"], b["rho"]), "T": rel_l2(a["T"], b["T"])}
    for k, scale in (("U", np.sqrt(rt)), ("q", np.asarray(b["rho"]) * rt ** 1.5)):
        den = max(np.linalg.norm(b[k]), floor * np.linalg.norm(scale))
        out[k] = float(np.linalg.norm(np.asarray(a[k]) - np.asarray(b[k])) / den)
    return out
