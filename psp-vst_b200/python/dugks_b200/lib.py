"""ctypes binding of the C ABI in include/dugks.h (libdugks_b200.so).

``Solver`` mirrors the reference's fvDVM class (src/fvDVM/fvDVM/fvDVM.H:80-409):
construct it from a flattened case, then ``evolution(dt)`` advances one time
step (fvDVM::evolution, fvDVM.C:2128-2174) and ``get_co_num(dt)`` is
fvDVM::getCoNum (fvDVM.C:2177-2185).  Errors raise :class:`DugksError`.
The library is required: there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "..", "lib", "libdugks_b200.so"))
# the bounds-checked build of the same sources (-DDUGKS_CHECK): indices read
# from device tables are range-checked, a bad one returns DUGKS_ERR_ARG
CHECK_LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "..", "lib", "libdugks_b200_check.so"))

FP64 = 0
FP32C = 1
PATCH_MAXWELL_WALL = 1
PATCH_FAR_FIELD = 2
LS_MAGSF, LS_INVDIST, LS_UNWEIGHTED = 0, 1, 2

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_OOM", 4: "ERR_TIMEOUT", 5: "ERR_NAN", 6: "ERR_STATE",
          7: "ERR_UNSUPPORTED"}


class DugksError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)


class Mesh(C.Structure):
    _fields_ = [("n_cells", C.c_int32), ("n_internal_faces", C.c_int32), ("n_boundary_faces", C.c_int32),
                ("n_solution_dims", C.c_int32), ("owner", _i64p), ("neighbour", _i64p),
                ("cell_centres", _dp), ("cell_volumes", _dp), ("face_centres", _dp), ("face_areas", _dp),
                ("n_patches", C.c_int32), ("patch_start", _i32p)]


class DVSet(C.Structure):
    _fields_ = [("n_per_dim", C.c_int32), ("xis", _dp), ("weights", _dp), ("xi_max", C.c_double)]


class DVList(C.Structure):
    _fields_ = [("n_dv", C.c_int32), ("xi", _dp), ("weights", _dp), ("xi_max", C.c_double)]


class Gas(C.Structure):
    _fields_ = [("R", C.c_double), ("omega", C.c_double), ("Tref", C.c_double), ("mu_ref", C.c_double),
                ("Pr", C.c_double), ("K_inner", C.c_int32)]


class BC(C.Structure):
    _fields_ = [("patch_type", _i32p), ("rho", _dp), ("U", _dp), ("T", _dp), ("p", _dp)]


class Adapt(C.Structure):
    _fields_ = [("max_co", C.c_double), ("max_delta_t", C.c_double)]


class Shard(C.Structure):
    """Velocity-space shard of a solver (dugks_dv_shard): rank of world;
    use_nccl with the NCCL unique id rank 0 made (nccl_unique_id())."""
    _fields_ = [("rank", C.c_int32), ("world", C.c_int32), ("use_nccl", C.c_int32), ("nccl_id", C.c_ubyte * 128)]


def shard(rank: int, world: int, nccl_id: bytes | None = None) -> Shard:
    s = Shard(rank, world, 1 if nccl_id is not None else 0)
    if nccl_id is not None:
        if len(nccl_id) != 128:
            raise ValueError("an NCCL unique id is 128 bytes")
        C.memmove(s.nccl_id, nccl_id, 128)
    return s


def _load_torch_nccl() -> None:
    # The library opens libnccl.so.2 by soname when a shard uses NCCL; load
    # torch (and with it the NCCL it was built with) first, so that the
    # process holds one NCCL and torch.distributed can still start.
    try:
        import torch  # noqa: F401
    except ImportError:
        pass


def nccl_unique_id() -> bytes:
    """A new NCCL unique id (rank 0 makes it and sends it to the other ranks)."""
    _load_torch_nccl()
    buf = (C.c_ubyte * 128)()
    st = load().dugks_nccl_unique_id(buf)
    if st != 0:
        raise DugksError(st, "ncclGetUniqueId failed or NCCL is not available")
    return bytes(buf)


def dv_rows(n_rows: int, rank: int, world: int) -> tuple[int, int]:
    """The DV rows rank owns: rows*rank/world .. rows*(rank+1)/world, as
    dugks_create_sharded assigns them."""
    return n_rows * rank // world, n_rows * (rank + 1) // world


class Objective(C.Structure):
    """dugks_objective: time-averaged boundary energy and momentum flux."""
    _fields_ = [("energy_weight", _dp), ("momentum_weight", _dp), ("n_steps", C.c_int32),
                ("window_start", C.c_int32), ("dt", C.c_double), ("max_snapshots", C.c_int32),
                ("reserved", C.c_int32 * 3)]


class AdjointStats(C.Structure):
    _fields_ = [("forward_steps", C.c_int64), ("reverse_steps", C.c_int64), ("snapshots", C.c_int32),
                ("reserved", C.c_int32), ("ms_total", C.c_double), ("ms_forward", C.c_double),
                ("device_bytes", C.c_double)]


class Options(C.Structure):
    _fields_ = [("precision", C.c_int32), ("ls_weighting", C.c_int32), ("device", C.c_int32),
                ("tile_cells", C.c_int32), ("dv_chunks", C.c_int32), ("macro_flux", C.c_int32),
                ("reserved", C.c_int32 * 10)]


# every symbol include/dugks.h declares, with its ctypes signature
SIGNATURES = {
    "dugks_abi_version": (C.c_int, []),
    "dugks_default_options": (None, [C.POINTER(Options)]),
    "dugks_mesh_geometry": (C.c_int, [C.c_int32, _dp, C.c_int32, _i64p, _i64p, _i64p, C.c_int32, _i64p, C.c_int32,
                                      _dp, _dp, _dp, _dp]),
    "dugks_create": (C.c_int, [C.POINTER(Mesh), C.POINTER(DVSet), C.POINTER(Gas), C.POINTER(BC),
                               C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "dugks_set_macros": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "dugks_step": (C.c_int, [C.c_void_p, C.c_int32, _dp]),
    "dugks_co_num": (C.c_int, [C.c_void_p, C.c_double, _dp, _dp]),
    "dugks_step_adaptive": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Adapt), _dp, _dp]),
    "dugks_get_macros": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "dugks_get_face_macros": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "dugks_get_boundary_rho": (C.c_int, [C.c_void_p, _dp]),
    "dugks_get_df": (C.c_int, [C.c_void_p, _i32p, C.c_int32, _dp, _dp]),
    "dugks_get_state": (C.c_int, [C.c_void_p, _dp, _dp]),
    "dugks_set_state": (C.c_int, [C.c_void_p, _dp, _dp, C.c_double]),
    "dugks_step_record_size": (C.c_int64, [C.c_void_p]),
    "dugks_get_step_record": (C.c_int, [C.c_void_p, _dp]),
    "dugks_set_step_record": (C.c_int, [C.c_void_p, _dp]),
    "dugks_adjoint_run": (C.c_int, [C.c_void_p, C.POINTER(Objective), _dp, _dp, _dp, _dp, C.POINTER(AdjointStats)]),
    "dugks_objective_run": (C.c_int, [C.c_void_p, C.POINTER(Objective), _dp, C.POINTER(AdjointStats)]),
    "dugks_boundary_fluxes": (C.c_int, [C.c_void_p, C.c_double, _dp]),
    "dugks_checkpoint_forward_steps": (C.c_int64, [C.c_int32, C.c_int32]),
    "dugks_layout": (C.c_int, [C.c_void_p, _i32p, _i32p, _i32p]),
    "dugks_n_dv": (C.c_int32, [C.c_void_p]),
    "dugks_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, _dp, C.POINTER(C.c_void_p)]),
    "dugks_batch_step": (C.c_int, [C.c_void_p, C.c_int32]),
    "dugks_batch_last_ms": (C.c_int, [C.c_void_p, _dp]),
    "dugks_batch_graph_kernels": (C.c_int64, [C.c_void_p]),
    "dugks_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "dugks_batch_destroy": (None, [C.c_void_p]),
    "dugks_nccl_unique_id": (C.c_int, [C.POINTER(C.c_ubyte)]),
    "dugks_create_sharded": (C.c_int, [C.POINTER(Mesh), C.POINTER(DVSet), C.POINTER(Gas), C.POINTER(BC),
                                       C.POINTER(Options), C.POINTER(Shard), C.POINTER(C.c_void_p)]),
    "dugks_dv_range": (C.c_int, [C.c_void_p, _i32p, _i32p]),
    "dugks_create_dv_list": (C.c_int, [C.POINTER(Mesh), C.POINTER(DVList), C.POINTER(Gas), C.POINTER(BC),
                                       C.POINTER(Options), C.POINTER(Shard), C.POINTER(C.c_void_p)]),
    "dugks_shard_phase": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.POINTER(_dp), _i64p]),
    "dugks_last_step_ms": (C.c_int, [C.c_void_p, _dp]),
    "dugks_step_timed": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp]),
    "dugks_kernel_launches": (C.c_int64, [C.c_void_p]),
    "dugks_last_error": (C.c_char_p, [C.c_void_p]),
    "dugks_destroy": (None, [C.c_void_p]),
    "dugks_cell_macros_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                            C.c_void_p, C.POINTER(Gas), C.c_double, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_int32]),
}

_lib = None


def load(path: str | None = None):
    """Load libdugks_b200.so (built by __graft_entry__.build()); raises if absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} not found: build the CUDA library first (python -c 'import __graft_entry__ as g; g.build()')")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def ptr(a: np.ndarray | None, ctype=C.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def mesh_geometry(pm) -> dict:
    """OpenFOAM primitiveMesh geometry of a polyMesh via the library's host routine."""
    lib = load()
    nF = pm.n_faces
    Cf = np.zeros((nF, 3))
    Sf = np.zeros((nF, 3))
    Cc = np.zeros((pm.n_cells, 3))
    V = np.zeros(pm.n_cells)
    pts = np.ascontiguousarray(pm.points, dtype=np.float64)
    fo = np.ascontiguousarray(pm.face_offsets, dtype=np.int64)
    fp = np.ascontiguousarray(pm.face_points, dtype=np.int64)
    own = np.ascontiguousarray(pm.owner, dtype=np.int64)
    nei = np.ascontiguousarray(pm.neighbour, dtype=np.int64)
    st = lib.dugks_mesh_geometry(len(pts), ptr(pts), nF, ptr(fo, C.c_int64), ptr(fp, C.c_int64), ptr(own, C.c_int64),
                                 pm.n_internal_faces, ptr(nei, C.c_int64), pm.n_cells, ptr(Cf), ptr(Sf), ptr(Cc), ptr(V))
    if st != 0:
        raise DugksError(st, "dugks_mesh_geometry failed")
    return {"Cf": Cf, "Sf": Sf, "C": Cc, "V": V}


class Solver:
    """fvDVM-shaped wrapper over one dugks_handle."""

    def __init__(self, case, precision: int = FP64, ls_weighting: int = LS_MAGSF, device: int = 0,
                 tile_cells: int = 0, dv_chunks: int = 0, shard: Shard | None = None, macro_flux: bool | None = None,
                 lib_path: str | None = None):
        # lib_path: another build of the library, e.g. CHECK_LIB_PATH
        self.lib = load(lib_path)
        self.case = case
        fc = case.flat
        self._keep = []

        def keep(a, dtype):
            a = np.ascontiguousarray(a, dtype=dtype)
            self._keep.append(a)
            return a

        own = keep(fc["owner"], np.int64)
        nei = keep(fc["neighbour"], np.int64)
        cc = keep(fc["C"], np.float64)
        vv = keep(fc["V"], np.float64)
        cf = keep(fc["Cf"], np.float64)
        sf = keep(fc["Sf"], np.float64)
        ps = keep(fc["patch_start"], np.int32)
        self.mesh = Mesh(case.n_cells, fc["n_internal"], fc["n_boundary"], case.D, ptr(own, C.c_int64),
                         ptr(nei, C.c_int64), ptr(cc), ptr(vv), ptr(cf), ptr(sf), len(fc["patch_type"]),
                         ptr(ps, C.c_int32))
        xis = keep(case.xis, np.float64)
        ws = keep(case.weights, np.float64)
        self.dv = DVSet(len(xis), ptr(xis), ptr(ws), case.xi_max)
        g = case.gas
        self.gas = Gas(g["R"], g["omega"], g["Tref"], g["muRef"], g["Pr"], int(g.get("K", 0)))
        pt = keep(fc["patch_type"], np.int32)
        rb = keep(fc["rho_b"], np.float64)
        ub = keep(fc["U_b"], np.float64)
        tb = keep(fc["T_b"], np.float64)
        pb = keep(fc.get("p_b", np.zeros(len(fc["T_b"]))), np.float64)
        self.bc = BC(ptr(pt, C.c_int32), ptr(rb), ptr(ub), ptr(tb), ptr(pb))
        opt = Options()
        self.lib.dugks_default_options(C.byref(opt))
        opt.precision = precision
        opt.ls_weighting = ls_weighting
        opt.device = device
        opt.tile_cells = tile_cells
        opt.dv_chunks = dv_chunks
        if macro_flux is None:
            macro_flux = getattr(case, "macro_flux", False)
        opt.macro_flux = 1 if macro_flux else 0
        h = C.c_void_p()
        if getattr(case, "dv_w", None) is not None:
            dxi, dw = case.dv_set()
            dxi = keep(dxi.reshape(-1), np.float64)
            dw = keep(dw, np.float64)
            self.dv_list = DVList(len(dw), ptr(dxi), ptr(dw), case.xi_max)
            if shard is not None and shard.use_nccl:
                _load_torch_nccl()
            st = self.lib.dugks_create_dv_list(C.byref(self.mesh), C.byref(self.dv_list), C.byref(self.gas),
                                               C.byref(self.bc), C.byref(opt),
                                               C.byref(shard) if shard is not None else None, C.byref(h))
        elif shard is None:
            st = self.lib.dugks_create(C.byref(self.mesh), C.byref(self.dv), C.byref(self.gas), C.byref(self.bc),
                                       C.byref(opt), C.byref(h))
        else:
            if shard.use_nccl:
                _load_torch_nccl()
            st = self.lib.dugks_create_sharded(C.byref(self.mesh), C.byref(self.dv), C.byref(self.gas),
                                               C.byref(self.bc), C.byref(opt), C.byref(shard), C.byref(h))
        self.h = h
        if st != 0:
            msg = self.lib.dugks_last_error(h).decode() if h.value else "dugks_create failed"
            self.close()
            raise DugksError(st, msg)
        self.n_dv = self.lib.dugks_n_dv(self.h)
        first, nloc = C.c_int32(), C.c_int32()
        self._check(self.lib.dugks_dv_range(self.h, C.byref(first), C.byref(nloc)))
        self.dv_first, self.n_dv_local = first.value, nloc.value
        self.set_macros(case.rho0, case.U0, case.T0)

    def _check(self, st):
        if st != 0:
            raise DugksError(st, self.lib.dugks_last_error(self.h).decode())

    def set_macros(self, rho, U, T):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        U = np.ascontiguousarray(U, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        self._check(self.lib.dugks_set_macros(self.h, ptr(rho), ptr(U), ptr(T)))

    def evolution(self, dt: float):
        self.step(1, dt)

    def step(self, n: int, dt):
        dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (n,)))
        self._check(self.lib.dugks_step(self.h, n, ptr(dts)))

    def step_adaptive(self, n: int, dt: float, max_co: float, max_delta_t: float = 1e300):
        """n steps with the adjustable time step (setDeltaTvar); dt is the
        last step's time step.  Returns (last dt, array of the n dts)."""
        ad = Adapt(max_co, max_delta_t)
        d = C.c_double(dt)
        hist = np.zeros(max(n, 1))
        self._check(self.lib.dugks_step_adaptive(self.h, n, C.byref(ad), C.byref(d), ptr(hist)))
        return d.value, hist[:n]

    def shard_phase(self, phase: int, dt: float = 0.0) -> tuple[int, int]:
        """dugks_shard_phase: (device address, count) of the doubles the host
        sums over all shards after phases 0 and 1; (0, 0) after phase 2."""
        p, n = _dp(), C.c_int64()
        self._check(self.lib.dugks_shard_phase(self.h, phase, dt, C.byref(p), C.byref(n)))
        return (C.cast(p, C.c_void_p).value or 0, n.value) if phase < 2 else (0, 0)

    def step_timed(self, n: int, dt) -> np.ndarray:
        """n steps with CUDA events around every stage: [passA, face combine,
        passB, cell combine, total] milliseconds summed over the steps."""
        dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (n,)))
        out = np.zeros(5)
        self._check(self.lib.dugks_step_timed(self.h, n, ptr(dts), ptr(out)))
        return out

    def layout(self) -> dict:
        """dugks_layout: cells per tile, tiles and DV chunks the handle uses."""
        t, n, c = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self.lib.dugks_layout(self.h, C.byref(t), C.byref(n), C.byref(c)))
        return {"tile_cells": t.value, "n_tiles": n.value, "dv_chunks": c.value}

    def kernel_launches(self) -> int:
        return int(self.lib.dugks_kernel_launches(self.h))

    def last_step_ms(self) -> float:
        v = C.c_double()
        self._check(self.lib.dugks_last_step_ms(self.h, C.byref(v)))
        return v.value

    def get_co_num(self, dt: float):
        a, b = C.c_double(), C.c_double()
        self._check(self.lib.dugks_co_num(self.h, dt, C.byref(a), C.byref(b)))
        return a.value, b.value

    def macros(self) -> dict:
        n = self.case.n_cells
        rho, T = np.zeros(n), np.zeros(n)
        U, q = np.zeros((n, 3)), np.zeros((n, 3))
        self._check(self.lib.dugks_get_macros(self.h, ptr(rho), ptr(U), ptr(T), ptr(q)))
        return {"rho": rho, "U": U, "T": T, "q": q}

    def face_macros(self) -> dict:
        nF = self.case.flat["n_internal"] + self.case.flat["n_boundary"]
        rho, T = np.zeros(nF), np.zeros(nF)
        U, q = np.zeros((nF, 3)), np.zeros((nF, 3))
        self._check(self.lib.dugks_get_face_macros(self.h, ptr(rho), ptr(U), ptr(T), ptr(q)))
        return {"rho": rho, "U": U, "T": T, "q": q}

    def boundary_rho(self) -> np.ndarray:
        out = np.zeros(self.case.flat["n_boundary"])
        self._check(self.lib.dugks_get_boundary_rho(self.h, ptr(out)))
        return out

    def df(self, cells) -> tuple[np.ndarray, np.ndarray]:
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        g = np.zeros((len(cells), self.n_dv_local))
        hh = np.zeros((len(cells), self.n_dv_local))
        self._check(self.lib.dugks_get_df(self.h, ptr(cells, C.c_int32), len(cells), ptr(g), ptr(hh)))
        return g, hh

    def state(self) -> tuple[np.ndarray, np.ndarray]:
        g = np.zeros((self.n_dv_local, self.case.n_cells))
        hh = np.zeros((self.n_dv_local, self.case.n_cells))
        self._check(self.lib.dugks_get_state(self.h, ptr(g), ptr(hh)))
        return g, hh

    def set_state(self, g, hh, dt_prev: float, record=None):
        """Load g~, h~; with the step record of the run that produced them
        the next steps continue bit for bit."""
        g = np.ascontiguousarray(g, dtype=np.float64)
        hh = np.ascontiguousarray(hh, dtype=np.float64)
        self._check(self.lib.dugks_set_state(self.h, ptr(g), ptr(hh), dt_prev))
        if record is not None:
            rec = np.ascontiguousarray(record, dtype=np.float64)
            if rec.size != self.lib.dugks_step_record_size(self.h):
                raise ValueError("step record of another mesh")
            self._check(self.lib.dugks_set_step_record(self.h, ptr(rec)))

    def step_record(self) -> np.ndarray:
        """Per-cell rho, U, T, q, tau and the Courant sums of the last step
        (dugks_get_step_record)."""
        rec = np.zeros(self.lib.dugks_step_record_size(self.h))
        self._check(self.lib.dugks_get_step_record(self.h, ptr(rec)))
        return rec

    def adjoint(self, n_steps: int, dt: float, energy_weight=None, momentum_weight=None, window_start: int = 0,
                max_snapshots: int = 64) -> dict:
        """dugks_adjoint_run: the objective J (boundary energy and momentum
        flux averaged over steps window_start .. n_steps-1 of a fixed-dt run
        from the current state) and its gradient with respect to the T and U
        patch values of every boundary face and muRef.  The solver's state is
        left where it started.  Returns J, dT_b [nb], dU_b [nb, 3], dmu and
        the run's statistics."""
        nb = self.case.flat["n_boundary"]
        ew = None if energy_weight is None else np.ascontiguousarray(np.reshape(energy_weight, nb), dtype=np.float64)
        mw = None if momentum_weight is None else np.ascontiguousarray(np.reshape(momentum_weight, 3 * nb),
                                                                         dtype=np.float64)
        obj = Objective(ptr(ew), ptr(mw), int(n_steps), int(window_start), float(dt), int(max_snapshots))
        J, dmu = C.c_double(), C.c_double()
        dT, dU = np.zeros(nb), np.zeros((nb, 3))
        stats = AdjointStats()
        self._check(self.lib.dugks_adjoint_run(self.h, C.byref(obj), C.byref(J), ptr(dT), ptr(dU), C.byref(dmu),
                                               C.byref(stats)))
        return {"J": J.value, "dT_b": dT, "dU_b": dU, "dmu": dmu.value,
                "stats": {k: getattr(stats, k) for k in ("forward_steps", "reverse_steps", "snapshots", "ms_total",
                                                         "ms_forward", "device_bytes")}}

    def boundary_fluxes(self, dt: float) -> np.ndarray:
        """dugks_boundary_fluxes: [n_boundary, 5] mass, momentum (3) and
        energy flux through every boundary face in the next step (along Sf,
        out of the gas); the state does not advance."""
        out = np.zeros((self.case.flat["n_boundary"], 5))
        self._check(self.lib.dugks_boundary_fluxes(self.h, float(dt), ptr(out)))
        return out

    def objective(self, n_steps: int, dt: float, energy_weight=None, momentum_weight=None,
                  window_start: int = 0) -> tuple[float, dict]:
        """dugks_objective_run: J of a forward run of n_steps (the solver
        advances) and the run's statistics."""
        nb = self.case.flat["n_boundary"]
        ew = None if energy_weight is None else np.ascontiguousarray(np.reshape(energy_weight, nb), dtype=np.float64)
        mw = None if momentum_weight is None else np.ascontiguousarray(np.reshape(momentum_weight, 3 * nb),
                                                                         dtype=np.float64)
        obj = Objective(ptr(ew), ptr(mw), int(n_steps), int(window_start), float(dt), 1)
        J = C.c_double()
        stats = AdjointStats()
        self._check(self.lib.dugks_objective_run(self.h, C.byref(obj), C.byref(J), C.byref(stats)))
        return J.value, {"ms_total": stats.ms_total, "device_bytes": stats.device_bytes}

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.dugks_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent solvers stepped together through one CUDA graph
    (dugks_batch_create / dugks_batch_step); solvers[i] steps with dt[i]."""

    def __init__(self, solvers, dt):
        self.lib = load()
        self.solvers = list(solvers)
        hs = (C.c_void_p * len(self.solvers))(*[s.h.value for s in self.solvers])
        self._dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(self.solvers),)))
        b = C.c_void_p()
        st = self.lib.dugks_batch_create(hs, len(self.solvers), ptr(self._dt), C.byref(b))
        self.b = b
        if st != 0:
            msg = self.lib.dugks_batch_last_error(b).decode() if b.value else "dugks_batch_create failed"
            self.close()
            raise DugksError(st, msg)

    def step(self, n: int):
        st = self.lib.dugks_batch_step(self.b, n)
        if st != 0:
            raise DugksError(st, self.lib.dugks_batch_last_error(self.b).decode())

    def last_ms(self) -> float:
        v = C.c_double()
        self.lib.dugks_batch_last_ms(self.b, C.byref(v))
        return v.value

    def graph_kernels(self) -> int:
        return int(self.lib.dugks_batch_graph_kernels(self.b))

    def close(self):
        if getattr(self, "b", None) is not None and self.b.value:
            self.lib.dugks_batch_destroy(self.b)
        self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune_batch(cases, dt, precision: int = FP32C, tiles=(0, 96, 64), chunk_scales=(0.25, 0.5, 1.0, 2.0),
               steps: int = 4, warmup: int = 2, device: int = 0):
    """Autotuner of the batched launch.  Every candidate is a cell count per
    tile (0: the automatic 128, shrunk to fit) and a factor on each case's
    automatic DV-chunk count; it is measured as what it will run as -- the
    whole batch of cases in one graph, CUDA-event time of `steps` steps after
    `warmup` -- and the fastest wins.  Returns (best, table): best holds the
    tile and scale and the per-case Solver keyword arguments, table every
    candidate's milliseconds per step."""
    dts = np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(cases),))
    table = []
    best = None
    for tile in tiles:
        base = [Solver(c, precision=precision, device=device, tile_cells=tile) for c in cases]
        auto = [s.layout()["dv_chunks"] for s in base]
        for scale in chunk_scales:
            if scale == 1.0:
                solvers = base
            else:
                solvers = [Solver(c, precision=precision, device=device, tile_cells=tile,
                                  dv_chunks=max(1, int(round(scale * a)))) for c, a in zip(cases, auto)]
            kwargs = [{"tile_cells": tile, "dv_chunks": s.layout()["dv_chunks"]} for s in solvers]
            b = Batch(solvers, dts)
            b.step(warmup)
            b.step(steps)
            ms = b.last_ms() / steps
            b.close()
            table.append({"tile_cells": tile, "chunk_scale": scale, "ms_per_step": ms})
            if best is None or ms < best["ms_per_step"]:
                best = {"tile_cells": tile, "chunk_scale": scale, "ms_per_step": ms, "solver_kwargs": kwargs}
            if solvers is not base:
                for s in solvers:
                    s.close()
        for s in base:
            s.close()
    return best, table

