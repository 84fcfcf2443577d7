"""Benchmark of the B200 DUGKS step (dugksFoam fvDVM::evolution).

Default workload: flow past a sphere on a cubed-sphere mesh (6 x 24 x 24 x
32 cells = 110,592, radial stretch 1.12, r in [1, 10]), 16^3 Gauss-Hermite
DVs (4,096), far field at Ma 0.5, Kn 0.1 on the diameter, isothermal diffuse
wall; FP64.  Synthetic mesh and initial state (uniform free stream).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  Multi-GPU, by default replicas (every rank
advances its own copy of the workload; the step has no cross-rank
exchange), so value = all ranks' cell-DV updates / the slowest rank's time,
weak scaling.  --dv-shard splits one workload's DV rows over the ranks
instead (NCCL all-reduce of the raw face and cell moments, two per step):
value = the workload's cell-DV updates / the slowest rank's time, strong
scaling.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "psp-vst_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "cell·DV updates/s: FP32-comp vs FP64 at ≤1e-6 macro rel-L2; % HBM peak; adjoint"
UNIT = "cell·DV updates/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["ball", "cavity", "cube", "batch", "adjoint"], default="ball",
                   help="batch: 64 seeded cavities of uneven size through one CUDA graph (FP32c), "
                        "against the same cases stepped one at a time")
    p.add_argument("--precision", choices=["fp64", "fp32c"], default=None,
                   help="default fp64; fp32c for --workload batch")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp32c", action="store_true")
    p.add_argument("--no-adjoint", action="store_true", help="skip the short adjoint measurement of the default run")
    p.add_argument("--no-batch", action="store_true", help="skip the short batch measurement of the default run")
    p.add_argument("--no-cube", action="store_true",
                   help="skip the mixed-precision sub-line of the default run (64^3 cube, 20^3 DVs, FP64 and FP32c)")
    p.add_argument("--cube-steps", type=int, default=40,
                   help="steps after which the cube sub-line compares FP32c with FP64")
    p.add_argument("--cpu-sample-ndv", type=int, default=8, help="1-D DV count of the CPU baseline sample")
    p.add_argument("--ndv1d", type=int, default=0, help="override the 1-D DV count (profiling of small cases)")
    p.add_argument("--ball-m", type=int, default=24,
                   help="--workload ball: cells per cube-face edge (profiling of small cases; default 24)")
    p.add_argument("--ball-nr", type=int, default=32, help="--workload ball: radial cells (default 32)")
    p.add_argument("--cube-n", type=int, default=64, help="--workload cube: cells per side")
    p.add_argument("--kn", type=float, default=0.1, help="--workload cube: Knudsen number")
    p.add_argument("--tune", action="store_true",
                   help="--workload batch: pick tile size and DV-chunk scale with the batch autotuner first")
    p.add_argument("--fd-dirs", type=int, default=0,
                   help="--workload adjoint: central-difference checks on this many random directions")
    p.add_argument("--adjoint-n", type=int, default=0,
                   help="--workload adjoint: cavity side (default 128), or the ball's cells per cube-face edge")
    p.add_argument("--adjoint-case", choices=["cavity", "ball"], default="cavity",
                   help="--workload adjoint: the lid-driven cavity, or far-field flow past the sphere")
    p.add_argument("--dv-shard", action="store_true",
                   help="N>1: shard the DV rows of one workload over the ranks (NCCL) instead of replicas")
    a = p.parse_args()
    if a.precision is None:
        a.precision = "fp32c" if a.workload == "batch" else "fp64"
    return a


def build_case(name, ndv1d=0, cube_n=64, kn=0.1, geometry=None, ball_m=24, ball_nr=32):
    """The workload's case and its config description.  geometry: a
    function of the PolyMesh giving its cell and face geometry (default:
    the library's dugks_mesh_geometry; the reference arm passes the
    oracle's restatement, which gives the same numbers bit for bit)."""
    from dugks_b200 import case as cs
    if name == "ball":
        c = cs.ball_case(ball_m, ball_nr, 1.12, ndv1d or 16, kn=0.1, mach=0.5, flatten=False)
        cfg = {"workload": f"ball: cubed sphere 6x{ball_m}x{ball_m}x{ball_nr} ({6 * ball_m * ball_m * ball_nr} cells), "
                           f"stretch 1.12, r 1..10, {ndv1d or 16}^3 GH DVs, far field Ma 0.5, Kn 0.1 (diameter), "
                           "diffuse isothermal wall"}
    elif name == "cube":
        c = cs.cube_case(cube_n, ndv1d or 20, kn=kn, flatten=False)
        cfg = {"workload": f"cube: {cube_n}^3 lid-driven cube, {ndv1d or 20}^3 GH DVs, Kn {kn}, lid 50 m/s"}
    else:
        c = cs.cavity_case(61, ndv1d or 28, flatten=False)
        cfg = {"workload": "cavity: 61x61 lid-driven cavity, 28^2 GH DVs, Kn 0.075, lid 50 m/s"}
    c.flatten(geometry(c.mesh) if geometry is not None else None)
    cfg["cells"] = c.n_cells
    cfg["n_dv"] = c.n_dv
    cfg["dt"] = c.dt
    cfg["cfl"] = 0.5
    return c, cfg


def state_arrays(case) -> int:
    """DF arrays a step must move per (cell, DV): g and h, or g alone when h
    is identically zero (D = 3 and KInner = 0 make K + 3 - D = 0 in every
    formula that feeds h, and the library's passes then carry g alone)."""
    return 1 if case.D == 3 and int(case.gas.get("K", 0)) == 0 else 2


def run_config(cfg, precision, world, shard, nv_loc, nc):
    """The config object both arms print for the same workload."""
    rs = 8 if precision == "fp64" else 4
    return dict(cfg, precision=precision,
                parallelism=f"dv-shard x{world} (NCCL all-reduce of raw moments)" if shard
                else f"replicas x{world}",
                l2="inputs larger than L2 (state %.2f GB per GPU)" % (2 * rs * nc * nv_loc / 1e9))


def profiled_traffic(kernel: str, precision: str):
    """DRAM bytes per cell.DV update of a pass kernel, from the committed
    ncu summary of the same kernel with the same 16^3 DV set on a smaller
    cubed sphere (6 x 16^3 = 24,576 cells; the full launch is too large to
    capture; traffic per update is set by the tile layout, alike on both
    meshes), or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_ball24576_dv4096_{precision}.md")
    try:
        with open(path) as f:
            for ln in f:
                if ln.startswith("traffic_bytes_per_update:"):
                    return float(ln.split(":")[1])
    except OSError:
        pass
    return None


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_uuid(dev: int):
    try:
        import torch
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


def oracle_rate(case, threads: int, steps: int, warmup: int, xi=None, w=None):
    """cell.DV updates/s and ms per step of the CPU oracle on `case` (or on
    its mesh with the DV set xi, w), `threads` OpenMP threads."""
    import oracle_bind as ob
    o = ob.Oracle(case, threads=threads, xi=xi, w=w)
    for _ in range(warmup):
        o.evolution(case.dt)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.evolution(case.dt)
    t = time.perf_counter() - t0
    n = case.n_cells * o.n_dv * steps
    o.close()
    return n / t, 1e3 * t / steps


def dv_sample(case, n1d: int):
    """A smaller Gauss-Hermite set of the same form for a bounded CPU sample."""
    from dugks_b200 import quadrature
    C = math.sqrt(2.0 * case.gas["R"] * case.gas["Tref"])
    xis, w = quadrature.gauss_hermite_half_range(C, n1d)
    return quadrature.tensor_product(xis, w, case.D)


def oracle_bytes(case, n_dv: int) -> int:
    """Host memory of the oracle's per-(DV, cell) and per-(DV, face) arrays."""
    fl = case.flat
    return 8 * n_dv * (4 * case.n_cells + 2 * (fl["n_internal"] + fl["n_boundary"]))


def host_available_bytes() -> int:
    try:
        return os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        return 0


def cpu_baseline(case_name: str, n1d: int, steps: int, warmup: int, one_thread: bool = True):
    """The CPU restatement of the step (the reference itself cannot be built
    here: it needs OpenFOAM, MPI and legacy TBB) on all host cores, on a
    bounded sample of the workload: the same mesh with an n1d^D DV set; and
    on one thread, as the reference runs each rank (fvDVM.C:41)."""
    import oracle_bind as ob
    c, _ = build_case(case_name, geometry=ob.geometry)
    xi, w = dv_sample(c, n1d)
    cores = os.cpu_count() or 1
    rate, ms = oracle_rate(c, cores, steps, warmup, xi, w)
    out = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"same mesh ({c.n_cells} cells) with a {n1d}^{c.D} = {len(w)}-DV Gauss-Hermite set, "
                     f"{steps} steps after {warmup} warm-up, OpenMP over DVs/faces/cells ({cores} threads)",
           "ms_per_sample_step": ms}
    if one_thread:
        r1, ms1 = oracle_rate(c, 1, 1, 0, xi, w)
        out["single_thread"] = {"value": r1, "unit": UNIT, "cores": 1, "ms_per_sample_step": ms1,
                                "sample": f"the same {len(w)}-DV sample, 1 step, 1 thread (the reference's "
                                          f"NUM_THREADS 1 per rank, fvDVM.C:41)"}
    return out


def max_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    """The largest x over all ranks of the default process group (x itself
    without one): multi-GPU times are the slowest rank's."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world: int, cells: int, dvs: int, steps: int, seconds: float) -> float:
    """Whole-job cell.DV updates/s of `world` replicas that each advanced
    cells x dvs pairs `steps` times, timed by the slowest rank."""
    return world * cells * dvs * steps / seconds


def batch_cases(seed: int = 20261203, n: int = 64):
    """The batched workload: n lid-driven cavities, side N from {32, 48, 64,
    96, 128, 192, 256}, Kn log-uniform in [0.01, 10], lid speed uniform in
    [10, 100] m/s, wall T uniform in [250, 350] K, 28^2 GH DVs; seeded."""
    import numpy as np
    from dugks_b200 import case as cs
    rng = np.random.default_rng(seed)
    sizes = rng.choice([32, 48, 64, 96, 128, 192, 256], size=n)
    kn = 10.0 ** rng.uniform(-2.0, 1.0, size=n)
    lid = rng.uniform(10.0, 100.0, size=n)
    tw = rng.uniform(250.0, 350.0, size=n)
    return [cs.cavity_case(int(N), 28, kn=float(k), u_lid=float(u), T_wall=float(t))
            for N, k, u, t in zip(sizes, kn, lid, tw)]


def run_batch(args):
    """--workload batch on one GPU: aggregate cell.DV updates/s of the
    batched graph, beside the same cases stepped one at a time."""
    import torch
    from dugks_b200 import lib as dl
    torch.cuda.set_device(0)
    prec = dl.FP64 if args.precision == "fp64" else dl.FP32C
    print(json.dumps(batch_line(args.steps, args.warmup, prec, args.tune)), flush=True)


def batch_line(steps: int, warmup: int, prec: int, tune: bool = False) -> dict:
    """The batch of batch_cases() through one CUDA graph, timed with CUDA
    events over `steps` steps after `warmup`; the same cases stepped one at
    a time; end to end with every case's macros to the host; and the
    graph's own cost on cases whose kernels do almost nothing."""
    import torch
    from dugks_b200 import lib as dl
    seed = 20261203
    cases = batch_cases(seed)
    tuning = None
    if tune:
        t0 = time.perf_counter()
        best, table = dl.tune_batch(cases, [c.dt for c in cases], precision=prec)
        tuning = {"chosen": {"tile_cells": best["tile_cells"], "chunk_scale": best["chunk_scale"]},
                  "candidates": table, "tuning_seconds": time.perf_counter() - t0}
        solvers = [dl.Solver(c, precision=prec, **kw) for c, kw in zip(cases, best["solver_kwargs"])]
    else:
        solvers = [dl.Solver(c, precision=prec) for c in cases]
    pairs = sum(c.n_cells * c.n_dv for c in cases)
    K = max(2, steps - steps % 2)
    W = max(4, warmup + warmup % 2)
    batch = dl.Batch(solvers, [c.dt for c in cases])
    batch.step(W)
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_uuid(0))
    sampler.start()
    time.sleep(0.4)
    l0 = sum(s.kernel_launches() for s in solvers)
    batch.step(K)
    launches = sum(s.kernel_launches() for s in solvers) - l0
    clocks = sampler.stop()
    t_ms = batch.last_ms()
    value = pairs * K / (t_ms / 1e3)
    # one at a time: each case's own K steps, CUDA events on its stream
    seq_ms = 0.0
    best = {"value": 0.0, "cells": 0}   # the fastest case alone (the largest cavities)
    for s, c in zip(solvers, cases):
        ms = float(s.step_timed(K, c.dt)[4])
        seq_ms += ms
        r = c.n_cells * c.n_dv * K / (ms / 1e3)
        if r > best["value"]:
            best = {"value": r, "cells": c.n_cells}
    seq = pairs * K / (seq_ms / 1e3)
    # end to end: two steps per call, then every case's macros to the host
    te0 = time.perf_counter()
    for _ in range(K // 2):
        batch.step(2)
        for s in solvers:
            s.macros()
    te = time.perf_counter() - te0
    rs = 8 if prec == dl.FP64 else 4
    peak, peak_kind = measured_peaks()
    # the graph's own cost: the same 64 branches of kernels on 4x4 cavities
    # with 6^2 DVs, whose kernels do almost nothing; its time per step
    # bounds what a persistent kernel over all cases could save
    from dugks_b200 import case as cs
    tiny = [cs.cavity_case(4, 6) for _ in cases]
    tsol = [dl.Solver(c, precision=prec) for c in tiny]
    tb = dl.Batch(tsol, [c.dt for c in tiny])
    tb.step(W)
    tb.step(K)
    floor_ms = tb.last_ms() / K
    floor = {"ms_per_step": floor_ms, "kernels_per_step": tb.graph_kernels() // 2,
             "us_per_kernel": 1e3 * floor_ms / max(1, tb.graph_kernels() // 2),
             "share_of_batch_step": floor_ms / (t_ms / K),
             "workload": "64 cavities of 4x4 cells x 6^2 DVs in the same graph structure"}
    tb.close()
    for s_ in tsol:
        s_.close()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W,
        "ms_per_step": t_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == dl.FP64 else "f32 storage / f64 moments", "data": "synthetic",
        "config": {"workload": "batch: 64 lid-driven cavities, N in {32..256}, Kn log-U[0.01,10], lid U[10,100] m/s, "
                               "T_wall U[250,350] K, 28^2 GH DVs, each at its own CFL-0.5 dt, one CUDA graph "
                               "(a branch per case)",
                   "cases": len(cases), "cells": sum(c.n_cells for c in cases), "pairs": pairs, "seed": seed,
                   "precision": "fp64" if prec == dl.FP64 else "fp32c", "parallelism": "one GPU",
                   "l2": "inputs larger than L2 (state %.2f GB)" % (4 * rs * pairs / 1e9)},
        "one_at_a_time": {"value": seq, "ms_per_step": seq_ms / K, "speedup_of_batch": value / seq,
                          "fastest_case_alone": best},
        "e2e": {"value": pairs * K / te, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": sum(72 * c.n_cells for c in cases) // 2},
        "gpu_launches": launches,
        "graph_kernels_per_two_steps": batch.graph_kernels(),
        "graph_floor": floor,
        "autotune": tuning,
        "step_roofline": {"bytes_per_update": 6 * rs, "achieved": 6 * rs * pairs / (t_ms / K / 1e3) / 1e9,
                          "frac": 6 * rs * pairs / (t_ms / K / 1e3) / 1e9 / peak, "peak": peak,
                          "peak_kind": peak_kind},
        "clocks": clocks,
    }
    batch.close()
    for s_ in solvers:
        s_.close()
    return line


def sphere_loads(solver, case, steps_done):
    """Drag and wall heat flux of the ball after steps_done steps: the
    x-momentum and energy flux of the next step's relaxed DFs through the
    sphere's wall faces (area vectors out of the gas, into the sphere),
    from dugks_boundary_fluxes (the state does not advance)."""
    import numpy as np
    fl = case.flat
    nb = fl["n_boundary"]
    wall = np.zeros(nb, bool)
    for p, t in enumerate(fl["patch_type"]):
        if t == 1:
            wall[fl["patch_start"][p]:fl["patch_start"][p + 1]] = True
    F = solver.boundary_fluxes(case.dt)
    drag, heat = float(F[wall, 1].sum()), float(F[wall, 4].sum())
    area = float(np.linalg.norm(fl["Sf"][fl["n_internal"]:][wall], axis=1).sum())
    return {"after_steps": steps_done, "drag_N": drag, "wall_heat_W": heat, "wall_area_m2": area,
            "mean_wall_heat_flux_W_m2": heat / area, "wall_mass_flux_kg_s": float(F[wall, 0].sum()),
            "note": "fluxes of step %d into the sphere wall" % (steps_done + 1)}


def cube_line(n: int = 64, n1d: int = 20, kn: float = 0.1, steps: int = 40, timed: int = 5, device: int = 0):
    """The mixed-precision configuration on one GPU: lid-driven cube of n^3
    cells, n1d^3 Gauss-Hermite DVs, lid 50 m/s.  FP64 and FP32c (FP32
    deviation storage, FP64 relaxation and moment sums) each advance
    `steps` steps from the same uniform start; steps 3..2+timed are timed
    with CUDA events; then FP32c's rho, U, T, q are compared with FP64's by
    plain relative L2.  The two solvers run one after the other (the FP64
    state and face values take about 160 GB at 64^3 x 20^3)."""
    import numpy as np
    from dugks_b200 import case as cs
    from dugks_b200 import lib as dl
    c = cs.cube_case(n, n1d, kn=kn)
    nc, nv = c.n_cells, c.n_dv
    out = {"workload": f"cube: {n}^3 lid-driven cube, {n1d}^3 GH DVs, Kn {kn}, lid 50 m/s",
           "cells": nc, "n_dv": nv, "dt": c.dt, "steps": steps, "timed_steps": timed}
    peak, peak_kind = measured_peaks()
    mac = {}
    for name, prec, rs in (("fp64", dl.FP64, 8), ("fp32c", dl.FP32C, 4)):
        try:
            s = dl.Solver(c, precision=prec, device=device)
        except dl.DugksError as e:
            out[name] = {"error": str(e)}
            continue
        s.step(2, c.dt)
        st = s.step_timed(timed, c.dt)
        s.step(steps - 2 - timed, c.dt)
        mac[name] = s.macros()
        ms = float(st[4]) / timed
        out[name] = {"value": nc * nv / (ms / 1e3), "ms_per_step": ms,
                     "pass_a_ms": float(st[0]) / timed, "pass_b_ms": float(st[2]) / timed,
                     "step_roofline_frac": 3 * state_arrays(c) * rs * nc * nv / (ms / 1e3) / 1e9 / peak}
        s.close()
        del s
    if "fp64" in mac and "fp32c" in mac:
        a, b = mac["fp32c"], mac["fp64"]
        out["fp32c_rel_l2_vs_fp64"] = {k: float(np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k]))
                                       for k in ("rho", "U", "T", "q")}
        out["fp32c_speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["fp32c"]["ms_per_step"]
    return out


def adjoint_case(n: int = 128, seed: int = 20261203):
    """The adjoint workload: n x n lid-driven cavity, 32^2 GH DVs, Kn 0.1,
    lid 50 m/s, every wall face at its own temperature 273 K + N(0, 5 K)
    (seeded); returns the case and the objective's weights (wall heat flux
    on every wall face, x-momentum flux on the lid) and lid mask."""
    import numpy as np
    from dugks_b200 import case as cs
    c = cs.cavity_case(n, 32, kn=0.1)
    fl = dict(c.flat)
    nb = fl["n_boundary"]
    rng = np.random.default_rng(seed)
    fl["T_b"] = 273.0 + rng.normal(0.0, 5.0, nb)
    c.flat = fl
    lid = np.zeros(nb, bool)
    lid[fl["patch_start"][0]:fl["patch_start"][1]] = True
    fw = np.zeros((nb, 3))
    fw[lid, 0] = 1.0
    return c, np.ones(nb), fw, lid


def run_adjoint(args):
    print(json.dumps(adjoint_line(args)), flush=True)


def adjoint_ball_case(m: int = 8, seed: int = 20261203):
    """The adjoint on a curved mesh: flow past the sphere (cubed sphere 6 x
    m x m x m, stretch 1.12, 8^3 GH DVs, Ma 0.5, Kn 0.1), every wall face at
    its own temperature 273 K + N(0, 5 K) (seeded); objective = heat load
    into the sphere + drag (x-momentum flux into it)."""
    import numpy as np
    from dugks_b200 import case as cs
    c = cs.ball_case(m, m, 1.12, 8, kn=0.1, mach=0.5)
    fl = dict(c.flat)
    nb = fl["n_boundary"]
    wall = np.zeros(nb, bool)
    for p, t in enumerate(fl["patch_type"]):
        if t == 1:
            wall[fl["patch_start"][p]:fl["patch_start"][p + 1]] = True
    rng = np.random.default_rng(seed)
    T_b = np.array(fl["T_b"], dtype=float)
    T_b[wall] = 273.0 + rng.normal(0.0, 5.0, int(wall.sum()))
    fl["T_b"] = T_b
    c.flat = fl
    fw = np.zeros((nb, 3))
    fw[wall, 0] = 1.0
    return c, wall.astype(float), fw, wall


def adjoint_line(args):
    """--workload adjoint on one GPU: forward + reverse steps of the FP64
    adjoint (binomial checkpointing, <= 64 device snapshots), objective
    averaged over the last quarter of the steps; optionally central
    differences (h = 1e-6 relative) of the objective along random
    directions in (512 wall temperatures, lid speed, Kn)."""
    import copy

    import numpy as np
    import torch
    from dugks_b200 import lib as dl
    torch.cuda.set_device(0)
    ball = getattr(args, "adjoint_case", "cavity") == "ball"
    n_side = args.adjoint_n or (8 if ball else 128)
    # lid: the faces whose x velocity is the "speed" parameter (the lid, or the sphere)
    case, hw, fw, lid = adjoint_ball_case(n_side) if ball else adjoint_case(n_side)
    N = max(4, args.steps)
    window = N - N // 4
    snaps = 64
    solver = dl.Solver(case)
    nc, nv = case.n_cells, solver.n_dv
    W = max(3, args.warmup)
    solver.adjoint(W, case.dt, hw, fw, window_start=W - 1, max_snapshots=2)
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_uuid(0))
    sampler.start()
    time.sleep(0.4)
    l0 = solver.kernel_launches()
    r = solver.adjoint(N, case.dt, hw, fw, window_start=window, max_snapshots=snaps)
    launches = solver.kernel_launches() - l0
    clocks = sampler.stop()
    st = r["stats"]
    # the plain forward rate of the same solver, for the cost ratio
    fwd = solver.step_timed(20, case.dt)
    fwd_ms = float(fwd[4]) / 20
    rev_ms = (st["ms_total"] - st["ms_forward"]) / N
    ms_per_step = st["ms_total"] / N
    nb = case.flat["n_boundary"]
    wall_T = case.flat["T_b"]
    mu = case.gas["muRef"]
    grad = {"dJ_dT_wall_l2": float(np.linalg.norm(r["dT_b"])),
            "dJ_dU_lid": float(np.sum(r["dU_b"][lid, 0])),
            "dJ_dKn_relative": float(r["dmu"] * mu)}
    fd = None
    if args.fd_dirs > 0:
        rng = np.random.default_rng(20261204)
        h = 1e-6
        errs = []
        for _ in range(args.fd_dirs):
            dT = rng.normal(size=nb) * wall_T
            dU = rng.normal() * 50.0
            dmu = rng.normal() * mu
            dUb = np.zeros((nb, 3))
            dUb[lid, 0] = dU
            ad = float(r["dT_b"] @ dT + np.sum(r["dU_b"] * dUb) + r["dmu"] * dmu)
            J = []
            for sgn in (1.0, -1.0):
                cc = copy.copy(case)
                cc.flat = dict(case.flat)
                cc.gas = dict(case.gas)
                cc.flat["T_b"] = wall_T + sgn * h * dT
                cc.flat["U_b"] = case.flat["U_b"] + sgn * h * dUb
                cc.gas["muRef"] = mu + sgn * h * dmu
                J.append(dl.Solver(cc).objective(N, case.dt, hw, fw, window_start=window)[0])
            fdv = (J[0] - J[1]) / (2 * h)
            errs.append(abs(fdv - ad) / abs(ad))
        fd = {"directions": args.fd_dirs, "h_relative": h, "max_rel_err": max(errs), "rel_errs": errs}
    solver.close()
    peak, peak_kind = measured_peaks()
    line = {
        "metric": METRIC, "value": nc * nv * N / (st["ms_total"] / 1e3),
        "unit": "cell·DV forward+reverse steps/s", "n_gpus": 1, "steps": N, "warmup": W,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": (f"adjoint: flow past the sphere, cubed sphere 6x{n_side}x{n_side}x{n_side}, 8^3 GH DVs, "
                                f"Ma 0.5, Kn 0.1, {int(lid.sum())} wall faces at 273 K + N(0, 5 K), objective = sphere "
                                f"heat load + drag averaged over the last {N - window} of {N} steps") if ball else
                               (f"adjoint: {n_side}x{n_side} lid-driven cavity, 32^2 GH DVs, Kn 0.1, lid 50 m/s, "
                                f"{nb} wall faces at 273 K + N(0, 5 K), objective = wall heat flux + lid shear "
                                f"averaged over the last {N - window} of {N} steps"),
                   "cells": nc, "dvs": nv, "snapshots": st["snapshots"], "precision": "fp64",
                   "l2": "state %.2f GB, the record and adjoint arrays %.2f GB more"
                         % (16 * nc * nv / 1e9, st["device_bytes"] / 1e9)},
        "J": r["J"], "gradient": grad,
        "adjoint": {"forward_steps_incl_recompute": st["forward_steps"], "ms_forward_total": st["ms_forward"],
                    "reverse_ms_per_step": rev_ms, "forward_ms_per_step": fwd_ms,
                    "adjoint_step_over_forward_step": ms_per_step / fwd_ms,
                    "device_gb": st["device_bytes"] / 1e9},
        "fd_check": fd,
        "gpu_launches": launches,
        "step_roofline": {"bytes_per_update": 48, "achieved": 48 * nc * nv / (ms_per_step / 1e3) / 1e9,
                          "frac": 48 * nc * nv / (ms_per_step / 1e3) / 1e9 / peak, "peak": peak,
                          "peak_kind": peak_kind},
        "clocks": clocks,
    }
    return line


def run_reference(args):
    """The reference arm: the CPU oracle (the reference dugksFoam cannot be
    built here: OpenFOAM, MPI and legacy TBB are absent) on the same
    workload and config as the CUDA arm, W warm-up and K timed steps on all
    host cores.  It loads no library of this repository: the mesh geometry
    comes from the oracle's own restatement.  When the host cannot hold the
    oracle's arrays, or the full DV set would not finish within a few
    minutes, each step is a bounded sample instead (the same mesh with an
    8^D Gauss-Hermite set), and `cpu_baseline.sample` says so."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle_bind as ob
    world = int(os.environ.get("WORLD_SIZE", "1"))
    case, cfg = build_case(args.workload, args.ndv1d, args.cube_n, args.kn, geometry=ob.geometry,
                           ball_m=args.ball_m, ball_nr=args.ball_nr)
    nc, nv = case.n_cells, case.n_dv
    K, W = args.steps, max(3, args.warmup)
    config = run_config(cfg, args.precision, world, args.dv_shard and world > 1, nv, nc)
    cores = os.cpu_count() or 1
    budget_s = 300.0   # warm-up + timed steps of the full workload
    full = oracle_bytes(case, nv) < 0.6 * host_available_bytes()
    rate = ms = None
    if full:
        o = ob.Oracle(case, threads=cores)
        t0 = time.perf_counter()
        o.evolution(case.dt)
        t1 = time.perf_counter() - t0
        if t1 * (W + K - 1) <= budget_s:
            for _ in range(W - 1):
                o.evolution(case.dt)
            t0 = time.perf_counter()
            for _ in range(K):
                o.evolution(case.dt)
            t = time.perf_counter() - t0
            rate, ms = nc * nv * K / t, 1e3 * t / K
            sample = (f"the full workload ({nc} cells x {nv} DVs), {K} steps after {W} warm-up, OpenMP over "
                      f"DVs/faces/cells ({cores} threads)")
        o.close()
        del o
    if rate is None:
        why = "host memory" if not full else "time"
        xi, w = dv_sample(case, 8)
        rate, ms = oracle_rate(case, cores, K, W, xi, w)
        sample = (f"bounded by {why}: same mesh ({nc} cells) with an 8^{case.D} = {len(w)}-DV Gauss-Hermite set "
                  f"per step, {K} steps after {W} warm-up, OpenMP over DVs/faces/cells ({cores} threads)")
    cb = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    xi, w = dv_sample(case, 8)
    r1, ms1 = oracle_rate(case, 1, 1, 0, xi, w)
    cb["single_thread"] = {"value": r1, "unit": UNIT, "cores": 1, "ms_per_sample_step": ms1,
                           "sample": f"same mesh with an 8^{case.D} = {len(w)}-DV set, 1 step, 1 thread (the "
                                     f"reference's NUM_THREADS 1 per rank, fvDVM.C:41)"}
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config, "cpu_baseline": cb,
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "batch":
        if int(os.environ.get("WORLD_SIZE", "1")) > 1:
            raise SystemExit("--workload batch runs on one GPU")
        run_batch(args)
        return
    if args.workload == "adjoint":
        if int(os.environ.get("WORLD_SIZE", "1")) > 1:
            raise SystemExit("--workload adjoint runs on one GPU")
        run_adjoint(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    from dugks_b200 import lib as dl
    case, cfg = build_case(args.workload, args.ndv1d, args.cube_n, args.kn, ball_m=args.ball_m,
                           ball_nr=args.ball_nr)
    prec = dl.FP64 if args.precision == "fp64" else dl.FP32C
    shard = None
    if world > 1 and args.dv_shard:
        from dugks_b200 import shard as sh
        shard = sh.init_nccl_shard(rank, world)
    solver = dl.Solver(case, precision=prec, device=local, shard=shard)
    nv, nc = solver.n_dv, case.n_cells
    nv_loc = solver.n_dv_local
    # whole-job rate: replicas each advance the whole workload; shards share one
    job_rate = (lambda k, sec: nc * nv * k / sec) if shard is not None else \
        (lambda k, sec: replica_rate(world, nc, nv, k, sec))
    K, W = args.steps, max(3, args.warmup)

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up
    solver.step(W, case.dt)
    barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_uuid(local)) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.4)
    l0 = solver.kernel_launches()
    stage = solver.step_timed(K, case.dt)            # CUDA events on the library's stream
    launches = solver.kernel_launches() - l0
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop() if sampler else None
    t_ms = max_over_ranks(float(stage[4]), dist)
    value = job_rate(K, t_ms / 1e3)

    # end to end through the public API with host buffers: each step is
    # fvDVM::evolution (dt passed by value) followed by the copy of the
    # cell macros rho, U, T, q (and tau) back into host fields
    barrier()
    te0 = time.perf_counter()
    for _ in range(K):
        solver.step(1, case.dt)
        solver.macros()
    te = max_over_ranks(time.perf_counter() - te0, dist)
    e2e = job_rate(K, te)

    rs = 8 if prec == dl.FP64 else 4
    arr = state_arrays(case)
    peak, peak_kind = measured_peaks()
    a_ms, b_ms = stage[0] / K, stage[2] / K
    # per-launch figures of this rank's kernels (its DV block)
    if b_ms >= a_ms:
        kname, kbytes, kms = "pass B (face relaxation, flux, update, cell moments)", 2 * arr * rs * nc * nv_loc, b_ms
        tpu = profiled_traffic("k_pass_b", args.precision) if args.workload == "ball" else None
    else:
        kname, kbytes, kms = "pass A (reconstruction, face moments)", arr * rs * nc * nv_loc, a_ms
        tpu = profiled_traffic("k_pass_a", args.precision) if args.workload == "ball" else None
    achieved = kbytes / (kms / 1e3) / 1e9
    traffic = tpu * nc * nv_loc if tpu is not None else None
    step_bytes = 3 * arr * rs * nc * nv_loc
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t_ms / K, "higher_is_better": True, "scaling": "strong" if shard is not None else "weak",
        "vs_baseline": None,
        "dtype": "f64" if prec == dl.FP64 else "f32 storage / f64 moments", "data": "synthetic",
        "config": run_config(cfg, args.precision, world, shard is not None, nv_loc, nc),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 8, "d2h_bytes_per_step": 72 * nc + 16},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": kbytes,
                     "traffic_source": "ncu DRAM read+write per update of the same kernel on a 6x16^3 cubed "
                                       "sphere with the same DV set, times this launch's updates"
                     if traffic is not None else None},
        "step_roofline": {"bytes_per_update": 3 * arr * rs, "h_identically_zero": arr == 1,
                          "achieved": step_bytes / (t_ms / K / 1e3) / 1e9,
                          "frac": step_bytes / (t_ms / K / 1e3) / 1e9 / peak},
        "stage_ms_per_step": {"pass_a": a_ms, "face_combine": stage[1] / K, "pass_b": b_ms,
                              "cell_combine": stage[3] / K},
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_fp32c and prec == dl.FP64:
        # the FP32-compensated path on the same workload, and its macros'
        # rel-L2 against this FP64 run after the same steps
        import numpy as np
        ref = solver.macros()
        steps_done = W + 2 * K
        if args.workload == "ball":
            line["sphere"] = sphere_loads(solver, case, steps_done)
        del solver
        s32 = dl.Solver(case, precision=dl.FP32C, device=local)
        s32.step(W, case.dt)
        st32 = s32.step_timed(K, case.dt)
        s32.step(steps_done - W - K, case.dt)
        m32 = s32.macros()
        rel = {k: float(np.linalg.norm(m32[k] - ref[k]) / np.linalg.norm(ref[k])) for k in ("rho", "U", "T", "q")}
        v32 = nc * nv * K / (st32[4] / 1e3)
        line["fp32c"] = {"value": v32, "ms_per_step": st32[4] / K, "speedup_vs_fp64": v32 / value,
                         "rel_l2_vs_fp64_after_%d_steps" % steps_done: rel,
                         "step_roofline_frac": 3 * 4 * arr * nc * nv / (st32[4] / K / 1e3) / 1e9 / peak}
        del s32
    else:
        del solver
    default_ball = args.workload == "ball" and not args.ndv1d and args.ball_m == 24 and args.ball_nr == 32
    if rank == 0 and world == 1 and not args.no_cube and default_ball:
        # the mixed-precision configuration itself: FP32c against FP64 on the
        # 64^3 x 20^3 cube
        line["cube"] = cube_line(steps=max(8, args.cube_steps), device=local)
    if rank == 0 and world == 1 and not args.no_adjoint and args.workload == "ball":
        # the adjoint configuration (128x128 cavity, 32^2 DVs, FP64) over a
        # short horizon: forward + reverse steps with <= 64 snapshots
        import types
        sub = adjoint_line(types.SimpleNamespace(adjoint_n=128, steps=100, warmup=3, fd_dirs=0))
        line["adjoint"] = {k: sub[k] for k in ("value", "unit", "steps", "ms_per_step", "adjoint", "J", "gradient",
                                                "gpu_launches")}
        line["adjoint"]["workload"] = sub["config"]["workload"]
    if rank == 0 and world == 1 and not args.no_batch and args.workload == "ball":
        # the batched configuration: 64 seeded cavities through one graph,
        # beside the same cases stepped one at a time
        sub = batch_line(8, 4, dl.FP32C)
        line["batch"] = {k: sub[k] for k in ("value", "unit", "steps", "ms_per_step", "one_at_a_time", "e2e",
                                              "gpu_launches", "graph_kernels_per_two_steps", "graph_floor",
                                              "step_roofline", "dtype")}
        line["batch"]["workload"] = sub["config"]["workload"]
        line["batch"]["pairs"] = sub["config"]["pairs"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload, args.cpu_sample_ndv, 2, 1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
