#!/usr/bin/env python
"""Time-to-converge of the B200 SIMPLE solver on the 2048 x 1024 density
workload: mixed precision vs FP64 on the GPU, with the reference's CPU path
timed beside it.

One "step" is one full solve from the initial state to the outer iteration
after which the full-system pressure drop stays within 1e-5 (relative) of
the converged FP64 value dP*.  dP* and the iteration counts k64 / kmix are
found first by untimed calibration runs (FP64 and mixed, each run until the
pressure drop is stationary).  The timed steps then run exactly kmix (mixed)
and k64 (FP64) outer iterations from a reset state; value = mixed seconds.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank solves its own replica (seed + rank): the
path does not shard, so the replicas run independently with no collective
on the data path; the line reports the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "coldplate-solver_b200"))

METRIC = "time-to-converge 2048×1024 (ΔP rel err ≤1e-5): mixed vs FP64 GPU; adjoint/fwd"
DP_TOL = 1e-5
# outer iterations of the FP64 solve of the default workload (2048 x 1024,
# seed 0), measured by this script's calibration run on a B200; used only by
# the reference arm, which has no GPU run to count them from
DEFAULT_K64 = 153
# the pressure solver of the timed workload: pressureSolverType 4 with the
# reference's default pTol and maxPressureIter (SIMPLE.h); type 4 is the
# reference's AMG-CG (relative tolerance), here multigrid-PCG
BENCH_KNOBS = dict(pressureSolverType=4, maxPressureIter=30, pTol=1e-6)
# adjoint: relative residual of the adjoint system; at 2048 x 1024, 1e-6
# leaves the gradient within 3e-5 (relative) of a 1e-11 solve on every cell
# whose gradient is above 1% of the largest
ADJ_TOL = 1e-6
ADJ_MAX_ITER = 2000
# ncu captures of the dominant kernels (profiles/): DRAM bytes read + written
PCG_MG_CAPTURE_BYTES = (850.3 + 1406.4) * 1e6     # k_pcg_mg<float>, one launch
PCG_MG_CAPTURE_ITERS = 30
THERMAL_CAPTURE_BYTES_PER_CELL_ITER = 702.0        # k_th_bicgstab, 512 x 256 x 12 capture


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ny", type=int, default=1024)
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--max-iter", type=int, default=3000)
    ap.add_argument("--cpu-sample-iters", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-fields", type=int, default=64)
    ap.add_argument("--batch-outer", type=int, default=200)
    ap.add_argument("--no-thermal", action="store_true")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def flush_l2(torch):
    """Write 512 MB (> 126 MB L2) between timed solves."""
    buf = torch.empty(64 * 1024 * 1024, dtype=torch.float64, device="cuda")
    buf.fill_(1.0)
    torch.cuda.synchronize()
    del buf


def first_stable_iter(dp: np.ndarray, dp_star: float, tol: float = DP_TOL) -> int:
    """1-based count of iterations after which |dP_k - dP*| <= tol |dP*| for all k."""
    bad = np.nonzero(np.abs(dp - dp_star) > tol * abs(dp_star))[0]
    return int(bad[-1] + 2) if bad.size else 1


def calibrate(Simple, case, prec: str, max_iter: int):
    """Untimed run until the full pressure drop is stationary (relative
    change over 200 iterations below 1e-9, or residual epsilon 1e-12)."""
    prm = case.params(precision=prec, maxIterations=max_iter, epsilon=1e-14, historyCapacity=max_iter,
                      chunk=100)
    with Simple(cellType=case.cellType, **prm) as g:
        done = 0
        while done < max_iter:
            rep = g.step(100)
            done = rep["iter"]
            h = g.history()
            dp = h["fullTotal"]
            if rep["done"]:
                break
            if len(dp) > 400 and abs(dp[-1] - dp[-201]) <= 1e-9 * abs(dp[-1]):
                break
        h = g.history()
    return h


# ------------------------------------------------------------------ CPU baseline
def cpu_baseline(case, n_iter: int, k_converge: int) -> dict | None:
    """The reference's own CPU path (oracle/_ref/ref_f32, built from its
    sources) on this workload, all host threads, a bounded sample of outer
    iterations; time-to-converge extrapolated with the FP64 iteration count.
    Without AMGCL the reference runs pressureSolverType 4 as its Jacobi-PCG
    (SIMPLE.cpp:167-185), which needs far more outer iterations than k, so
    the extrapolation is a lower bound on its time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import REF_DIR, write_case
    cores = os.cpu_count() or 1
    exe = os.path.join(REF_DIR, "ref_f32")
    # without AMGCL the reference resolves pressureSolverType 4 to its PCG
    # at load time (SIMPLE.cpp:167-185)
    prm = case.params(maxIterations=n_iter, epsilon=1e-30, pressureSolverType=1)
    if os.path.exists(exe):
        from oracle import ref_overrides
        with tempfile.TemporaryDirectory() as d:
            write_case(d, case.cellType, case.hy, case.hx, case.U, case.Ht)
            out = subprocess.run([exe, d, d, *ref_overrides(prm, threads=cores), "time_only=1"],
                                 capture_output=True, text=True, timeout=3600).stdout
        secs = [float(l.split()[2]) for l in out.splitlines() if l.startswith("ITER")]
        kind, used = "reference", cores
    else:
        from oracle import Oracle
        o = Oracle("f32", prm, cellType=case.cellType, hy=case.hy, hx=case.hx, U=case.U, Ht=case.Ht)
        secs = []
        for _ in range(n_iter):
            t = time.perf_counter()
            o.run(1)
            secs.append(time.perf_counter() - t)
        kind, used = "port", 1
    if not secs:
        return None
    s_per_it = float(np.mean(secs[1:] if len(secs) > 1 else secs))
    return {"value": s_per_it * k_converge, "unit": "s", "cores": used, "kind": kind,
            "sample": f"{len(secs)} outer iterations of the same workload, {s_per_it:.3f} s each, "
                      f"extrapolated to {k_converge} iterations (lower bound: without AMGCL the "
                      f"reference's pressure solver is Jacobi-PCG)",
            "s_per_outer_iteration": s_per_it}


# ------------------------------------------------------------------ reference arm
def reference_arm(args, case, rank: int):
    if rank != 0:
        return
    k = DEFAULT_K64
    if k is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "outer-iteration count of this workload not yet measured on a B200"}))
        return
    times = []
    for s in range(args.warmup + args.steps):
        cb = cpu_baseline(case, max(1, args.cpu_sample_iters), k)
        if cb is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU build missing"}))
            return
        if s >= args.warmup:
            times.append(cb)
    v = float(np.mean([t["value"] for t in times]))
    line = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"density_field {args.nx}x{args.ny} seed {args.seed}"},
            "impl": "reference",
            "cpu_baseline": {k2: times[-1][k2] for k2 in ("kind", "cores", "sample")} | {"value": v, "unit": "s"},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------ ranks
def replica_seed(seed: int, rank: int) -> int:
    """Each rank solves its own replica of the workload (the path does not
    shard): the density field of seed + rank."""
    return seed + rank


def max_over_ranks(x: float, dist, device: str) -> float:
    """The job's time is its slowest replica's: max of x over the ranks (one
    all-reduce, which every rank calls at the same point)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ batched solves
BATCH_SINGLE_OUTER = 20


def batch_leg(Simple, torch, args) -> dict:
    """--batch-fields density fields (64 by default: Nx in 256-1024, Ny in
    128-512, U_in in 0.2-1.0 m/s, mixed precision, epsilon 1e-6) advanced by
    the batched kernel for --batch-outer outer iterations (200) with the
    autotuned tile, against the same
    fields solved one after the other (BATCH_SINGLE_OUTER iterations each).
    Most of these fields never reach epsilon 1e-6 with the reference's SIMPLE
    iteration (their residual RMS levels off near 1e-5), so the leg times a
    fixed number of iterations and reports cell-iterations per second."""
    from coldplate_b200 import Batch, cases
    nf, nout = args.batch_fields, args.batch_outer
    cs = cases.batch(nf, seed=args.seed, **BENCH_KNOBS)
    cells = [c.cellType.shape[0] * c.cellType.shape[1] for c in cs]
    prm = dict(precision="mixed", epsilon=1e-6, maxIterations=nout, historyCapacity=nout)
    fields = [Simple(cellType=c.cellType, **c.params(**prm)) for c in cs]
    try:
        with Batch(fields) as b:
            tune = b.autotune(3)
            flush_l2(torch)
            torch.cuda.synchronize()
            rep = b.run(nout)
            its = [len(f.history()["iter"]) for f in fields]
    finally:
        for f in fields:
            f.close()
    work = float(sum(n * k for n, k in zip(cells, its)))
    t = rep["device_ms"] / 1e3
    # the same fields solved alone (one context, cp_step) for a few iterations each
    t1, work1 = 0.0, 0.0
    for c, n in zip(cs, cells):
        with Simple(cellType=c.cellType, **c.params(**{**prm, "maxIterations": BATCH_SINGLE_OUTER + 2})) as s:
            r = s.step(BATCH_SINGLE_OUTER)
            t1 += r["device_ms"] / 1e3
            work1 += n * BATCH_SINGLE_OUTER
    return {"workload": f"{nf} density fields, Nx 256-1024, Ny 128-512, U_in 0.2-1.0 m/s, seed {args.seed}, "
                        f"mixed, {nout} outer iterations",
            "cells": int(sum(cells)), "t_s": t, "launches": rep["launches"],
            "tile": [rep["tileRows"], rep["tileCols"]], "autotune_trial_ms": tune["device_ms"],
            "cell_iterations_per_s": work / t,
            "sequential_single_cell_iterations_per_s": work1 / t1,
            "speedup_vs_sequential": (work / t) / (work1 / t1),
            "fields_done": rep["fieldsDone"]}


# ------------------------------------------------------------------ 3-D thermal solve + p-norm adjoint
THERMAL_FLOW_ITERS = 300
THERMAL_P = 8.0
THERMAL_STEPS = 3


def thermal_leg(Simple, torch, args) -> dict:
    """The conjugate-heat-transfer solve on a 1024 x 512 density flow (mixed
    precision, THERMAL_FLOW_ITERS outer iterations, untimed): 1024 x 512 x 12
    cells (8 base-plate + 4 channel layers, cases.THERMAL_3D), hotspot power
    map, the reference's rtol 1e-6; then the p-norm (p = 8) adjoint
    gradient.  Device times from CUDA events on the solver's stream; e2e
    through the public calls with host arrays (inputs up, T back)."""
    from coldplate_b200 import Thermal, cases
    from coldplate_b200.thermal import inputs_from_flow
    Ny, Nx = 512, 1024
    c = cases.density_field(Ny, Nx, seed=args.seed, **BENCH_KNOBS)
    with Simple(cellType=c.cellType, **c.params(precision="mixed", maxIterations=THERMAL_FLOW_ITERS + 2,
                                                 epsilon=1e-30)) as s:
        s.step(THERMAL_FLOW_ITERS)
        fl = inputs_from_flow(s, c.cellType)
    q0 = cases.power_map(Ny, Nx, args.seed) * 1e4
    prm = dict(Nx=Nx, Ny=Ny, dx=c.hx, dy=c.hy, rtol=1e-6, maxiter=5000, **cases.THERMAL_3D)
    n = Nx * Ny * (prm["nz_solid"] + prm["nz_fluid"])
    levels, a, b = 1, Nx, Ny              # 2 x 2 column aggregates down to one column
    while a > 1 or b > 1:
        a, b, levels = (a + 1) // 2, (b + 1) // 2, levels + 1
    fwd, adj = [], []
    with Thermal(**prm) as th:
        th.set_inputs(q0=q0, **fl)
        for k in range(args.warmup + THERMAL_STEPS):
            flush_l2(torch)
            torch.cuda.synchronize()
            r = th.solve()
            flush_l2(torch)
            torch.cuda.synchronize()
            J, g, ra = th.pnorm_gradient(THERMAL_P)
            if k >= args.warmup:
                fwd.append(r)
                adj.append(ra)
        tb_max, _ = th.objective(THERMAL_P)
        # end to end: host inputs up, solve, T and the objective back
        e2e = []
        for k in range(1 + THERMAL_STEPS):
            flush_l2(torch)
            t0 = time.perf_counter()
            th.set_inputs(q0=q0, **fl)
            th.solve()
            T = th.T
            th.objective(THERMAL_P)
            if k >= 1:
                e2e.append(time.perf_counter() - t0)
    t_f = max(r["device_ms"] for r in fwd) / 1e3
    t_a = max(r["device_ms"] for r in adj) / 1e3
    its_f = max(r["iterations"] for r in fwd)
    its_a = max(r["iterations"] for r in adj)
    # algorithmic bytes per cell and BiCGStab iteration, FP64 words, every
    # vector and coefficient once per phase that needs it: level 0 85.5 (the
    # two vector updates fused with pre-smoothing, 8 and 7; two residual
    # restrictions, 9.25 each; two prolongation + post-smoothing sweeps, 12
    # each; two operator applications, 10 each; the solution update, 8) and
    # the coarse levels 18.7 (27.25 / 4 per V-cycle, twice, times 4/3)
    bytes_iter = 104 * 8 * n
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = bytes_iter * its_f / t_f / 1e9
    return {"workload": f"density flow 1024x512 seed {args.seed} ({THERMAL_FLOW_ITERS} mixed SIMPLE iterations) "
                        f"-> 1024x512x12 CHT (8 plate + 4 channel layers), hotspot power map, rtol 1e-6, "
                        f"p-norm p={THERMAL_P:g}",
            "cells": n, "t_forward_s": t_f, "forward_iterations": its_f,
            "t_adjoint_s": t_a, "adjoint_iterations": its_a, "adjoint_over_forward": t_a / t_f,
            "Tb_max_C": tb_max, "Tb_pnorm_C": J, "max_abs_dJ_dgamma": float(np.abs(g).max()),
            "residual_forward": max(r["residual"] for r in fwd),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "kernel": "k_th_bicgstab<false> (assembly and factorisation inside the time)",
                         "traffic": THERMAL_CAPTURE_BYTES_PER_CELL_ITER * n * its_f,
                         "algorithmic_bytes": bytes_iter * its_f,
                         "traffic_source": "ncu capture at 512x256x12 (10 iterations), scaled by cells x iterations; "
                                           "L2 holds more of the smaller case, so this is a lower bound",
                         "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
            "e2e": {"value": float(np.mean(e2e)), "unit": "s", "h2d_bytes_per_step": int(4 * 8 * Nx * Ny),
                    "d2h_bytes_per_step": int(T.nbytes + 16)},
            # launches: assembly, fill, a Galerkin coarsening per coarse level, a
            # z-factorisation per level, the persistent solver; the adjoint adds
            # the p-norm, its right-hand side and the sensitivity
            "multigrid_levels": levels,
            "gpu_launches_per_forward": 2 + (levels - 1) + levels + 1,
            "gpu_launches_per_adjoint": 2 + levels + 1 + 1}


# ------------------------------------------------------------------ our arm
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    from coldplate_b200 import cases
    case = cases.density_field(args.ny, args.nx, seed=replica_seed(args.seed, rank), **BENCH_KNOBS)
    if args.impl == "reference":
        return reference_arm(args, case, rank)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from coldplate_b200 import Simple, build
    build.build()

    # ---- calibration (untimed): dP*, k64, kmix
    hmx = calibrate(Simple, case, "mixed", args.max_iter)
    h64 = calibrate(Simple, case, "fp64", args.max_iter)
    dp_star = float(h64["fullTotal"][-1])
    k64 = first_stable_iter(h64["fullTotal"], dp_star)
    kmix = first_stable_iter(hmx["fullTotal"], dp_star)
    dp_mix_final = float(hmx["fullTotal"][-1])

    # ---- timed solves (device time, CUDA events inside cp_step)
    def timed_solves(prec: str, k: int, n_warm: int, n_steps: int, adjoint: bool = False):
        """Forward solves of k outer iterations from a reset state; with
        adjoint=True each is followed by the adjoint gradient at its state."""
        prm = case.params(precision=prec, maxIterations=k + 10, epsilon=1e-30, historyCapacity=k + 10,
                          chunk=max(32, min(k, 512)))
        out, adj = [], []
        with Simple(cellType=case.cellType, **prm) as g:
            for s in range(n_warm + n_steps):
                g.reset()
                flush_l2(torch)
                if dist:
                    dist.barrier()
                torch.cuda.synchronize()
                rep = g.step(k)
                torch.cuda.synchronize()
                if adjoint:
                    flush_l2(torch)
                    _, arep = g.adjoint_dp_dgamma(max_iter=ADJ_MAX_ITER, tol=ADJ_TOL)
                if s >= n_warm:
                    out.append(rep["device_ms"] / 1e3)
                    if adjoint:
                        adj.append(arep)
            dp_end = g.history()["fullTotal"][k - 1]
        return out, dp_end, adj

    with ClockSampler(local) as clk:
        t_mix, dp_mix_k, adj_reps = timed_solves("mixed", kmix, args.warmup, args.steps, adjoint=True)
        t_64, dp_64_k, _ = timed_solves("fp64", k64, 1, 1)
    clocks = clk.summary()
    t_mixed = max(t_mix)
    t_adj = max(r["device_ms"] for r in adj_reps) / 1e3
    t_mixed = max_over_ranks(t_mixed, dist, "cuda")

    # ---- per-kernel device times and the roofline of the dominant kernel
    prm = case.params(precision="mixed", maxIterations=100000, epsilon=1e-30, historyCapacity=100000)
    with Simple(cellType=case.cellType, **prm) as g:
        g.step(50)
        kt = g.kernel_times(20)
    nP = (args.ny) * (args.nx - 1)
    w_mix = 4
    pcg_ms = kt["ms"]["pcg"] / max(kt["launches"]["pcg"], 1)
    pcg_iters = kt["pcgIterations"] / max(kt["launches"]["pcg"], 1)
    # 23 w per unknown per multigrid-PCG iteration: 8 w for the CG vectors
    # (read x, r, p, dE, dN; write x, r, p) and 15 w for the V(1,1) cycle
    # (fine-level restriction and prolongation-smoothing, 11.25 w, times 4/3
    # for the coarse levels)
    pcg_bytes = pcg_iters * 23 * w_mix * nP
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = pcg_bytes / (pcg_ms * 1e-3) / 1e9
    # DRAM traffic of one launch from the ncu capture of this kernel on this
    # workload (profiles/k_pcg_mg_float_density_2048x1024.md: 850.3 + 1406.4 MB
    # for a launch of 30 CG iterations, taken with 16 x 64 float tiles; the
    # 32 x 64 tiles read the same arrays with less halo), scaled to this
    # line's CG iterations
    traffic = PCG_MG_CAPTURE_BYTES * pcg_iters / PCG_MG_CAPTURE_ITERS
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "algorithmic_bytes": pcg_bytes, "kernel": "k_pcg_mg<float>",
                "traffic_source": "ncu capture (2048x1024, 30 CG iterations) scaled by CG iterations",
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}

    # ---- batched solves: 64 density fields of random size in one persistent kernel
    batch_line = None
    if not args.no_batch:
        batch_line = batch_leg(Simple, torch, args)

    # ---- 3-D thermal solve and its p-norm adjoint on a 1024 x 512 density flow
    thermal_line = None
    if not args.no_thermal:
        thermal_line = thermal_leg(Simple, torch, args)

    # ---- end to end through the public API with host buffers
    e2e_t = []
    gamma_host = torch.from_numpy(1.0 - case.cellType).pin_memory().numpy()
    prm = case.params(precision="mixed", maxIterations=kmix + 10, epsilon=1e-30, historyCapacity=kmix + 10,
                      chunk=max(32, min(kmix, 512)))
    with Simple(cellType=case.cellType, **prm) as g:
        for s in range(1 + args.steps):
            flush_l2(torch)
            t0 = time.perf_counter()
            g.reset()
            g.set_gamma(gamma_host)
            g.step(kmix)
            p = g.get("p")
            u = g.get("u")
            v = g.get("v")
            dp = g.history()["fullTotal"][-1]
            t1 = time.perf_counter()
            if s >= 1:
                e2e_t.append(t1 - t0)
    h2d = gamma_host.nbytes
    d2h = p.nbytes + u.nbytes + v.nbytes + 8

    if rank == 0:
        cb = None if args.no_cpu_baseline else cpu_baseline(case, args.cpu_sample_iters, k64)
        iters_per_launch = 8
        line = {
            "metric": METRIC, "value": t_mixed, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_mixed * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner / f64 fields+reductions",
            "data": "synthetic",
            "config": {"workload": f"density_field {args.nx}x{args.ny} seed {args.seed} (SOU, 2.5-D, "
                                   f"Brinkman alpha_max 1e9, q 0.1, U_in {case.U} m/s)",
                       "flush": "512 MB L2 flush before every timed solve",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "t_fp64_s": max(t_64), "t_mixed_s": t_mixed, "mixed_over_fp64": t_mixed / max(t_64),
            "adjoint": {"t_s": t_adj, "over_forward_mixed": t_adj / t_mixed, "over_forward_fp64": t_adj / max(t_64),
                        "iterations": int(max(r["iterations"] for r in adj_reps)),
                        "residual": float(max(r["residual"] for r in adj_reps)), "tol": ADJ_TOL,
                        "solver": "FGMRES(30), transposed-SIMPLE preconditioner, FP64 Krylov vectors"},
            "k_fp64": k64, "k_mixed": kmix, "dp_star_pa": dp_star,
            "dp_rel_err_mixed_final": abs(dp_mix_final - dp_star) / abs(dp_star),
            "dp_rel_err_mixed_at_k": abs(dp_mix_k - dp_star) / abs(dp_star),
            "dp_rel_err_fp64_at_k": abs(dp_64_k - dp_star) / abs(dp_star),
            "calibration_iters": {"fp64": int(len(h64["fullTotal"])), "mixed": int(len(hmx["fullTotal"]))},
            "kernel_ms_per_outer_iteration": {k2: v2 / max(kt["iterations"], 1) for k2, v2 in kt["ms"].items()},
            "pcg_iterations_per_outer": pcg_iters,
            "jacobi_sweeps_per_outer": kt["jacobiSweeps"] / max(kt["iterations"], 1),
            "roofline": roofline,
            "cpu_baseline": cb,
            "e2e": {"value": float(np.mean(e2e_t)), "unit": "s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "batch": batch_line,
            "thermal": thermal_line,
            "clocks": clocks,
            "gpu_launches": int((args.steps) * kmix * iters_per_launch),
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
