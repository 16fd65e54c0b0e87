"""Check the adjoint gradient dΔP/dγ against central finite differences.

    PYTHONPATH=coldplate-solver_b200 python -m coldplate_b200.fdcheck \
        [--ny 256 --nx 512 --seed 0 --cells 32 --h 1e-4]

Works on the density workload of ``cases.density_field`` (FP64 form,
pressureSolverType 4).  The base state is run until the full-system
pressure drop is stationary to ``--stationary`` (relative change over 100
outer iterations) or ``--base-iters``; the adjoint gradient is taken there.

Each finite difference restarts two solves from the base state, one with
the cell's γ raised by h and one with it lowered by h, and steps them in
lockstep until the DIFFERENCE D = ΔP(+h) - ΔP(-h) is stationary to
``--dtol`` (relative change over 100 iterations).  On large grids the SIMPLE
iteration has a slow tail (at 2048 x 1024 ΔP still moves by about 2e-9 per
100 iterations after 12,000 iterations), so neither solve converges to the
1e-13 that an h = 1e-4 difference of raw pressure drops would need.  The
tail is common to both solves and cancels in D, which converges much
sooner.  Cells are drawn with a seeded generator from γ in [0.05, 0.95], at
least 3 cells from the walls and away from the inlet and outlet buffers.
Beside the central difference it reports the one-sided quotients.  Where
velocities sit on the reference's +-3 U_in clamp the pressure drop is only
piecewise smooth in gamma: the one-sided slopes can differ by several per
cent however small h is (a kink), the central difference is their average,
and a derivative exists only in the generalised sense; the check then
reports whether the adjoint lies between the one-sided slopes.  Prints one
line per cell and a JSON summary line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import cases
from .solver import Simple


def run_stationary(s: Simple, tol: float, max_iter: int, chunk: int = 100) -> tuple[float, int, float]:
    """Iterate until |ΔP_k - ΔP_{k-100}| <= tol |ΔP_k|; returns (ΔP, iterations, last relative change)."""
    done = 0
    rel = float("inf")
    while done < max_iter:
        s.step(chunk)
        h = s.history()["fullTotal"]
        done = len(h)
        if done > 100:
            rel = abs(h[-1] - h[-101]) / max(abs(h[-1]), 1e-300)
            if rel <= tol:
                break
    h = s.history()["fullTotal"]
    return float(h[-1]), len(h), rel


def pick_cells(gamma: np.ndarray, k: int, rng, margin: int = 3, buffer: int = 32) -> list[tuple[int, int]]:
    Ny, Nx = gamma.shape
    b = min(buffer, Nx // 8) + 2
    ok = np.zeros_like(gamma, dtype=bool)
    ok[margin + max(1, Ny // 128):Ny - margin - max(1, Ny // 128), b:Nx - b] = True
    ok &= (gamma >= 0.05) & (gamma <= 0.95)
    cand = np.argwhere(ok)
    idx = rng.choice(len(cand), size=min(k, len(cand)), replace=False)
    return [tuple(int(x) for x in cand[q]) for q in idx]


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cells", type=int, default=32)
    ap.add_argument("--h", type=float, default=1e-4)
    ap.add_argument("--stationary", type=float, default=1e-13)
    ap.add_argument("--base-iters", type=int, default=6000)
    ap.add_argument("--fd-iters", type=int, default=6000)
    ap.add_argument("--dtol", type=float, default=1e-7)
    ap.add_argument("--adjoint-tol", type=float, default=1e-10)
    a = ap.parse_args(argv)

    case = cases.density_field(a.ny, a.nx, seed=a.seed, pressureSolverType=4, maxPressureIter=30, pTol=1e-6)
    gamma = 1.0 - case.cellType
    cap = max(a.base_iters, a.fd_iters) + 200
    prm = case.params(precision="fp64", maxIterations=cap + 10, epsilon=1e-30, historyCapacity=cap + 10)
    t0 = time.time()
    with Simple(gamma=gamma, **prm) as base:
        J0, n0, rel0 = run_stationary(base, a.stationary, a.base_iters)
        grad, rep = base.adjoint_dp_dgamma(max_iter=5000, tol=a.adjoint_tol)
        state = {f: base.get(f) for f in ("u", "v", "p")}
    print(f"base: dP {J0:.12g} Pa after {n0} iterations (stationary {rel0:.1e}); adjoint {rep['iterations']} "
          f"iterations, residual {rep['residual']:.1e}, {rep['device_ms']:.0f} ms", flush=True)
    rng = np.random.default_rng(a.seed + 1)
    cells = pick_cells(gamma, a.cells, rng)
    scale = float(np.abs(grad).max())
    rows = []
    with Simple(gamma=gamma, **prm) as sp, Simple(gamma=gamma, **prm) as sm, Simple(gamma=gamma, **prm) as s0:
        for (i, j) in cells:
            for s, sgn in ((sp, 1.0), (sm, -1.0), (s0, 0.0)):
                g = gamma.copy()
                g[i, j] += sgn * a.h
                s.set_gamma(g)
                for f, v in state.items():
                    s.set(f, v)
                s.reset_loop()
            n, drel = 0, float("inf")
            while n < a.fd_iters:
                for s in (sp, sm, s0):
                    s.step(100)
                hp, hm, h0 = (s.history()["fullTotal"] for s in (sp, sm, s0))
                D = hp - hm
                n = len(D)
                if n > 100:
                    drel = abs(D[-1] - D[-101]) / max(abs(D[-1]), 1e-300)
                    if drel <= a.dtol:
                        break
            fd = D[-1] / (2.0 * a.h)
            # one-sided quotients against the unperturbed solve stepped alongside
            fwd, bwd = (hp[-1] - h0[-1]) / a.h, (h0[-1] - hm[-1]) / a.h
            kink = abs(fwd - bwd) / max(abs(fd), 1e-300)
            inside = min(fwd, bwd) - 1e-6 * abs(fd) <= grad[i, j] <= max(fwd, bwd) + 1e-6 * abs(fd)
            err = abs(fd - grad[i, j])
            rel_err = err / max(abs(fd), 1e-300)
            rows.append(dict(cell=[i, j], gamma=float(gamma[i, j]), fd=fd, fwd=fwd, bwd=bwd, kink=kink,
                             adjoint=float(grad[i, j]), adjoint_between_one_sided=bool(inside),
                             rel_err=rel_err, err_over_scale=err / scale, iters=n, d_stationary=drel))
            print(f"cell ({i:4d},{j:4d}) gamma {gamma[i, j]:.3f}: fd {fd: .6e} adjoint {grad[i, j]: .6e} "
                  f"rel err {rel_err:.1e}; one-sided {fwd: .4e} / {bwd: .4e} (kink {kink:.1e}, adjoint "
                  f"{'inside' if inside else 'OUTSIDE'}); iters {n}, D stationary {drel:.1e}", flush=True)
    rel = np.array([r["rel_err"] for r in rows])
    sig = np.array([abs(r["fd"]) >= 1e-2 * scale for r in rows])
    out = {"workload": f"density_field {a.nx}x{a.ny} seed {a.seed}", "cells": len(rows), "h": a.h,
           "dp_pa": J0, "base_iterations": n0, "adjoint_iterations": rep["iterations"],
           "max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
           "max_fd_iters": int(max(r["iters"] for r in rows)),
           "smooth_cells": int(sum(r["kink"] <= 1e-3 for r in rows)),
           "max_rel_err_smooth_cells": max([r["rel_err"] for r in rows if r["kink"] <= 1e-3], default=None),
           "adjoint_between_one_sided": int(sum(r["adjoint_between_one_sided"] for r in rows)),
           "adjoint_residual": rep["residual"],
           "max_d_stationary": float(max(r["d_stationary"] for r in rows)),
           "max_rel_err_significant": float(rel[sig].max()) if sig.any() else None,
           "significant_cells": int(sig.sum()), "max_err_over_scale": float(max(r["err_over_scale"] for r in rows)),
           "wall_s": time.time() - t0}
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
