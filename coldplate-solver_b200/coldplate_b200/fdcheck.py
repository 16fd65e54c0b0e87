"""Check the adjoint gradient dΔP/dγ against central finite differences.

    PYTHONPATH=coldplate-solver_b200 python -m coldplate_b200.fdcheck \
        [--case density|constricted] [--ny 256 --nx 512 --seed 0 --cells 32 --h 1e-4]
        [--ptol 1e-6 --momentum-tol T --max-momentum-iter K]

Works on the density workload of ``cases.density_field`` (or the
constricted channel of ``cases.constricted_channel``), FP64 form,
pressureSolverType 4.  The base state is run until the full-system pressure
drop is stationary to ``--stationary`` (relative change over 100 outer
iterations) or ``--base-iters``; the adjoint gradient is taken there.

Each finite difference restarts two solves from the base state, one with
the cell's γ raised by h and one with it lowered by h, and steps them in
lockstep with an unperturbed solve until the DIFFERENCE D = ΔP(+h) - ΔP(-h)
is stationary to ``--dtol`` (relative change over 100 iterations).

Where the flow has faces with zero flux (a jet's symmetry plane, stagnant
corners; the clamped passages of the reference's +-3 max(U_in, 0.1) velocity
clamp create them), the upwind switch of those faces, and the clamp of face
averages between clamped velocities, sit exactly on their kink: the +h and
-h solves take different branches there, so the one-sided quotients against
the base differ by a term that does not shrink with h, while their average,
the central difference, is the mean of the branches' derivatives, which the
adjoint takes at such faces.  The tool reports both; the adjoint is compared
with the central difference.

The inner solves' tolerances (``--ptol``, ``--momentum-tol`` and their
iteration caps) do not move the fixed point, but with loose ones the
iteration may never settle on it: at 256 x 128 with pTol 1e-6 and the
default momentum tolerance, the state keeps wandering by about 1e-6 Pa of
ΔP (the pressure and momentum stop rules switch between counts from one
outer iteration to the next), which is about 1e-4 of the difference D at
h = 1e-4.  With pTol 1e-12 and momentumTol 1e-14 it reaches its fixed point
exactly (the same ΔP to 2e-12) and D is stationary to the bit.  Cells are
drawn with a seeded generator from γ in
[0.05, 0.95], at least 3 cells from the walls and away from the inlet and
outlet buffers.  Prints one line per cell and a JSON summary line.
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


def clamped_unknowns(s: Simple, maxVel: float) -> int:
    """Velocity unknowns at the clamp bound in the current state."""
    M, N = s.M, s.N
    u, v = s.get("u")[1:M, 1:N - 1], s.get("v")[1:M - 1, 1:N]
    return int((np.abs(u) >= maxVel * (1 - 1e-12)).sum() + (np.abs(v) >= maxVel * (1 - 1e-12)).sum())


class FiniteDifferences:
    """Three solvers (gamma + h, gamma - h, gamma) restarted from one base
    state for each cell and stepped in lockstep."""

    def __init__(self, gamma: np.ndarray, prm: dict, state: dict):
        self.gamma, self.state = gamma, state
        self.s = [Simple(gamma=gamma, **prm) for _ in range(3)]

    def close(self):
        for s in self.s:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def cell(self, i: int, j: int, h: float, dtol: float, max_iter: int) -> dict:
        for s, sgn in zip(self.s, (1.0, -1.0, 0.0)):
            g = self.gamma.copy()
            g[i, j] += sgn * h
            s.set_gamma(g)
            for f, v in self.state.items():
                s.set(f, v)
            s.reset_loop()
        n, drel = 0, float("inf")
        while n < max_iter:
            for s in self.s:
                s.step(100)
            hp, hm, h0 = (s.history()["fullTotal"] for s in self.s)
            D = hp - hm
            n = len(D)
            if n > 100:
                drel = abs(D[-1] - D[-101]) / max(abs(D[-1]), 1e-300)
                if drel <= dtol:
                    break
        return {"fd": D[-1] / (2.0 * h), "fwd": (hp[-1] - h0[-1]) / h, "bwd": (h0[-1] - hm[-1]) / h,
                "iters": n, "d_stationary": drel}


def make_case(name: str, ny: int, nx: int, seed: int, **knobs):
    """The FD workloads, FP64 form, pressureSolverType 4; `knobs` override
    the inner tolerances (pTol, maxPressureIter, momentumTol, ...)."""
    kw = dict(pressureSolverType=4, maxPressureIter=30, pTol=1e-6)
    kw.update(knobs)
    if name == "constricted":
        return cases.constricted_channel(ny, nx, **kw)
    return cases.density_field(ny, nx, seed=seed, **kw)


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--case", choices=["density", "constricted"], default="density")
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
    ap.add_argument("--adjoint-model", type=int, default=0, help="cp_adjoint_model: 0 auto, 1 equations, 2 fixed point")
    ap.add_argument("--ptol", type=float, default=1e-6)
    ap.add_argument("--max-pressure-iter", type=int, default=30)
    ap.add_argument("--momentum-tol", type=float, default=None, help="default: the SIMPLE.h value")
    ap.add_argument("--max-momentum-iter", type=int, default=None, help="default: the SIMPLE.h value")
    a = ap.parse_args(argv)

    knobs = dict(pTol=a.ptol, maxPressureIter=a.max_pressure_iter)
    if a.momentum_tol is not None:
        knobs["momentumTol"] = a.momentum_tol
    if a.max_momentum_iter is not None:
        knobs["maxMomentumIter"] = a.max_momentum_iter
    case = make_case(a.case, a.ny, a.nx, a.seed, **knobs)
    gamma = 1.0 - case.cellType
    cap = max(a.base_iters, a.fd_iters) + 200
    prm = case.params(precision="fp64", maxIterations=cap + 10, epsilon=1e-30, historyCapacity=cap + 10,
                      adjointModel=a.adjoint_model)
    t0 = time.time()
    with Simple(gamma=gamma, **prm) as base:
        J0, n0, rel0 = run_stationary(base, a.stationary, a.base_iters)
        grad, rep = base.adjoint_dp_dgamma(max_iter=20000, tol=a.adjoint_tol)
        state = {f: base.get(f) for f in ("u", "v", "p")}
        nclamp = clamped_unknowns(base, 3.0 * max(abs(case.U), 0.1))
    print(f"base: dP {J0:.12g} Pa after {n0} iterations (stationary {rel0:.1e}), {nclamp} velocities on the "
          f"clamp; adjoint (model {rep['model']}) {rep['iterations']} iterations, residual {rep['residual']:.1e}, "
          f"{rep['device_ms']:.0f} ms", flush=True)
    rng = np.random.default_rng(a.seed + 1)
    cells = pick_cells(gamma, a.cells, rng, buffer=32 if a.case == "density" else 8)
    scale = float(np.abs(grad).max())
    rows = []
    with FiniteDifferences(gamma, prm, state) as fdc:
        for (i, j) in cells:
            r = fdc.cell(i, j, a.h, a.dtol, a.fd_iters)
            fd, fwd, bwd = r["fd"], r["fwd"], r["bwd"]
            err = abs(fd - grad[i, j])
            rel_err = err / max(abs(fd), 1e-300)
            rows.append(dict(cell=[i, j], gamma=float(gamma[i, j]), adjoint=float(grad[i, j]), rel_err=rel_err,
                             err_over_scale=err / scale, **r))
            print(f"cell ({i:4d},{j:4d}) gamma {gamma[i, j]:.3f}: fd {fd: .6e} adjoint {grad[i, j]: .6e} "
                  f"rel err {rel_err:.1e}; one-sided {fwd: .4e} / {bwd: .4e}; iters {r['iters']}, "
                  f"D stationary {r['d_stationary']:.1e}", flush=True)
    rel = np.array([r["rel_err"] for r in rows])
    sig = np.array([abs(r["fd"]) >= 1e-2 * scale for r in rows])
    out = {"workload": f"{a.case} {a.nx}x{a.ny} seed {a.seed}", "cells": len(rows), "h": a.h,
           "dp_pa": J0, "base_iterations": n0, "clamped_velocities": nclamp,
           "adjoint_iterations": rep["iterations"], "adjoint_residual": rep["residual"], "adjoint_model": rep["model"],
           "max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
           "max_rel_err_significant": float(rel[sig].max()) if sig.any() else None,
           "significant_cells": int(sig.sum()), "max_err_over_scale": float(max(r["err_over_scale"] for r in rows)),
           "max_fd_iters": int(max(r["iters"] for r in rows)),
           "max_d_stationary": float(max(r["d_stationary"] for r in rows)),
           "wall_s": time.time() - t0}
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
