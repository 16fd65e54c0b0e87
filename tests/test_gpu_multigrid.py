"""The multigrid-preconditioned CG (pressureSolverType 4, the reference's GPU
default) solves the same pressure-correction system as the reference's PCG:
compared with a direct sparse solve of that system assembled on the host
from dE, dN and the mass imbalance (pressure_solver.cpp:706-742)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from _helpers import gpu_for, oracle_for, rel_l2, small_cases

pytestmark = pytest.mark.gpu


def pressure_system(dE, dN, uS, vS, rho, hx, hy):
    """Assemble the reference's pressure-correction matrix and rhs on
    i in [1, M-1], j in [1, N-2] (M+1 = rows of dE)."""
    M = dE.shape[0] - 1
    N = dE.shape[1]
    nI, nJ = M - 1, N - 2
    idx = lambda i, j: (i - 1) * nJ + (j - 1)
    rows, cols, vals = [], [], []
    b = np.zeros(nI * nJ)
    for i in range(1, M):
        for j in range(1, N - 1):
            aE = rho * dE[i, j] * hy
            aW = rho * dE[i, j - 1] * hy if j > 1 else 0.0
            aN = rho * dN[i, j] * hx if i < M - 1 else 0.0
            aS = rho * dN[i - 1, j] * hx if i > 1 else 0.0
            aP = aE + aW + aN + aS
            if aP < 1e-20:
                aP = 1.0
            k = idx(i, j)
            rows.append(k); cols.append(k); vals.append(aP)
            if j + 1 <= N - 2:
                rows.append(k); cols.append(idx(i, j + 1)); vals.append(-aE)
            if j > 1:
                rows.append(k); cols.append(idx(i, j - 1)); vals.append(-aW)
            if i < M - 1:
                rows.append(k); cols.append(idx(i + 1, j)); vals.append(-aN)
            if i > 1:
                rows.append(k); cols.append(idx(i - 1, j)); vals.append(-aS)
            b[k] = rho * uS[i, j - 1] * hy - rho * uS[i, j] * hy + rho * vS[i - 1, j] * hx - rho * vS[i, j] * hx
    A = sp.csr_matrix((vals, (rows, cols)), shape=(nI * nJ, nI * nJ))
    return A, b, nI, nJ


@pytest.mark.parametrize("name", ["straight", "network", "density"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_multigrid_pcg_solves_the_pressure_system(name, prec):
    case = small_cases()[name]
    o = oracle_for(case)
    o.run(15)
    o.momentum(True)
    o.momentum(False)
    dE, dN, uS, vS = o.get("dE"), o.get("dN"), o.get("uStar"), o.get("vStar")
    A, b, nI, nJ = pressure_system(dE, dN, uS, vS, 1000.0, case.hx, case.hy)
    x = spl.spsolve(A.tocsc(), b)
    tol = 1e-13 if prec == "fp64" else 1e-7     # relative to ||b|| for types 2 / 4
    with gpu_for(case, pressureSolverType=4, maxPressureIter=200, pTol=tol, precision=prec) as g:
        for f, a in (("dE", dE), ("dN", dN), ("uStar", uS), ("vStar", vS)):
            g.set(f, a)
        it, _ = g.solvePressureSystem()
        ps = g.get("pStar")[1:-1, 1:-2].reshape(-1)
    if prec == "fp64":
        assert it < 200
    assert rel_l2(ps, x) <= (1e-8 if prec == "fp64" else 1e-3), (it, rel_l2(ps, x))


def test_multigrid_and_jacobi_pcg_reach_the_same_fixed_point():
    """Solver type changes the path, not the converged pressure drop."""
    case = small_cases()["density"]
    out = {}
    for t in (1, 4):
        with gpu_for(case, pressureSolverType=t, maxPressureIter=400, pTol=1e-14, maxIterations=3000,
                     epsilon=1e-14) as g:
            g.step(3000)
            out[t] = g.history()["fullTotal"][-1]
    assert abs(out[4] - out[1]) <= 1e-7 * abs(out[1]), out


@pytest.mark.parametrize("ptol", [1e-3, 1e-6])
def test_multigrid_pcg_stops_on_the_relative_residual(ptol):
    """Types 2 / 4 take pTol as AMGCL's CG does: stop after the first
    iteration with ||b - A x|| <= pTol ||b|| and report the iterations done."""
    case = small_cases()["density"]
    o = oracle_for(case)
    o.run(15)
    o.momentum(True)
    o.momentum(False)
    dE, dN, uS, vS = o.get("dE"), o.get("dN"), o.get("uStar"), o.get("vStar")
    A, b, nI, nJ = pressure_system(dE, dN, uS, vS, 1000.0, case.hx, case.hy)

    def solve(max_it):
        with gpu_for(case, pressureSolverType=4, maxPressureIter=max_it, pTol=ptol, precision="fp64") as g:
            for f, a in (("dE", dE), ("dN", dN), ("uStar", uS), ("vStar", vS)):
                g.set(f, a)
            it, _ = g.solvePressureSystem()
            x = g.get("pStar")[1:-1, 1:-2].reshape(-1)
        return it, np.linalg.norm(b - A @ x) / np.linalg.norm(b)

    it, rel = solve(200)
    assert 1 <= it < 200 and rel <= ptol * 1.001, (it, rel)
    if it > 1:
        it2, rel2 = solve(it - 1)
        assert it2 == it - 1 and rel2 > ptol * 0.999, (it2, rel2)


def test_smoothed_aggregation_cycle_matches_its_oracle():
    """pressureSolverType 4 runs smoothed aggregation (3 x 3 aggregates,
    9-point Galerkin levels, weights 2/3 and 0.8, V(1,1) with Jacobi 0.9):
    the GPU's FP64 CG iteration count equals that of the same cycle in the
    oracle (oracle/pressure_sa.py) on a 512 x 256 density state, whose
    hierarchy has two grid-wide levels and CTA levels below."""
    from coldplate_b200 import cases
    from pressure_sa import Level, galerkin, pcg, pressure_stencil, vcycle
    case = cases.density_field(256, 512, seed=0)
    o = oracle_for(case, pressureSolverType=1, maxPressureIter=200)
    o.run(30)
    o.momentum(True)
    o.momentum(False)
    dE, dN, uS, vS = o.get("dE"), o.get("dN"), o.get("uStar"), o.get("vStar")
    A, b, nI, nJ = pressure_system(dE, dN, uS, vS, 1000.0, case.hx, case.hy)
    St = pressure_stencil(dE, dN, 1000.0, case.hx, case.hy)
    levels, Al = [], St
    while Al[(0, 0)].size > 64:
        lv = Level(Al, 2.0 / 3.0 if not levels else 0.8)
        levels.append(lv)
        Al = galerkin(lv)
    levels.append(Level(Al, None))
    _, it_o = pcg(St, b.reshape(nI, nJ), lambda r: vcycle(levels, r, 0.9), tol=1e-6, maxit=200)
    with gpu_for(case, pressureSolverType=4, maxPressureIter=200, pTol=1e-6, precision="fp64") as g:
        for f, a in (("dE", dE), ("dN", dN), ("uStar", uS), ("vStar", vS)):
            g.set(f, a)
        it, _ = g.solvePressureSystem()
        x = g.get("pStar")[1:-1, 1:-2].reshape(-1)
    assert len(levels) >= 4 and it_o <= 20
    assert abs(it - it_o) <= 1, (it, it_o)
    assert np.linalg.norm(b - A @ x) <= 1e-6 * 1.001 * np.linalg.norm(b)
