"""The adjoint gradient on the density workload (cases.density_field) at
converged states, against central finite differences (h = 1e-4) of
converged FP64 solves restarted from the base state and stepped until the
difference is stationary (coldplate_b200.fdcheck): within 1e-4 relative on
every checked cell, seeded cells with gamma in [0.05, 0.95] away from the
walls and the inlet and outlet buffers.

256 x 128: no velocity on the clamp; the AUTO model is the equations model.
The inner solves run to pTol 1e-12 and momentumTol 1e-14 so that the
iteration reaches its fixed point exactly (the fixed point does not depend
on them); with pTol 1e-6 and the default momentum tolerance the state keeps
wandering by about 1e-6 Pa of dP, about 1e-4 of the FD difference.

512 x 256: thousands of velocities sit on the +-3 max(U_in, 0.1) clamp once
the iteration has reached its fixed point (about 50,000 outer iterations);
AUTO takes the fixed-point model.
"""
import numpy as np
import pytest

from coldplate_b200 import Simple, cases
from coldplate_b200.fdcheck import FiniteDifferences, clamped_unknowns, pick_cells, run_stationary

pytestmark = pytest.mark.gpu

TOL = 1e-4
TIGHT = dict(pTol=1e-12, maxPressureIter=200, momentumTol=1e-14, maxMomentumIter=50)


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    return built_lib


def _check(ny, nx, ncells, base_iters, fd_iters, stationary, dtol, model, min_clamped, **knobs):
    kw = dict(pressureSolverType=4, maxPressureIter=30, pTol=1e-6)
    kw.update(knobs)
    case = cases.density_field(ny, nx, seed=0, **kw)
    gamma = 1.0 - case.cellType
    cap = max(base_iters, fd_iters) + 200
    prm = case.params(precision="fp64", maxIterations=cap + 10, epsilon=1e-30, historyCapacity=cap + 10)
    with Simple(gamma=gamma, **prm) as base:
        J0, n0, rel0 = run_stationary(base, stationary, base_iters)
        grad, rep = base.adjoint_dp_dgamma(max_iter=20000, tol=1e-11)
        state = {f: base.get(f) for f in ("u", "v", "p")}
        nclamp = clamped_unknowns(base, 3.0 * max(abs(case.U), 0.1))
    assert rel0 <= stationary, (n0, rel0)
    assert rep["converged"] and rep["model"] == model, rep
    assert nclamp >= min_clamped, nclamp
    cells = pick_cells(gamma, ncells, np.random.default_rng(1))
    out = []
    with FiniteDifferences(gamma, prm, state) as fdc:
        for (i, j) in cells:
            r = fdc.cell(i, j, 1e-4, dtol, fd_iters)
            fd, fwd, bwd, adj = r["fd"], r["fwd"], r["bwd"], float(grad[i, j])
            out.append(dict(cell=(i, j), fd=fd, adjoint=adj, rel=abs(adj - fd) / abs(fd), fwd=fwd, bwd=bwd,
                            case="smooth" if abs(fwd - bwd) <= 1e-2 * abs(fd) else "kink: one-sided slopes differ",
                            fd_iters=r["iters"], d_stationary=r["d_stationary"]))
    print(out)
    assert all(o["d_stationary"] <= dtol for o in out), out
    bad = [o for o in out if not o["rel"] <= TOL]
    assert not bad, (bad, out)


def test_density_256x128_equations_model():
    _check(128, 256, 32, 4000, 4000, 1e-14, 1e-10, model=1, min_clamped=0, **TIGHT)


def test_density_512x256_fixed_point_model():
    _check(256, 512, 2, 60000, 20000, 1e-13, 1e-8, model=2, min_clamped=1000)
