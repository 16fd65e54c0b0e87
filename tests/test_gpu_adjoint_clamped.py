"""The adjoint gradient where the reference's velocity clamp is active.

At the converged state of the constricted channel (cases.constricted_channel)
velocities sit on the +-3 max(U_in, 0.1) clamp.  The adjoint differentiates
the fixed point the reference iteration reaches there (frozen Jacobi sweep
count and clamped set); it must agree with central differences (h = 1e-4) of
converged FP64 forward solves, restarted from the base state and stepped
until the difference is stationary, within 1e-4 relative on every checked
cell.  The one-sided quotients are reported: they differ from each other
because faces with zero flux in the jet behind the gap sit on the upwind
switch (and faces between clamped velocities on the clamp), where the map
has a kink; the central difference and the adjoint take the mean of the two
branches there.
"""
import numpy as np
import pytest

from coldplate_b200 import Simple, cases
from coldplate_b200.fdcheck import FiniteDifferences, clamped_unknowns, pick_cells, run_stationary

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    return built_lib


def _check(case, cells, base_iters, fd_iters, min_clamped):
    gamma = 1.0 - case.cellType
    cap = max(base_iters, fd_iters) + 200
    prm = case.params(precision="fp64", maxIterations=cap + 10, epsilon=1e-30, historyCapacity=cap + 10)
    with Simple(gamma=gamma, **prm) as base:
        J0, n0, rel0 = run_stationary(base, 1e-14, base_iters)
        grad, rep = base.adjoint_dp_dgamma(max_iter=20000, tol=1e-13)
        state = {f: base.get(f) for f in ("u", "v", "p")}
        nclamp = clamped_unknowns(base, 3.0 * max(abs(case.U), 0.1))
    assert nclamp >= min_clamped, nclamp
    assert rep["model"] == 2 and rep["clampedUnknowns"] >= min_clamped, rep   # the fixed-point model
    assert rep["converged"], rep
    out = []
    with FiniteDifferences(gamma, prm, state) as fdc:
        for (i, j) in cells:
            r = fdc.cell(i, j, 1e-4, 1e-9, fd_iters)
            fd, fwd, bwd, adj = r["fd"], r["fwd"], r["bwd"], float(grad[i, j])
            smooth = abs(fwd - bwd) <= 1e-2 * abs(fd)
            ok = abs(adj - fd) <= TOL * abs(fd)
            out.append(dict(cell=(i, j), fd=fd, adjoint=adj, rel=abs(adj - fd) / abs(fd), fwd=fwd, bwd=bwd,
                            case="smooth" if smooth else "kink: one-sided slopes differ", ok=ok))
    print(out)
    bad = [o for o in out if not o["ok"]]
    assert not bad, (bad, out)
    return out


def test_adjoint_on_the_constricted_channel():
    """Cells on the gamma = 0.5 faces of the block, both sides of the gap:
    the adjoint within 1e-4 of the central difference on each (the test
    records whether the one-sided quotients differ, a kink)."""
    case = cases.constricted_channel(32, 96, pressureSolverType=4, maxPressureIter=30, pTol=1e-6)
    _check(case, [(12, 45), (19, 50), (5, 39), (25, 39)], 40000, 40000, min_clamped=50)
