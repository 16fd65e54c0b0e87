"""The adjoint operator entry by entry.

On a 12 x 36 constricted channel with 42 velocities on the clamp and zero-
flux faces in the jet behind the gap, the fixed-point adjoint's J_X^T (each
row by cp_adjoint_probe on a unit vector), dJ/dX and the adjoint solution
lambda are compared with the same quantities of the fixed-point model
restated on the FP64 oracle (tests/_frozen_model.py), differentiated by
central differences.
"""
import numpy as np
import pytest

from coldplate_b200 import Simple, cases
from coldplate_b200.fdcheck import run_stationary

from _frozen_model import FrozenModel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    return built_lib


def test_fixed_point_adjoint_operator_matches_the_model_jacobian():
    case = cases.constricted_channel(12, 36, gap=2, pressureSolverType=1, maxPressureIter=2000, pTol=1e-15)
    prm = case.params(precision="fp64", maxIterations=400000, epsilon=1e-30, historyCapacity=400010, adjointModel=2)
    with Simple(gamma=1.0 - case.cellType, **prm) as g:
        J0, n0, rel0 = run_stationary(g, 1e-15, 200000)
        dj, meta = g.adjoint_probe(1)
        lam, meta2 = g.adjoint_probe(2, max_iter=20000, tol=1e-13)
        assert meta["model"] == 2 and meta2["converged"], (meta, meta2)
        state = {f: g.get(f) for f in ("u", "v", "p")}
        fm = FrozenModel(case, case.params(maxIterations=10 ** 7, epsilon=1e-30), state, meta["sweepsU"],
                         meta["sweepsV"])
        assert fm.cu.sum() == meta2["clampedUnknowns"] and fm.cu.sum() > 0
        zero = {"u": np.zeros((g.M + 1, g.N)), "v": np.zeros((g.M, g.N + 1)), "p": np.zeros((g.M + 1, g.N + 1))}
        rows = np.zeros((len(fm.keys), len(fm.keys)))
        for k, (f, a) in enumerate(fm.keys):
            x = {q: z.copy() for q, z in zero.items()}
            x[f][a] = 1.0
            y, _ = g.adjoint_probe(0, x)
            rows[k] = fm.pack(y)
    GX, JX = fm.jacobians()
    # the model's equations vanish at the state (it is a fixed point)
    assert np.abs(fm.G(fm.X0)).max() <= 1e-10, np.abs(fm.G(fm.X0)).max()
    # J_X^T rows: columns of clamped velocities hold a kink (a face average
    # on the clamp) and never reach the gradient; the rest agree to rounding
    # and the FD truncation
    cols = np.ones(GX.shape[1], bool)
    cols[:fm.nu][fm.cu] = False
    rowscale = np.abs(GX).max(axis=1)
    rel = (np.abs(rows - GX)[:, cols].max(axis=1) / rowscale).max()
    assert rel <= 1e-5, rel
    assert np.abs(fm.pack(dj) - JX).max() <= 1e-6 * np.abs(JX).max()
    lam_m = np.linalg.solve(GX.T, JX)
    assert np.abs(fm.pack(lam) - lam_m).max() <= 1e-6 * np.abs(lam_m).max()
