"""Discrete adjoint dJ/dgamma of the full-system pressure drop against
central finite differences (h = 1e-4) of converged FP64 forward solves, on
cells with gamma in [0.05, 0.95] away from walls, inlet and outlet."""
import numpy as np
import pytest

from coldplate_b200 import Simple, cases

pytestmark = pytest.mark.gpu

KN = dict(pressureSolverType=4, maxPressureIter=60, pTol=1e-16, momentumTol=1e-14, epsilon=1e-30)


def converged_dp(case, gamma, n=4000):
    with Simple(gamma=gamma, **case.params(maxIterations=n + 10, **KN)) as s:
        s.step(n)
        h = s.history()["fullTotal"]
    assert abs(h[-1] - h[-200]) <= 1e-12 * abs(h[-1]), (h[-1], h[-200])
    return h[-1]


def pick_cells(gamma, k, rng, margin=3, buffer=8):
    Ny, Nx = gamma.shape
    cand = [(i, j) for i in range(margin, Ny - margin) for j in range(buffer, Nx - buffer)
            if 0.05 <= gamma[i, j] <= 0.95]
    idx = rng.choice(len(cand), size=min(k, len(cand)), replace=False)
    return [cand[q] for q in idx]


@pytest.mark.parametrize("prec", ["fp64"])
def test_adjoint_matches_finite_differences(prec):
    case = cases.density_field(24, 48, seed=4)
    gamma = 1.0 - case.cellType
    with Simple(gamma=gamma, **case.params(maxIterations=4010, precision=prec, **KN)) as s:
        s.step(4000)
        J0 = s.history()["fullTotal"][-1]
        grad, rep = s.adjoint_dp_dgamma(max_iter=3000, tol=1e-11)
    assert rep["converged"], rep
    assert abs(rep["J"] - J0) <= 1e-9 * abs(J0)
    rng = np.random.default_rng(0)
    h = 1e-4
    scale = np.abs(grad).max()
    for (i, j) in pick_cells(gamma, 8, rng):
        gp = gamma.copy(); gp[i, j] += h
        gm = gamma.copy(); gm[i, j] -= h
        fd = (converged_dp(case, gp) - converged_dp(case, gm)) / (2 * h)
        err = abs(fd - grad[i, j])
        assert err <= 1e-4 * max(abs(fd), 1e-2 * scale), ((i, j), fd, grad[i, j], err)


def test_autograd_function():
    import torch

    from coldplate_b200.autograd import PressureDrop
    case = cases.density_field(16, 32, seed=2)
    gamma = torch.tensor(1.0 - case.cellType, dtype=torch.float64, requires_grad=True)
    knobs = case.params(**KN)
    dp = PressureDrop.apply(gamma, knobs, 4000)
    dp.backward()
    assert gamma.grad is not None and gamma.grad.shape == gamma.shape
    assert torch.isfinite(gamma.grad).all()
    with Simple(gamma=gamma.detach().numpy(), **case.params(maxIterations=4010, **KN)) as s:
        s.step(4000)
        g2, _ = s.adjoint_dp_dgamma(tol=1e-10)
    np.testing.assert_allclose(gamma.grad.numpy(), g2, rtol=1e-6, atol=1e-9 * np.abs(g2).max())

