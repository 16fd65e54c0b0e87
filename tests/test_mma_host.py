"""The in-process optimiser step's host parts against the reference
optimiser's own functions (tests/golden/mma.npz, made by
tests/golden/make_mma_golden.py): the density filter
(mma_optimizer.py:370-388) and four consecutive MMA updates
(mma_optimizer.py:589-718); and the filter's transpose from autograd."""
import os

import numpy as np
import torch

from coldplate_b200.mma import MMAState, density_filter, mma_update

Z = np.load(os.path.join(os.path.dirname(__file__), "golden", "mma.npz"))


def test_density_filter_matches_the_reference():
    x = torch.from_numpy(Z["x0"])
    for r in (1.5, 3.0):
        np.testing.assert_allclose(density_filter(x, r).numpy(), Z[f"filter_r{r}"], rtol=0, atol=1e-13)
    assert torch.equal(density_filter(x, 0.0), x)


def test_density_filter_transpose():
    rng = np.random.default_rng(3)
    a = torch.tensor(rng.standard_normal((24, 40)), requires_grad=True)
    w = torch.tensor(rng.standard_normal((24, 40)))
    y = density_filter(a, 3.0)
    (gt,) = torch.autograd.grad((y * w).sum(), a)
    # <F a, w> = <a, F^T w> for a second input through the same linear map
    b = torch.tensor(rng.standard_normal((24, 40)))
    assert abs(float((density_filter(b, 3.0) * w).sum() - (b * gt).sum())) <= 1e-10 * float(w.abs().sum())


def test_mma_updates_match_the_reference():
    M, N = Z["x0"].shape
    xmin, xmax = torch.from_numpy(Z["xmin"]), torch.from_numpy(Z["xmax"])
    x = torch.from_numpy(np.clip(Z["x0"], Z["xmin"], Z["xmax"]))
    st = MMAState()
    dg = torch.full((M * N,), 1.0 / (M * N), dtype=torch.float64)
    for k in range(4):
        xn = mma_update(x, torch.from_numpy(Z[f"df0_{k}"]), float(Z[f"g_{k}"]), dg, xmin, xmax, st)
        np.testing.assert_allclose(xn.numpy(), Z[f"x_{k + 1}"], rtol=0, atol=1e-9)
        x = xn.reshape(M, N)
