"""torch.autograd.Function for the pressure drop of a density field.

    dp = PressureDrop.apply(gamma, knobs)   # gamma: Ny x Nx tensor, 1 fluid .. 0 solid
    dp.backward()                           # gamma.grad = dJ/dgamma (discrete adjoint)

Forward: a GPU SIMPLE solve (libcoldplate.so) of the field to convergence,
J = full-system total-pressure drop.  Backward: the discrete adjoint at the
converged state, which keeps only that state and recomputes the
coefficients.  This is the in-process replacement for the optimiser's
subprocess call (run_solvers.py:248) for the flow part of the objective.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import Simple


class PressureDrop(torch.autograd.Function):
    @staticmethod
    def forward(ctx, gamma: torch.Tensor, knobs: dict, max_outer: int = 20000, adj_tol: float = 1e-10):
        g = gamma.detach().to("cpu", torch.float64).numpy()
        prm = dict(knobs)
        prm.setdefault("maxIterations", max_outer)
        solver = Simple(gamma=g, **prm)
        rep = solver.runIterations()
        ctx.solver = solver
        ctx.adj_tol = adj_tol
        ctx.gshape = gamma.shape
        ctx.gdevice, ctx.gdtype = gamma.device, gamma.dtype
        return torch.tensor(rep["fullTotalDrop"], dtype=gamma.dtype, device=gamma.device)

    @staticmethod
    def backward(ctx, grad_out):
        solver = ctx.solver
        g, rep = solver.adjoint_dp_dgamma(tol=ctx.adj_tol)
        solver.close()
        if not rep["converged"]:
            raise RuntimeError(f"adjoint did not converge: {rep}")
        grad = torch.from_numpy(np.ascontiguousarray(g)).to(ctx.gdevice, ctx.gdtype)
        return grad_out * grad, None, None, None
