"""torch.autograd.Functions for the optimiser's two objectives.

    dp = PressureDrop.apply(gamma, knobs)   # gamma: Ny x Nx tensor, 1 fluid .. 0 solid
    dp.backward()                           # gamma.grad = dJ/dgamma (discrete adjoint)

    J = ThermalPNorm.apply(gamma, u_xy, v_xy, q0, params, p)
    J.backward()                            # gamma.grad = dJ/dgamma of the bottom p-norm

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


class ThermalPNorm(torch.autograd.Function):
    """J = bottom-layer p-norm of the 3-D thermal solve (include/cp_thermal.h)
    for gamma (Ny x Nx tensor) with the velocities u_xy, v_xy and the heat
    flux q0 (arrays, held fixed) and the cp_thermal_params fields in
    ``params``.  Backward: the discrete adjoint of the assembled system
    (cp_thermal_pnorm_gradient); the fluid mask (gamma > 0.01) has no
    derivative and is held fixed."""

    @staticmethod
    def forward(ctx, gamma: torch.Tensor, u_xy, v_xy, q0, params: dict, p: float = 8.0):
        from .thermal import Thermal
        g = gamma.detach().to("cpu", torch.float64).numpy()
        th = Thermal(**params)
        th.set_inputs(g, u_xy, v_xy, q0)
        rep = th.solve()
        if not rep["converged"]:
            th.close()
            raise RuntimeError(f"thermal solve did not converge: {rep}")
        J, grad, arep = th.pnorm_gradient(p)
        th.close()
        if not arep["converged"]:
            raise RuntimeError(f"thermal adjoint did not converge: {arep}")
        ctx.grad = torch.from_numpy(np.ascontiguousarray(grad)).to(gamma.device, gamma.dtype)
        return torch.tensor(J, dtype=gamma.dtype, device=gamma.device)

    @staticmethod
    def backward(ctx, grad_out):
        return grad_out * ctx.grad, None, None, None, None, None
