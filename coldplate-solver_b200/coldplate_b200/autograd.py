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

Device memory: PressureDrop keeps the converged u, v, p as host arrays
between forward and backward and builds a fresh context for the adjoint, so
a forward-only call (a line search, a no_grad evaluation) leaves nothing on
the GPU.  ThermalPNorm keeps its thermal context from forward to backward
when gamma needs a gradient (the adjoint needs the temperature) and frees it
in backward, or when the autograd graph is dropped; without a gradient it
frees it at once.  gamma crosses to the host once per call (the C ABI takes
host arrays; 8 MB at 2048 x 1024).
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import Simple


def _host(gamma: torch.Tensor) -> np.ndarray:
    return np.ascontiguousarray(gamma.detach().to("cpu", torch.float64).numpy())


class PressureDrop(torch.autograd.Function):
    """J = full-system total-pressure drop of the converged flow through
    gamma.  `sink` (a dict, optional) receives the converged u, v, p."""

    @staticmethod
    def forward(ctx, gamma: torch.Tensor, knobs: dict, max_outer: int = 20000, adj_tol: float = 1e-10,
                sink: dict | None = None):
        g = _host(gamma)
        prm = dict(knobs)
        prm.setdefault("maxIterations", max_outer)
        solver = Simple(gamma=g, **prm)
        try:
            rep = solver.runIterations()
            state = {f: solver.get(f) for f in ("u", "v", "p")}
        except BaseException:
            solver.close()
            raise
        if sink is not None:
            sink.update(state)
        ctx.solver = None
        if ctx.needs_input_grad[0]:
            ctx.state, ctx.gamma_host, ctx.prm, ctx.adj_tol = state, g, prm, adj_tol
            # with an inlet ramp the adjoint needs the solve's iteration count
            # (the ramped inlet velocity), which a fresh context does not have
            if prm.get("enableInletRamp"):
                ctx.solver = solver
        if ctx.solver is None:
            solver.close()
        ctx.gdevice, ctx.gdtype = gamma.device, gamma.dtype
        return torch.tensor(rep["fullTotalDrop"], dtype=gamma.dtype, device=gamma.device)

    @staticmethod
    def backward(ctx, grad_out):
        solver = ctx.solver or Simple(gamma=ctx.gamma_host, **ctx.prm)
        try:
            if ctx.solver is None:
                for f, a in ctx.state.items():
                    solver.set(f, a)
            g, rep = solver.adjoint_dp_dgamma(tol=ctx.adj_tol, max_iter=20000)
        finally:
            solver.close()
            ctx.solver, ctx.state = None, None
        if not rep["converged"]:
            raise RuntimeError(f"adjoint did not converge: {rep}")
        grad = torch.from_numpy(np.ascontiguousarray(g)).to(ctx.gdevice, ctx.gdtype)
        return grad_out * grad, None, None, None, None


class ThermalPNorm(torch.autograd.Function):
    """J = bottom-layer p-norm of the 3-D thermal solve (include/cp_thermal.h)
    for gamma (Ny x Nx tensor) with the velocities u_xy, v_xy and the heat
    flux q0 (arrays, held fixed) and the cp_thermal_params fields in
    ``params``.  Backward: the discrete adjoint of the assembled system
    (cp_thermal_pnorm_gradient), run only when a gradient is asked for; the
    fluid mask (gamma > 0.01) has no derivative and is held fixed."""

    @staticmethod
    def forward(ctx, gamma: torch.Tensor, u_xy, v_xy, q0, params: dict, p: float = 8.0):
        from .thermal import Thermal
        th = Thermal(**params)
        th.set_inputs(_host(gamma), u_xy, v_xy, q0)
        rep = th.solve()
        if not rep["converged"]:
            th.close()
            raise RuntimeError(f"thermal solve did not converge: {rep}")
        _, J = th.objective(p)
        if ctx.needs_input_grad[0]:
            ctx.th, ctx.p = th, p
        else:
            th.close()
        ctx.gdevice, ctx.gdtype = gamma.device, gamma.dtype
        return torch.tensor(J, dtype=gamma.dtype, device=gamma.device)

    @staticmethod
    def backward(ctx, grad_out):
        th = ctx.th
        try:
            _, grad, arep = th.pnorm_gradient(ctx.p)
        finally:
            th.close()
            ctx.th = None
        if not arep["converged"]:
            raise RuntimeError(f"thermal adjoint did not converge: {arep}")
        g = torch.from_numpy(np.ascontiguousarray(grad)).to(ctx.gdevice, ctx.gdtype)
        return grad_out * g, None, None, None, None, None
