"""In-process MMA topology-optimisation step on the GPU solvers.

The reference's optimiser (mma_optimizer.py) evaluates every design by
writing geometry files and running the flow and thermal executables as
subprocesses (evaluate_objective, :442-495, through run_solvers.py:193-340),
and takes its sensitivity from a separate 2-D conduction adjoint that reads
the thermal result files back (compute_sensitivities, :498-571).  Here one
MMA iteration runs in the process, on tensors:

  density filter      the reference's density_filter_fast (:370-388): a box
                      filter of size 2 ceil(r) + 1 with mirrored edges
                      (scipy.ndimage.uniform_filter, mode "reflect"), written
                      in torch so its transpose comes from autograd
  full fluid domain   the design block placed between the inlet and outlet
                      buffers, walls solid, as write_geometry builds it
                      (:256-305)
  flow                coldplate_b200.autograd.PressureDrop (GPU SIMPLE solve;
                      backward = discrete adjoint)
  thermal             coldplate_b200.autograd.ThermalPNorm on the design
                      block with the flow's cell-centred velocities (held
                      fixed, as the reference's adjoint holds them)
  objective           f0 = w_peak * (bottom-layer p-norm of T, p = 8: a
                      smooth stand-in for the peak temperature that the
                      reference estimates as T_avg + T_range / 2)
                      + w_dp * dP / dp_scale (0 by default, as in the
                      reference, whose objective has no pressure term)
  constraint          g = mean(gamma_phys) - vol_frac_target (:856-858)
  update              mma_update: the reference's single-constraint MMA
                      (:589-718), in torch
  walls               rows [0, n_wall) and the last n_wall rows of the
                      design stay solid (:780-800, :880-882)

The sensitivities are the exact derivatives of this f0 and g with respect
to the design variables, through the filter; the reference instead feeds
the gradient with respect to the filtered field straight into MMA.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from .autograd import PressureDrop, ThermalPNorm


# ------------------------------------------------------------------ filter
def _mirror_index(n: int, h: int, device) -> torch.Tensor:
    """Indices of a length-n axis padded by h on both sides with mirrored
    edges (d c b a | a b c d | d c b a); h <= n."""
    i = torch.arange(-h, n + h, device=device)
    i = torch.where(i < 0, -i - 1, i)
    return torch.where(i >= n, 2 * n - 1 - i, i)


def density_filter(x: torch.Tensor, radius: float) -> torch.Tensor:
    """Box filter of size 2 ceil(radius) + 1 along each axis with mirrored
    edges: the reference's density_filter_fast (mma_optimizer.py:370-388,
    scipy.ndimage.uniform_filter(x, size, mode="reflect")).  radius <= 0
    returns x.  Differentiable."""
    if radius <= 0:
        return x.clone()
    h = int(math.ceil(radius))
    s = 2 * h + 1
    M, N = x.shape
    if h > min(M, N):
        raise ValueError(f"filter radius {radius} exceeds the design size {M} x {N}")
    y = x.index_select(0, _mirror_index(M, h, x.device))
    y = y.index_select(1, _mirror_index(N, h, x.device))
    k = torch.full((1, 1, s, 1), 1.0 / s, dtype=x.dtype, device=x.device)
    y = torch.nn.functional.conv2d(y[None, None], k)                       # along rows
    y = torch.nn.functional.conv2d(y, k.transpose(2, 3))                   # along columns
    return y[0, 0]


# ------------------------------------------------------------------ MMA
@dataclass
class MMAState:
    """History of the moving asymptotes (mma_optimizer.py:574-584)."""
    xold1: torch.Tensor | None = None
    xold2: torch.Tensor | None = None
    low: torch.Tensor | None = None
    upp: torch.Tensor | None = None
    iter: int = 0


def mma_update(x: torch.Tensor, df0dx: torch.Tensor, g: float, dgdx: torch.Tensor, xmin: torch.Tensor,
               xmax: torch.Tensor, state: MMAState, move_limit: float = 0.2, asyinit: float = 0.5,
               asydecr: float = 0.7, asyincr: float = 1.2) -> torch.Tensor:
    """One step of the method of moving asymptotes (Svanberg 1987) for one
    objective and one constraint g(x) <= 0, as the reference's mma_update
    (mma_optimizer.py:589-718) sets it up: asymptotes from the last two
    designs (shrunk where the move oscillates, widened where it is
    monotone), move limits, the convex separable approximation, and its
    one-dimensional dual solved by bisection on the multiplier.  Flat
    tensors of the design size; returns the new design."""
    x, df0, dg = x.reshape(-1), df0dx.reshape(-1), dgdx.reshape(-1)
    lo_b, hi_b = xmin.reshape(-1), xmax.reshape(-1)
    span = torch.clamp(hi_b - lo_b, min=1e-10)
    if state.iter < 2 or state.low is None:
        low, upp = x - asyinit * span, x + asyinit * span
    else:
        trend = (x - state.xold1) * (state.xold1 - state.xold2)
        fac = torch.where(trend < 0, torch.full_like(x, asydecr),
                          torch.where(trend > 0, torch.full_like(x, asyincr), torch.zeros_like(x)))
        low = torch.where(trend != 0, x - fac * (state.xold1 - state.low), x - asyinit * span)
        upp = torch.where(trend != 0, x + fac * (state.upp - state.xold1), x + asyinit * span)
    low = torch.minimum(torch.maximum(low, x - 10.0 * span), x - 0.01 * span)
    upp = torch.maximum(torch.minimum(upp, x + 10.0 * span), x + 0.01 * span)
    a = torch.maximum(lo_b, torch.maximum(low + 0.1 * (x - low), x - move_limit * span))
    b = torch.minimum(hi_b, torch.minimum(upp - 0.1 * (upp - x), x + move_limit * span))
    ux2, xl2 = (upp - x) ** 2, (x - low) ** 2
    p0 = torch.clamp(df0, min=0.0) * ux2 + 1e-6 * span
    q0 = torch.clamp(-df0, min=0.0) * xl2 + 1e-6 * span
    p1 = torch.clamp(dg, min=0.0) * ux2
    q1 = torch.clamp(-dg, min=0.0) * xl2
    g_lin = g - float(torch.dot(dg, x))

    def x_of(lam: float) -> torch.Tensor:
        sp, sq = torch.sqrt(p0 + lam * p1), torch.sqrt(q0 + lam * q1)
        xn = (sp * low + sq * upp) / torch.clamp(sp + sq, min=1e-20)
        return torch.minimum(torch.maximum(xn, a), b)

    def g_of(lam: float) -> float:
        return float(torch.dot(dg, x_of(lam))) + g_lin

    if g_of(0.0) <= 0.0:
        lam = 0.0
    else:
        lo, hi = 0.0, 1e6
        while g_of(hi) > 0.0 and hi < 1e12:
            hi *= 10.0
        for _ in range(100):
            mid = 0.5 * (lo + hi)
            if g_of(mid) > 0.0:
                lo = mid
            else:
                hi = mid
            if hi - lo < 1e-10:
                break
        lam = 0.5 * (lo + hi)
    xnew = x_of(lam)
    state.xold2 = state.xold1.clone() if state.xold1 is not None else x.clone()
    state.xold1 = x.clone()
    state.low, state.upp = low, upp
    state.iter += 1
    return xnew


# ------------------------------------------------------------------ the optimisation problem
@dataclass
class MMAProblem:
    """One cold-plate design problem.  The flow domain is Ny x (n_in +
    design columns + n_out); the design block sits between the buffers."""
    flow_knobs: dict                  # cp_params names of the flow solve (grid, fluid, solver settings)
    thermal_params: dict              # cp_thermal_params of the design block (Nx = design columns)
    q0: np.ndarray                    # bottom heat flux of the design block [W/m^2]
    n_in: int = 0
    n_out: int = 0
    inlet_cell_type: np.ndarray | None = None    # buffer geometry (cellType), fluid when None
    outlet_cell_type: np.ndarray | None = None
    vol_frac_target: float = 0.4
    w_peak: float = 1.0
    w_dp: float = 0.0
    dp_scale: float = 1.0
    pnorm: float = 8.0
    filter_radius: float = 3.0
    n_wall: int = 1
    move_limit: float = 0.2
    asyinit: float = 0.5
    asydecr: float = 0.7
    asyincr: float = 1.2
    max_outer: int = 20000
    adj_tol: float = 1e-8
    history: list = field(default_factory=list)

    def full_gamma(self, gamma_design: torch.Tensor) -> torch.Tensor:
        """The flow domain's gamma: buffers, the design block, solid top
        and bottom rows (write_geometry, mma_optimizer.py:269-297)."""
        Ny, nd = gamma_design.shape
        dev, dt = gamma_design.device, gamma_design.dtype
        gin = (torch.ones(Ny, self.n_in, dtype=dt, device=dev) if self.inlet_cell_type is None else
               1.0 - torch.as_tensor(self.inlet_cell_type, dtype=dt, device=dev))
        gout = (torch.ones(Ny, self.n_out, dtype=dt, device=dev) if self.outlet_cell_type is None else
                1.0 - torch.as_tensor(self.outlet_cell_type, dtype=dt, device=dev))
        g = torch.cat([gin, gamma_design, gout], dim=1)
        mask = torch.ones_like(g)
        mask[0] = 0.0
        mask[-1] = 0.0
        return g * mask

    def objective(self, gamma_phys: torch.Tensor) -> tuple[torch.Tensor, dict]:
        """f0 of a filtered design (with the autograd graph) and metrics:
        the in-process counterpart of evaluate_objective
        (mma_optimizer.py:442-495)."""
        gfull = self.full_gamma(gamma_phys)
        knobs = dict(self.flow_knobs)
        knobs.setdefault("maxIterations", self.max_outer)
        flow: dict = {}
        dp = PressureDrop.apply(gfull, knobs, self.max_outer, self.adj_tol, flow)
        # the converged flow's cell-centred velocities on the design block
        # (output.cpp:90-107, cropped like u_thermal.txt / v_thermal.txt)
        u, v = flow["u"], flow["v"]
        Ny, Nx = gfull.shape
        sl = slice(self.n_in, Nx - self.n_out)
        u_xy = np.ascontiguousarray(0.5 * (u[1:Ny + 1, 0:Nx] + u[1:Ny + 1, 1:Nx + 1])[:, sl])
        v_xy = np.ascontiguousarray(0.5 * (v[0:Ny, 1:Nx + 1] + v[1:Ny + 1, 1:Nx + 1])[:, sl])
        T = ThermalPNorm.apply(gamma_phys, u_xy, v_xy, self.q0, self.thermal_params, self.pnorm)
        f0 = self.w_peak * T
        if self.w_dp != 0.0:
            f0 = f0 + self.w_dp * dp / self.dp_scale
        return f0, {"Tb_pnorm": float(T), "dP": float(dp)}

    def iterate(self, gamma: torch.Tensor, state: MMAState) -> tuple[torch.Tensor, dict]:
        """One MMA iteration (the body of run_optimization's loop,
        mma_optimizer.py:829-882) on the design gamma (Ny x design
        columns): filter, objective, volume constraint, sensitivities by
        autograd through the filter, MMA update, walls.  Returns the new
        design and this iteration's record."""
        x = gamma.detach().clone().requires_grad_(True)
        phys = density_filter(x, self.filter_radius).clamp(0.0, 1.0)
        wall = torch.ones_like(phys)
        wall[:self.n_wall] = 0.0
        wall[phys.shape[0] - self.n_wall:] = 0.0
        phys = phys * wall
        f0, metrics = self.objective(phys)
        vol = phys.mean()
        g = float(vol) - self.vol_frac_target
        df0dx, = torch.autograd.grad(f0, x, retain_graph=True)
        dgdx, = torch.autograd.grad(vol, x)
        xmin = torch.zeros_like(x)
        xmax = torch.ones_like(x)
        xmax[:self.n_wall] = 0.0
        xmax[x.shape[0] - self.n_wall:] = 0.0
        xnew = mma_update(x.detach(), df0dx, g, dgdx, xmin, xmax, state, self.move_limit, self.asyinit,
                          self.asydecr, self.asyincr).reshape(x.shape)
        xnew = xnew * wall
        rec = {"f0": float(f0), "vol_frac": float(vol), "g": g,
               "max_change": float((xnew - gamma.detach()).abs().max()), **metrics}
        self.history.append(rec)
        return xnew, rec
