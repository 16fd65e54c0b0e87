"""One in-process MMA iteration (coldplate_b200.mma) on the GPU solvers:
the replacement of the reference optimiser's evaluate_objective /
compute_sensitivities subprocess round trip (mma_optimizer.py:442-571).

A 24 x 40 flow domain (4-column inlet and outlet buffers around a 24 x 32
design block), the density workload's physics, the 8 + 4 layer thermal
stack on the design block with a hotspot power map."""
import numpy as np
import pytest
import torch

from coldplate_b200 import cases
from coldplate_b200.mma import MMAProblem, MMAState, density_filter

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    return built_lib


def _problem(**over) -> tuple[MMAProblem, torch.Tensor]:
    Ny, nd, nb = 24, 32, 4
    c = cases.density_field(Ny, nd + 2 * nb, seed=5, pressureSolverType=4, maxPressureIter=60, pTol=1e-14,
                            epsilon=1e-11)
    knobs = c.params()
    thermal = dict(Nx=nd, Ny=Ny, dx=c.hx, dy=c.hy, rtol=1e-11, maxiter=4000, **cases.THERMAL_3D)
    q0 = cases.power_map(Ny, nd, 5) * 1e4
    prm = dict(flow_knobs=knobs, thermal_params=thermal, q0=q0, n_in=nb, n_out=nb, filter_radius=1.5,
               n_wall=1, max_outer=8000, adj_tol=1e-10, vol_frac_target=0.6)
    prm.update(over)
    gam = torch.from_numpy(np.ascontiguousarray((1.0 - c.cellType)[:, nb:nb + nd]))
    return MMAProblem(**prm), gam


def test_one_mma_iteration_in_process():
    prob, gam = _problem(w_peak=1.0, w_dp=1.0, dp_scale=1e4)
    st = MMAState()
    xnew, rec = prob.iterate(gam, st)
    assert np.isfinite(rec["f0"]) and rec["Tb_pnorm"] > 25.0 and rec["dP"] > 0.0
    assert xnew.shape == gam.shape and torch.isfinite(xnew).all()
    assert float((xnew - gam).abs().max()) <= prob.move_limit + 1e-12
    assert float(xnew[0].abs().max()) == 0.0 and float(xnew[-1].abs().max()) == 0.0
    assert float(xnew.min()) >= 0.0 and float(xnew.max()) <= 1.0
    # a second iteration uses the asymptote history
    xnew2, rec2 = prob.iterate(xnew, st)
    assert st.iter == 2 and torch.isfinite(xnew2).all() and np.isfinite(rec2["f0"])


def test_sensitivity_through_filter_and_flow_adjoint():
    """f0 = dP / 1e4 (w_peak 0): the autograd gradient through the filter,
    the full-domain assembly and the flow adjoint against a central
    difference of f0 along a smooth direction of the design interior."""
    prob, gam = _problem(w_peak=0.0, w_dp=1.0, dp_scale=1e4)
    x = gam.clone().requires_grad_(True)

    def f0_of(z):
        phys = density_filter(z, prob.filter_radius).clamp(0.0, 1.0)
        phys = torch.cat([torch.zeros_like(phys[:1]), phys[1:-1], torch.zeros_like(phys[:1])])
        return prob.objective(phys)[0]

    f = f0_of(x)
    (g,) = torch.autograd.grad(f, x)
    Ny, nd = gam.shape
    yy, xx = np.mgrid[0:Ny, 0:nd]
    d = np.sin(np.pi * yy / (Ny - 1)) * np.cos(2 * np.pi * xx / nd) * ((gam.numpy() > 0.05) & (gam.numpy() < 0.95))
    d = torch.from_numpy(d)
    h = 1e-4
    with torch.no_grad():
        fd = (float(f0_of(gam + h * d)) - float(f0_of(gam - h * d))) / (2 * h)
    ad = float((g * d).sum())
    assert abs(ad - fd) <= 1e-4 * abs(fd), (ad, fd)
