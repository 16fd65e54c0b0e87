"""Known answers of the physics on the straight channel (64 x 256 cells,
fluid rows 8-55 between 8-row Brinkman walls, FOU, uniform inlet), checked
on the FP64 oracle (CPU) and on the GPU solve.  The reference ships no
tests, so these are derived from the flow itself:

- plane Poiseuille: at Re ~ 10 (U 0.02 m/s) the flow is developed after
  about 0.3 mm, and the centreline pressure gradient is 12 mu U / h^2 with
  h between the 48 fluid rows and 50 (the Brinkman wall lets the profile
  reach into the first solid cell); the peak velocity is about 1.5 U and
  the flow rate through a developed column equals the inlet's;
- mass conservation: inlet and outlet patch mass fluxes agree at
  convergence (SIMPLE.cpp:543-621 prints the same balance);
- mirror symmetry: the geometry and boundary conditions are symmetric
  about the channel's centre line, so u and p are mirror images and v is
  odd, up to the rounding the iteration amplifies (the reference's CSR row
  order is not mirror-symmetric).
"""
import numpy as np
import pytest

from _helpers import gpu_for, oracle_for

MU = 1e-3
FLUID_ROWS = 48


def poiseuille_checks(case, u, p):
    M, N = u.shape[0] - 1, p.shape[1] - 1
    hx, hy, U = case.hx, case.hy, case.U
    x = (np.arange(1, N) - 0.5) * hx
    sel = (x > 0.3 * x[-1]) & (x < 0.9 * x[-1])
    slope = np.polyfit(x[sel], p[M // 2, 1:N][sel], 1)[0]
    ratio = -slope * (FLUID_ROWS * hy) ** 2 / (12.0 * MU * U)
    # h_eff = 48 / sqrt(ratio) cells: between 48 and 50.6
    assert 0.90 <= ratio <= 1.0, ratio
    prof = u[1:M, int(0.7 * N)]
    assert 1.40 <= prof.max() / U <= 1.52, prof.max() / U
    assert abs(prof.sum() * hy / (U * FLUID_ROWS * hy) - 1.0) <= 1e-3


def balance_and_symmetry_checks(u, v, p, mass_in, mass_out, tol):
    assert abs(mass_in - mass_out) <= 1e-4 * abs(mass_in), (mass_in, mass_out)
    M = u.shape[0] - 1
    assert np.abs(u[1:M] - u[1:M][::-1]).max() <= tol * np.abs(u).max()
    assert np.abs(p[1:M] - p[1:M][::-1]).max() <= tol * np.abs(p).max()
    # v is odd; measured against the velocity scale (max |v| is 7 % of max |u|)
    assert np.abs(v[1:M - 1] + v[1:M - 1][::-1]).max() <= tol * np.abs(u).max()


def test_oracle_plane_poiseuille():
    from coldplate_b200 import cases
    case = cases.straight_channel(64, 256, U=0.02)
    o = oracle_for(case, maxIterations=6000)
    h = o.run(6000)
    assert len(h) < 6000
    poiseuille_checks(case, o.get("u"), o.get("p"))


def test_oracle_mass_balance_and_mirror_symmetry():
    from coldplate_b200 import cases
    case = cases.straight_channel(64, 256)
    o = oracle_for(case, maxIterations=3000)
    h = o.run(3000)
    assert len(h) < 3000
    balance_and_symmetry_checks(o.get("u"), o.get("v"), o.get("p"), h[-1, 13], h[-1, 14], 1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_plane_poiseuille(precision):
    from coldplate_b200 import cases
    case = cases.straight_channel(64, 256, U=0.02)
    with gpu_for(case, maxIterations=6000, precision=precision) as g:
        rep = g.runIterations()
        assert rep["stop_reason"] == 1 or (precision == "mixed" and rep["stop_reason"] == 2), rep
        poiseuille_checks(case, g.get("u"), g.get("p"))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_mass_balance_and_mirror_symmetry(precision):
    from coldplate_b200 import cases
    case = cases.straight_channel(64, 256)
    with gpu_for(case, maxIterations=3000, precision=precision) as g:
        rep = g.runIterations()
        assert rep["stop_reason"] == 1 or (precision == "mixed" and rep["stop_reason"] == 2), rep
        h = g.history()
        tol = 1e-5 if precision == "fp64" else 1e-4
        balance_and_symmetry_checks(g.get("u"), g.get("v"), g.get("p"), h["inMassFlux"][-1], h["outMassFlux"][-1],
                                    tol)
