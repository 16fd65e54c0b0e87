"""The seeded synthetic workloads (coldplate_b200.cases) against the
configurations they stand in for: sizes, parameter ranges, the physics
knobs each one names, determinism in the seed, and a fluid path from inlet
to outlet (without one the pressure drop is not a channel flow's)."""
import numpy as np
import pytest
from scipy import ndimage

from coldplate_b200 import cases


def runs(col: np.ndarray) -> list[int]:
    """Lengths of the runs of True in a 1-D boolean array."""
    out, n = [], 0
    for v in col:
        if v:
            n += 1
        elif n:
            out.append(n)
            n = 0
    if n:
        out.append(n)
    return out


def percolates(fluid: np.ndarray) -> bool:
    lab, _ = ndimage.label(fluid)
    return bool(set(lab[:, 0][lab[:, 0] > 0]) & set(lab[:, -1][lab[:, -1] > 0]))


def test_straight_channel_is_config_1():
    c = cases.straight_channel()
    assert (c.Ny, c.Nx) == (64, 256) and c.hx == c.hy == 1e-5 and c.U == 0.5
    fluid = c.cellType < 0.5
    assert np.all(fluid[8:56]) and not fluid[:8].any() and not fluid[56:].any()
    k = c.params()
    assert (k["rho"], k["eta"]) == (1000.0, 1e-3)
    assert k["convectionScheme"] == 0 and k["uvAlpha"] == 0.7 and k["pAlpha"] == 0.3
    assert k["pTol"] == 1e-8 and k["maxIterations"] == 2000 and k["epsilon"] == 1e-7
    assert k["momentumSolverType"] == 1 and k["pressureSolverType"] == 1


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_network_is_config_2(seed):
    c = cases.random_network(512, 1024, seed=seed)
    assert (c.Ny, c.Nx) == (512, 1024)
    assert 0.3 <= c.U <= 1.0 and c.Ht == 2e-4
    k = c.params()
    assert k["convectionScheme"] == 1 and k["enableTwoPointFiveD"] == 1
    assert set(np.unique(c.cellType)) <= {0.0, 1.0}          # binary geometry
    fluid = c.cellType < 0.5
    inlets = runs(fluid[:, 0])
    assert 1 <= len(inlets) <= 6 and min(inlets) >= 8        # 3-6 walkers of width 8-24, merged where they meet
    assert percolates(fluid)
    assert np.array_equal(c.cellType, cases.random_network(512, 1024, seed=seed).cellType)
    assert not np.array_equal(c.cellType, cases.random_network(512, 1024, seed=seed + 10).cellType)


def test_density_field_is_config_3():
    c = cases.density_field()
    assert (c.Ny, c.Nx) == (1024, 2048) and c.Ht == 2e-4
    k = c.params()
    assert k["convectionScheme"] == 1 and k["enableTwoPointFiveD"] == 1
    assert k["eta"] / k["brinkmanKMin"] == pytest.approx(1e9)  # alpha_max 1e9 kg/m^3 s
    assert k["brinkmanQ"] == 0.1
    gam = 1.0 - c.cellType
    assert gam.min() >= 0.0 and gam.max() <= 1.0
    assert np.all(gam[8:-8, :32] == 1.0) and np.all(gam[8:-8, -32:] == 1.0)   # inlet / outlet buffers
    assert np.all(gam[:8] == 0.0) and np.all(gam[-8:] == 0.0)                 # walls Ny / 128 rows
    inner = gam[8:-8, 32:-32]
    # a continuous density through the tanh projection (beta 8 leaves most
    # cells between the phases), about 70 % above 0.5 for the field
    # standardised to mean 0.6
    assert 0.6 <= (inner > 0.5).mean() <= 0.8
    assert ((inner > 0.05) & (inner < 0.95)).mean() > 0.3
    assert (inner < 0.05).any() and (inner > 0.95).any()
    assert percolates(gam > 0.5)


def test_density_field_correlation_length():
    """The Gaussian random field's correlation: the autocorrelation of the
    field at a lag of the correlation length (32 cells) is exp(-1/2) for a
    kernel of sigma 32 / sqrt 2 (C(r) = exp(-r^2 / (4 sigma^2)))."""
    g = cases.gaussian_random_field(512, 1024, 32.0, np.random.default_rng(3))
    g = (g - g.mean()) / g.std()
    lag = 32
    c = np.mean(g[:, :-lag] * g[:, lag:])
    assert c == pytest.approx(np.exp(-0.5), abs=0.08)


def test_batch_is_config_4():
    cs = cases.batch(64, seed=0)
    assert len(cs) == 64
    for c in cs:
        assert 256 <= c.Nx <= 1024 and 128 <= c.Ny <= 512
        assert 0.2 <= c.U <= 1.0
        assert c.params()["epsilon"] == 1e-6
    sizes = {(c.Ny, c.Nx) for c in cs}
    assert len(sizes) > 50                                    # uneven grid sizes
    again = cases.batch(64, seed=0)
    assert all(np.array_equal(a.cellType, b.cellType) and a.U == b.U for a, b in zip(cs, again))


def test_thermal_settings_are_config_5():
    t = cases.THERMAL_3D
    assert (t["nz_solid"], t["nz_fluid"]) == (8, 4)
    assert (t["k_s"], t["k_f"], t["Cp"], t["T_inlet"]) == (400.0, 0.6, 4180.0, 25.0)
