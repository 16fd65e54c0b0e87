"""Seeded synthetic cold-plate geometries and run settings.

Nothing here is read from a dataset: every geometry is generated from a
numpy seed.  The settings follow the reference's SIMPLE.h defaults except
where a workload states otherwise; all cells are dx = dy = 10 um, water
rho = 1000 kg/m^3, mu = 1e-3 Pa s.

Workloads
  straight_channel  Ny x Nx straight channel, solid walls Ny/8 rows thick
                    top and bottom, FOU, uniform inlet (256 x 64 by default)
  random_network    binary channel network from a Manhattan/diagonal router
                    (3-6 inlets, widths 8-24 cells, split/merge probability
                    0.3), SOU, 2.5-D sink with Ht = 200 um
  density_field     continuous density: a Gaussian random field (correlation
                    length 32 cells, mean 0.6, std 0.2) through a tanh
                    projection (beta 8, eta 0.5), Brinkman alpha_max 1e9 with
                    q = 0.1, SOU, 2.5-D;
                    fluid inlet/outlet buffers keep the boundary patches pure
                    fluid so the pressure drop is defined
  constricted_channel  a channel narrowed to a gap that carries the flow
                    above the reference's velocity clamp (adjoint tests)
  batch             density fields of random sizes (Nx 256-1024, Ny 128-512)
                    and inlet velocities (0.2-1.0 m/s)
  THERMAL_3D,       the 3-D conjugate-heat-transfer settings on the flow's
  power_map         plane (8 + 4 layers) and a hotspot heat-flux map

Values are rounded to float32 so the reference's float and double builds
read identical geometries from the text files.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

H = 1e-5          # cell size [m]
RHO, MU = 1000.0, 1e-3


@dataclass
class Case:
    name: str
    cellType: np.ndarray          # Ny x Nx, 0 fluid .. 1 solid
    U: float                      # inlet velocity [m/s]
    Ht: float = 0.0               # out-of-plane height [m]
    hy: float = H
    hx: float = H
    knobs: dict = field(default_factory=dict)   # SIMPLE.h / cp_params names

    @property
    def Ny(self) -> int:
        return int(self.cellType.shape[0])

    @property
    def Nx(self) -> int:
        return int(self.cellType.shape[1])

    def params(self, **over) -> dict:
        """Full knob dict for coldplate_b200.Simple / the oracle."""
        d = dict(Ny=self.Ny, Nx=self.Nx, hy=self.hy, hx=self.hx, targetVel=self.U, Ht_channel=self.Ht)
        d.update(self.knobs)
        d.update(over)
        return d


def _base_knobs(Nx: int) -> dict:
    # core sampling planes at 25 % and 75 % of the length (the SIMPLE.h
    # defaults of 10 mm / 50 mm lie outside small domains)
    return dict(rho=RHO, eta=MU, pressureSolverType=1, momentumSolverType=1,
                usePressureDropConvergence=0, saveStateInterval=0,
                xPlaneCoreInlet=0.25 * Nx * H, xPlaneCoreOutlet=0.75 * Nx * H)


def _f32(a: np.ndarray) -> np.ndarray:
    return np.asarray(a, dtype=np.float32).astype(np.float64)


# ------------------------------------------------------------------ workloads
def straight_channel(Ny: int = 64, Nx: int = 256, U: float = 0.5, **over) -> Case:
    ct = np.zeros((Ny, Nx))
    w = max(1, Ny // 8)
    ct[:w] = 1.0
    ct[Ny - w:] = 1.0
    knobs = _base_knobs(Nx)
    knobs.update(convectionScheme=0, uvAlpha=0.7, pAlpha=0.3, pTol=1e-8, maxPressureIter=30,
                 epsilon=1e-7, maxIterations=2000, brinkmanKMin=1e-14, brinkmanQ=1.0,
                 enableTwoPointFiveD=0)
    knobs.update(over)
    return Case("straight_channel", _f32(ct), U, 0.0, knobs=knobs)


def _carve(fluid: np.ndarray, y: float, x: int, w: int) -> None:
    Ny = fluid.shape[0]
    lo = int(round(y - w / 2))
    fluid[max(lo, 0):min(lo + w, Ny), x] = True


def random_network(Ny: int = 512, Nx: int = 1024, seed: int = 0, **over) -> Case:
    """Binary channel network: walkers from 3-6 inlets move east with
    Manhattan jogs and diagonal runs, split with probability 0.3 and merge
    where they meet; the outlet column collects everything."""
    rng = np.random.default_rng(seed)
    wall = max(2, Ny // 64)
    fluid = np.zeros((Ny, Nx), dtype=bool)
    n_in = int(rng.integers(3, 7))
    walkers = []
    for _ in range(n_in):
        w = int(rng.integers(8, 25))
        y = float(rng.uniform(wall + w / 2 + 1, Ny - wall - w / 2 - 1))
        walkers.append([y, 0, w, 0.0])  # y, x, width, slope
    x = 0
    seg_end = {}
    while walkers and x < Nx:
        new = []
        for k, wk in enumerate(walkers):
            y, _, w, slope = wk
            key = id(wk)
            if seg_end.get(key, -1) <= x:
                r = rng.random()
                if r < 0.4:
                    slope = 0.0
                elif r < 0.7:
                    slope = float(rng.choice([-1.0, 1.0]))          # diagonal
                else:
                    slope = float(rng.choice([-1.0, 1.0])) * 4.0    # Manhattan jog
                seg_end[key] = x + int(rng.integers(16, 65))
                if rng.random() < 0.3 and len(walkers) + len(new) < 12:
                    w2 = int(rng.integers(8, 25))
                    new.append([y, x, w2, -slope if slope != 0 else float(rng.choice([-1.0, 1.0]))])
            y = float(np.clip(y + slope, wall + w / 2 + 1, Ny - wall - w / 2 - 1))
            wk[0], wk[1], wk[3] = y, x, slope
            if abs(slope) > 1.0:     # vertical jog: carve the whole span
                for yy in np.arange(y - abs(slope), y + abs(slope) + 1):
                    _carve(fluid, yy, x, w)
            _carve(fluid, y, x, w)
        walkers.extend(new)
        # merge walkers that overlap
        walkers.sort(key=lambda q: q[0])
        merged = []
        for wk in walkers:
            if merged and abs(wk[0] - merged[-1][0]) < (wk[2] + merged[-1][2]) / 2 + wall:
                continue
            merged.append(wk)
        walkers = merged
        x += 1
    # open tiny solid islands (single cells) so the network has clean walls
    solid = ~fluid
    nb = np.zeros_like(solid, dtype=np.int32)
    nb[1:, :] += solid[:-1, :]
    nb[:-1, :] += solid[1:, :]
    nb[:, 1:] += solid[:, :-1]
    nb[:, :-1] += solid[:, 1:]
    solid &= nb >= 2
    solid[:wall] = True
    solid[Ny - wall:] = True
    U = float(rng.uniform(0.3, 1.0))
    knobs = _base_knobs(Nx)
    knobs.update(convectionScheme=1, enableTwoPointFiveD=1, twoPointFiveDConvectionFactor=1.2,
                 pTol=1e-8, maxPressureIter=30, epsilon=1e-7, maxIterations=20000)
    knobs.update(over)
    return Case("random_network", _f32(solid.astype(np.float64)), U, 2e-4, knobs=knobs)


def gaussian_random_field(Ny: int, Nx: int, corr: float, rng: np.random.Generator) -> np.ndarray:
    """White noise convolved (FFT) with a Gaussian of correlation length
    `corr` cells (kernel sigma = corr / sqrt 2), min-max normalised to [0, 1]."""
    w = rng.standard_normal((Ny, Nx))
    sig = corr / np.sqrt(2.0)
    ky = np.fft.fftfreq(Ny)[:, None]
    kx = np.fft.fftfreq(Nx)[None, :]
    Hk = np.exp(-2.0 * np.pi ** 2 * sig ** 2 * (kx ** 2 + ky ** 2))
    g = np.real(np.fft.ifft2(np.fft.fft2(w) * Hk))
    g -= g.min()
    g /= max(g.max(), 1e-300)
    return g


def tanh_projection(g: np.ndarray, beta: float = 8.0, eta: float = 0.5) -> np.ndarray:
    return (np.tanh(beta * eta) + np.tanh(beta * (g - eta))) / (np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta)))


def density_gamma(Ny: int, Nx: int, seed: int, corr: float = 32.0, buffer: int = 32,
                  wall: int | None = None, mean: float = 0.6, std: float = 0.2) -> np.ndarray:
    """gamma (1 fluid .. 0 solid) of the density workload.  The random field
    is standardised to the given mean and standard deviation before the
    projection: with mean 0.6 about 70 % of the cells lie above eta = 0.5,
    so the fluid phase percolates from inlet to outlet (a field centred on
    eta sits at the 2-D percolation threshold and forces the flow through
    Brinkman solid)."""
    rng = np.random.default_rng(seed)
    g = gaussian_random_field(Ny, Nx, corr, rng)
    g = mean + std * (g - g.mean()) / max(g.std(), 1e-300)
    gam = tanh_projection(g)
    gam = np.clip(gam, 0.0, 1.0)
    b = min(buffer, Nx // 8)
    gam[:, :b] = 1.0
    gam[:, Nx - b:] = 1.0
    wall = max(1, Ny // 128) if wall is None else wall
    gam[:wall] = 0.0
    gam[Ny - wall:] = 0.0
    return gam


def density_field(Ny: int = 1024, Nx: int = 2048, seed: int = 0, U: float = 0.5, **over) -> Case:
    gam = density_gamma(Ny, Nx, seed)
    knobs = _base_knobs(Nx)
    knobs.update(convectionScheme=1, enableTwoPointFiveD=1, twoPointFiveDConvectionFactor=1.2,
                 brinkmanKMin=MU / 1e9, brinkmanQ=0.1, pTol=1e-8, maxPressureIter=30,
                 epsilon=1e-7, maxIterations=100000)
    knobs.update(over)
    return Case("density_field", _f32(1.0 - gam), U, 2e-4, knobs=knobs)


def constricted_channel(Ny: int = 32, Nx: int = 96, gap: int = 6, U: float = 0.5, **over) -> Case:
    """A straight channel (one solid wall row top and bottom) blocked over
    16 columns in the middle except for a gap of `gap` rows, with a row and a
    column of gamma = 0.5 along the block's faces; the density workload's
    physics (SOU, 2.5-D, Brinkman alpha_max 1e9, q 0.1).  The gap carries the
    flow at more than 3 U_in, so the reference's +-3 max(U_in, 0.1) velocity
    clamp is active at the converged state."""
    gam = np.ones((Ny, Nx))
    gam[:1] = 0.0
    gam[Ny - 1:] = 0.0
    c0, c1 = Nx // 2 - 8, Nx // 2 + 8
    lo = (Ny - gap) // 2
    gam[1:lo, c0:c1] = 0.0
    gam[lo + gap:Ny - 1, c0:c1] = 0.0
    gam[lo - 1, c0:c1] = 0.5
    gam[lo + gap, c0:c1] = 0.5
    gam[1:lo, c0 - 1] = 0.5
    gam[lo + gap:Ny - 1, c0 - 1] = 0.5
    knobs = _base_knobs(Nx)
    knobs.update(convectionScheme=1, enableTwoPointFiveD=1, twoPointFiveDConvectionFactor=1.2,
                 brinkmanKMin=MU / 1e9, brinkmanQ=0.1, pTol=1e-8, maxPressureIter=30,
                 epsilon=1e-7, maxIterations=100000)
    knobs.update(over)
    return Case("constricted_channel", _f32(1.0 - gam), U, 2e-4, knobs=knobs)


def batch(n: int = 64, seed: int = 0, **over) -> list[Case]:
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        Nx = int(rng.integers(256, 1025))
        Ny = int(rng.integers(128, 513))
        U = float(rng.uniform(0.2, 1.0))
        c = density_field(Ny, Nx, seed=int(rng.integers(0, 2 ** 31)), U=U, epsilon=1e-6, **over)
        c.name = f"batch{k}"
        out.append(c)
    return out


# the conjugate-heat-transfer workload on a converged density flow: 8 base
# plate and 4 channel layers, water, T_in 25 C, 200 um channels on a 0.5 mm plate
THERMAL_3D = dict(nz_solid=8, nz_fluid=4, k_s=400.0, k_f=0.6, rho=1000.0, Cp=4180.0, T_inlet=25.0,
                  H_t=2e-4, H_b=5e-4)


def power_map(Ny: int, Nx: int, seed: int) -> np.ndarray:
    """Heat flux [W/cm^2] (the unit of the reference's power_map.txt): 20
    W/cm^2 background plus 4-12 Gaussian hotspots with sigma U[20, 80] cells
    and peak U[50, 300] W/cm^2 at uniformly drawn centres."""
    rng = np.random.default_rng(seed)
    q = np.full((Ny, Nx), 20.0)
    y, x = np.mgrid[0:Ny, 0:Nx]
    for _ in range(int(rng.integers(4, 13))):
        cy, cx = rng.uniform(0, Ny), rng.uniform(0, Nx)
        sig, peak = rng.uniform(20.0, 80.0), rng.uniform(50.0, 300.0)
        q += peak * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * sig * sig))
    return q


WORKLOADS = {
    "straight_channel": straight_channel,
    "random_network": random_network,
    "density_field": density_field,
}
