"""CPU restatement of the reference's 3-D conjugate-heat-transfer assembly
(ThermalSolver/thermal_solver.cpp), test infrastructure only: tests, the
smoke check and bench.py's CPU baseline use it as the checker, nothing in the
product calls it.

The reference assembles, per cell (i, j, k) of an Nx x Ny x Nz grid (k = 0 the
bottom of the base plate, idx = k Nx Ny + j Nx + i), a 7-point finite-volume
row (thermal_solver.cpp:420-520):
  * x and y faces: diffusion with the harmonic mean of the cell
    conductivities, plus first-order upwind advection between two fluid
    cells with the face velocity (u_P + u_nb)/2 scaled by the Poiseuille
    factor of the layer; inlet (i = 0) Dirichlet T_in at half a cell with
    the advective inflow, outflow terms at i = Nx-1 and j = Ny-1;
  * z faces: diffusion only, conductivity averaged by layer thickness; the
    heat flux q0 enters the bottom layer;
  * conductivity: k_s in the base plate, RAMP k_f + (k_s - k_f)(1 - g) /
    (1 + qk g) above (thermal_solver.cpp:267-295); a cell is fluid above the
    base plate when gamma > 0.01;
  * the diagonal gets + 1e-12.
The sums run in the reference's order, so the assembled matrix and right-hand
side agree with the reference's to the last bit; the system is then solved
with scipy.  Pinned against the reference's own assembly (built against the
AMGCL stand-in in refbuild/shim, which dumps A, b and a tight solution) by
tests/test_thermal_oracle.py.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class ThermalParams:
    """thermal_solver.cpp:148-200 (defaults as there)."""
    Nx: int = 0
    Ny: int = 0
    nz_solid: int = 2
    nz_fluid: int = 7
    dx: float = 0.0
    dy: float = 0.0
    H_b: float = 0.0005
    H_t: float = 0.004
    k_s: float = 400.0
    k_f: float = 0.6
    rho: float = 998.0
    Cp: float = 4180.0
    T_inlet: float = 30.0
    k_interp_mode: int = 1
    qk: float = 1.0

    @property
    def Nz(self) -> int:
        return self.nz_solid + self.nz_fluid


def kval_layer(p: ThermalParams, g: np.ndarray) -> np.ndarray:
    """Conductivity of a fluid-layer cell from gamma (thermal_solver.cpp:267-295)."""
    g = np.clip(g, 0.0, 1.0)
    if p.k_interp_mode == 1:
        num = 1.0 - g
        den = 1.0 + p.qk * g
        return p.k_f + (p.k_s - p.k_f) * num / den
    if p.k_interp_mode == 2:
        return p.k_s * p.k_f / ((1.0 - g) * p.k_f + g * p.k_s + 1e-30)
    return p.k_s * (1.0 - g) + p.k_f * g


def assemble(p: ThermalParams, gamma: np.ndarray, u_xy: np.ndarray, v_xy: np.ndarray, q0: np.ndarray):
    """(A (scipy CSR), b): the reference's system for gamma (Ny x Nx, 1 = fluid),
    cell-centred velocities u_xy, v_xy (Ny x Nx, m/s) and bottom heat flux q0
    (Ny x Nx, W/m^2)."""
    import scipy.sparse as sp

    Nx, Ny, Nz = p.Nx, p.Ny, p.Nz
    # the reference keeps the domain length (cols * dx) and divides it again
    # (thermal_solver.cpp:186-187, 729)
    dx, dy = (Nx * p.dx) / Nx, (Ny * p.dy) / Ny
    rhoCp = p.rho * p.Cp
    T_in = p.T_inlet
    dz_s, dz_f = p.H_b / p.nz_solid, p.H_t / p.nz_fluid
    dz = np.array([dz_s] * p.nz_solid + [dz_f] * p.nz_fluid)
    n = Nx * Ny * Nz
    idx = np.arange(n).reshape(Nz, Ny, Nx)

    gam = np.asarray(gamma, dtype=np.float64)
    kf_layer = kval_layer(p, gam)
    K = np.empty((Nz, Ny, Nx))
    REG = np.zeros((Nz, Ny, Nx), dtype=bool)
    PO = np.zeros(Nz)
    for k in range(Nz):
        if k < p.nz_solid:
            K[k] = p.k_s
        else:
            K[k] = kf_layer
            REG[k] = gam > 0.01
            z = (k - p.nz_solid + 0.5) * dz_f / p.H_t
            PO[k] = 4.0 * z * (1 - z)
    gcl = np.clip(gam, 0.0, 1.0)

    def harm(a, b):
        return 2 * a * b / (a + b + 1e-30)

    diag = np.zeros((Nz, Ny, Nx))
    b = np.zeros((Nz, Ny, Nx))
    rows, cols, vals = [], [], []

    def add_off(mask, nb_shift, value):
        r = idx[mask]
        c = idx[mask] + nb_shift
        rows.append(r)
        cols.append(c)
        vals.append(value[mask])

    for k in range(Nz):
        dzk = dz[k]
        Ax, Ay, Az = dy * dzk, dx * dzk, dx * dy
        po = PO[k]
        kP = K[k]
        fl = k >= p.nz_solid
        g = gcl if fl else np.zeros((Ny, Nx))
        uP = np.where(g > 0.01, u_xy * po, 0.0)
        vP = np.where(g > 0.01, v_xy * po, 0.0)
        reg = REG[k]
        d = diag[k]
        bb = b[k]
        I = np.broadcast_to(np.arange(Nx), (Ny, Nx))
        J = np.broadcast_to(np.arange(Ny)[:, None], (Ny, Nx))
        off = {}   # neighbour -> summed off-diagonal value (2 entries at most, summed like the reference)
        # x faces
        # west
        m = I > 0
        kW = np.roll(kP, 1, axis=1)
        D = harm(kP, kW) * Ax / dx
        d += np.where(m, D, 0.0)
        offW = np.where(m, -D, 0.0)
        regW = np.roll(reg, 1, axis=1)
        adv = m & reg & regW
        uW = np.roll(u_xy, 1, axis=1) * po
        F = rhoCp * 0.5 * (uP + uW) * Ax
        d += np.where(adv, np.maximum(-F, 0.0), 0.0)
        offW = np.where(adv, offW + (-np.maximum(F, 0.0)), offW)
        off["W"] = (m, -1, offW)
        inl = (I == 0) & reg
        Dbc = 2.0 * kP * Ax / dx
        Fbc = rhoCp * uP * Ax
        d += np.where(inl, Dbc, 0.0)
        bb += np.where(inl, Dbc * T_in, 0.0)
        bb += np.where(inl & (Fbc > 0), Fbc * T_in, 0.0)
        d += np.where(inl & ~(Fbc > 0), -Fbc, 0.0)
        # east
        m = I < Nx - 1
        kE = np.roll(kP, -1, axis=1)
        D = harm(kP, kE) * Ax / dx
        d += np.where(m, D, 0.0)
        offE = np.where(m, -D, 0.0)
        regE = np.roll(reg, -1, axis=1)
        adv = m & reg & regE
        uE = np.roll(u_xy, -1, axis=1) * po
        F = rhoCp * 0.5 * (uP + uE) * Ax
        d += np.where(adv, np.maximum(F, 0.0), 0.0)
        offE = np.where(adv, offE + (-np.maximum(-F, 0.0)), offE)
        off["E"] = (m, 1, offE)
        outl = (I == Nx - 1) & reg & (uP > 0)
        d += np.where(outl, rhoCp * uP * Ax, 0.0)
        # y faces
        m = J > 0
        kS = np.roll(kP, 1, axis=0)
        D = harm(kP, kS) * Ay / dy
        d += np.where(m, D, 0.0)
        offS = np.where(m, -D, 0.0)
        regS = np.roll(reg, 1, axis=0)
        adv = m & reg & regS
        vS = np.roll(v_xy, 1, axis=0) * po
        F = rhoCp * 0.5 * (vP + vS) * Ay
        d += np.where(adv, np.maximum(-F, 0.0), 0.0)
        offS = np.where(adv, offS + (-np.maximum(F, 0.0)), offS)
        off["S"] = (m, -Nx, offS)
        m = J < Ny - 1
        kN = np.roll(kP, -1, axis=0)
        D = harm(kP, kN) * Ay / dy
        d += np.where(m, D, 0.0)
        offN = np.where(m, -D, 0.0)
        regN = np.roll(reg, -1, axis=0)
        adv = m & reg & regN
        vN = np.roll(v_xy, -1, axis=0) * po
        F = rhoCp * 0.5 * (vP + vN) * Ay
        d += np.where(adv, np.maximum(F, 0.0), 0.0)
        offN = np.where(adv, offN + (-np.maximum(-F, 0.0)), offN)
        off["N"] = (m, Nx, offN)
        topo = (J == Ny - 1) & reg & (vP > 0)
        d += np.where(topo, rhoCp * vP * Ay, 0.0)
        # z faces (diffusion only)
        if k > 0:
            kN_ = K[k - 1]
            dzP, dzN = dz[k], dz[k - 1]
            kfz = (dzP + dzN) / (dzP / kP + dzN / kN_)
            D = kfz * Az / (0.5 * (dzP + dzN))
            d += D
            off["B"] = (np.ones((Ny, Nx), dtype=bool), -Nx * Ny, -D)
        else:
            bb += q0 * Az
        if k < Nz - 1:
            kN_ = K[k + 1]
            dzP, dzN = dz[k], dz[k + 1]
            kfz = (dzP + dzN) / (dzP / kP + dzN / kN_)
            D = kfz * Az / (0.5 * (dzP + dzN))
            d += D
            off["T"] = (np.ones((Ny, Nx), dtype=bool), Nx * Ny, -D)
        for (mask, shift, value) in off.values():
            r = idx[k][mask]
            rows.append(r)
            cols.append(r + shift)
            vals.append(value[mask])
        rows.append(idx[k].ravel())
        cols.append(idx[k].ravel())
        vals.append((d + 1e-12).ravel())
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return A, b.ravel()


def solve(p: ThermalParams, gamma, u_xy, v_xy, q0) -> np.ndarray:
    """T (Nz x Ny x Nx) of the reference's system, by a sparse direct solve."""
    import scipy.sparse.linalg as spl
    A, b = assemble(p, gamma, u_xy, v_xy, q0)
    return spl.spsolve(A.tocsc(), b).reshape(p.Nz, p.Ny, p.Nx)


def pnorm(T: np.ndarray, pexp: float) -> float:
    """(mean over the bottom layer of T^p)^(1/p) (thermal_solver.cpp:346-362)."""
    Tb = T[0]
    return float(np.power(np.sum(np.power(Tb, pexp)) / Tb.size, 1.0 / pexp))


def dk_dgamma(p: ThermalParams, g: np.ndarray) -> np.ndarray:
    """dk/dgamma above the base plate at the clamped gamma; for RAMP the
    reference's dk_dgamma (thermal_solver.cpp:317-321)."""
    g = np.clip(g, 0.0, 1.0)
    if p.k_interp_mode == 1:
        den = 1.0 + p.qk * g
        return (p.k_s - p.k_f) * (-(1.0 + p.qk)) / (den * den)
    if p.k_interp_mode == 2:
        den = (1.0 - g) * p.k_f + g * p.k_s + 1e-30
        return -p.k_s * p.k_f * (p.k_s - p.k_f) / (den * den)
    return np.full_like(g, p.k_f - p.k_s)


def pnorm_gradient(p: ThermalParams, gamma, u_xy, v_xy, q0, pexp: float):
    """(J, dJ/dgamma (Ny x Nx), T, lambda) of J = (mean over the bottom
    layer of T^p)^(1/p) by the discrete adjoint of the assembled system:
    A^T lambda = dJ/dT, dJ/dgamma = -lambda^T dR/dgamma for R = A T - b,
    with velocities and fluid masks fixed.  gamma enters through the
    conductivity of the cells above the base plate: the x/y face
    conductances harm(k_P, k_N) A / h, the inlet conductance 2 k Ax / dx and
    the z conductances.  The reference computes no sensitivity
    (thermal_solver.cpp:377-378 fills zeros), so this is pinned by central
    finite differences of J (tests/test_thermal_oracle.py)."""
    import scipy.sparse.linalg as spl
    Nx, Ny, Nz, nzS = p.Nx, p.Ny, p.Nz, p.nz_solid
    A, b = assemble(p, gamma, u_xy, v_xy, q0)
    T = spl.spsolve(A.tocsc(), b)
    Tb = T[:Nx * Ny]
    J = float(np.power(np.sum(np.power(Tb, pexp)) / Tb.size, 1.0 / pexp))
    rhs = np.zeros_like(T)
    rhs[:Nx * Ny] = np.power(Tb / J, pexp - 1.0) / (Nx * Ny)
    lam = spl.spsolve(A.T.tocsc(), rhs)
    T3, L3 = T.reshape(Nz, Ny, Nx), lam.reshape(Nz, Ny, Nx)
    dx, dy = (Nx * p.dx) / Nx, (Ny * p.dy) / Ny
    dz = np.array([p.H_b / p.nz_solid] * p.nz_solid + [p.H_t / p.nz_fluid] * p.nz_fluid)
    gam = np.asarray(gamma, dtype=np.float64)
    K = np.empty((Nz, Ny, Nx))
    K[:nzS] = p.k_s
    K[nzS:] = kval_layer(p, gam)
    fluid = gam > 0.01

    def dharm(a, c):            # d/da of 2ac / (a + c + 1e-30)
        s_ = a + c + 1e-30
        return 2.0 * c * (c + 1e-30) / (s_ * s_)

    acc = np.zeros((Ny, Nx))
    for k in range(nzS, Nz):
        t, lm, kk = T3[k], L3[k], K[k]
        gx = dy * dz[k] / dx       # Ax / dx
        gy = dx * dz[k] / dy       # Ay / dy
        acc[:, 1:] += (lm[:, 1:] - lm[:, :-1]) * (t[:, 1:] - t[:, :-1]) * dharm(kk[:, 1:], kk[:, :-1]) * gx
        acc[:, :-1] += (lm[:, :-1] - lm[:, 1:]) * (t[:, :-1] - t[:, 1:]) * dharm(kk[:, :-1], kk[:, 1:]) * gx
        acc[1:, :] += (lm[1:, :] - lm[:-1, :]) * (t[1:, :] - t[:-1, :]) * dharm(kk[1:, :], kk[:-1, :]) * gy
        acc[:-1, :] += (lm[:-1, :] - lm[1:, :]) * (t[:-1, :] - t[1:, :]) * dharm(kk[:-1, :], kk[1:, :]) * gy
        acc[:, 0] += np.where(fluid[:, 0], lm[:, 0] * (t[:, 0] - p.T_inlet) * 2.0 * gx, 0.0)
    for k in range(nzS - 1, Nz - 1):
        kL, kU, dL, dU = K[k], K[k + 1], dz[k], dz[k + 1]
        den = dL / kL + dU / kU
        dkf = (dL + dU) * (dU / (kU * kU)) / (den * den)
        if k >= nzS:
            dkf = dkf + (dL + dU) * (dL / (kL * kL)) / (den * den)
        acc += (L3[k] - L3[k + 1]) * (T3[k] - T3[k + 1]) * dkf * (dx * dy) / (0.5 * (dL + dU))
    return J, -dk_dgamma(p, gam) * acc, T3, L3


def read_dump(path: str):
    """n, CSR (ptr, col, val), b, x written by the AMGCL stand-in."""
    import scipy.sparse as sp
    with open(path, "rb") as f:
        n, nnz = np.frombuffer(f.read(8), dtype=np.int32)
        ptr = np.frombuffer(f.read(4 * (n + 1)), dtype=np.int32)
        col = np.frombuffer(f.read(4 * nnz), dtype=np.int32)
        val = np.frombuffer(f.read(8 * nnz), dtype=np.float64)
        b = np.frombuffer(f.read(8 * n), dtype=np.float64)
        x = np.frombuffer(f.read(8 * n), dtype=np.float64)
    return sp.csr_matrix((val, col, ptr), shape=(n, n)), b, x


def write_case(case_dir: str, geometry: np.ndarray, u_xy: np.ndarray, v_xy: np.ndarray, dx: float, dy: float,
               qf: float, Ht: float, power_map_wcm2: np.ndarray | None = None) -> None:
    """The reference thermal solver's inputs (thermal_solver.cpp:700-755):
    thermal_params.txt (M N dx dy qf Ht), geometry_thermal.txt (0 fluid, 1
    solid), u_thermal.txt, v_thermal.txt and optionally power_map.txt (W/cm^2)."""
    import os
    os.makedirs(case_dir, exist_ok=True)
    Ny, Nx = geometry.shape
    with open(os.path.join(case_dir, "thermal_params.txt"), "w") as f:
        f.write(f"{Ny} {Nx} {dx:.17g} {dy:.17g} {qf:.17g} {Ht:.17g}\n")
    np.savetxt(os.path.join(case_dir, "geometry_thermal.txt"), geometry, fmt="%.17g")
    np.savetxt(os.path.join(case_dir, "u_thermal.txt"), u_xy, fmt="%.17g")
    np.savetxt(os.path.join(case_dir, "v_thermal.txt"), v_xy, fmt="%.17g")
    if power_map_wcm2 is not None:
        np.savetxt(os.path.join(case_dir, "power_map.txt"), power_map_wcm2, fmt="%.17g")
