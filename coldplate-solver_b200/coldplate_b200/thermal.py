"""The 3-D conjugate-heat-transfer solve on the GPU (include/cp_thermal.h).

Mirrors the reference's ThermalSolver3D (ThermalSolver/thermal_solver.cpp):
the same parameters and defaults (struct Params, :148-200), inputs gamma
(1 fluid .. 0 solid), the cell-centred velocities u_xy / v_xy and the bottom
heat flux q0 on the Ny x Nx plane, ``solve()`` (:422), ``T`` (Nz x Ny x Nx),
``compute_pnorm_objective`` (:345-358) and ``compute_optimization_results``
(:361-386), whose sensitivity here is the discrete adjoint instead of the
reference's zeros.  ``load_case`` reads a case directory the way the
reference's main() does (:675-772).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._native import CpThermalParams, CpThermalReport, check, lib

_PARAM_NAMES = [f for f, _ in CpThermalParams._fields_]


def default_thermal_params() -> CpThermalParams:
    p = CpThermalParams()
    lib().cp_thermal_params_default(ctypes.byref(p))
    return p


def _plane(a, Ny: int, Nx: int, name: str) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != (Ny, Nx):
        raise ValueError(f"{name} must be {Ny} x {Nx}, got {a.shape}")
    return a


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _report(r: CpThermalReport) -> dict:
    return {"iterations": r.iterations, "converged": bool(r.converged), "residual": r.residual,
            "device_ms": r.device_ms}


class Thermal:
    """One thermal problem resident on the GPU.  Keyword arguments are the
    fields of cp_thermal_params (Nx, Ny, dx, dy required)."""

    def __init__(self, **kw):
        p = default_thermal_params()
        for k, v in kw.items():
            if k not in _PARAM_NAMES:
                raise TypeError(f"unknown thermal parameter {k!r}")
            setattr(p, k, v)
        self.params = p
        h = ctypes.c_void_p()
        check(lib().cp_thermal_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.Nx, self.Ny, self.Nz = p.Nx, p.Ny, p.nz_solid + p.nz_fluid

    # -- lifetime
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().cp_thermal_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- inputs, solve, outputs
    def set_inputs(self, gamma, u_xy, v_xy, q0) -> None:
        """gamma (1 fluid, 0 solid), velocities [m/s], bottom flux [W/m^2]; Ny x Nx each."""
        a = [_plane(x, self.Ny, self.Nx, n) for x, n in ((gamma, "gamma"), (u_xy, "u_xy"), (v_xy, "v_xy"),
                                                          (q0, "q0"))]
        check(lib().cp_thermal_set_inputs(self._h, *[_dptr(x) for x in a]))

    def solve(self) -> dict:
        r = CpThermalReport()
        check(lib().cp_thermal_solve(self._h, ctypes.byref(r)))
        return _report(r)

    @property
    def T(self) -> np.ndarray:
        out = np.empty((self.Nz, self.Ny, self.Nx))
        check(lib().cp_thermal_get_T(self._h, _dptr(out)))
        return out

    def objective(self, pnorm_exp: float = 10) -> tuple[float, float]:
        """(Tb_max, Tb_pnorm) of the bottom layer."""
        mx, pn = ctypes.c_double(), ctypes.c_double()
        check(lib().cp_thermal_objective(self._h, float(pnorm_exp), ctypes.byref(mx), ctypes.byref(pn)))
        return mx.value, pn.value

    def compute_pnorm_objective(self, pnorm_exp: float = 10) -> float:
        return self.objective(pnorm_exp)[1]

    def pnorm_gradient(self, pnorm_exp: float = 10) -> tuple[float, np.ndarray, dict]:
        """(J, dJ/dgamma (Ny x Nx), adjoint-solve report)."""
        g = np.empty((self.Ny, self.Nx))
        J = ctypes.c_double()
        r = CpThermalReport()
        check(lib().cp_thermal_pnorm_gradient(self._h, float(pnorm_exp), ctypes.byref(J), _dptr(g),
                                              ctypes.byref(r)))
        return J.value, g, _report(r)

    def save_outputs(self, export_dir: str, gamma, pnorm_exp: float | None = None) -> list[str]:
        """The reference's thermal result files from the current solution
        (coldplate_b200.output.save_thermal_outputs): thermal_metrics.txt,
        k_thermal.txt, T_bottom.txt, and with pnorm_exp given also
        dJ_dgamma.txt from the adjoint, in the format the optimiser reads.
        gamma is the field passed to set_inputs."""
        from . import output
        p = self.params
        dz = [p.H_b / p.nz_solid] * p.nz_solid + [p.H_t / p.nz_fluid] * p.nz_fluid
        g = self.pnorm_gradient(pnorm_exp)[1] if pnorm_exp is not None else None
        return output.save_thermal_outputs(export_dir, self.T, gamma, p.dx, p.dy, dz, p.nz_solid, p.k_s, p.k_f,
                                           p.qk, dJ_dgamma=g)

    def compute_optimization_results(self, pnorm_exp: float = 10) -> dict:
        """Tb_max, Tb_pnorm and dJ_dgamma (Ny x Nx) of the current solution."""
        mx, _ = self.objective(pnorm_exp)
        J, g, _ = self.pnorm_gradient(pnorm_exp)
        return {"Tb_max": mx, "Tb_pnorm": J, "dJ_dgamma": g}


def _read_2d(path: str) -> np.ndarray | None:
    """read_2d (thermal_solver.cpp:210-221): whitespace-separated rows,
    blank and '#' lines skipped; None when the file cannot be opened."""
    if not os.path.exists(path):
        return None
    rows = []
    with open(path) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            row = [float(x) for x in line.split()]
            if row:
                rows.append(row)
    if not rows:
        return np.zeros((0, 0))
    cols = len(rows[0])
    return np.array([r[:cols] + [0.0] * (cols - len(r)) for r in rows])


def load_case(case_dir: str, qk: float = 1.0, k_interp_mode: int = 1) -> tuple[dict, dict]:
    """(parameters, inputs) of a case directory as the reference's main()
    builds them (thermal_solver.cpp:700-772): thermal_params.txt
    ``M N dx dy qf Ht``; geometry_thermal.txt (0 fluid, 1 solid) sets the
    grid and gamma = 1 - value; u_thermal.txt / v_thermal.txt; power_map.txt
    in W/cm^2 when its size matches the grid, otherwise the uniform qf."""
    with open(os.path.join(case_dir, "thermal_params.txt")) as f:
        tok = f.read().split()
    dx, dy, qf, Ht = (float(x) for x in tok[2:6])
    geo = _read_2d(os.path.join(case_dir, "geometry_thermal.txt"))
    if geo is None or geo.size == 0:
        raise FileNotFoundError(f"{case_dir}/geometry_thermal.txt could not be loaded")
    Ny, Nx = geo.shape
    gamma = 1.0 - geo
    u_xy, v_xy = np.zeros((Ny, Nx)), np.zeros((Ny, Nx))
    u = _read_2d(os.path.join(case_dir, "u_thermal.txt"))
    v = _read_2d(os.path.join(case_dir, "v_thermal.txt"))
    if u is not None and u.size:
        r, c = min(Ny, u.shape[0]), min(Nx, u.shape[1])
        u_xy[:r, :c] = u[:r, :c]
        v_xy[:r, :c] = v[:r, :c]
    pm = _read_2d(os.path.join(case_dir, "power_map.txt"))
    if pm is not None and pm.shape == (Ny, Nx):
        q0 = pm * 10000.0
    else:
        q0 = np.full((Ny, Nx), qf)
    prm = dict(Nx=Nx, Ny=Ny, dx=dx, dy=dy, H_t=Ht, qk=qk, k_interp_mode=k_interp_mode)
    return prm, dict(gamma=gamma, u_xy=u_xy, v_xy=v_xy, q0=q0)


def inputs_from_flow(simple, cellType, n_in_buffer: int = 0, n_out_buffer: int = 0) -> dict:
    """gamma, u_xy, v_xy of the thermal domain from a flow solve: the
    cell-centred velocities (u averaged over the west/east faces, v over
    south/north, output.cpp:90-107) and gamma = 1 - cellType, cropped to
    columns n_in_buffer .. Nx - n_out_buffer - 1 like the reference's
    u_thermal / v_thermal / geometry_thermal files (output.cpp:171-198,
    GeometryGenerator_V6.py:512), without their text rounding."""
    ct = np.asarray(cellType, dtype=np.float64)
    Ny, Nx = ct.shape
    u, v = simple.get("u"), simple.get("v")
    uC = 0.5 * (u[1:Ny + 1, 0:Nx] + u[1:Ny + 1, 1:Nx + 1])
    vC = 0.5 * (v[0:Ny, 1:Nx + 1] + v[1:Ny + 1, 1:Nx + 1])
    sl = slice(n_in_buffer, Nx - n_out_buffer)
    return dict(gamma=np.ascontiguousarray(1.0 - ct[:, sl]), u_xy=np.ascontiguousarray(uC[:, sl]),
                v_xy=np.ascontiguousarray(vC[:, sl]))
