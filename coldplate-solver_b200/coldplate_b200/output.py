"""The reference's on-disk result formats, written from this library's fields
and history, so that tools that read the reference's ExportFiles/ (plotting
scripts, the MMA driver, the thermal post-processor) take GPU results
unchanged.

Formats (Utilities/output.cpp):
  * matrices, saveMatrix (:48-72): one text row per matrix row, values
    tab-separated, printed as C++ streams print a float by default (six
    significant digits, %g style);
  * saveAll (:74-200): the staggered u, v, p; cell-centred u_full, v_full,
    pressure_full, u_resid_full, v_resid_full; the pressure-gradient
    magnitude and the thermal crops u_thermal, v_thermal, pressure_thermal,
    p_gradient (columns N_in_buffer .. Nx - N_out_buffer - 1).  The VTK file
    that saveAll also writes is not produced;
  * the per-iteration logs of initLogFiles / writeIterationLogs (:302-364):
    residuals.txt and pressure_drop_history.txt.
The reference keeps every field in float; the values are rounded to float
and combined in float in the reference's order, so the files match the
reference's byte for byte on the same state.
"""
from __future__ import annotations

import os

import numpy as np


def _fmt(x: np.float32) -> str:
    # C++ operator<<(float) with default flags: %g with six significant digits
    return "%.6g" % float(x)


def save_matrix(path: str, a) -> None:
    """saveMatrix (output.cpp:48-72) for a 2-D array."""
    a = np.asarray(a, dtype=np.float32)
    with open(path, "w") as f:
        for row in a:
            f.write("\t".join(_fmt(x) for x in row))
            f.write("\n")


def save_all(export_dir: str, u, v, p, hx: float, hy: float, n_in_buffer: int = 0, n_out_buffer: int = 0,
             u_old=None, v_old=None) -> list[str]:
    """The text files of saveAll (output.cpp:74-200) for staggered fields
    u (M+1 x N), v (M x N+1), p (M+1 x N+1).  u_old / v_old (the fields at
    the start of the last iteration) are needed for u_resid_full and
    v_resid_full; without them those two files are not written.  Returns
    the file names written."""
    f32 = np.float32
    u, v, p = (np.asarray(x, dtype=f32) for x in (u, v, p))
    M, N = p.shape[0] - 1, p.shape[1] - 1
    rows, cols = M - 1, N - 1
    os.makedirs(export_dir, exist_ok=True)
    out = []

    def put(name, a):
        save_matrix(os.path.join(export_dir, name + ".txt"), a)
        out.append(name + ".txt")

    put("u", u)
    put("v", v)
    put("p", p)
    half = f32(0.5)
    # cell centres: u averaged over the west/east faces, v over south/north
    uC = half * (u[1:rows + 1, 0:cols] + u[1:rows + 1, 1:cols + 1])
    vC = half * (v[0:rows, 1:cols + 1] + v[1:rows + 1, 1:cols + 1])
    pC = p[1:rows + 1, 1:cols + 1].copy()
    put("u_full", uC)
    put("v_full", vC)
    put("pressure_full", pC)
    if u_old is not None and v_old is not None:
        uo, vo = np.asarray(u_old, dtype=f32), np.asarray(v_old, dtype=f32)
        duW = u[1:rows + 1, 0:cols] - uo[1:rows + 1, 0:cols]
        duE = u[1:rows + 1, 1:cols + 1] - uo[1:rows + 1, 1:cols + 1]
        dvS = v[0:rows, 1:cols + 1] - vo[0:rows, 1:cols + 1]
        dvN = v[1:rows + 1, 1:cols + 1] - vo[1:rows + 1, 1:cols + 1]
        put("u_resid_full", half * (np.abs(duW) + np.abs(duE)))
        put("v_resid_full", half * (np.abs(dvS) + np.abs(dvN)))
    # pressure gradient magnitude: central differences inside, one-sided at the edges
    hx32, hy32 = f32(hx), f32(hy)
    gx = np.zeros_like(pC)
    gy = np.zeros_like(pC)
    if cols > 1:
        gx[:, 1:cols - 1] = (pC[:, 2:] - pC[:, :-2]) / (f32(2.0) * hx32)
        gx[:, 0] = (pC[:, 1] - pC[:, 0]) / hx32
        gx[:, cols - 1] = (pC[:, cols - 1] - pC[:, cols - 2]) / hx32
    if rows > 1:
        gy[1:rows - 1, :] = (pC[2:, :] - pC[:-2, :]) / (f32(2.0) * hy32)
        gy[0, :] = (pC[1, :] - pC[0, :]) / hy32
        gy[rows - 1, :] = (pC[rows - 1, :] - pC[rows - 2, :]) / hy32
    gmag = np.sqrt(gx * gx + gy * gy)
    n_th = cols - n_in_buffer - n_out_buffer
    if n_th > 0:
        sl = slice(n_in_buffer, n_in_buffer + n_th)
        put("u_thermal", uC[:, sl])
        put("v_thermal", vC[:, sl])
        put("pressure_thermal", pC[:, sl])
        put("p_gradient", gmag[:, sl])
    return out


RESID_HEADER = ("Iter MassRMS U_RMS V_RMS MassRMSn U_RMSn V_RMSn NormEnabled "
                "Core_dP_AfterInletBuffer(Pa) Full_dP_FullSystem(Pa) CFL CFL_ratio")
DP_HEADER = "Iter Core_Total(Pa) Full_Total(Pa) Core_Static(Pa) Full_Static(Pa)"


def write_logs(export_dir: str, hist: dict, normalized: bool = False, vel_floor: float = 1e-6,
               mass_floor: float = 1e-12, cfl: float = 0.1, cfl_ratio: float = 0.0) -> None:
    """residuals.txt and pressure_drop_history.txt (output.cpp:302-364) from
    history rows (``Simple.history()`` or the same columns).  The normalised
    columns divide by the first RMS above its floor, as the reference's
    bookkeeping does (iterations.cpp:628-656); cfl / cfl_ratio are the
    pseudo-time controller's values, which stay at their initial 0.1 / 0
    while pseudo-time stepping is off (the only mode this library runs)."""
    f32 = np.float32
    os.makedirs(export_dir, exist_ok=True)
    n = len(hist["iter"])

    # RMS0: the first RMS above its floor, the floor itself until then
    floors = {"residMass_RMS": f32(max(mass_floor, 1e-30)), "residU_RMS": f32(max(vel_floor, 1e-30)),
              "residV_RMS": f32(max(vel_floor, 1e-30))}
    rms0 = {c: None for c in floors}
    with open(os.path.join(export_dir, "residuals.txt"), "w") as fr, \
            open(os.path.join(export_dir, "pressure_drop_history.txt"), "w") as fd:
        fr.write(RESID_HEADER + "\n")
        fd.write(DP_HEADER + "\n")
        for k in range(n):
            it = int(hist["iter"][k])
            m, uu, vv = (f32(hist[c][k]) for c in ("residMass_RMS", "residU_RMS", "residV_RMS"))
            for c, x in (("residMass_RMS", m), ("residU_RMS", uu), ("residV_RMS", vv)):
                if rms0[c] is None and x > floors[c]:
                    rms0[c] = x
            r0 = {c: (rms0[c] if rms0[c] is not None else floors[c]) for c in floors}
            # rms / rms0 in float (output.cpp:339-341)
            mn = m / r0["residMass_RMS"] if r0["residMass_RMS"] > 0 else f32(0.0)
            un = uu / r0["residU_RMS"] if r0["residU_RMS"] > 0 else f32(0.0)
            vn = vv / r0["residV_RMS"] if r0["residV_RMS"] > 0 else f32(0.0)
            core, full = f32(hist["coreTotal"][k]), f32(hist["fullTotal"][k])
            cs, fs = f32(hist["coreStatic"][k]), f32(hist["fullStatic"][k])
            fr.write(" ".join([str(it), _fmt(m), _fmt(uu), _fmt(vv), _fmt(mn), _fmt(un), _fmt(vn),
                               "1" if normalized else "0", _fmt(core), _fmt(full), _fmt(f32(cfl)),
                               _fmt(f32(cfl_ratio))]) + "\n")
            fd.write(" ".join([str(it), _fmt(core), _fmt(full), _fmt(cs), _fmt(fs)]) + "\n")


# ---------------------------------------------------------------- thermal files
def _seqsum(a: np.ndarray) -> float:
    """Left-to-right float64 sum (the reference's accumulation loops)."""
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    return float(np.cumsum(a)[-1]) if a.size else 0.0


def thermal_metrics(T, gamma, dx: float, dy: float, dz_cells, nz_solid: int) -> dict:
    """compute_thermal_metrics (ThermalSolver/thermal_output.cpp:135-323) for
    T (Nz x Ny x Nx), gamma (Ny x Nx, 1 fluid), the cell sizes and the layer
    thicknesses: volume-weighted averages, standard deviations, ranges,
    uniformity indices and gradient statistics of the base plate, the fluid,
    the solid fins and the whole domain, summed in the reference's loop
    order."""
    T = np.asarray(T, dtype=np.float64)
    Nz, Ny, Nx = T.shape
    dz = np.asarray(dz_cells, dtype=np.float64)
    V = (dx * dy) * dz                                  # per layer, as dx * dy * dz_k
    Vc = np.broadcast_to(V[:, None, None], T.shape)
    TV = T * Vc
    base = np.zeros(T.shape, dtype=bool)
    base[:nz_solid] = True
    fl2 = np.asarray(gamma, dtype=np.float64) > 0.01
    fluid = np.zeros(T.shape, dtype=bool)
    fluid[nz_solid:] = fl2[None]
    solid = ~base & ~fluid
    z = 0.0

    def avg(mask):
        sv = _seqsum(np.where(mask, Vc, z))
        return (_seqsum(np.where(mask, TV, z)) / sv if sv > 0 else 0.0), sv

    m = {}
    m["T_avg_base"], sVb = avg(base)
    m["T_avg_fluid"], sVf = avg(fluid)
    m["T_avg_solid"], _ = avg(solid)
    m["T_avg_global"], sVg = avg(np.ones(T.shape, dtype=bool))

    def rng(mask, sv):
        return float(T[mask].max() - T[mask].min()) if sv > 0 else 0.0

    m["T_range_base"] = rng(base, sVb)
    m["T_range_fluid"] = rng(fluid, sVf)
    m["T_range_global"] = rng(np.ones(T.shape, dtype=bool), sVg)

    def std(mask, mean, sv):
        d = T - mean
        s = _seqsum(np.where(mask, Vc * d * d, z))
        return float(np.sqrt(s / sv if sv > 0 else 0.0))

    m["T_std_base"] = std(base, m["T_avg_base"], sVb)
    m["T_std_fluid"] = std(fluid, m["T_avg_fluid"], sVf)
    m["T_std_global"] = std(np.ones(T.shape, dtype=bool), m["T_avg_global"], sVg)

    def unif(s, a):
        return 0.0 if a <= 0.0 else max(0.0, min(1.0, 1.0 - s / a))

    m["T_uniformity_base"] = unif(m["T_std_base"], m["T_avg_base"])
    m["T_uniformity_global"] = unif(m["T_std_global"], m["T_avg_global"])
    # gradients: central differences inside, one-sided at the faces
    # (compute_gradient_components, thermal_output.cpp:64-108)
    gx = np.empty_like(T)
    gy = np.empty_like(T)
    gz = np.empty_like(T)
    gx[:, :, 1:-1] = (T[:, :, 2:] - T[:, :, :-2]) / (2.0 * dx)
    gx[:, :, 0] = (T[:, :, 1] - T[:, :, 0]) / dx
    gx[:, :, -1] = (T[:, :, -1] - T[:, :, -2]) / dx
    gy[:, 1:-1, :] = (T[:, 2:, :] - T[:, :-2, :]) / (2.0 * dy)
    gy[:, 0, :] = (T[:, 1, :] - T[:, 0, :]) / dy
    gy[:, -1, :] = (T[:, -1, :] - T[:, -2, :]) / dy
    for k in range(Nz):
        if k == 0:
            gz[k] = (T[1] - T[0]) / dz[0]
        elif k == Nz - 1:
            gz[k] = (T[k] - T[k - 1]) / dz[Nz - 1]
        else:
            gz[k] = (T[k + 1] - T[k - 1]) / (2.0 * (0.5 * (dz[k - 1] + dz[k])))
    g = np.sqrt(gx * gx + gy * gy + gz * gz)
    flat = int(np.argmax(g))
    m["grad_max"] = float(g.ravel()[flat])
    m["grad_max_k"], m["grad_max_j"], m["grad_max_i"] = (int(v) for v in np.unravel_index(flat, T.shape))
    m["grad_avg"] = _seqsum(g * Vc) / sVg if sVg > 0 else 0.0
    m["grad_max_base"] = float(g[:nz_solid].max())
    m["grad_avg_base"] = _seqsum(np.where(base, g * Vc, z)) / sVb if sVb > 0 else 0.0
    return m


def save_thermal_metrics(export_dir: str, m: dict) -> None:
    """thermal_metrics.txt in the layout of save_thermal_metrics
    (thermal_output.cpp:326-371), values as C++ fixed with 4 decimals."""
    f4 = "%.4f"
    lines = ["# Thermal Metrics - Volume-Weighted Statistics", "# All temperatures in [C]", "#",
             "# Average Temperatures",
             "T_avg_base    " + f4 % m["T_avg_base"], "T_avg_fluid   " + f4 % m["T_avg_fluid"],
             "T_avg_solid   " + f4 % m["T_avg_solid"], "T_avg_global  " + f4 % m["T_avg_global"], "#",
             "# Standard Deviations",
             "T_std_base    " + f4 % m["T_std_base"], "T_std_fluid   " + f4 % m["T_std_fluid"],
             "T_std_global  " + f4 % m["T_std_global"], "#",
             "# Temperature Ranges (max - min)",
             "T_range_base  " + f4 % m["T_range_base"], "T_range_fluid " + f4 % m["T_range_fluid"],
             "T_range_global" + f4 % m["T_range_global"], "#",
             "# Uniformity Indices (1 = uniform, 0 = non-uniform)",
             "T_uniformity_base   " + f4 % m["T_uniformity_base"],
             "T_uniformity_global " + f4 % m["T_uniformity_global"], "#",
             "# Thermal Gradients [C/m]",
             "grad_max          " + f4 % m["grad_max"], "grad_avg          " + f4 % m["grad_avg"],
             "grad_max_base     " + f4 % m["grad_max_base"], "grad_avg_base     " + f4 % m["grad_avg_base"],
             "grad_max_loc      %d %d %d" % (m["grad_max_i"], m["grad_max_j"], m["grad_max_k"])]
    with open(os.path.join(export_dir, "thermal_metrics.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")


def _save_fixed(path: str, a, decimals: int) -> None:
    fmt = "%%.%df" % decimals
    with open(path, "w") as f:
        for row in np.asarray(a, dtype=np.float64):
            f.write("\t".join(fmt % x for x in row) + "\n")


def save_thermal_outputs(export_dir: str, T, gamma, dx: float, dy: float, dz_cells, nz_solid: int,
                         k_s: float, k_f: float, qk: float, dJ_dgamma=None) -> list[str]:
    """The text files the reference's thermal main() writes
    (thermal_solver.cpp:777-787): thermal_metrics.txt, k_thermal.txt (the
    RAMP conductivity of the channel layer, fixed 6 decimals,
    thermal_output.cpp:530-570) and T_bottom.txt (the k = 0 layer, fixed 4
    decimals, :621-650).  With dJ_dgamma given, also dJ_dgamma.txt as the
    optimiser's adjoint step writes it (tab-separated %.10e,
    AdjointMethod/thermal_adjoint.py:156).  dx, dy are the cell sizes as given;
    the domain length is divided again as the reference does
    (thermal_solver.cpp:186-187).  The VTK files are not written."""
    os.makedirs(export_dir, exist_ok=True)
    T = np.asarray(T, dtype=np.float64)
    Nz, Ny, Nx = T.shape
    dxr, dyr = (Nx * dx) / Nx, (Ny * dy) / Ny
    save_thermal_metrics(export_dir, thermal_metrics(T, gamma, dxr, dyr, dz_cells, nz_solid))
    g = np.clip(np.asarray(gamma, dtype=np.float64), 0.0, 1.0)
    k = k_f + (k_s - k_f) * (1.0 - g) / (1.0 + qk * g)
    _save_fixed(os.path.join(export_dir, "k_thermal.txt"), k, 6)
    _save_fixed(os.path.join(export_dir, "T_bottom.txt"), T[0], 4)
    out = ["thermal_metrics.txt", "k_thermal.txt", "T_bottom.txt"]
    if dJ_dgamma is not None:
        with open(os.path.join(export_dir, "dJ_dgamma.txt"), "w") as f:
            for row in np.asarray(dJ_dgamma, dtype=np.float64):
                f.write("\t".join("%.10e" % x for x in row) + "\n")
        out.append("dJ_dgamma.txt")
    return out
