"""Command-line replacement of the reference's thermal post-processor.

    PYTHONPATH=coldplate-solver_b200 python -m coldplate_b200.thermal_main [directory] [qk] [mode] [--pnorm P]

Same arguments as ``thermal_solver.exe [directory] [qk] [mode]``
(ThermalSolver/thermal_solver.cpp:675-691: directory default
../ExportFiles, RAMP parameter qk default 1, interpolation mode default 1).
Reads the case the way its main() does (thermal_params.txt,
geometry_thermal.txt, u_thermal.txt, v_thermal.txt, power_map.txt), solves
on the GPU, and writes thermal_metrics.txt, k_thermal.txt and T_bottom.txt
into the directory (thermal_solver.cpp:777-787).  With --pnorm P it also
writes dJ_dgamma.txt, the adjoint gradient of the bottom p-norm, which the
reference leaves to its Python adjoint step.  The VTK files are not
written.  Exit status 0 on success, 1 when the inputs cannot be read (as the
reference), 2 when the solve does not converge.
"""
from __future__ import annotations

import argparse
import os
import sys


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(prog="thermal_main")
    ap.add_argument("directory", nargs="?", default="../ExportFiles")
    ap.add_argument("qk", nargs="?", type=float, default=1.0)
    ap.add_argument("mode", nargs="?", type=int, default=1)
    ap.add_argument("--pnorm", type=float, default=None, help="also write dJ_dgamma.txt for this p")
    ap.add_argument("--rtol", type=float, default=None, help="solver tolerance (default: the reference's 1e-6)")
    a = ap.parse_args(argv)

    from .thermal import Thermal, load_case
    if not os.path.exists(os.path.join(a.directory, "thermal_params.txt")):
        print(f"Error: Cannot open {a.directory}/thermal_params.txt", file=sys.stderr)
        return 1
    try:
        prm, inp = load_case(a.directory, qk=a.qk, k_interp_mode=a.mode)
    except FileNotFoundError as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    if a.rtol is not None:
        prm["rtol"] = a.rtol
    with Thermal(**prm) as th:
        print(f"Grid: {th.Nx}x{th.Ny}x{th.Nz} = {th.Nx * th.Ny * th.Nz} DOFs")
        th.set_inputs(**inp)
        rep = th.solve()
        print(f"  BiCGStab + multigrid: {rep['iterations']} iters, res={rep['residual']:.3e} "
              f"({rep['device_ms'] / 1e3:.3f}s on the GPU)")
        if not rep["converged"]:
            print("Error: the thermal solve did not converge", file=sys.stderr)
            return 2
        files = th.save_outputs(a.directory, inp["gamma"], pnorm_exp=a.pnorm)
    for f in files:
        print(f"Saved: {a.directory}/{f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
