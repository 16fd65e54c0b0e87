"""Time the 3-D thermal solve and its p-norm adjoint on a synthetic case.

    PYTHONPATH=coldplate-solver_b200 python -m coldplate_b200.thermal_run \\
        [--ny 512] [--nx 1024] [--seed 0] [--rtol 1e-6] [--maxiter 2000] [--repeat 3] [--no-adjoint]

The case: the density geometry of the flow workloads (gamma from
cases.density_gamma), channel velocity 0.5 gamma m/s along x with a small
random cross-flow, the hotspot power map, and the 8 + 4 layer settings of
cases.THERMAL_3D.  Prints one JSON line with device times (CUDA events on
the solver's stream) of the last repeat.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import cases
from .thermal import Thermal


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--rtol", type=float, default=1e-6)
    ap.add_argument("--maxiter", type=int, default=2000)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--no-adjoint", action="store_true")
    a = ap.parse_args()
    Ny, Nx = a.ny, a.nx
    gam = cases.density_gamma(Ny, Nx, a.seed)
    rng = np.random.default_rng(a.seed)
    u = 0.5 * gam
    v = 0.02 * (rng.random((Ny, Nx)) - 0.5) * gam
    q0 = cases.power_map(Ny, Nx, a.seed) * 1e4
    prm = dict(Nx=Nx, Ny=Ny, dx=cases.H, dy=cases.H, rtol=a.rtol, maxiter=a.maxiter, **cases.THERMAL_3D)
    out = {"case": f"{Nx}x{Ny}x{prm['nz_solid'] + prm['nz_fluid']} seed {a.seed}", "rtol": a.rtol}
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        for _ in range(a.repeat):
            r = th.solve()
            out["forward"] = r
            if not a.no_adjoint:
                J, g, ra = th.pnorm_gradient(8)
                out["adjoint"] = ra
                out["J"] = J
        out["Tb_max"], out["Tb_pnorm"] = th.objective(8)
    out["forward_ms_per_iteration"] = out["forward"]["device_ms"] / max(out["forward"]["iterations"], 1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
