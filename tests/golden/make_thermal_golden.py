"""Generate the golden fixtures of the thermal parity tests.

Runs the reference's thermal solver (ThermalSolver/thermal_solver.cpp, built
by oracle/refbuild/build_ref.sh into oracle/_ref/thermal_ref_pin against the
AMGCL API stand-in, which dumps the assembled system and a tight solution)
on two small seeded cases, a uniform heat flux and a power map, and stores
the inputs, the CSR matrix, the right-hand side, the solution and the text
files its main() wrote.  The oracle's assembly must reproduce the system bit
for bit, and the writers of coldplate_b200.output the files byte for byte.

    python tests/golden/make_thermal_golden.py          (needs oracle/_ref/)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "coldplate-solver_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from coldplate_b200 import cases  # noqa: E402
from thermal_oracle import read_dump, write_case  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "thermal_ref_pin")
CASE = dict(Ny=10, Nx=22, dx=2e-5, dy=2e-5, qf=5.0e5, Ht=2e-4)
FILES = ("thermal_metrics.txt", "k_thermal.txt", "T_bottom.txt")


def inputs(seed):
    Ny, Nx = CASE["Ny"], CASE["Nx"]
    gam = cases.density_gamma(Ny, Nx, seed, buffer=3)
    rng = np.random.default_rng(seed)
    u = gam * (0.4 + 0.2 * rng.random((Ny, Nx))) - 0.05 * rng.random((Ny, Nx))
    v = 0.1 * (rng.random((Ny, Nx)) - 0.5) * gam
    pm = 20.0 + 80.0 * rng.random((Ny, Nx))
    return gam, u, v, pm


def main():
    for name, seed, with_map in (("thermal_uniform", 3, False), ("thermal_map", 8, True)):
        gam, u, v, pm = inputs(seed)
        with tempfile.TemporaryDirectory() as d:
            case = os.path.join(d, "case")
            write_case(case, 1.0 - gam, u, v, CASE["dx"], CASE["dy"], CASE["qf"], CASE["Ht"],
                       pm if with_map else None)
            dump = os.path.join(d, "dump.bin")
            subprocess.run([REF, case], check=True, capture_output=True, timeout=600,
                           env=dict(os.environ, CP_AMGCL_SHIM_DUMP=dump, OMP_NUM_THREADS="1"))
            A, b, x = read_dump(dump)
            texts = {f: open(os.path.join(case, f), "rb").read() for f in FILES}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), geometry=1.0 - gam, u=u, v=v,
                            power_map=pm if with_map else np.zeros((0, 0)), indptr=A.indptr, indices=A.indices,
                            data=A.data, b=b, x=x, case=np.array([CASE[k] for k in ("Ny", "Nx", "dx", "dy", "qf", "Ht")]),
                            **{f.replace(".txt", ""): np.frombuffer(t, dtype=np.uint8) for f, t in texts.items()})
        print("wrote", name)


if __name__ == "__main__":
    main()
