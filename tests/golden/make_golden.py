"""Generate the golden fixtures of the CPU parity tests.

Runs the reference solver's own sources (built by oracle/refbuild/build_ref.sh
into oracle/_ref/, float as shipped and re-typed double, both with
-ffp-contract=off) on three small seeded cases and stores, per case and
precision, the geometry, the run settings, the per-iteration history and the
final fields.  The oracle restatement must reproduce them bit for bit.

    python tests/golden/make_golden.py          (needs oracle/_ref/)
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "coldplate-solver_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from coldplate_b200 import cases  # noqa: E402
from oracle import run_reference, write_case  # noqa: E402

N_ITER = 40
FIELDS = ("u", "v", "p", "uStar", "vStar", "pStar", "dE", "dN")


def golden_cases():
    return {
        "straight": cases.straight_channel(16, 48),
        "network": cases.random_network(32, 64, seed=5),
        "density": cases.density_field(24, 40, seed=2),
    }


def main():
    for name, case in golden_cases().items():
        prm = case.params(maxIterations=N_ITER, epsilon=1e-12)
        for prec, binary in (("f32", "ref_f32_pin"), ("f64", "ref_f64_pin")):
            with tempfile.TemporaryDirectory() as d:
                write_case(d, case.cellType, case.hy, case.hx, case.U, case.Ht)
                res = run_reference(binary, d, prm)
            out = os.path.join(HERE, f"{name}_{prec}.npz")
            np.savez_compressed(
                out, cellType=case.cellType, hy=case.hy, hx=case.hx, U=case.U, Ht=case.Ht,
                params=json.dumps(prm), history=res.history,
                **{f"field_{k}": res.fields[k] for k in FIELDS})
            print(out, res.history.shape)


if __name__ == "__main__":
    main()
