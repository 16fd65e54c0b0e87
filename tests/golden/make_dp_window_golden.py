"""Generate tests/golden/dp_window.json: where the reference's own outer loop
stops under its pressure-drop window rule (SIMPLE.cpp:449-491).

For each case and window setting, the reference solver's sources (re-typed
double build, oracle/_ref/ref_f64_pin) run SIMPLE::runIterations() itself
(harness option run_native=1), which writes ExportFiles/residuals.txt one row
per completed iteration; the row count is the stop iteration.

    python tests/golden/make_dp_window_golden.py          (needs oracle/_ref/)
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "coldplate-solver_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from coldplate_b200 import cases  # noqa: E402
from oracle import REF_DIR, ref_overrides, write_case  # noqa: E402

MAX_ITER = 600
# (rampSteps, dpConvergenceWindow, dpConvergencePercent)
WINDOWS = ((50, 40, 1.0), (20, 30, 0.5), (100, 60, 0.2))


def window_cases():
    return {"density": cases.density_field(40, 80, seed=1), "network": cases.random_network(48, 96, seed=3)}


def window_params(case, ramp, window, pct):
    return case.params(usePressureDropConvergence=1, rampSteps=ramp, dpConvergenceWindow=window,
                       dpConvergencePercent=pct, epsilon=1e-30, maxIterations=MAX_ITER)


def reference_stop(binary, case, prm) -> int:
    with tempfile.TemporaryDirectory() as d:
        write_case(d, case.cellType, case.hy, case.hx, case.U, case.Ht)
        subprocess.run([os.path.join(REF_DIR, binary), d, d, *ref_overrides(prm), "run_native=1"], check=True,
                       stdout=subprocess.DEVNULL, timeout=600)
        with open(os.path.join(d, "ExportFiles", "residuals.txt")) as f:
            return sum(1 for line in f if line[:1].isdigit())


def main():
    out = []
    for name, case in window_cases().items():
        for ramp, window, pct in WINDOWS:
            n = reference_stop("ref_f64_pin", case, window_params(case, ramp, window, pct))
            out.append({"case": name, "rampSteps": ramp, "window": window, "percent": pct, "stop": n})
            print(out[-1])
    with open(os.path.join(HERE, "dp_window.json"), "w") as f:
        json.dump({"max_iter": MAX_ITER, "runs": out}, f, indent=1)


if __name__ == "__main__":
    main()
