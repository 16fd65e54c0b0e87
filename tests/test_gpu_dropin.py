"""The compiled drop-in: the reference's own outer loop over the library.

oracle/_ref/ref_dropin is the reference's sources as shipped with
Utilities/iterations.cpp replaced by coldplate-solver_b200/dropin/
iterations_gpu.cpp and linked against libcoldplate.so (built by
oracle/refbuild/build_ref.sh).  Run through SIMPLE::runIterations() itself
(harness option run_native=1), it must write residuals.txt and
pressure_drop_history.txt that match the ones the Python path
(coldplate_b200.Simple, the same library through ctypes) writes for the same
case, and its default-on pressure-drop window rule must stop the loop where
the reference does (tests/golden/dp_window.json).
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from oracle import REF_DIR, ref_overrides, write_case

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_dp_window_golden import window_cases, window_params  # noqa: E402

pytestmark = pytest.mark.gpu
EXE = os.path.join(REF_DIR, "ref_dropin")


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    if not os.path.exists(EXE):
        pytest.fail("oracle/_ref/ref_dropin is missing: build it with oracle/refbuild/build_ref.sh")
    return built_lib


def _run_dropin(case, prm) -> tuple[np.ndarray, np.ndarray]:
    with tempfile.TemporaryDirectory() as d:
        write_case(d, case.cellType, case.hy, case.hx, case.U, case.Ht)
        subprocess.run([EXE, d, d, *ref_overrides(prm), "run_native=1"], check=True, stdout=subprocess.DEVNULL,
                       timeout=600)
        ex = os.path.join(d, "ExportFiles")
        return (np.loadtxt(os.path.join(ex, "residuals.txt"), comments=("#", "I", "i"), ndmin=2),
                np.loadtxt(os.path.join(ex, "pressure_drop_history.txt"), comments=("#", "I", "i"), ndmin=2))


def _logs_of(g) -> tuple[np.ndarray, np.ndarray]:
    with tempfile.TemporaryDirectory() as d:
        g.writeIterationLogs(d)
        return (np.loadtxt(os.path.join(d, "residuals.txt"), comments=("#", "I", "i"), ndmin=2),
                np.loadtxt(os.path.join(d, "pressure_drop_history.txt"), comments=("#", "I", "i"), ndmin=2))


# SIMPLE.h float members the case does not set, at their defaults
_FLOAT_DEFAULTS = dict(uvAlpha=0.7, pAlpha=0.3, momentumTol=1e-6, residNormFloorVel=1e-6, residNormFloorMass=1e-12,
                       twoPointFiveDSinkMultiplier=1.0)


def _as_float32(prm: dict) -> dict:
    """The parameters as the reference's float build holds them (its members
    are float): the drop-in passes those values on, so the Python path runs
    with the same ones."""
    out = {**_FLOAT_DEFAULTS, **prm}
    return {k: float(np.float32(v)) if isinstance(v, float) else v for k, v in out.items()}


def test_reference_loop_over_the_library_matches_the_python_path():
    from coldplate_b200 import Simple
    case = window_cases()["density"]
    prm = case.params(maxIterations=60, epsilon=1e-30, usePressureDropConvergence=0)
    res_d, dp_d = _run_dropin(case, prm)
    with Simple(cellType=case.cellType, **_as_float32(prm)) as g:
        g.step(60)
        res_p, dp_p = _logs_of(g)
    assert res_d.shape == res_p.shape == (60, res_p.shape[1]), (res_d.shape, res_p.shape)
    assert dp_d.shape == dp_p.shape
    np.testing.assert_array_equal(res_d[:, 0], res_p[:, 0])
    # residual RMS columns (mass, u, v) and the core / full pressure drops
    np.testing.assert_allclose(res_d[:, 1:4], res_p[:, 1:4], rtol=2e-5, atol=0)
    np.testing.assert_allclose(dp_d[:, 1:5], dp_p[:, 1:5], rtol=2e-5, atol=1e-6)


def test_reference_window_rule_stops_the_loop_over_the_library():
    golden = json.load(open(os.path.join(HERE, "golden", "dp_window.json")))
    run = next(r for r in golden["runs"] if r["case"] == "density" and r["rampSteps"] == 50)
    case = window_cases()["density"]
    prm = window_params(case, run["rampSteps"], run["window"], run["percent"])
    res_d, _ = _run_dropin(case, prm)
    assert len(res_d) == run["stop"]
