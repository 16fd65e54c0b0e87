"""The pressure-drop window stop rule on the GPU (the default stop rule of
the reference, SIMPLE.h:98, SIMPLE.cpp:449-491) against the reference: the
FP64 solve through the C ABI must stop for the window rule at the iteration
where the reference's own runIterations() stopped
(tests/golden/dp_window.json), with the core and full pressure drops of
every iteration within 1e-9 (relative) of the FP64 oracle's."""
import json
import os
import sys

import numpy as np
import pytest

from oracle import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_dp_window_golden import window_cases, window_params  # noqa: E402

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(HERE, "golden", "dp_window.json")))
CASES = window_cases()
DP_TOL = 1e-9


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    return built_lib


@pytest.mark.parametrize("run", GOLDEN["runs"], ids=lambda r: f"{r['case']}-{r['rampSteps']}-{r['window']}")
def test_gpu_stops_on_the_window_rule_where_the_reference_does(run):
    from coldplate_b200 import Simple
    case = CASES[run["case"]]
    prm = window_params(case, run["rampSteps"], run["window"], run["percent"])
    with Simple(cellType=case.cellType, **prm, historyCapacity=GOLDEN["max_iter"]) as g:
        rep = g.runIterations()
        h = g.history()
    assert rep["stop_reason"] == 3, rep          # CP_STOP_DP_WINDOW
    assert rep["iter"] == run["stop"]
    o = Oracle("f64", prm, cellType=case.cellType, hy=case.hy, hx=case.hx, U=case.U, Ht=case.Ht)
    ho = o.run(run["stop"])
    for col, k in (("coreTotal", 9), ("fullTotal", 10)):
        err = np.abs(h[col] - ho[:, k]) / np.maximum(np.abs(ho[:, k]), 1e-300)
        assert err.max() <= DP_TOL, (col, float(err.max()), int(err.argmax()))
