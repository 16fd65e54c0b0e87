"""The pressure-drop window stop rule (SIMPLE.cpp:449-491, on by default in
the reference, SIMPLE.h:98) as restated in oracle.dp_window_stop, applied to
FP64 oracle histories, against where the reference's own runIterations()
stopped (tests/golden/dp_window.json, made by
tests/golden/make_dp_window_golden.py)."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_dp_window_golden import window_cases, window_params  # noqa: E402
from oracle import Oracle, dp_window_stop  # noqa: E402

GOLDEN = json.load(open(os.path.join(HERE, "golden", "dp_window.json")))
CASES = window_cases()


@pytest.mark.parametrize("run", GOLDEN["runs"], ids=lambda r: f"{r['case']}-{r['rampSteps']}-{r['window']}")
def test_window_rule_stops_where_the_reference_stops(run):
    case = CASES[run["case"]]
    prm = window_params(case, run["rampSteps"], run["window"], run["percent"])
    o = Oracle("f64", prm, cellType=case.cellType, hy=case.hy, hx=case.hx, U=case.U, Ht=case.Ht)
    h = o.run(GOLDEN["max_iter"])
    assert dp_window_stop(h[:, 9], run["rampSteps"], run["window"], run["percent"]) == run["stop"]
    assert run["stop"] < GOLDEN["max_iter"]
