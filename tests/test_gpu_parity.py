"""Parity of the CUDA path (through the C ABI) with the FP64 oracle.

The oracle is the C restatement of the reference SIMPLE iteration re-typed
to double (pinned bit for bit against the reference sources in the CPU
tests).  Tolerance: relative L2 <= 1e-8 on u, v, p, u*, v*, p', dE, dN and
on the history columns; iteration counts must match exactly.
"""
import numpy as np
import pytest

from _helpers import FIELD_NAMES, gpu_for, oracle_for, rel_l2, small_cases

pytestmark = pytest.mark.gpu

TOL = 1e-8
CASES = small_cases()


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    return built_lib


def _compare_fields(g, o, tol=TOL):
    errs = {}
    for name in FIELD_NAMES:
        errs[name] = rel_l2(g.get(name), o.get(name))
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, f"fields beyond {tol}: {bad} (all: {errs})"
    return errs


@pytest.mark.parametrize("name", list(CASES))
def test_one_iteration(name):
    case = CASES[name]
    o = oracle_for(case)
    hist_o = o.run(1)
    with gpu_for(case) as g:
        g.step(1)
        _compare_fields(g, o, tol=1e-11)
        hg = g.history()
        assert int(hg["itersU"][0]) == int(o.scalars()["itersU"])
        assert int(hg["itersV"][0]) == int(o.scalars()["itersV"])
        assert int(hg["pIters"][0]) == int(hist_o[0, 8])


def test_teacher_forced_trajectory():
    """Every outer iteration of a 40-iteration oracle trajectory: load the
    oracle state (u, v, p) into the GPU, run one GPU iteration, compare with
    the oracle's next state.  This checks each step along the whole
    transient, independently of how the iteration amplifies rounding."""
    for name in CASES:
        case = CASES[name]
        o = oracle_for(case)
        with gpu_for(case) as g:
            for k in range(40):
                state = {f: o.get(f) for f in ("u", "v", "p")}
                hist_o = o.run(1)
                for f, a in state.items():
                    g.set(f, a)
                g.reset_loop()
                g.step(1)
                errs = {f: rel_l2(g.get(f), o.get(f)) for f in FIELD_NAMES}
                assert max(errs.values()) <= 1e-10, (name, k, errs)
                hg = g.history()
                assert int(hg["pIters"][0]) == int(hist_o[0, 8]), (name, k)
                assert int(hg["itersU"][0]) == int(o.scalars()["itersU"]), (name, k)
                assert int(hg["itersV"][0]) == int(o.scalars()["itersV"]), (name, k)
                for kk, col in ((2, "residU_RMS"), (3, "residV_RMS"), (4, "residMass_RMS"),
                                (9, "coreTotal"), (10, "fullTotal"), (11, "coreStatic"), (12, "fullStatic")):
                    ref = hist_o[0, kk]
                    assert abs(hg[col][0] - ref) <= 1e-9 * max(abs(ref), 1e-300), (name, k, col)


@pytest.mark.parametrize("name", ["network", "density"])
def test_fifty_iterations_free_running(name):
    """Free-running 50 iterations on the cases whose iteration does not
    amplify rounding (the straight channel does: see test_sensitivity)."""
    case = CASES[name]
    o = oracle_for(case)
    hist_o = o.run(50)
    with gpu_for(case) as g:
        g.step(50)
        _compare_fields(g, o)
        hg = g.history()
        n = len(hist_o)
        assert len(hg["iter"]) == n
        np.testing.assert_array_equal(hg["pIters"][:n], hist_o[:, 8])
        for k, col in ((2, "residU_RMS"), (3, "residV_RMS"), (4, "residMass_RMS"), (5, "residU_max"),
                       (6, "residV_max"), (7, "residMass_max"), (9, "coreTotal"), (10, "fullTotal"),
                       (11, "coreStatic"), (12, "fullStatic"), (13, "inMassFlux"), (14, "outMassFlux")):
            assert rel_l2(hg[col][:n], hist_o[:, k]) <= TOL, col


def test_converged_straight_channel():
    """Straight channel 256 x 64 (FOU, epsilon 1e-7) run to convergence on
    both.  The reference iteration amplifies rounding during the transient,
    so the two runs stop a few iterations apart; both reach the residual
    stop rule and the same pressure drop to the stopping accuracy."""
    from coldplate_b200 import cases
    case = cases.straight_channel(64, 256)
    o = oracle_for(case, maxIterations=3000)
    hist_o = o.run(3000)
    with gpu_for(case, maxIterations=3000) as g:
        rep = g.runIterations()
        assert rep["stop_reason"] == 1  # residual
        assert abs(rep["iter"] - len(hist_o)) <= 0.05 * len(hist_o)
        assert abs(rep["fullTotalDrop"] - hist_o[-1, 10]) <= 1e-3 * abs(hist_o[-1, 10])
        for f in ("u", "p"):
            assert rel_l2(g.get(f), o.get(f)) <= 1e-3, f


@pytest.mark.parametrize("name", ["network", "density"])
def test_dispatch_boundary(name):
    """solveU/VMomentumImplicit and solvePressureSystem one by one on a state
    taken from the oracle after 20 iterations."""
    case = CASES[name]
    o = oracle_for(case)
    o.run(20)
    with gpu_for(case) as g:
        for f in ("u", "v", "p"):
            g.set(f, o.get(f))
        # the oracle's next step starts by re-applying the BCs, which the
        # state already satisfies; compare the three sub-solves
        itU_g, rU_g = g.solveUMomentumImplicit()
        itV_g, rV_g = g.solveVMomentumImplicit()
        itU_o, rU_o = o.momentum(True)
        itV_o, rV_o = o.momentum(False)
        assert (itU_g, itV_g) == (itU_o, itV_o)
        assert abs(rU_g - rU_o) <= 1e-9 * max(abs(rU_o), 1e-30)
        assert abs(rV_g - rV_o) <= 1e-9 * max(abs(rV_o), 1e-30)
        for f in ("dE", "dN"):
            assert rel_l2(g.get(f), o.get(f)) <= 1e-12, f
        # uStar/vStar: interior unknowns (the reference applies BCs to them
        # only later in calculateStep)
        for f in ("uStar", "vStar"):
            a, b = g.get(f), o.get(f)
            assert rel_l2(a[1:-1, 1:-1], b[1:-1, 1:-1]) <= 1e-11, f
        # pressure: feed the oracle's u*, v* into both
        g.set("uStar", o.get("uStar"))
        g.set("vStar", o.get("vStar"))
        itP_g, rm_g = g.solvePressureSystem()
        itP_o, rm_o = o.pressure()
        assert itP_g == itP_o
        assert abs(rm_g - rm_o) <= 1e-12 * max(abs(rm_o), 1e-30)
        assert rel_l2(g.get("pStar"), o.get("pStar")) <= 1e-10


def test_mixed_precision_converges_to_fp64():
    """Mixed precision reaches the FP64 fixed point: after 4000 iterations of
    the density case the full pressure drop agrees with FP64 within 1e-5."""
    case = CASES["density"]
    with gpu_for(case, maxIterations=4000, epsilon=1e-14) as g64:
        r64 = g64.step(4000)
        h64 = g64.history()["fullTotal"]
    with gpu_for(case, maxIterations=4000, epsilon=1e-14, precision="mixed") as g32:
        r32 = g32.step(4000)
    dp64, dp32 = r64["fullTotalDrop"], r32["fullTotalDrop"]
    # FP64 itself is stationary to well below the tolerance
    assert abs(h64[-1] - h64[-500]) <= 1e-6 * abs(dp64)
    assert abs(dp32 - dp64) <= 1e-5 * abs(dp64), (dp32, dp64)
