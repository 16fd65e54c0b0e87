"""Parity at the benchmark sizes: the 2048 x 1024 density workload (the
timed bench case: row pitch 2080, multi-block grid strides) and the
1024 x 512 random-network workload.

The state is taken after 40 mixed-precision multigrid iterations on the GPU
(a developed flow, not the initial one).  From it, the FP64 form with the
reference's Jacobi-PCG (pressureSolverType 1) and the FP64 oracle each run
one outer iteration, teacher-forced: both start from the same u, v, p, for
two consecutive steps.  Every field must agree within relative L2 1e-10, the
Jacobi and PCG iteration counts exactly, the residuals and pressure drops
within 1e-9.  The three solver-dispatch calls (cp_momentum_u/v,
cp_pressure) are then compared one by one on the oracle's state.
"""
import numpy as np
import pytest

from _helpers import FIELD_NAMES, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    return built_lib


def _cases():
    from coldplate_b200 import cases
    return {"density_2048x1024": cases.density_field(1024, 2048, seed=0, pressureSolverType=4, pTol=1e-6,
                                                     maxPressureIter=30),
            "network_1024x512": cases.random_network(512, 1024, seed=0, pressureSolverType=4, pTol=1e-6,
                                                     maxPressureIter=30)}


@pytest.mark.parametrize("name", ["density_2048x1024", "network_1024x512"])
def test_teacher_forced_at_full_size(name):
    from coldplate_b200 import Simple
    from oracle import Oracle
    case = _cases()[name]
    with Simple(cellType=case.cellType, **case.params(precision="mixed", maxIterations=100, epsilon=1e-30)) as g:
        g.step(40)
        state = {f: g.get(f) for f in ("u", "v", "p")}
    prm = case.params(pressureSolverType=1, maxIterations=100, epsilon=1e-30)
    o = Oracle("f64", prm, cellType=case.cellType, hy=case.hy, hx=case.hx, U=case.U, Ht=case.Ht)
    for f, a in state.items():
        o.set(f, a)
    with Simple(cellType=case.cellType, **prm) as g:
        assert g.get("u").shape == (case.Ny + 2, case.Nx + 1)
        for k in range(2):
            state = {f: o.get(f) for f in ("u", "v", "p")}
            hist_o = o.run(1)
            for f, a in state.items():
                g.set(f, a)
            g.reset_loop()
            g.step(1)
            errs = {f: rel_l2(g.get(f), o.get(f)) for f in FIELD_NAMES}
            assert max(errs.values()) <= 1e-10, (name, k, errs)
            hg = g.history()
            sc = o.scalars()
            assert (int(hg["itersU"][0]), int(hg["itersV"][0]), int(hg["pIters"][0])) == \
                (int(sc["itersU"]), int(sc["itersV"]), int(hist_o[0, 8])), (name, k)
            for kk, col in ((2, "residU_RMS"), (3, "residV_RMS"), (4, "residMass_RMS"), (9, "coreTotal"),
                            (10, "fullTotal"), (11, "coreStatic"), (12, "fullStatic")):
                ref = hist_o[0, kk]
                assert abs(hg[col][0] - ref) <= 1e-9 * max(abs(ref), 1e-300), (name, k, col, hg[col][0], ref)
        # the dispatch boundary on the oracle's state
        for f in ("u", "v", "p"):
            g.set(f, o.get(f))
        itU_g, rU_g = g.solveUMomentumImplicit()
        itV_g, rV_g = g.solveVMomentumImplicit()
        itU_o, rU_o = o.momentum(True)
        itV_o, rV_o = o.momentum(False)
        assert (itU_g, itV_g) == (itU_o, itV_o)
        assert abs(rU_g - rU_o) <= 1e-9 * abs(rU_o) and abs(rV_g - rV_o) <= 1e-9 * abs(rV_o)
        for f in ("dE", "dN"):
            assert rel_l2(g.get(f), o.get(f)) <= 1e-12, f
        for f in ("uStar", "vStar"):
            assert rel_l2(g.get(f)[1:-1, 1:-1], o.get(f)[1:-1, 1:-1]) <= 1e-11, f
        g.set("uStar", o.get("uStar"))
        g.set("vStar", o.get("vStar"))
        itP_g, rm_g = g.solvePressureSystem()
        itP_o, rm_o = o.pressure()
        assert itP_g == itP_o
        assert abs(rm_g - rm_o) <= 1e-12 * abs(rm_o)
        assert rel_l2(g.get("pStar"), o.get("pStar")) <= 1e-10
        assert np.isfinite(g.get("pStar")).all()
