"""Batched solves (cp_batch_*): several fields of different grid sizes,
geometries and inlet velocities advanced by one persistent kernel.  Each
field must follow the same trajectory as the same field solved alone
(cp_step); only the order of the global sums differs, so the FP64 form
agrees to rounding and every iteration count is identical.  Both schedules
are covered: cell tiles (pressureSolverType 2, the 2 x 2 aggregation cycle)
and teams of CTAs (pressureSolverType 4, the single-field smoothed-
aggregation iteration per team)."""
import numpy as np
import pytest

from _helpers import rel_l2
from coldplate_b200 import Batch, CpError, Simple, cases

pytestmark = pytest.mark.gpu

KN = dict(pressureSolverType=2, maxPressureIter=20, pTol=1e-6)
STOP_RESIDUAL = 1
# cell tiles: every field on the 2 x 2 cycle (type 2); teams: type 4
MODES = {"tiles": dict(pressureSolverType=2), "teams": dict(pressureSolverType=4)}


def small_batch(n=4, seed=5, **over):
    rng = np.random.default_rng(seed)
    shapes = [(24, 48), (40, 96), (33, 70), (16, 130), (50, 64), (28, 200)]
    out = []
    for q in range(n):
        Ny, Nx = shapes[q % len(shapes)]
        U = float(rng.uniform(0.2, 1.0))
        out.append(cases.density_field(Ny, Nx, seed=int(rng.integers(0, 2 ** 31)), U=U, **{**KN, **over}))
    return out


def open_fields(cs, prec, **over):
    return [Simple(cellType=c.cellType, **c.params(precision=prec, **over)) for c in cs]


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_matches_single_field_solves(prec, mode):
    cs = small_batch(5, **MODES[mode])
    n_it = 40
    over = dict(maxIterations=n_it + 10, epsilon=1e-30, historyCapacity=n_it + 10)
    singles = []
    for c in cs:
        with Simple(cellType=c.cellType, **c.params(precision=prec, **over)) as s:
            s.step(n_it)
            singles.append((s.history(), {f: s.get(f) for f in ("u", "v", "p")}))
    fields = open_fields(cs, prec, maxIterations=n_it, epsilon=1e-30, historyCapacity=n_it + 10)
    try:
        with Batch(fields) as b:
            rep = b.run(n_it + 5)
        assert rep["fieldsDone"] == len(cs) and rep["outerIterations"] == n_it
        assert (rep["teamCtas"] > 0) == (mode == "teams"), rep
        tol = 1e-9 if prec == "fp64" else 1e-5
        for q, (f, (h1, fl1)) in enumerate(zip(fields, singles)):
            h2 = f.history()
            assert len(h2["iter"]) == n_it
            if prec == "fp64":
                for col in ("pIters", "itersU", "itersV"):
                    np.testing.assert_array_equal(h2[col], h1[col][:n_it], err_msg=f"field {q} {col}")
            np.testing.assert_allclose(h2["fullTotal"], h1["fullTotal"][:n_it], rtol=tol, err_msg=f"field {q}")
            for name in ("u", "v", "p"):
                assert rel_l2(f.get(name), fl1[name]) <= tol, (q, name, rel_l2(f.get(name), fl1[name]))
    finally:
        for f in fields:
            f.close()


@pytest.mark.parametrize("mode", sorted(MODES))
def test_fields_stop_on_their_own_rules(mode):
    """Different maxIterations per field: each stops where its single solve does."""
    cs = small_batch(3, seed=9, **MODES[mode])
    limits = [7, 19, 33]
    fields = [Simple(cellType=c.cellType, **c.params(maxIterations=m, epsilon=1e-30, historyCapacity=64))
              for c, m in zip(cs, limits)]
    try:
        with Batch(fields) as b:
            rep = b.run(200)
        assert rep["fieldsDone"] == 3 and rep["outerIterations"] == max(limits)
        for c, m, f in zip(cs, limits, fields):
            assert len(f.history()["iter"]) == m
            with Simple(cellType=c.cellType, **c.params(maxIterations=m, epsilon=1e-30, historyCapacity=64)) as s:
                s.runIterations()
                ref = s.history()["fullTotal"]
            np.testing.assert_allclose(f.history()["fullTotal"], ref, rtol=1e-9)
    finally:
        for f in fields:
            f.close()


@pytest.mark.parametrize("mode", sorted(MODES))
def test_batch_converges_like_single_field_solves(mode):
    """Run to the residual tolerance: every field stops for the same reason
    and at (within rounding of the stop test) the same iteration as alone."""
    cs = small_batch(3, seed=11, **MODES[mode])
    over = dict(maxIterations=4000, epsilon=1e-5, historyCapacity=4000)
    fields = open_fields(cs, "mixed", **over)
    try:
        with Batch(fields) as b:
            rep = b.run(4000)
        assert rep["fieldsDone"] == 3
        for q, (c, f) in enumerate(zip(cs, fields)):
            h = f.history()
            reason = f.step(0)["stop_reason"]
            with Simple(cellType=c.cellType, **c.params(precision="mixed", **over)) as s:
                r1 = s.runIterations()
                n1 = len(s.history()["iter"])
            assert reason == r1["stop_reason"], (q, reason, r1["stop_reason"])
            assert abs(len(h["iter"]) - n1) <= 2, (q, len(h["iter"]), n1)
            if reason == STOP_RESIDUAL:
                assert h["error"][-1] <= 1e-5
    finally:
        for f in fields:
            f.close()


def test_autotune_picks_a_tile_and_resets_the_fields():
    cs = small_batch(3, seed=2)
    fields = open_fields(cs, "mixed", maxIterations=100, epsilon=1e-30, historyCapacity=128)
    try:
        with Batch(fields) as b:
            best = b.autotune(3)
            assert best["tileRows"] * best["tileCols"] >= 256 and best["device_ms"] > 0
            for f in fields:
                assert len(f.history()["iter"]) == 0
            rep = b.run(10)
            assert rep["tileRows"] == best["tileRows"] and rep["tileCols"] == best["tileCols"]
            assert rep["outerIterations"] == 10
            with pytest.raises(CpError) as e:
                b.set_team(4)
            assert e.value.status == 2
    finally:
        for f in fields:
            f.close()


def test_autotune_picks_a_team_and_resets_the_fields():
    cs = small_batch(3, seed=2, **MODES["teams"])
    fields = open_fields(cs, "mixed", maxIterations=100, epsilon=1e-30, historyCapacity=128)
    try:
        with Batch(fields) as b:
            best = b.autotune(3)
            assert best["teamCtas"] >= 1 and best["tileRows"] == 0 and best["device_ms"] > 0
            for f in fields:
                assert len(f.history()["iter"]) == 0
            rep = b.run(10)
            assert rep["teamCtas"] == best["teamCtas"] and rep["outerIterations"] == 10
            with pytest.raises(CpError):
                b.set_team(0)
    finally:
        for f in fields:
            f.close()


def test_team_sizes_agree():
    """Teams of 1, 3 and 37 CTAs (more fields than teams: the queue hands the
    next field to the first free team) give the same FP64 trajectories up to
    the order of the sums, with identical iteration counts."""
    cs = small_batch(5, seed=4, **MODES["teams"])
    n_it = 25
    out = []
    for ctas in (1, 3, 37):
        fields = open_fields(cs, "fp64", maxIterations=n_it, epsilon=1e-30, historyCapacity=n_it + 10)
        try:
            with Batch(fields) as b:
                b.set_team(ctas)
                rep = b.run(n_it)
            assert rep["teamCtas"] == ctas and rep["fieldsDone"] == len(cs)
            out.append([(f.history(), f.get("p")) for f in fields])
        finally:
            for f in fields:
                f.close()
    for run in out[1:]:
        for q, ((h0, p0), (h1, p1)) in enumerate(zip(out[0], run)):
            for col in ("pIters", "itersU", "itersV"):
                np.testing.assert_array_equal(h1[col], h0[col], err_msg=f"field {q} {col}")
            np.testing.assert_allclose(h1["fullTotal"], h0["fullTotal"], rtol=1e-10, err_msg=f"field {q}")
            assert rel_l2(p1, p0) <= 1e-10


def test_batch_rejects_mixed_precisions_and_jacobi_pcg():
    cs = small_batch(2)
    a = Simple(cellType=cs[0].cellType, **cs[0].params(precision="fp64"))
    b = Simple(cellType=cs[1].cellType, **cs[1].params(precision="mixed"))
    c = Simple(cellType=cs[1].cellType, **cs[1].params(pressureSolverType=1))
    try:
        with pytest.raises(CpError) as e:
            Batch([a, b])
        assert e.value.status == 1
        with pytest.raises(CpError) as e:
            Batch([a, c])
        assert e.value.status == 2
        with pytest.raises(CpError):
            Batch([a, a])
    finally:
        for f in (a, b, c):
            f.close()
