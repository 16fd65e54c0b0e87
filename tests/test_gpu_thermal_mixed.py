"""The mixed-precision thermal solve (precision = CP_PREC_MIXED: a float
V-cycle inside the FP64 BiCGStab, restarted from its iterate while the FP64
residual b - A T is above rtol) against the FP64 oracle
(oracle/thermal_oracle.py: the reference's assembly, solved by a sparse
direct solve) and against the FP64 GPU solve."""
import numpy as np
import pytest

from test_gpu_thermal import full_size_case, gpu_solve, inputs, oracle_params

pytestmark = pytest.mark.gpu

MIXED = 1


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_mixed_temperature_matches_oracle(mode):
    from thermal_oracle import solve
    Ny, Nx = 20, 44
    gam, u, v, q0 = inputs(Ny, Nx, 3)
    prm = dict(Nx=Nx, Ny=Ny, dx=2e-5, dy=2e-5, H_t=2e-4, rtol=1e-12, maxiter=5000, k_interp_mode=mode, qk=3.0,
               precision=MIXED)
    T, rep = gpu_solve(prm, gam, u, v, q0)
    To = solve(oracle_params(**prm), gam, u, v, q0)
    assert rep["converged"] and rep["residual"] <= 1e-12 and rep["iterations"] > 0
    assert np.linalg.norm(T - To) <= 1e-9 * np.linalg.norm(To), np.abs(T - To).max()


def test_mixed_gradient_matches_oracle():
    """The p-norm adjoint solved with the float V-cycle (A^T, same hierarchy)."""
    from thermal_oracle import pnorm_gradient

    from coldplate_b200 import Thermal, cases
    Ny, Nx = 24, 48
    gam, u, v, q0 = inputs(Ny, Nx, 9, "graded")
    prm = dict(Nx=Nx, Ny=Ny, dx=1e-5, dy=1e-5, rtol=1e-12, maxiter=5000, precision=MIXED, **cases.THERMAL_3D)
    Jo, go, _, _ = pnorm_gradient(oracle_params(**prm), gam, u, v, q0, 8.0)
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        assert th.solve()["converged"]
        J, g, rep = th.pnorm_gradient(8)
    assert rep["converged"]
    assert J == pytest.approx(Jo, rel=1e-11)
    assert np.abs(g - go).max() <= 1e-8 * np.abs(go).max(), np.abs(g - go).max() / np.abs(go).max()


def test_mixed_full_size_true_residual_and_objective():
    """At 1024 x 512 x 12 and rtol 1e-6 (the measured workload's tolerance)
    the mixed solve meets rtol on the oracle's own CPU assembly of the
    reference system, with no slack for a drifting recursive residual, and
    its p-norm and adjoint gradient agree with the FP64 solve's."""
    from thermal_oracle import assemble

    from coldplate_b200 import Thermal, cases
    gam, u, v, q0 = full_size_case()
    base = dict(Nx=1024, Ny=512, dx=1e-5, dy=1e-5, rtol=1e-6, maxiter=5000, **cases.THERMAL_3D)
    out = {}
    for prec in (0, MIXED):
        with Thermal(precision=prec, **base) as th:
            th.set_inputs(gam, u, v, q0)
            rep = th.solve()
            T = th.T.ravel()
            J, g, arep = th.pnorm_gradient(8)
        assert rep["converged"] and arep["converged"], (prec, rep, arep)
        out[prec] = (T, J, g, rep)
    A, b = assemble(oracle_params(**base), gam, u, v, q0)
    T = out[MIXED][0]
    res = np.linalg.norm(b - A @ T) / np.linalg.norm(b)
    assert res <= 1.0001e-6, (res, out[MIXED][3])
    J64, Jmx = out[0][1], out[MIXED][1]
    assert abs(Jmx - J64) <= 1e-6 * abs(J64), (Jmx, J64)
    g64, gmx = out[0][2], out[MIXED][2]
    assert np.abs(gmx - g64).max() <= 1e-3 * np.abs(g64).max(), np.abs(gmx - g64).max() / np.abs(g64).max()


def test_mixed_restart_reports_the_true_residual():
    """A tolerance near the FP64 floor: the mixed solve restarts from its
    iterate until the residual it computes on entry meets rtol, and reports
    that residual, which the oracle's assembly confirms."""
    from thermal_oracle import assemble

    from coldplate_b200 import Thermal, cases
    Ny, Nx = 64, 128
    gam, u, v, q0 = inputs(Ny, Nx, 7)
    prm = dict(Nx=Nx, Ny=Ny, dx=1e-5, dy=1e-5, rtol=1e-12, maxiter=20000, precision=MIXED, **cases.THERMAL_3D)
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        rep = th.solve()
        T = th.T.ravel()
    A, b = assemble(oracle_params(**prm), gam, u, v, q0)
    res = np.linalg.norm(b - A @ T) / np.linalg.norm(b)
    assert rep["converged"], rep
    assert res <= 1.01e-12 and rep["residual"] <= 1e-12, (res, rep)


def test_mixed_rejects_unknown_precision():
    from coldplate_b200 import Thermal
    from coldplate_b200._native import CpError
    with pytest.raises(CpError):
        Thermal(Nx=8, Ny=8, dx=1e-5, dy=1e-5, precision=7)
