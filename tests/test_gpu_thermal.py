"""The GPU thermal solve and its p-norm adjoint against the oracle
(oracle/thermal_oracle.py: the reference's assembly, solved by a sparse
direct solve; its adjoint gradient pinned by central differences)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def inputs(Ny, Nx, seed, kind="density"):
    from coldplate_b200 import cases
    rng = np.random.default_rng(seed)
    if kind == "graded":
        gam = 0.05 + 0.9 * rng.random((Ny, Nx))
    else:
        gam = cases.density_gamma(Ny, Nx, seed, buffer=4)
    u = gam * (0.4 + 0.2 * rng.random((Ny, Nx))) - 0.05 * rng.random((Ny, Nx))
    v = 0.1 * (rng.random((Ny, Nx)) - 0.5) * gam
    q0 = (20.0 + 80.0 * rng.random((Ny, Nx))) * 1e4
    return gam, u, v, q0


def oracle_params(**kw):
    from thermal_oracle import ThermalParams
    keep = {k: v for k, v in kw.items() if k in ThermalParams.__dataclass_fields__}
    return ThermalParams(**keep)


def gpu_solve(prm, gam, u, v, q0):
    from coldplate_b200 import Thermal
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        rep = th.solve()
        return th.T, rep


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("uniform", [True, False])
def test_temperature_matches_oracle(mode, uniform):
    from thermal_oracle import solve
    Ny, Nx = 20, 44
    gam, u, v, q0 = inputs(Ny, Nx, 3)
    if uniform:
        q0 = np.full((Ny, Nx), 5.0e5)
    prm = dict(Nx=Nx, Ny=Ny, dx=2e-5, dy=2e-5, H_t=2e-4, rtol=1e-12, maxiter=5000, k_interp_mode=mode, qk=3.0)
    T, rep = gpu_solve(prm, gam, u, v, q0)
    To = solve(oracle_params(**prm), gam, u, v, q0)
    assert rep["converged"] and rep["residual"] <= 1e-12 and rep["iterations"] > 0
    assert np.linalg.norm(T - To) <= 1e-9 * np.linalg.norm(To), np.abs(T - To).max()


def test_plate_and_channel_layers_of_the_3d_workload():
    """The 8 + 4 layer settings, the hotspot power map and p = 8."""
    from thermal_oracle import solve

    from coldplate_b200 import Thermal, cases
    Ny, Nx = 48, 96
    gam, u, v, _ = inputs(Ny, Nx, 5)
    q0 = cases.power_map(Ny, Nx, 5) * 1e4
    prm = dict(Nx=Nx, Ny=Ny, dx=1e-5, dy=1e-5, rtol=1e-12, maxiter=5000, **cases.THERMAL_3D)
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        rep = th.solve()
        T = th.T
        mx, pn = th.objective(8)
        assert th.compute_pnorm_objective(8) == pn
    To = solve(oracle_params(**prm), gam, u, v, q0)
    assert rep["converged"]
    assert T.shape == (12, Ny, Nx)
    assert np.linalg.norm(T - To) <= 1e-9 * np.linalg.norm(To)
    assert mx == T[0].max()
    assert pn == pytest.approx(np.mean(T[0] ** 8) ** (1 / 8), rel=1e-13)


@pytest.mark.parametrize("kind,mode", [("graded", 1), ("graded", 2), ("graded", 0), ("density", 1)])
def test_pnorm_gradient_matches_oracle(kind, mode):
    from thermal_oracle import pnorm_gradient

    from coldplate_b200 import Thermal
    Ny, Nx = 16, 28
    gam, u, v, q0 = inputs(Ny, Nx, 9, kind)
    prm = dict(Nx=Nx, Ny=Ny, dx=2e-5, dy=2e-5, H_t=2e-4, rtol=1e-12, maxiter=5000, k_interp_mode=mode, qk=3.0)
    Jo, go, _, _ = pnorm_gradient(oracle_params(**prm), gam, u, v, q0, 8.0)
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        th.solve()
        J, g, rep = th.pnorm_gradient(8)
        res = th.compute_optimization_results(8)
    assert rep["converged"]
    assert J == pytest.approx(Jo, rel=1e-11)
    assert np.abs(g - go).max() <= 1e-8 * np.abs(go).max(), np.abs(g - go).max() / np.abs(go).max()
    assert np.array_equal(res["dJ_dgamma"], g) and res["Tb_pnorm"] == J


def test_pnorm_gradient_against_gpu_central_differences():
    """dJ/dgamma against central differences of J from the GPU's own forward
    solves, on a density geometry of 8 + 4 layers."""
    from coldplate_b200 import Thermal, cases
    Ny, Nx = 24, 48
    gam, u, v, q0 = inputs(Ny, Nx, 2)
    prm = dict(Nx=Nx, Ny=Ny, dx=1e-5, dy=1e-5, rtol=1e-13, maxiter=20000, **cases.THERMAL_3D)
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        th.solve()
        J, g, _ = th.pnorm_gradient(8)

        def Jof(gm):
            th.set_inputs(gm, u, v, q0)
            th.solve()
            return th.objective(8)[1]

        inside = np.argwhere((gam > 0.05) & (gam < 0.95))
        pick = inside[np.random.default_rng(1).choice(len(inside), size=min(6, len(inside)), replace=False)]
        for j, i in pick:
            h = 1e-5
            gp, gm = gam.copy(), gam.copy()
            gp[j, i] += h
            gm[j, i] -= h
            fd = (Jof(gp) - Jof(gm)) / (2 * h)
            assert abs(fd - g[j, i]) <= 1e-4 * np.abs(g).max(), (j, i, fd, g[j, i])


def test_repeated_solves_are_bitwise_identical():
    from coldplate_b200 import Thermal
    Ny, Nx = 32, 64
    gam, u, v, q0 = inputs(Ny, Nx, 4)
    prm = dict(Nx=Nx, Ny=Ny, dx=1e-5, dy=1e-5, H_t=2e-4, rtol=1e-10, maxiter=5000)
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        r1 = th.solve()
        T1 = th.T
        _, g1, _ = th.pnorm_gradient(8)
        r2 = th.solve()
        T2 = th.T
        _, g2, _ = th.pnorm_gradient(8)
    assert r1["iterations"] == r2["iterations"]
    assert np.array_equal(T1, T2) and np.array_equal(g1, g2)


def test_state_and_input_errors():
    from coldplate_b200 import CpError, Thermal
    Ny, Nx = 6, 10
    gam, u, v, q0 = inputs(Ny, Nx, 1, "graded")
    with Thermal(Nx=Nx, Ny=Ny, dx=1e-5, dy=1e-5) as th:
        with pytest.raises(CpError) as e:
            th.solve()
        assert e.value.status == 7
        bad = u.copy()
        bad[2, 3] = np.nan
        with pytest.raises(CpError) as e:
            th.set_inputs(gam, bad, v, q0)
        assert e.value.status == 3
        with pytest.raises(ValueError):
            th.set_inputs(gam[:, :-1], u, v, q0)
        th.set_inputs(gam, u, v, q0)
        with pytest.raises(CpError) as e:
            th.pnorm_gradient(8)
        assert e.value.status == 7
        th.solve()
        with pytest.raises(CpError) as e:
            th.pnorm_gradient(0.5)
        assert e.value.status == 1


def test_maxiter_stops_unconverged():
    from coldplate_b200 import Thermal
    Ny, Nx = 32, 64
    gam, u, v, q0 = inputs(Ny, Nx, 4)
    with Thermal(Nx=Nx, Ny=Ny, dx=1e-5, dy=1e-5, H_t=2e-4, rtol=1e-14, maxiter=3) as th:
        th.set_inputs(gam, u, v, q0)
        rep = th.solve()
    assert rep["iterations"] == 3 and not rep["converged"]


def test_case_directory_and_flow_inputs(tmp_path):
    """A case written in the reference's files solves like the arrays it
    holds; the thermal inputs of a flow solve are its cell-centred
    velocities."""
    from thermal_oracle import solve, write_case

    from coldplate_b200 import Simple, Thermal, cases
    from coldplate_b200.thermal import inputs_from_flow, load_case
    c = cases.density_field(24, 48, seed=2, U=0.4, pressureSolverType=4)
    with Simple(cellType=c.cellType, **c.params(maxIterations=20, epsilon=1e-30)) as s:
        s.step(20)
        fl = inputs_from_flow(s, c.cellType)
        u, v = s.get("u"), s.get("v")
    assert np.allclose(fl["u_xy"][3, 5], 0.5 * (u[4, 5] + u[4, 6]))
    assert np.allclose(fl["v_xy"][3, 5], 0.5 * (v[3, 6] + v[4, 6]))
    q0 = cases.power_map(24, 48, 1)
    write_case(str(tmp_path), 1.0 - fl["gamma"], fl["u_xy"], fl["v_xy"], 1e-5, 1e-5, 1e5, 2e-4, q0)
    prm, inp = load_case(str(tmp_path))
    prm.update(rtol=1e-12, maxiter=5000)
    with Thermal(**prm) as th:
        th.set_inputs(**inp)
        th.solve()
        T = th.T
    To = solve(oracle_params(**prm), inp["gamma"], inp["u_xy"], inp["v_xy"], inp["q0"])
    assert np.linalg.norm(T - To) <= 1e-9 * np.linalg.norm(To)


def test_autograd_function_matches_the_adjoint_call():
    import torch

    from coldplate_b200 import Thermal, cases
    from coldplate_b200.autograd import ThermalPNorm
    Ny, Nx = 16, 32
    gam, u, v, q0 = inputs(Ny, Nx, 6)
    prm = dict(Nx=Nx, Ny=Ny, dx=1e-5, dy=1e-5, rtol=1e-12, maxiter=5000, **cases.THERMAL_3D)
    g = torch.tensor(gam, dtype=torch.float64, requires_grad=True)
    J = ThermalPNorm.apply(g, u, v, q0, prm, 8.0)
    (2.0 * J).backward()
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        th.solve()
        Jr, gr, _ = th.pnorm_gradient(8)
    assert float(J.detach()) == Jr
    assert np.array_equal(g.grad.numpy(), 2.0 * gr)


def test_result_files_from_a_gpu_solve(tmp_path):
    """The reference's thermal files written from a GPU solve agree with the
    same files written from the oracle's temperature field (the solves
    differ at their tolerance only), and dJ_dgamma.txt holds the gradient."""
    from thermal_oracle import solve

    from coldplate_b200 import Thermal, cases, output
    Ny, Nx = 20, 40
    gam, u, v, q0 = inputs(Ny, Nx, 7)
    prm = dict(Nx=Nx, Ny=Ny, dx=1e-5, dy=1e-5, rtol=1e-12, maxiter=5000, **cases.THERMAL_3D)
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        th.solve()
        files = th.save_outputs(str(tmp_path / "gpu"), gam, pnorm_exp=8)
        _, g, _ = th.pnorm_gradient(8)
    assert files == ["thermal_metrics.txt", "k_thermal.txt", "T_bottom.txt", "dJ_dgamma.txt"]
    To = solve(oracle_params(**prm), gam, u, v, q0)
    p = oracle_params(**prm)
    dz = [p.H_b / p.nz_solid] * p.nz_solid + [p.H_t / p.nz_fluid] * p.nz_fluid
    output.save_thermal_outputs(str(tmp_path / "ora"), To, gam, 1e-5, 1e-5, dz, p.nz_solid, p.k_s, p.k_f, p.qk)
    for name in ("k_thermal.txt", "T_bottom.txt"):
        a = np.loadtxt(tmp_path / "gpu" / name)
        b = np.loadtxt(tmp_path / "ora" / name)
        assert np.allclose(a, b, rtol=0, atol=2e-4), name
    assert np.allclose(np.loadtxt(tmp_path / "gpu" / "dJ_dgamma.txt"), g, rtol=1e-9, atol=0)
    mg = {l.split()[0]: l.split()[1:] for l in open(tmp_path / "gpu" / "thermal_metrics.txt") if not l.startswith("#")}
    mo = {l.split()[0]: l.split()[1:] for l in open(tmp_path / "ora" / "thermal_metrics.txt") if not l.startswith("#")}
    assert mg.keys() == mo.keys()
    assert abs(float(mg["T_avg_base"][0]) - float(mo["T_avg_base"][0])) <= 2e-4


def full_size_case(seed=0):
    """The 3-D workload's size (1024 x 512 x 12) with the density geometry,
    a channel flow of 0.5 gamma m/s and the hotspot power map."""
    from coldplate_b200 import cases
    Ny, Nx = 512, 1024
    gam = cases.density_gamma(Ny, Nx, seed)
    rng = np.random.default_rng(seed)
    u = 0.5 * gam
    v = 0.02 * (rng.random((Ny, Nx)) - 0.5) * gam
    q0 = cases.power_map(Ny, Nx, seed) * 1e4
    return gam, u, v, q0


def test_full_size_residual_against_the_oracle_matrix():
    """At 1024 x 512 x 12 the GPU temperature satisfies the oracle's own
    assembly of the reference system to the requested tolerance:
    ||b - A T|| / ||b|| within 1.5 rtol, with A and b built on the CPU."""
    from thermal_oracle import assemble

    from coldplate_b200 import Thermal, cases
    gam, u, v, q0 = full_size_case()
    prm = dict(Nx=1024, Ny=512, dx=1e-5, dy=1e-5, rtol=1e-9, maxiter=5000, **cases.THERMAL_3D)
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        rep = th.solve()
        T = th.T.ravel()
    A, b = assemble(oracle_params(**prm), gam, u, v, q0)
    res = np.linalg.norm(b - A @ T) / np.linalg.norm(b)
    # the kernel stops on its recursive residual; the true one may drift a little above it
    assert rep["converged"] and res <= 1.5e-9, (res, rep)


def test_full_size_gradient_directional_derivative():
    """At 1024 x 512 x 12 the adjoint gradient's directional derivative
    along a smooth random perturbation of gamma (cells inside (0.05, 0.95),
    so the fluid mask does not move) matches central differences of J from
    GPU forward solves."""
    from coldplate_b200 import Thermal, cases
    gam, u, v, q0 = full_size_case(1)
    prm = dict(Nx=1024, Ny=512, dx=1e-5, dy=1e-5, rtol=1e-10, maxiter=8000, **cases.THERMAL_3D)
    rng = np.random.default_rng(5)
    d = cases.gaussian_random_field(512, 1024, 16.0, rng) - 0.5
    d *= (gam > 0.05) & (gam < 0.95)
    with Thermal(**prm) as th:
        th.set_inputs(gam, u, v, q0)
        assert th.solve()["converged"]
        _, g, rep = th.pnorm_gradient(8)
        assert rep["converged"]

        def Jof(gm):
            th.set_inputs(gm, u, v, q0)
            assert th.solve()["converged"]
            return th.objective(8)[1]

        h = 1e-4
        fd = (Jof(gam + h * d) - Jof(gam - h * d)) / (2 * h)
    ad = float(np.sum(g * d))
    assert abs(fd - ad) <= 1e-4 * abs(ad), (fd, ad)


def test_thermal_main_writes_the_reference_files(tmp_path):
    """python -m coldplate_b200.thermal_main <dir> [qk] [mode] --pnorm 8 on a
    case written in the reference's files: the result files appear and
    T_bottom.txt matches the oracle's solution at its printed precision."""
    from thermal_oracle import solve, write_case

    from coldplate_b200 import cases
    from coldplate_b200.thermal import load_case
    from coldplate_b200.thermal_main import main
    Ny, Nx = 16, 36
    gam, u, v, _ = inputs(Ny, Nx, 12)
    write_case(str(tmp_path), 1.0 - gam, u, v, 1e-5, 1e-5, 4e5, 2e-4, cases.power_map(Ny, Nx, 12))
    assert main([str(tmp_path), "3", "1", "--pnorm", "8", "--rtol", "1e-12"]) == 0
    for f in ("thermal_metrics.txt", "k_thermal.txt", "T_bottom.txt", "dJ_dgamma.txt"):
        assert (tmp_path / f).exists(), f
    prm, inp = load_case(str(tmp_path), qk=3.0)
    To = solve(oracle_params(**prm), inp["gamma"], inp["u_xy"], inp["v_xy"], inp["q0"])
    assert np.allclose(np.loadtxt(tmp_path / "T_bottom.txt"), To[0], rtol=0, atol=6e-5)
