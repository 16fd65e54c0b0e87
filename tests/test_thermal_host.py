"""Host side of the thermal solve without a GPU: parameter defaults and
checks, and the case-directory reader against the reference's file rules
(thermal_solver.cpp:210-221, 700-772)."""
import numpy as np
import pytest


def test_defaults_are_the_reference_defaults(built_lib):
    """cp_thermal_params_default() = struct Params (thermal_solver.cpp:148-183)."""
    from coldplate_b200.thermal import default_thermal_params
    p = default_thermal_params()
    expect = dict(nz_solid=2, nz_fluid=7, H_b=5e-4, H_t=4e-3, k_s=400.0, k_f=0.6, rho=998.0, Cp=4180.0,
                  T_inlet=30.0, rtol=1e-6, maxiter=1000, k_interp_mode=1, qk=1.0, precision=0)
    for k, v in expect.items():
        assert getattr(p, k) == pytest.approx(v), k


@pytest.mark.parametrize("over", [dict(Nx=1), dict(Ny=0), dict(nz_solid=0), dict(nz_fluid=70),
                                  dict(nz_solid=8, nz_fluid=9), dict(dx=0.0),
                                  dict(k_f=-1.0), dict(k_interp_mode=3), dict(maxiter=-1),
                                  dict(rtol=float("nan")), dict(T_inlet=float("inf")), dict(precision=2),
                                  dict(precision=-1)])
def test_bad_parameters_are_rejected_before_any_device_work(built_lib, over):
    from coldplate_b200 import CpError, Thermal
    kw = dict(Nx=8, Ny=6, dx=1e-5, dy=1e-5)
    kw.update(over)
    with pytest.raises(CpError) as e:
        Thermal(**kw)
    assert e.value.status == 1, over


def test_create_without_gpu_fails_loudly(built_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from coldplate_b200 import CpError, Thermal
    with pytest.raises(CpError) as e:
        Thermal(Nx=8, Ny=6, dx=1e-5, dy=1e-5)
    assert e.value.status == 6


def test_unknown_parameter_is_a_type_error(built_lib):
    from coldplate_b200 import Thermal
    with pytest.raises(TypeError):
        Thermal(Nx=8, Ny=6, dx=1e-5, dy=1e-5, kappa=1.0)


def test_load_case_reads_like_the_reference(tmp_path):
    from thermal_oracle import write_case

    from coldplate_b200.thermal import load_case
    rng = np.random.default_rng(4)
    Ny, Nx = 5, 7
    geom = (rng.random((Ny, Nx)) > 0.5).astype(float)
    u, v = rng.random((Ny, Nx)), rng.random((Ny, Nx)) - 0.5
    pm = 10.0 + rng.random((Ny, Nx))
    d = tmp_path / "c"
    write_case(str(d), geom, u, v, 2e-5, 3e-5, 4.0e5, 1.5e-4, pm)
    prm, inp = load_case(str(d), qk=3.0, k_interp_mode=2)
    assert prm == dict(Nx=Nx, Ny=Ny, dx=2e-5, dy=3e-5, H_t=1.5e-4, qk=3.0, k_interp_mode=2)
    assert np.array_equal(inp["gamma"], 1.0 - geom)
    assert np.array_equal(inp["u_xy"], u) and np.array_equal(inp["v_xy"], v)
    assert np.array_equal(inp["q0"], pm * 10000.0)
    # a power map of another size, or none, gives the uniform flux qf
    np.savetxt(d / "power_map.txt", pm[:, :-1])
    assert np.all(load_case(str(d))[1]["q0"] == 4.0e5)
    (d / "power_map.txt").unlink()
    assert np.all(load_case(str(d))[1]["q0"] == 4.0e5)
    # comment and blank lines are skipped; short velocity files fill what they cover
    with open(d / "u_thermal.txt", "w") as f:
        f.write("# header\n\n1 2\n3 4\n")
    u2 = load_case(str(d))[1]["u_xy"]
    assert np.array_equal(u2[:2, :2], [[1, 2], [3, 4]]) and np.all(u2[2:] == 0) and np.all(u2[:, 2:] == 0)


def test_power_map_statistics():
    from coldplate_b200 import cases
    q = cases.power_map(512, 1024, 7)
    assert q.shape == (512, 1024)
    assert q.min() >= 20.0 and q.max() <= 20.0 + 12 * 300.0
    assert q.max() > 70.0
    assert np.array_equal(q, cases.power_map(512, 1024, 7))


def test_thermal_main_reports_missing_inputs_like_the_reference(tmp_path, capsys):
    """The command-line replacement exits 1 on a directory without
    thermal_params.txt, before touching the GPU (thermal_solver.cpp:700-704)."""
    from coldplate_b200.thermal_main import main
    assert main([str(tmp_path)]) == 1
    assert "Cannot open" in capsys.readouterr().err


def test_inputs_from_flow_crop_matches_the_flow_writer(tmp_path):
    """inputs_from_flow takes the same columns and the same cell-centred
    averages as the u_thermal / v_thermal files of output.save_all (up to
    the files' float rounding), with inlet and outlet buffers."""
    from coldplate_b200 import output
    from coldplate_b200.thermal import inputs_from_flow
    rng = np.random.default_rng(3)
    Ny, Nx, nin, nout = 6, 14, 2, 3
    M, N = Ny + 1, Nx + 1
    fields = {"u": rng.random((M + 1, N)), "v": rng.random((M, N + 1)), "p": rng.random((M + 1, N + 1))}

    class Flow:
        def get(self, name):
            return fields[name]

    ct = (rng.random((Ny, Nx)) > 0.5).astype(float)
    fl = inputs_from_flow(Flow(), ct, nin, nout)
    assert fl["gamma"].shape == (Ny, Nx - nin - nout)
    assert np.array_equal(fl["gamma"], 1.0 - ct[:, nin:Nx - nout])
    output.save_all(str(tmp_path), fields["u"], fields["v"], fields["p"], 1e-5, 1e-5, nin, nout)
    # the files print six significant digits
    assert np.allclose(np.loadtxt(tmp_path / "u_thermal.txt"), fl["u_xy"], rtol=1e-5, atol=1e-6)
    assert np.allclose(np.loadtxt(tmp_path / "v_thermal.txt"), fl["v_xy"], rtol=1e-5, atol=1e-6)


def test_thermal_metrics_without_fluid():
    """No fluid cell: the fluid averages, deviation and range are zero, as
    the reference's guards give (thermal_output.cpp:239-246)."""
    from coldplate_b200 import output
    T = 30.0 + np.arange(2 * 3 * 4, dtype=float).reshape(2, 3, 4)
    m = output.thermal_metrics(T, np.zeros((3, 4)), 1e-5, 1e-5, [1e-4, 1e-4], 1)
    assert m["T_avg_fluid"] == 0.0 and m["T_std_fluid"] == 0.0 and m["T_range_fluid"] == 0.0
    assert m["T_avg_solid"] > 0.0 and m["T_range_global"] == T.max() - T.min()
    assert m["grad_max"] > 0.0
    assert 0 <= m["grad_max_k"] < 2 and 0 <= m["grad_max_j"] < 3 and 0 <= m["grad_max_i"] < 4
