"""The thermal oracle (oracle/thermal_oracle.py) against the reference's own
thermal solver: ThermalSolver/thermal_solver.cpp built against the AMGCL API
stand-in (oracle/refbuild/shim/amgcl), which dumps the system the reference
assembled and its tight solution.  The restated assembly must give the same
matrix and right-hand side bit for bit."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "thermal_ref_pin")


def thermal_inputs(Ny, Nx, seed):
    """A seeded density geometry with cell-centred velocities of both signs."""
    from coldplate_b200 import cases
    gam = cases.density_gamma(Ny, Nx, seed, buffer=4)
    rng = np.random.default_rng(seed)
    u = gam * (0.4 + 0.2 * rng.random((Ny, Nx))) - 0.05 * rng.random((Ny, Nx))
    v = 0.1 * (rng.random((Ny, Nx)) - 0.5) * gam
    pm = 20.0 + 80.0 * rng.random((Ny, Nx))        # W/cm^2
    return gam, u, v, pm


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("with_map", [False, True])
def test_assembly_matches_the_reference_bit_for_bit(tmp_path, with_map):
    from thermal_oracle import ThermalParams, assemble, read_dump, solve, write_case
    Ny, Nx, dx, dy, qf, Ht = 20, 44, 2e-5, 2e-5, 5.0e5, 2e-4
    gam, u, v, pm = thermal_inputs(Ny, Nx, 3)
    case = str(tmp_path / "case")
    geom = 1.0 - gam                       # the file holds 0 = fluid, 1 = solid
    write_case(case, geom, u, v, dx, dy, qf, Ht, pm if with_map else None)
    gam = 1.0 - geom                       # what the reference reads back (thermal_solver.cpp:738)
    dump = str(tmp_path / "dump.bin")
    subprocess.run([REF, case], check=True, capture_output=True, text=True, timeout=600,
                   env=dict(os.environ, CP_AMGCL_SHIM_DUMP=dump, OMP_NUM_THREADS="1"))
    A_ref, b_ref, x_ref = read_dump(dump)
    p = ThermalParams(Nx=Nx, Ny=Ny, dx=dx, dy=dy, H_t=Ht)
    q0 = pm * 10000.0 if with_map else np.full((Ny, Nx), qf)
    A, b = assemble(p, gam, u, v, q0)
    A_ref.sort_indices()
    assert np.array_equal(A.indptr, A_ref.indptr) and np.array_equal(A.indices, A_ref.indices)
    assert np.array_equal(A.data, A_ref.data), np.abs(A.data - A_ref.data).max()
    assert np.array_equal(b, b_ref)
    T = solve(p, gam, u, v, q0).ravel()
    assert np.linalg.norm(T - x_ref) <= 1e-10 * np.linalg.norm(x_ref)


def fd_case(kind):
    """Small thermal inputs for the gradient checks: a graded density field
    (every column fluid, gamma in [0.05, 0.95]) or a channel geometry with
    solid fins (gamma 0 / 1 with graded buffers)."""
    from coldplate_b200 import cases
    Ny, Nx = 12, 20
    rng = np.random.default_rng(11)
    if kind == "graded":
        gam = 0.05 + 0.9 * rng.random((Ny, Nx))
    else:
        gam = cases.density_gamma(Ny, Nx, 5, buffer=3)
    u = gam * (0.3 + 0.2 * rng.random((Ny, Nx)))
    v = 0.05 * (rng.random((Ny, Nx)) - 0.5) * gam
    q0 = (20.0 + 80.0 * rng.random((Ny, Nx))) * 1e4
    return gam, u, v, q0


@pytest.mark.parametrize("kind,mode", [("graded", 1), ("graded", 2), ("graded", 0), ("fins", 1)])
def test_adjoint_gradient_matches_central_differences(kind, mode):
    """The oracle's discrete-adjoint dJ/dgamma of the bottom p-norm (p = 8)
    against central differences of J from exact sparse solves, at columns
    whose gamma lies inside (0.02, 0.98) (the fluid mask and the clamp do not
    move under the step).  Agreement is at the noise level of the sparse
    solves (about 1e-6 of the largest component)."""
    from thermal_oracle import ThermalParams, pnorm_gradient, solve
    gam, u, v, q0 = fd_case(kind)
    p = ThermalParams(Nx=gam.shape[1], Ny=gam.shape[0], dx=2e-5, dy=2e-5, H_t=2e-4, k_interp_mode=mode, qk=3.0)
    pexp = 8.0
    J, g, _, _ = pnorm_gradient(p, gam, u, v, q0, pexp)

    def Jof(gm):
        Tb = solve(p, gm, u, v, q0)[0]
        return float(np.power(np.mean(np.power(Tb, pexp)), 1.0 / pexp))

    inside = np.argwhere((gam > 0.02) & (gam < 0.98))
    rng = np.random.default_rng(0)
    pick = inside[rng.choice(len(inside), size=min(8, len(inside)), replace=False)]
    scale = np.abs(g).max()
    assert scale > 0
    for j, i in pick:
        h = 1e-6
        gp, gm = gam.copy(), gam.copy()
        gp[j, i] += h
        gm[j, i] -= h
        fd = (Jof(gp) - Jof(gm)) / (2 * h)
        assert abs(fd - g[j, i]) <= 1e-5 * scale + 1e-4 * abs(fd), (j, i, fd, g[j, i])


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("seed", [3, 8])
def test_thermal_result_files_match_the_reference_byte_for_byte(tmp_path, seed):
    """thermal_metrics.txt, k_thermal.txt and T_bottom.txt written by
    coldplate_b200.output from the reference's own temperature field equal
    the files the reference's main() wrote (thermal_output.cpp)."""
    from thermal_oracle import read_dump, write_case

    from coldplate_b200 import output
    Ny, Nx, dx, dy, qf, Ht = 20, 44, 2e-5, 2e-5, 5.0e5, 2e-4
    gam, u, v, pm = thermal_inputs(Ny, Nx, seed)
    case = str(tmp_path / "case")
    write_case(case, 1.0 - gam, u, v, dx, dy, qf, Ht, pm)
    gam = 1.0 - (1.0 - gam)
    dump = str(tmp_path / "dump.bin")
    subprocess.run([REF, case], check=True, capture_output=True, text=True, timeout=600,
                   env=dict(os.environ, CP_AMGCL_SHIM_DUMP=dump, OMP_NUM_THREADS="1"))
    _, _, x_ref = read_dump(dump)
    nzs, nzf, Hb = 2, 7, 5e-4
    T = x_ref.reshape(nzs + nzf, Ny, Nx)
    dz = [Hb / nzs] * nzs + [Ht / nzf] * nzf
    mine = str(tmp_path / "mine")
    files = output.save_thermal_outputs(mine, T, gam, dx, dy, dz, nzs, 400.0, 0.6, 1.0)
    assert files == ["thermal_metrics.txt", "k_thermal.txt", "T_bottom.txt"]
    for name in files:
        a = open(os.path.join(mine, name), "rb").read()
        b = open(os.path.join(case, name), "rb").read()
        assert a == b, name


def test_thermal_metrics_against_a_direct_restatement():
    """The vectorised metrics against plain loops in the reference's order."""
    from coldplate_b200 import output
    rng = np.random.default_rng(2)
    Nz, Ny, Nx, nzs = 5, 4, 6, 2
    T = 30 + 10 * rng.random((Nz, Ny, Nx))
    gam = (rng.random((Ny, Nx)) > 0.4).astype(float)
    dz = [1e-4, 1e-4, 5e-5, 5e-5, 5e-5]
    dx = dy = 1e-5
    m = output.thermal_metrics(T, gam, dx, dy, dz, nzs)
    s = sv = 0.0
    for k in range(Nz):
        for j in range(Ny):
            for i in range(Nx):
                if k >= nzs and gam[j, i] > 0.01:
                    V = dx * dy * dz[k]
                    s += T[k, j, i] * V
                    sv += V
    assert m["T_avg_fluid"] == s / sv
    ext = [output.thermal_metrics(T, gam, dx, dy, dz, nzs)["grad_max_i"]]
    assert 0 <= ext[0] < Nx


GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.mark.parametrize("name", ["thermal_uniform", "thermal_map"])
def test_oracle_and_writers_against_the_golden_fixtures(tmp_path, name):
    """The committed fixtures of the reference's thermal run
    (tests/golden/make_thermal_golden.py): the oracle's assembly equals the
    reference's matrix and right-hand side bit for bit, its solve matches the
    reference's tight solution, and the result-file writers reproduce the
    reference's files byte for byte from its temperature field.  Needs no
    reference build."""
    from thermal_oracle import ThermalParams, assemble, solve

    from coldplate_b200 import output
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    Ny, Nx, dx, dy, qf, Ht = z["case"]
    Ny, Nx = int(Ny), int(Nx)
    gam = 1.0 - z["geometry"]                       # as the reference reads it
    q0 = z["power_map"] * 10000.0 if z["power_map"].size else np.full((Ny, Nx), qf)
    p = ThermalParams(Nx=Nx, Ny=Ny, dx=dx, dy=dy, H_t=Ht)
    A, b = assemble(p, gam, z["u"], z["v"], q0)
    assert np.array_equal(A.indptr, z["indptr"]) and np.array_equal(A.indices, z["indices"])
    assert np.array_equal(A.data, z["data"])
    assert np.array_equal(b, z["b"])
    T = solve(p, gam, z["u"], z["v"], q0).ravel()
    assert np.linalg.norm(T - z["x"]) <= 1e-10 * np.linalg.norm(z["x"])
    dz = [p.H_b / p.nz_solid] * p.nz_solid + [p.H_t / p.nz_fluid] * p.nz_fluid
    files = output.save_thermal_outputs(str(tmp_path), z["x"].reshape(p.Nz, Ny, Nx), gam, dx, dy, dz, p.nz_solid,
                                        p.k_s, p.k_f, p.qk)
    for f in files:
        assert open(tmp_path / f, "rb").read() == z[f.replace(".txt", "")].tobytes(), f
