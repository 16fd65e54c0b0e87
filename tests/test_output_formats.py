"""The reference's result files (saveMatrix / saveAll / residuals.txt /
pressure_drop_history.txt, Utilities/output.cpp) written by
coldplate_b200.output match the files the reference itself writes, byte for
byte, on the same state: the reference build runs its own runIterations
(which logs every iteration and calls saveAll at the end) and the float
oracle, bit-identical to that build, supplies the state to our writers."""
import os
import subprocess

import numpy as np
import pytest

from _helpers import small_cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_f32_pin")


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", ["network", "density"])
def test_written_files_match_the_reference(tmp_path, name):
    from coldplate_b200 import output
    from oracle import Oracle, ref_overrides, write_case

    case = small_cases()[name]
    n = 15
    prm = case.params(maxIterations=n, epsilon=1e-30)
    ref_dir = str(tmp_path / "ref")
    write_case(ref_dir, case.cellType, case.hy, case.hx, case.U, case.Ht)
    subprocess.run([REF, ref_dir, ref_dir, *ref_overrides(prm, threads=1), "run_native=1"], check=True,
                   capture_output=True, text=True, timeout=600)
    ex_ref = os.path.join(ref_dir, "ExportFiles")

    o = Oracle("f32", prm, cellType=case.cellType, hy=case.hy, hx=case.hx, U=case.U, Ht=case.Ht)
    rows = o.run(n)
    hist = {c: rows[:, k] for k, c in enumerate(__import__("oracle").HIST_COLS)}
    ours = str(tmp_path / "ours")
    written = output.save_all(ours, o.get("u"), o.get("v"), o.get("p"), case.hx, case.hy,
                              u_old=o.get("uOld"), v_old=o.get("vOld"))
    output.write_logs(ours, hist)
    written += ["residuals.txt", "pressure_drop_history.txt"]
    assert len(written) == 14
    for fn in written:
        a = open(os.path.join(ex_ref, fn)).read()
        b = open(os.path.join(ours, fn)).read()
        assert a == b, (fn, a[:300], b[:300])


def test_matrix_format_is_the_cpp_stream_default(tmp_path):
    from coldplate_b200 import output
    p = str(tmp_path / "m.txt")
    output.save_matrix(p, np.array([[0.0, -0.0, 1e-5, 123456789.0], [0.1, -2.5, 1.0 / 3.0, 1e30]]))
    assert open(p).read() == "0\t-0\t1e-05\t1.23457e+08\n0.1\t-2.5\t0.333333\t1e+30\n"


@pytest.mark.gpu
def test_simple_writes_its_device_state(tmp_path):
    """Simple.saveAll / writeIterationLogs on a GPU solve: the files read back
    as the device fields rounded to float, one log row per iteration."""
    from coldplate_b200 import Simple
    case = small_cases()["density"]
    with Simple(cellType=case.cellType, **case.params(maxIterations=20, historyCapacity=20)) as s:
        s.step(12)
        u_old = s.get("u")
        v_old = s.get("v")
        s.step(1)
        names = s.saveAll(str(tmp_path), u_old=u_old, v_old=v_old)
        s.writeIterationLogs(str(tmp_path))
        for f in ("u", "v", "p"):
            back = np.loadtxt(str(tmp_path / f"{f}.txt"), delimiter="\t", ndmin=2)
            np.testing.assert_allclose(back, s.get(f).astype(np.float32), rtol=1e-5, atol=1e-30)
    assert "u_resid_full.txt" in names and "p_gradient.txt" in names
    lines = open(str(tmp_path / "residuals.txt")).read().splitlines()
    assert len(lines) == 14 and lines[0].startswith("Iter MassRMS")
