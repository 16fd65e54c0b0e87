"""The C ABI library without a GPU: it builds, loads, exports every function
the headers in include/ declare, and the ctypes structs match the C layout."""
import ctypes
import glob
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))


def declared_functions():
    names = set()
    for h in HEADERS:
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names.update(re.findall(r"^\s*(?:const\s+)?[a-z_]+\s*\*?\s*(cp_[a-z0-9_]+)\s*\(", src, flags=re.M))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("cp_create", "cp_destroy", "cp_step", "cp_run", "cp_momentum_u", "cp_momentum_v",
                 "cp_pressure", "cp_get_field", "cp_set_field", "cp_get_history", "cp_params_default",
                 "cp_last_error_string", "cp_pressure_noalloc", "cp_batch_run", "cp_thermal_solve",
                 "cp_thermal_pnorm_gradient"):
        assert must in names


def test_library_exports_every_declared_symbol(built_lib):
    lib = ctypes.CDLL(built_lib)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_defaults_are_the_reference_defaults(built_lib):
    """cp_params_default() = SIMPLE.h member initialisers."""
    from coldplate_b200 import default_params
    p = default_params()
    expect = dict(epsilon=1e-7, maxIterations=1000, saveStateInterval=1000, xPlaneCoreInlet=0.01,
                  xPlaneCoreOutlet=0.05, usePressureDropConvergence=1, dpConvergenceWindow=500,
                  dpConvergencePercent=1.0, numThreads=8, pressureSolverType=4, maxPressureIter=30,
                  pTol=1e-6, momentumSolverType=1, momentumTol=1e-6, maxMomentumIter=400,
                  momentumSorOmega=1.0, convectionScheme=0, enableTwoPointFiveD=0,
                  twoPointFiveDConvectionFactor=1.2, twoPointFiveDSinkMultiplier=1.0,
                  brinkmanKMin=1e-14, brinkmanQ=1.0, enablePseudoTimeStepping=0, rho=997.0,
                  eta=0.00089, enableInletRamp=0, rampSteps=1000, uvAlpha=0.7, pAlpha=0.3,
                  enableResidualViscosity=0, enableNormalizedResiduals=0, residNormFloorVel=1e-6,
                  residNormFloorMass=1e-12)
    for k, v in expect.items():
        assert getattr(p, k) == pytest.approx(v), k


def _c_offsets(struct_name, fields):
    prog = ["#include <stdio.h>", "#include <stddef.h>"] + [f'#include "{h}"' for h in HEADERS] + ["int main(void){"]
    prog.append(f'printf("%zu\\n", sizeof({struct_name}));')
    for f in fields:
        prog.append(f'printf("%zu\\n", offsetof({struct_name}, {f}));')
    prog.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write("\n".join(prog))
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    return [int(x) for x in out]


@pytest.mark.parametrize("which", ["params", "report", "adjoint", "batch", "timing", "thermal", "thermal_report"])
def test_ctypes_layout_matches_c(which):
    from coldplate_b200 import _native as nat
    cls, name = {"params": (nat.CpParams, "cp_params"), "report": (nat.CpIterReport, "cp_iter_report"),
                 "adjoint": (nat.CpAdjointReport, "cp_adjoint_report"),
                 "batch": (nat.CpBatchReport, "cp_batch_report"),
                 "timing": (nat.CpKernelTiming, "cp_kernel_timing"),
                 "thermal": (nat.CpThermalParams, "cp_thermal_params"),
                 "thermal_report": (nat.CpThermalReport, "cp_thermal_report")}[which]
    fields = cls._fields_
    c = _c_offsets(name, [f for f, _ in fields])
    assert c[0] == ctypes.sizeof(cls)
    assert c[1:] == [getattr(cls, f).offset for f, _ in fields]


def test_create_without_gpu_fails_loudly(built_lib):
    """On a machine without a GPU the product raises; it never falls back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from coldplate_b200 import CpError, Simple, cases
    c = cases.straight_channel(8, 16)
    with pytest.raises(CpError):
        Simple(cellType=c.cellType, **c.params())


def test_bad_parameters_are_rejected_before_any_device_work(built_lib):
    from coldplate_b200 import CpError, Simple, cases
    c = cases.straight_channel(8, 16)
    for over, code in ((dict(pressureSolverType=0), 2), (dict(pressureSolverType=3), 2),
                       (dict(pressureSolverType=5), 2),
                       (dict(momentumSolverType=0), 2), (dict(enablePseudoTimeStepping=1), 2),
                       (dict(enableResidualViscosity=1), 2), (dict(hx=-1.0), 1), (dict(Nx=2), 1),
                       (dict(uvAlpha=float("nan")), 1), (dict(precision=7), 1)):
        with pytest.raises(CpError) as e:
            Simple(cellType=c.cellType, **c.params(**over))
        assert e.value.status == code, over
