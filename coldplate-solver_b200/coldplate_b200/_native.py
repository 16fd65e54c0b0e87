"""ctypes binding of libcoldplate.so (the C ABI in include/cp_simple.h).

The library is built in-tree (see build.py) next to this package's parent
folder.  Loading it does not touch the GPU; every solver call does, and a
missing library or device raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(PKG_DIR), "libcoldplate.so")

CP_OK = 0
STATUS_NAMES = {0: "CP_OK", 1: "CP_ERR_BAD_PARAM", 2: "CP_ERR_UNSUPPORTED", 3: "CP_ERR_NONFINITE",
                5: "CP_ERR_TIMEOUT", 6: "CP_ERR_CUDA", 7: "CP_ERR_STATE"}
PREC_FP64, PREC_MIXED = 0, 1
STOP_NAMES = {0: "running", 1: "residual", 2: "max_iter", 3: "dp_window", 4: "error"}
FIELDS = {"u": 0, "v": 1, "p": 2, "uStar": 3, "vStar": 4, "pStar": 5, "dE": 6, "dN": 7, "gamma": 8,
          "alpha": 9, "cellType": 10}

_I, _D = ctypes.c_int, ctypes.c_double

# Field order and types mirror struct cp_params in include/cp_simple.h; the
# CPU test suite compares these offsets with the C compiler's.
PARAM_FIELDS = [
    ("Ny", _I), ("Nx", _I), ("hy", _D), ("hx", _D), ("targetVel", _D), ("N_in_buffer", _I),
    ("N_out_buffer", _I), ("Ht_channel", _D),
    ("epsilon", _D), ("maxIterations", _I), ("saveStateInterval", _I), ("reuseInitialFields", _I),
    ("xPlaneCoreInlet", _D), ("xPlaneCoreOutlet", _D),
    ("usePressureDropConvergence", _I), ("dpConvergenceWindow", _I), ("dpConvergencePercent", _D),
    ("usePressureDropSlopeGate", _I), ("dpSlopeWindowIters", _I), ("dpSlopeMaxDelta", _D),
    ("numThreads", _I), ("pressureSolverType", _I), ("parallelizeDirectSolver", _I),
    ("maxPressureIter", _I), ("pTol", _D), ("sorOmega", _D),
    ("momentumSolverType", _I), ("momentumTol", _D), ("maxMomentumIter", _I), ("momentumSorOmega", _D),
    ("convectionScheme", _I), ("enableTwoPointFiveD", _I), ("twoPointFiveDConvectionFactor", _D),
    ("twoPointFiveDSinkMultiplier", _D), ("brinkmanKMin", _D), ("brinkmanQ", _D),
    ("timeStepMultiplier", _D), ("enablePseudoTimeStepping", _I), ("pseudoCFL", _D),
    ("minPseudoSpeed", _D), ("useLocalPseudoTime", _I), ("pseudoControllerMode", _I),
    ("enableSER", _I), ("enableLineSearch", _I), ("enableCflRamp", _I),
    ("rho", _D), ("eta", _D), ("enableInletRamp", _I), ("rampSteps", _I), ("uvAlpha", _D), ("pAlpha", _D),
    ("enableResidualViscosity", _I), ("enableNormalizedResiduals", _I), ("residNormFloorVel", _D),
    ("residNormFloorMass", _D),
    ("precision", _I), ("historyCapacity", _I), ("chunk", _I), ("adjointModel", _I),
]


class CpParams(ctypes.Structure):
    _fields_ = PARAM_FIELDS


REPORT_FIELDS = [
    ("iter", _I), ("done", _I), ("stop_reason", _I), ("pressureIterations", _I),
    ("momentumItersU", _I), ("momentumItersV", _I),
    ("error", _D), ("residU", _D), ("residV", _D), ("residMass", _D),
    ("residU_RMS", _D), ("residV_RMS", _D), ("residMass_RMS", _D),
    ("residU_max", _D), ("residV_max", _D), ("residMass_max", _D),
    ("coreTotalDrop", _D), ("fullTotalDrop", _D), ("coreStaticDrop", _D), ("fullStaticDrop", _D),
    ("inletMassFlux", _D), ("outletMassFlux", _D), ("device_ms", _D),
]


class CpIterReport(ctypes.Structure):
    _fields_ = REPORT_FIELDS

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in REPORT_FIELDS}


KERNEL_KINDS = ("bc", "assemble", "jacobi", "mass", "pcg", "correct", "finalize")


class CpKernelTiming(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double * len(KERNEL_KINDS)), ("launches", ctypes.c_int * len(KERNEL_KINDS)),
                ("jacobiSweeps", ctypes.c_longlong), ("pcgIterations", ctypes.c_longlong),
                ("iterations", ctypes.c_int)]


class CpAdjointReport(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int), ("residual", ctypes.c_double),
                ("J", ctypes.c_double), ("device_ms", ctypes.c_double), ("model", ctypes.c_int),
                ("clampedUnknowns", ctypes.c_int)]


class CpBatchReport(ctypes.Structure):
    _fields_ = [("outerIterations", ctypes.c_int), ("fieldsDone", ctypes.c_int), ("launches", ctypes.c_int),
                ("tileRows", ctypes.c_int), ("tileCols", ctypes.c_int), ("device_ms", ctypes.c_double),
                ("teamCtas", ctypes.c_int)]


class CpThermalParams(ctypes.Structure):
    """struct cp_thermal_params (include/cp_thermal.h)."""
    _fields_ = [("Nx", _I), ("Ny", _I), ("nz_solid", _I), ("nz_fluid", _I), ("dx", _D), ("dy", _D),
                ("H_b", _D), ("H_t", _D), ("k_s", _D), ("k_f", _D), ("rho", _D), ("Cp", _D), ("T_inlet", _D),
                ("rtol", _D), ("maxiter", _I), ("k_interp_mode", _I), ("qk", _D), ("precision", _I)]


class CpThermalReport(ctypes.Structure):
    _fields_ = [("iterations", _I), ("converged", _I), ("residual", _D), ("device_ms", _D)]


# history row columns (cp_device.cuh HistCol)
HIST_COLS = ("iter", "error", "residU_RMS", "residV_RMS", "residMass_RMS", "residU_max", "residV_max",
             "residMass_max", "pIters", "coreTotal", "fullTotal", "coreStatic", "fullStatic",
             "inMassFlux", "outMassFlux", "itersU", "itersV", "residU", "residV", "residMass")

_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_L = ctypes.c_long

SIGNATURES = {
    "cp_params_default": (None, [ctypes.POINTER(CpParams)]),
    "cp_read_fluid_params": (_I, [ctypes.c_char_p, ctypes.POINTER(CpParams)]),
    "cp_create": (_I, [ctypes.POINTER(CpParams), ctypes.POINTER(_vp)]),
    "cp_destroy": (_I, [_vp]),
    "cp_set_cell_type": (_I, [_vp, _dp, _L, _L, _L, _L]),
    "cp_set_gamma": (_I, [_vp, _dp, _L, _L, _L, _L]),
    "cp_read_geometry": (_I, [_vp, ctypes.c_char_p]),
    "cp_get_field": (_I, [_vp, _I, _dp, _L, _L, _L, _L]),
    "cp_set_field": (_I, [_vp, _I, _dp, _L, _L, _L, _L]),
    "cp_step": (_I, [_vp, _I, ctypes.POINTER(CpIterReport)]),
    "cp_run": (_I, [_vp, ctypes.POINTER(CpIterReport)]),
    "cp_reset_loop": (_I, [_vp]),
    "cp_reset": (_I, [_vp]),
    "cp_kernel_times": (_I, [_vp, _I, ctypes.POINTER(CpKernelTiming)]),
    "cp_momentum_u": (_I, [_vp, _dp, _ip]),
    "cp_momentum_v": (_I, [_vp, _dp, _ip]),
    "cp_pressure": (_I, [_vp, _ip, _dp]),
    "cp_adjoint_dp_dgamma": (_I, [_vp, _dp, _L, _L, _L, _L, _I, _D, ctypes.POINTER(CpAdjointReport)]),
    "cp_adjoint_probe_len": (ctypes.c_size_t, [_vp]),
    "cp_adjoint_probe": (_I, [_vp, _I, _dp, _dp, _I, _D, _ip, ctypes.POINTER(CpAdjointReport)]),
    "cp_batch_create": (_I, [ctypes.POINTER(_vp), _I, ctypes.POINTER(_vp)]),
    "cp_batch_destroy": (_I, [_vp]),
    "cp_batch_set_tile": (_I, [_vp, _I, _I]),
    "cp_batch_set_team": (_I, [_vp, _I]),
    "cp_batch_run": (_I, [_vp, _I, ctypes.POINTER(CpBatchReport)]),
    "cp_batch_autotune": (_I, [_vp, _I, ctypes.POINTER(CpBatchReport)]),
    "cp_thermal_params_default": (None, [ctypes.POINTER(CpThermalParams)]),
    "cp_thermal_create": (_I, [ctypes.POINTER(CpThermalParams), ctypes.POINTER(_vp)]),
    "cp_thermal_destroy": (_I, [_vp]),
    "cp_thermal_set_inputs": (_I, [_vp, _dp, _dp, _dp, _dp]),
    "cp_thermal_solve": (_I, [_vp, ctypes.POINTER(CpThermalReport)]),
    "cp_thermal_get_T": (_I, [_vp, _dp]),
    "cp_thermal_objective": (_I, [_vp, _D, _dp, _dp]),
    "cp_thermal_pnorm_gradient": (_I, [_vp, _D, _dp, _dp, ctypes.POINTER(CpThermalReport)]),
    "cp_history_columns": (_I, []),
    "cp_get_history": (_I, [_vp, _dp, _I, _ip]),
    "cp_selftest_bounded_wait": (_I, [_I, _D, _ip]),
    "cp_status_string": (ctypes.c_char_p, [_I]),
    "cp_last_error_string": (ctypes.c_char_p, []),
}

_lib = None


class CpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with coldplate_b200.build.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != CP_OK:
        raise CpError(status, lib().cp_last_error_string().decode(errors="replace"))


def default_params() -> CpParams:
    p = CpParams()
    lib().cp_params_default(ctypes.byref(p))
    return p
