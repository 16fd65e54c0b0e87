"""ctypes front end of the CPU oracle (oracle/simple_oracle.c) and a runner
for the reference build in oracle/_ref/.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.

Two oracles live here:
  * ``Oracle`` - the C restatement of the reference SIMPLE iteration
    (float32 as shipped, or float64 re-typed), single threaded;
  * ``run_reference`` - the reference solver's own sources built against an
    Eigen API stand-in (oracle/refbuild/), used to pin the restatement and as
    the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

HIST_COLS = ("iter", "error", "residU_RMS", "residV_RMS", "residMass_RMS", "residU_max",
             "residV_max", "residMass_max", "pIters", "coreTotal", "fullTotal", "coreStatic",
             "fullStatic", "inMassFlux", "outMassFlux")

# Knobs of the reference's SIMPLE.h that the oracle models, with the values
# SIMPLE.h gives them (SIMPLE.h:68-448).  rho/eta are the SIMPLE.h fluid
# constants; callers override them per case.
ORACLE_DEFAULTS = dict(
    epsilon=1e-7, maxIterations=1000, maxPressureIter=30, pTol=1e-6, pressureSolverType=1,
    momentumSolverType=1, momentumTol=1e-6, maxMomentumIter=400, convectionScheme=0,
    enableTwoPointFiveD=0, twoPointFiveDConvectionFactor=1.2, twoPointFiveDSinkMultiplier=1.0,
    brinkmanKMin=1e-14, brinkmanQ=1.0, rho=997.0, eta=0.00089, uvAlpha=0.7, pAlpha=0.3,
    xPlaneCoreInlet=0.01, xPlaneCoreOutlet=0.05, enableInletRamp=0, rampSteps=1000,
    enableNormalizedResiduals=0, residNormFloorVel=1e-6, residNormFloorMass=1e-12,
)


class _Params(ctypes.Structure):
    _fields_ = [
        ("epsilon", ctypes.c_double), ("maxIterations", ctypes.c_int),
        ("maxPressureIter", ctypes.c_int), ("pTol", ctypes.c_double),
        ("pressureSolverType", ctypes.c_int), ("momentumSolverType", ctypes.c_int),
        ("momentumTol", ctypes.c_double), ("maxMomentumIter", ctypes.c_int),
        ("convectionScheme", ctypes.c_int), ("enableTwoPointFiveD", ctypes.c_int),
        ("twoPointFiveDConvectionFactor", ctypes.c_double),
        ("twoPointFiveDSinkMultiplier", ctypes.c_double), ("brinkmanKMin", ctypes.c_double),
        ("brinkmanQ", ctypes.c_double), ("rho", ctypes.c_double), ("eta", ctypes.c_double),
        ("uvAlpha", ctypes.c_double), ("pAlpha", ctypes.c_double),
        ("xPlaneCoreInlet", ctypes.c_double), ("xPlaneCoreOutlet", ctypes.c_double),
        ("enableInletRamp", ctypes.c_int), ("rampSteps", ctypes.c_int),
        ("enableNormalizedResiduals", ctypes.c_int), ("residNormFloorVel", ctypes.c_double),
        ("residNormFloorMass", ctypes.c_double),
    ]


_LIBS: dict[str, ctypes.CDLL] = {}


def build() -> None:
    """Compile the restatement (both precisions) with make."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib(prec: str) -> ctypes.CDLL:
    if prec not in ("f32", "f64"):
        raise ValueError(prec)
    if prec not in _LIBS:
        path = os.path.join(HERE, f"liboracle_{prec}.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        sfx = "_" + prec
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        sig = {
            "orc_create": (vp, [ctypes.POINTER(_Params), ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, dp]),
            "orc_create_from_case": (vp, [ctypes.POINTER(_Params), ctypes.c_char_p]),
            "orc_destroy": (None, [vp]),
            "orc_step": (ctypes.c_double, [vp, ip]),
            "orc_run": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.c_int]),
            "orc_get": (ctypes.c_int, [vp, ctypes.c_char_p, dp]),
            "orc_set": (ctypes.c_int, [vp, ctypes.c_char_p, dp]),
            "orc_dims": (ctypes.c_int, [vp, ip, ip]),
            "orc_scalars": (None, [vp, dp]),
            "orc_sample_plane": (None, [vp, ctypes.c_double, dp]),
            "orc_sample_patch": (None, [vp, ctypes.c_int, dp]),
            "orc_set_inlet_velocity": (None, [vp, ctypes.c_double]),
            "orc_wall_flags": (None, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_ubyte)]),
            "orc_assemble": (None, [vp, ctypes.c_int]),
            "orc_momentum": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_void_p]),
            "orc_pressure": (ctypes.c_int, [vp, ctypes.c_void_p]),
            "orc_velocity_bc": (None, [vp, ctypes.c_void_p, ctypes.c_void_p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name + sfx)
            fn.restype = res
            fn.argtypes = args
            setattr(lib, name, fn)
        _LIBS[prec] = lib
    return _LIBS[prec]


def _params(over: dict) -> _Params:
    d = dict(ORACLE_DEFAULTS)
    for k, v in over.items():
        if k in d:
            d[k] = v
    p = _Params()
    for name, ctype in _Params._fields_:
        setattr(p, name, int(d[name]) if ctype is ctypes.c_int else float(d[name]))
    return p


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """One SIMPLE state in the oracle (prec 'f32' as shipped or 'f64')."""

    def __init__(self, prec: str, params: dict, *, cellType=None, Ny=None, Nx=None, hy=None,
                 hx=None, U=None, Ht=0.0, case_dir=None):
        self.prec = prec
        self.lib = _lib(prec)
        self._prm = _params(params)
        if case_dir is not None:
            h = self.lib.orc_create_from_case(ctypes.byref(self._prm), case_dir.encode())
        else:
            ct = np.ascontiguousarray(cellType, dtype=np.float64)
            Ny, Nx = ct.shape
            h = self.lib.orc_create(ctypes.byref(self._prm), Ny, Nx, hy, hx, U, Ht, _dptr(ct))
        if not h:
            raise RuntimeError("oracle: bad case")
        self.h = h
        M, N = ctypes.c_int(), ctypes.c_int()
        self.lib.orc_dims(h, ctypes.byref(M), ctypes.byref(N))
        self.M, self.N = M.value, N.value

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.orc_destroy(h)
            self.h = None

    def shape(self, name: str):
        M, N = self.M, self.N
        return {"u": (M + 1, N), "v": (M, N + 1), "p": (M + 1, N + 1), "uStar": (M + 1, N),
                "vStar": (M, N + 1), "pStar": (M + 1, N + 1), "uOld": (M + 1, N),
                "vOld": (M, N + 1), "dE": (M + 1, N), "dN": (M, N + 1), "gamma": (M, N),
                "alpha": (M, N), "cellType": (M, N)}.get(name, (M + 1, N + 1))

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.shape(name), dtype=np.float64)
        if self.lib.orc_get(self.h, name.encode(), _dptr(out)) < 0:
            raise KeyError(name)
        return out

    def set(self, name: str, arr) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.shape(name))
        if self.lib.orc_set(self.h, name.encode(), _dptr(a)) < 0:
            raise KeyError(name)

    def step(self) -> tuple[float, int]:
        it = ctypes.c_int()
        e = self.lib.orc_step(self.h, ctypes.byref(it))
        return e, it.value

    def run(self, max_iter: int) -> np.ndarray:
        cap = max(int(max_iter), 1)
        hist = np.zeros((cap, len(HIST_COLS)), dtype=np.float64)
        n = self.lib.orc_run(self.h, int(max_iter), _dptr(hist), cap)
        return hist[:n]

    def scalars(self) -> dict:
        out = np.zeros(12)
        self.lib.orc_scalars(self.h, _dptr(out))
        keys = ("residU", "residV", "residMass", "residU_max", "residV_max", "residMass_max",
                "residU_RMS", "residV_RMS", "residMass_RMS", "itersU", "itersV", "itersP")
        return dict(zip(keys, out.tolist()))

    def sample_plane(self, x: float) -> np.ndarray:
        out = np.zeros(5)
        self.lib.orc_sample_plane(self.h, float(x), _dptr(out))
        return out

    def sample_patch(self, inlet: bool) -> np.ndarray:
        out = np.zeros(5)
        self.lib.orc_sample_patch(self.h, 1 if inlet else 0, _dptr(out))
        return out

    def set_inlet_velocity(self, v: float) -> None:
        self.lib.orc_set_inlet_velocity(self.h, float(v))

    def wall_flags(self, isU: bool) -> np.ndarray:
        M, N = self.M, self.N
        n = (M - 1) * (N - 2) if isU else (M - 2) * (N - 1)
        out = np.zeros(n, dtype=np.uint8)
        self.lib.orc_wall_flags(self.h, 1 if isU else 0, out.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
        return out.reshape((M - 1, N - 2) if isU else (M - 2, N - 1))

    def assemble(self, isU: bool) -> None:
        self.lib.orc_assemble(self.h, 1 if isU else 0)

    def _real(self):
        return ctypes.c_float() if self.prec == "f32" else ctypes.c_double()

    def momentum(self, isU: bool) -> tuple[int, float]:
        """solveUMomentumImplicit / solveVMomentumImplicit on the current state."""
        r = self._real()
        it = self.lib.orc_momentum(self.h, 1 if isU else 0, ctypes.byref(r))
        return it, float(r.value)

    def pressure(self) -> tuple[int, float]:
        """solvePressureSystem on the current u*, v*, dE, dN."""
        r = self._real()
        it = self.lib.orc_pressure(self.h, ctypes.byref(r))
        return it, float(r.value)


def dp_window_stop(core_dp, rampSteps: int, window: int, percent: float) -> int | None:
    """The pressure-drop window stop rule of SIMPLE::runIterations
    (SIMPLE.cpp:449-491), applied to a per-iteration core total-pressure-drop
    history: from iteration rampSteps on, the drops fill a circular buffer of
    `window` entries; once it is full, the loop stops after the first
    iteration whose buffer has a population standard deviation and a latest
    deviation from the mean both below `percent` % of max(|mean|, 1).
    Returns the number of completed iterations when the rule fires (the
    reference's loop exits after that iteration), or None."""
    buf = np.zeros(window)
    idx, filled = 0, False
    for it, d in enumerate(np.asarray(core_dp, dtype=np.float64)):
        if it < rampSteps:
            continue
        buf[idx] = d
        idx = (idx + 1) % window
        if idx == 0:
            filled = True
        if filled:
            s = 0.0
            for q in range(window):
                s += buf[q]
            mean = s / window
            var = 0.0
            for q in range(window):
                var += (buf[q] - mean) * (buf[q] - mean)
            denom = max(abs(mean), 1.0)
            std_pct = np.sqrt(var / window) / denom * 100.0
            latest_pct = abs(buf[(idx - 1 + window) % window] - mean) / denom * 100.0
            if std_pct < percent and latest_pct < percent:
                return it + 1
    return None


# --------------------------------------------------------------------------
# reference build (oracle/_ref)

def ref_available(name: str = "ref_f32_pin") -> bool:
    return os.path.exists(os.path.join(REF_DIR, name))


def write_case(case_dir: str, cellType: np.ndarray, hy: float, hx: float, U: float,
               Ht: float = 0.0) -> None:
    """ExportFiles/fluid_params.txt and geometry_fluid.txt in the reference's
    formats (SIMPLE.cpp:41-59, 653-662).  Values are written with 17
    significant digits so float and double parses recover the same numbers
    for float32-representable inputs."""
    ex = os.path.join(case_dir, "ExportFiles")
    os.makedirs(ex, exist_ok=True)
    Ny, Nx = cellType.shape
    with open(os.path.join(ex, "fluid_params.txt"), "w") as f:
        f.write(f"{Ny} {Nx} {hy:.17g} {hx:.17g} {U:.17g} 0 0 {Ht:.17g}\n")
    np.savetxt(os.path.join(ex, "geometry_fluid.txt"), np.asarray(cellType, dtype=np.float64),
               fmt="%.17g")


_REF_KEYS = ("rho", "eta", "brinkmanKMin", "brinkmanQ", "convectionScheme", "enableTwoPointFiveD",
             "twoPointFiveDConvectionFactor", "twoPointFiveDSinkMultiplier", "epsilon",
             "maxIterations", "maxPressureIter", "pTol", "momentumTol", "maxMomentumIter",
             "uvAlpha", "pAlpha", "xPlaneCoreInlet", "xPlaneCoreOutlet", "enableInletRamp",
             "rampSteps", "pressureSolverType", "momentumSolverType", "enableNormalizedResiduals",
             "usePressureDropConvergence", "dpConvergenceWindow", "dpConvergencePercent")


def ref_overrides(params: dict, threads: int = 1) -> list[str]:
    out = [f"{k}={params[k]!r}" if isinstance(params[k], float) else f"{k}={params[k]}"
           for k in _REF_KEYS if k in params]
    out.append(f"threads={threads}")
    return out


@dataclass
class RefResult:
    history: np.ndarray
    fields: dict


def read_fields(path: str) -> dict:
    out = {}
    with open(path, "rb") as f:
        while True:
            tag = f.read(16)
            if len(tag) < 16:
                break
            dims = np.frombuffer(f.read(8), dtype=np.int32)
            r, c = int(dims[0]), int(dims[1])
            out[tag.rstrip(b"\0").decode()] = np.frombuffer(f.read(8 * r * c), dtype=np.float64).reshape(r, c)
    return out


def run_reference(binary: str, case_dir: str, params: dict, threads: int = 1,
                  timeout: float = 600.0) -> RefResult:
    """Run oracle/_ref/<binary> on a case directory written by write_case()."""
    exe = os.path.join(REF_DIR, binary)
    with tempfile.TemporaryDirectory() as out:
        cmd = [exe, case_dir, out] + ref_overrides(params, threads)
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, timeout=timeout)
        hist = np.loadtxt(os.path.join(out, "history.txt"), skiprows=1, ndmin=2)
        return RefResult(history=hist[:, :len(HIST_COLS)], fields=read_fields(os.path.join(out, "fields.bin")))
