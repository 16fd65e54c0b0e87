"""Python mirror of the reference's SIMPLE solver interface over the C ABI.

``Simple`` follows class SIMPLE (SIMPLE.h:55-614): the parameters keep their
SIMPLE.h names (pressureSolverType, momentumSolverType, maxPressureIter,
uvAlpha, ...), the fields keep their staggered shapes (u (M+1) x N,
v M x (N+1), p (M+1) x (N+1)), and the entry points are the ones
iterations.cpp and SIMPLE.cpp call:

    runIterations()            SIMPLE.cpp:310      (whole loop, device-side stop rules)
    calculateStep()            iterations.cpp:82   (one outer iteration)
    solveUMomentumImplicit()   momentum_solver.cpp:362
    solveVMomentumImplicit()   momentum_solver.cpp:366
    solvePressureSystem()      pressure_solver.cpp:462

Every call runs the CUDA kernels in libcoldplate.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _native as nat


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_params(**knobs) -> nat.CpParams:
    """cp_params with the SIMPLE.h defaults, then the given overrides."""
    p = nat.default_params()
    names = {n for n, _ in nat.PARAM_FIELDS}
    for k, v in knobs.items():
        if k not in names:
            raise KeyError(f"unknown parameter {k!r}")
        if k == "precision" and isinstance(v, str):
            v = {"fp64": nat.PREC_FP64, "mixed": nat.PREC_MIXED}[v]
        setattr(p, k, v)
    return p


class Simple:
    """One field on the GPU.  ``knobs`` are cp_params / SIMPLE.h names."""

    def __init__(self, *, cellType=None, gamma=None, params: nat.CpParams | None = None, **knobs):
        self._lib = nat.lib()
        self.params = params if params is not None else make_params(**knobs)
        if params is not None and knobs:
            for k, v in knobs.items():
                setattr(self.params, k, v)
        h = ctypes.c_void_p()
        nat.check(self._lib.cp_create(ctypes.byref(self.params), ctypes.byref(h)))
        self._h = h
        self.M, self.N = self.params.Ny + 1, self.params.Nx + 1
        self.pressureIterations = 0
        if cellType is not None:
            self.set_cell_type(cellType)
        elif gamma is not None:
            self.set_gamma(gamma)

    # -------------------------------------------------------------- set-up
    @classmethod
    def from_case(cls, case_dir: str, **knobs) -> "Simple":
        """Load ExportFiles/fluid_params.txt and geometry_fluid.txt like the
        reference constructor (SIMPLE.cpp:18-29)."""
        p = make_params(**knobs)
        nat.check(nat.lib().cp_read_fluid_params(
            os.path.join(case_dir, "ExportFiles", "fluid_params.txt").encode(), ctypes.byref(p)))
        s = cls(params=p)
        nat.check(s._lib.cp_read_geometry(s._h, os.path.join(case_dir, "ExportFiles", "geometry_fluid.txt").encode()))
        return s

    def set_cell_type(self, cellType) -> None:
        a = np.ascontiguousarray(cellType, dtype=np.float64)
        nat.check(self._lib.cp_set_cell_type(self._h, _dptr(a), a.shape[0], a.shape[1], a.shape[1], 1))

    def set_gamma(self, gamma) -> None:
        a = np.ascontiguousarray(gamma, dtype=np.float64)
        nat.check(self._lib.cp_set_gamma(self._h, _dptr(a), a.shape[0], a.shape[1], a.shape[1], 1))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.cp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -------------------------------------------------------------- fields
    def shape(self, name: str) -> tuple[int, int]:
        M, N = self.M, self.N
        return {"u": (M + 1, N), "v": (M, N + 1), "p": (M + 1, N + 1), "uStar": (M + 1, N),
                "vStar": (M, N + 1), "pStar": (M + 1, N + 1), "dE": (M + 1, N), "dN": (M, N + 1),
                "gamma": (M, N), "alpha": (M, N), "cellType": (M, N)}[name]

    def get(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """The field as a float64 array of shape(name).  With `out` (a
        C-contiguous float64 array of that shape, e.g. a view of pinned host
        memory, which the copy then reaches by DMA) the field is written
        there and `out` is returned."""
        r, c = self.shape(name)
        if out is None:
            out = np.empty((r, c), dtype=np.float64)
        elif (out.dtype != np.float64 or out.shape != (r, c) or not out.flags.c_contiguous
              or not out.flags.writeable):
            raise ValueError(f"{name}: out must be a C-contiguous float64 array of shape {(r, c)}")
        nat.check(self._lib.cp_get_field(self._h, nat.FIELDS[name], _dptr(out), r, c, c, 1))
        return out

    def set(self, name: str, arr) -> None:
        r, c = self.shape(name)
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != (r, c):
            raise ValueError(f"{name}: shape {a.shape}, expected {(r, c)}")
        nat.check(self._lib.cp_set_field(self._h, nat.FIELDS[name], _dptr(a), r, c, c, 1))

    def __getattr__(self, name):
        if name in nat.FIELDS:
            return self.get(name)
        raise AttributeError(name)

    # -------------------------------------------------------------- loop
    def step(self, n: int = 1) -> dict:
        rep = nat.CpIterReport()
        nat.check(self._lib.cp_step(self._h, int(n), ctypes.byref(rep)))
        self.pressureIterations = rep.pressureIterations
        return rep.as_dict()

    def calculateStep(self) -> float:
        """One outer iteration; returns max(residU, residV, residMass)."""
        return self.step(1)["error"]

    def runIterations(self) -> dict:
        rep = nat.CpIterReport()
        nat.check(self._lib.cp_run(self._h, ctypes.byref(rep)))
        self.pressureIterations = rep.pressureIterations
        return rep.as_dict()

    def reset_loop(self) -> None:
        nat.check(self._lib.cp_reset_loop(self._h))

    def reset(self) -> None:
        """Back to the initial state (zero fields, empty history), no allocation."""
        nat.check(self._lib.cp_reset(self._h))

    def kernel_times(self, n: int) -> dict:
        """Run n outer iterations with a CUDA-event bracket around every launch."""
        t = nat.CpKernelTiming()
        nat.check(self._lib.cp_kernel_times(self._h, int(n), ctypes.byref(t)))
        return {"ms": dict(zip(nat.KERNEL_KINDS, list(t.ms))),
                "launches": dict(zip(nat.KERNEL_KINDS, list(t.launches))),
                "jacobiSweeps": t.jacobiSweeps, "pcgIterations": t.pcgIterations, "iterations": t.iterations}

    def history(self) -> dict:
        ncol = self._lib.cp_history_columns()
        cap = max(self.params.historyCapacity or self.params.maxIterations, 1)
        buf = np.zeros((cap, ncol), dtype=np.float64)
        n = ctypes.c_int()
        nat.check(self._lib.cp_get_history(self._h, _dptr(buf), cap, ctypes.byref(n)))
        rows = buf[: n.value]
        return {name: rows[:, k] for k, name in enumerate(nat.HIST_COLS)}

    # -------------------------------------------------------------- result files
    def saveAll(self, export_dir: str = "ExportFiles", u_old=None, v_old=None) -> list[str]:
        """The reference's result files (SIMPLE::saveAll, output.cpp:74-200)
        from the current fields; see coldplate_b200.output.  u_old / v_old
        (the fields before the last iteration) add u_resid_full /
        v_resid_full."""
        from . import output
        return output.save_all(export_dir, self.get("u"), self.get("v"), self.get("p"), self.params.hx,
                               self.params.hy, self.params.N_in_buffer, self.params.N_out_buffer, u_old, v_old)

    def writeIterationLogs(self, export_dir: str = "ExportFiles") -> None:
        """residuals.txt and pressure_drop_history.txt for the iterations run
        so far (output.cpp:302-364)."""
        from . import output
        output.write_logs(export_dir, self.history(), bool(self.params.enableNormalizedResiduals),
                          self.params.residNormFloorVel, self.params.residNormFloorMass)

    # -------------------------------------------------------------- adjoint
    def adjoint_dp_dgamma(self, max_iter: int = 2000, tol: float = 1e-10) -> tuple[np.ndarray, dict]:
        """dJ/dgamma (Ny x Nx) of the full-system total-pressure drop J at the
        current state (converge the forward solve first), by the discrete
        adjoint of the converged discretisation."""
        Ny, Nx = self.M - 1, self.N - 1
        g = np.empty((Ny, Nx), dtype=np.float64)
        rep = nat.CpAdjointReport()
        nat.check(self._lib.cp_adjoint_dp_dgamma(self._h, _dptr(g), Ny, Nx, Nx, 1, int(max_iter), float(tol),
                                                   ctypes.byref(rep)))
        return g, {name: getattr(rep, name) for name, _ in rep._fields_}

    def adjoint_probe(self, op: int, x: dict | None = None, max_iter: int = 2000,
                      tol: float = 1e-10) -> tuple[dict, dict]:
        """Verification of the adjoint at the current state (cp_adjoint_probe):
        op 0 J_X^T x, op 1 dJ/dX, op 2 the adjoint solution lambda.  x and the
        result are dicts of staggered arrays 'u' (M+1, N), 'v' (M, N+1) and
        'p' (M+1, N+1), zero outside the unknowns."""
        n = int(self._lib.cp_adjoint_probe_len(self._h))
        info = (ctypes.c_int * 4)()
        # the layout needs the pitch: ask with op 1 first when x must be packed
        y = np.zeros(n, dtype=np.float64)
        rep = nat.CpAdjointReport()
        M, N = self.M, self.N
        shapes = {"u": (M + 1, N), "v": (M, N + 1), "p": (M + 1, N + 1)}
        xin = None
        if op == 0:
            nat.check(self._lib.cp_adjoint_probe(self._h, 1, None, _dptr(y), 1, 1.0,
                                                  ctypes.cast(info, ctypes.POINTER(ctypes.c_int)), None))
            P = info[3]
            xin = np.zeros(n, dtype=np.float64)
            for b, f in enumerate(("u", "v", "p")):
                blk = xin[b * n // 3:(b + 1) * n // 3].reshape(-1, P)
                r, c = shapes[f]
                blk[:r, :c] = x[f]
        nat.check(self._lib.cp_adjoint_probe(self._h, int(op), None if xin is None else _dptr(xin), _dptr(y),
                                              int(max_iter), float(tol),
                                              ctypes.cast(info, ctypes.POINTER(ctypes.c_int)), ctypes.byref(rep)))
        P = info[3]
        out = {}
        for b, f in enumerate(("u", "v", "p")):
            blk = y[b * n // 3:(b + 1) * n // 3].reshape(-1, P)
            r, c = shapes[f]
            out[f] = blk[:r, :c].copy()
        meta = {"model": info[0], "sweepsU": info[1], "sweepsV": info[2], "pitch": P}
        if op == 2:
            meta.update({name: getattr(rep, name) for name, _ in rep._fields_})
        return out, meta

    # -------------------------------------------------------------- dispatch boundary
    def solveUMomentumImplicit(self) -> tuple[int, float]:
        r, it = ctypes.c_double(), ctypes.c_int()
        nat.check(self._lib.cp_momentum_u(self._h, ctypes.byref(r), ctypes.byref(it)))
        return it.value, r.value

    def solveVMomentumImplicit(self) -> tuple[int, float]:
        r, it = ctypes.c_double(), ctypes.c_int()
        nat.check(self._lib.cp_momentum_v(self._h, ctypes.byref(r), ctypes.byref(it)))
        return it.value, r.value

    def solvePressureSystem(self) -> tuple[int, float]:
        it, r = ctypes.c_int(), ctypes.c_double()
        nat.check(self._lib.cp_pressure(self._h, ctypes.byref(it), ctypes.byref(r)))
        return it.value, r.value


def partition_fields(work, n_parts: int) -> list[list[int]]:
    """Split fields of the given work (e.g. cells x expected outer
    iterations) into n_parts groups of nearly equal total work, one per GPU:
    largest first, each to the currently lightest group.  Fields are
    independent, so the groups need no exchange; every field lands in
    exactly one group.  Returns the field indices of each group, ascending."""
    if n_parts < 1:
        raise ValueError("n_parts must be >= 1")
    load = [0.0] * n_parts
    parts: list[list[int]] = [[] for _ in range(n_parts)]
    for q in sorted(range(len(work)), key=lambda i: (-float(work[i]), i)):
        k = min(range(n_parts), key=lambda r: (load[r], r))
        parts[k].append(q)
        load[k] += float(work[q])
    return [sorted(pq) for pq in parts]


class Batch:
    """Several ``Simple`` fields (grid sizes, geometries and inlet velocities
    may all differ) advanced together by one persistent kernel per launch
    (cp_batch_run).  Each field keeps its own stop rules, history and state:
    after ``run`` read results from the ``Simple`` objects as usual.  The
    fields must use pressureSolverType 2 or 4 and one precision, and must
    stay open while the batch exists.  When every field is type 4 the batch
    runs in team mode (teams of CTAs take whole fields from a queue and run
    the single-field smoothed-aggregation iteration); otherwise every field
    runs the 2 x 2 aggregation cycle over cell tiles."""

    def __init__(self, fields: list[Simple]):
        self._lib = nat.lib()
        self.fields = list(fields)
        arr = (ctypes.c_void_p * len(self.fields))(*[f._h.value for f in self.fields])
        h = ctypes.c_void_p()
        nat.check(self._lib.cp_batch_create(arr, len(self.fields), ctypes.byref(h)))
        self._h = h

    def set_tile(self, rows: int, cols: int) -> None:
        nat.check(self._lib.cp_batch_set_tile(self._h, int(rows), int(cols)))

    def set_team(self, ctas: int) -> None:
        """CTAs per team (team mode only)."""
        nat.check(self._lib.cp_batch_set_team(self._h, int(ctas)))

    def autotune(self, trial_outer: int = 4) -> dict:
        """Pick the fastest cell tile (team mode: team size) on trial_outer
        iterations; resets every field."""
        r = nat.CpBatchReport()
        nat.check(self._lib.cp_batch_autotune(self._h, int(trial_outer), ctypes.byref(r)))
        return {name: getattr(r, name) for name, _ in r._fields_}

    def run(self, max_outer: int) -> dict:
        r = nat.CpBatchReport()
        nat.check(self._lib.cp_batch_run(self._h, int(max_outer), ctypes.byref(r)))
        return {name: getattr(r, name) for name, _ in r._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.cp_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
