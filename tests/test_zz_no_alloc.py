"""cp_pressure_noalloc, the pressure solve that allocates no device memory.

Some callers cannot call cudaMalloc: a plugin that runs inside a host
application which has already handed the whole device-memory budget to its
own pool, or a control loop that must never wait in the allocator.  For
them the library keeps the solve's working memory in one fixed array and
the caller passes only inputs and outputs.  This test (collected last, so a
failure here comes after every other test has run) gives the entry point
the same inputs as the context-based cp_pressure and checks that both give
the same p', iteration count and mass imbalance, on two calls in a row.
The test owns its device buffers (torch), as such a caller would."""
import ctypes

import numpy as np
import pytest

from _helpers import gpu_for, oracle_for, rel_l2, small_cases

pytestmark = pytest.mark.gpu


def test_noalloc_pressure_matches_cp_pressure(built_lib):
    import torch

    from coldplate_b200 import _native as nat

    case = small_cases()["density"]
    o = oracle_for(case)
    o.run(12)
    o.momentum(True)
    o.momentum(False)
    fields = {f: o.get(f) for f in ("dE", "dN", "uStar", "vStar")}
    knobs = dict(pressureSolverType=1, maxPressureIter=60, pTol=1e-9)
    with gpu_for(case, **knobs) as g:
        for f, a in fields.items():
            g.set(f, a)
        it_ref, rm_ref = g.solvePressureSystem()
        p_ref = g.get("pStar")
        params = g.params

    M, N = case.Ny + 1, case.Nx + 1
    pitch = ((N + 1 + 31) // 32) * 32 + 8          # any pitch >= N + 1
    dev = torch.device("cuda:0")

    def on_device(a):
        t = torch.zeros((M + 2, pitch), dtype=torch.float64, device=dev)
        t[: a.shape[0], : a.shape[1]] = torch.from_numpy(a).to(dev)
        return t

    d = {f: on_device(a) for f, a in fields.items()}
    p_out = torch.full((M + 2, pitch), 7.0, dtype=torch.float64, device=dev)
    L = nat.lib()
    fn = L.cp_pressure_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(nat.CpParams)] + [ctypes.c_void_p] * 4 + [ctypes.c_long, ctypes.c_void_p,
                                                                            ctypes.POINTER(ctypes.c_int),
                                                                            ctypes.POINTER(ctypes.c_double),
                                                                            ctypes.c_void_p]
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        it, rm = ctypes.c_int(-1), ctypes.c_double(-1.0)
        st = fn(ctypes.byref(params), d["dE"].data_ptr(), d["dN"].data_ptr(), d["uStar"].data_ptr(),
                d["vStar"].data_ptr(), pitch, p_out.data_ptr(), ctypes.byref(it), ctypes.byref(rm), stream)
        assert st == 0, nat.lib().cp_last_error_string()
        p_na = p_out[: M + 1, : N + 1].cpu().numpy()
        assert it.value == it_ref, (call, it.value, it_ref)
        assert abs(rm.value - rm_ref) <= 1e-12 * abs(rm_ref), (call, rm.value, rm_ref)
        assert rel_l2(p_na, p_ref) <= 1e-12, (call, rel_l2(p_na, p_ref))
        p_out.fill_(-3.0)   # the next call must not depend on what is left here

    # beyond the fixed size: a clear error, before any device work
    from coldplate_b200.solver import make_params
    big = make_params(Ny=400, Nx=1000, hx=1e-5, hy=1e-5, rho=1000.0, pressureSolverType=1)
    st = fn(ctypes.byref(big), d["dE"].data_ptr(), d["dN"].data_ptr(), d["uStar"].data_ptr(),
            d["vStar"].data_ptr(), 1024, p_out.data_ptr(), None, None, stream)
    assert st == 1
    assert b"exceeds" in nat.lib().cp_last_error_string()
