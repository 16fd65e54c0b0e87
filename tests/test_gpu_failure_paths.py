"""Error paths of the flow solver, made without any GPU fault.

* Bounded waits: cp_selftest_bounded_wait runs a grid-barrier wait and an
  mbarrier wait on events that never come, with a 0.2 s limit; each must give
  up and leave CP_ERR_TIMEOUT in the device status word, and the device must
  stay usable afterwards.
* Non-finite input: a NaN in gamma is rejected at the host boundary with
  CP_ERR_NONFINITE.
* Non-finite state: a finite but huge velocity (1e300, set from the host)
  overflows inside the iteration; the finalize kernel detects it, the loop
  stops with CP_STOP_ERROR and cp_step returns CP_ERR_NONFINITE.
"""
import ctypes

import numpy as np
import pytest

from _helpers import gpu_for, small_cases

pytestmark = pytest.mark.gpu

CP_ERR_NONFINITE, CP_ERR_TIMEOUT, CP_STOP_ERROR = 3, 5, 4


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    return built_lib


@pytest.mark.parametrize("kind", [0, 1], ids=["grid_barrier", "mbarrier"])
def test_bounded_wait_gives_up_with_timeout(kind):
    from coldplate_b200 import _native as nat
    st = ctypes.c_int(-1)
    nat.check(nat.lib().cp_selftest_bounded_wait(kind, 0.2, ctypes.byref(st)))
    assert st.value == CP_ERR_TIMEOUT
    # the device is still usable
    case = small_cases()["density"]
    with gpu_for(case) as g:
        rep = g.step(2)
        assert rep["iter"] == 2 and np.isfinite(rep["fullTotalDrop"])


def test_selftest_rejects_bad_arguments():
    from coldplate_b200 import _native as nat
    st = ctypes.c_int(-1)
    assert nat.lib().cp_selftest_bounded_wait(2, 0.2, ctypes.byref(st)) == 1
    assert nat.lib().cp_selftest_bounded_wait(0, 0.0, ctypes.byref(st)) == 1


def test_nan_gamma_is_rejected():
    from coldplate_b200._native import CpError
    case = small_cases()["density"]
    with gpu_for(case) as g:
        gam = 1.0 - case.cellType
        gam[5, 7] = np.nan
        with pytest.raises(CpError) as e:
            g.set_gamma(gam)
        assert e.value.status == CP_ERR_NONFINITE


def test_overflowing_state_stops_with_error():
    from coldplate_b200 import _native as nat
    case = small_cases()["density"]
    with gpu_for(case) as g:
        g.step(3)
        u = g.get("u")
        u[10, 20] = 1e300
        g.set("u", u)
        rep = nat.CpIterReport()
        status = g._lib.cp_step(g._h, 5, ctypes.byref(rep))
        assert status == CP_ERR_NONFINITE
        assert rep.done == 1 and rep.stop_reason == CP_STOP_ERROR
