"""Failure detection on the device without a fault: the particle pass's waits on its TMA windows
are bounded (about a second) and report MPM_STATUS_TIMEOUT instead of hanging. The check runs the
same bounded mbarrier wait on a barrier that nothing completes, with a short limit, and then uses
the handle again to show the context stayed usable."""
import ctypes

import numpy as np
import pytest

from mpm_b200 import _lib, scenes
from mpm_b200.solver import Solver

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_the_context_stays_usable():
    sc = scenes.elastic_cube()
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    L = _lib.lib()
    timed_out = ctypes.c_int32(-1)
    _lib.check(L.mpm_check_bounded_wait(sol.h, 1 << 24, ctypes.byref(timed_out)), sol.h)
    assert timed_out.value == 1
    assert L.mpm_check_bounded_wait(sol.h, 0, ctypes.byref(timed_out)) == -1  # MPM_ERR_INVALID_ARG
    sol.step_fixed(sc.meta["dt"], 2)
    out = sol.download(("x",))
    assert np.all(np.isfinite(out["x"])) and sol.status() == 0
    sol.close()
