"""Failure detection without a GPU fault: in-kernel waits are bounded and
report through a status word the host turns into NBODY_ERR_TIMEOUT; the
context stays usable afterwards."""
import numpy as np
import pytest

import nbody_b200 as nb
import oracle as O
from nbody_b200 import _lib
from _util import derivs_rel

pytestmark = pytest.mark.gpu


def _selftest():
    import ctypes as C
    return _lib.bind("nbody_selftest_bounded_wait", [C.c_int, C.c_double])


def test_bounded_wait_reports_timeout_and_context_survives():
    f = _selftest()
    assert f(0, 20.0) == 4  # NBODY_ERR_TIMEOUT
    assert "gave up" in nb.load().nbody_last_error().decode()
    s = nb.plummer(700, seed=3)
    with nb.Engine(700, eps2=1e-4, dt=1.0) as e:   # the same context still computes correctly
        e.set_state(s)
        e.force_calculation()
        d = e.get_derivs()
    ea, ej = derivs_rel(d, O.force(s, 1e-4))
    assert ea <= 1e-12 and ej <= 1e-12


def test_selftest_rejects_bad_limit():
    f = _selftest()
    assert f(0, 0.0) == 1 and f(0, 1e6) == 1
