"""C-ABI library checks that need no GPU: the shared library loads, exports
every function include/nbody_cuda.h declares, validates its arguments, and
its host-side initial-condition generators behave."""
import ctypes as C

import numpy as np
import pytest

import nbody_b200 as nb
from nbody_b200 import _lib
from _util import GOLDEN_SIZES, golden


def test_library_loads_and_exports_header_symbols():
    L = nb.load()
    names = nb.header_functions()
    assert "nbody_force_calculation" in names and "nbody_create" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_config_defaults():
    cfg = _lib.NBodyConfig()
    assert nb.load().nbody_config_init(C.byref(cfg)) == 0
    assert cfg.eps2 == 1e-7 and cfg.precision == 0 and cfg.dt == 0.0
    assert cfg.eta == 1e-2 and cfg.eta0 == 1e-4


@pytest.mark.parametrize("field,value", [("n", 0), ("eps2", 0.0), ("eps2", -1.0), ("precision", 7),
                                         ("eta", 0.0), ("split_j", -1)])
def test_create_rejects_bad_config(field, value):
    L = nb.load()
    cfg = _lib.NBodyConfig()
    L.nbody_config_init(C.byref(cfg))
    cfg.n = 16
    setattr(cfg, field, value)
    h = C.c_void_p()
    assert L.nbody_create(C.byref(h), C.byref(cfg)) == 1  # NBODY_ERR_INVALID_ARG
    assert not h.value
    assert L.nbody_last_error()


def test_null_arguments_rejected():
    L = nb.load()
    assert L.nbody_create(None, None) == 1
    assert L.nbody_acc_jerk(None) == 1
    z = np.zeros(4)
    p = C.c_void_p(z.ctypes.data)
    assert L.nbody_force_calculation(4, 1e-7, 0, 0, 4, *([p] * 12), None) == 1
    assert L.nbody_force_calculation(4, 1e-7, 0, 2, 1, *([p] * 13)) == 1  # empty-reversed range


def test_status_strings():
    L = nb.load()
    for s in range(8):
        assert L.nbody_status_string(s)


def test_create_without_device_reports_it():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    L = nb.load()
    cfg = _lib.NBodyConfig()
    L.nbody_config_init(C.byref(cfg))
    cfg.n = 16
    h = C.c_void_p()
    assert L.nbody_create(C.byref(h), C.byref(cfg)) == 6  # NBODY_ERR_NO_DEVICE


@pytest.mark.parametrize("n", GOLDEN_SIZES)
def test_reference_ic_matches_reference(n):
    """The engine's copy of the reference initialiser reproduces the
    reference's bodies bit for bit (NaN velocities at n = 1, where the
    reference's virial rescale divides by a zero potential)."""
    g = golden(n)
    s = nb.reference_ic(n, 1e-7)
    for k in nb.FIELDS:
        assert np.array_equal(s[k], g[k], equal_nan=True), k


def test_plummer_moments():
    n = 20000
    s = nb.plummer(n, seed=1)
    m = s["m"]
    assert np.allclose(m, 1.0 / n)
    pos = np.stack([s["x"], s["y"], s["z"]])
    vel = np.stack([s["vx"], s["vy"], s["vz"]])
    assert np.abs((m * pos).sum(1)).max() < 1e-12
    assert np.abs((m * vel).sum(1)).max() < 1e-12
    T = 0.5 * (m * (vel ** 2).sum(0)).sum()
    assert abs(T - 0.25) < 0.02       # Henon units: T = -E = 1/4 within sampling noise
    r = np.sqrt((pos ** 2).sum(0))
    rh = np.median(r)                 # half-mass radius of a Plummer sphere = 0.769 in Henon units
    assert abs(rh - 0.769) < 0.03


def test_plummer_deterministic_and_seeded():
    a = nb.plummer(1000, 2)
    b = nb.plummer(1000, 2)
    c = nb.plummer(1000, 3)
    assert all(np.array_equal(a[k], b[k]) for k in nb.FIELDS)
    assert not np.array_equal(a["x"], c["x"])
