"""State files (nbody_write_state_file / nbody_read_state_file): host-only."""
import ctypes as C
import os

import numpy as np
import pytest

import nbody_b200 as nb
from nbody_b200 import _lib

_vp = C.c_void_p
_dp = C.POINTER(C.c_double)


def _fns():
    w = _lib.bind("nbody_write_state_file", [C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_double] + [_vp] * 7)
    r = _lib.bind("nbody_read_state_file", [C.c_char_p, C.c_int, C.POINTER(C.c_int), _dp, _dp, _dp] + [_vp] * 7)
    return w, r


def test_round_trip_bitwise(tmp_path):
    w, r = _fns()
    s = nb.plummer(777, seed=3)
    p = str(tmp_path / "s.bin").encode()
    assert w(p, 777, 0.125, 1 / 1024, 1e-4, *[_vp(s[k].ctypes.data) for k in nb.FIELDS]) == 0
    assert os.path.getsize(p) == 64 + 7 * 8 * 777
    n, t, dt, e2 = C.c_int(), C.c_double(), C.c_double(), C.c_double()
    assert r(p, 0, C.byref(n), C.byref(t), C.byref(dt), C.byref(e2), *([None] * 7)) == 0
    assert (n.value, t.value, dt.value, e2.value) == (777, 0.125, 1 / 1024, 1e-4)
    out = {k: np.empty(777) for k in nb.FIELDS}
    assert r(p, 777, C.byref(n), None, None, None, *[_vp(out[k].ctypes.data) for k in nb.FIELDS]) == 0
    for k in nb.FIELDS:
        assert np.array_equal(out[k], s[k])


def test_rejects_bad_files(tmp_path):
    w, r = _fns()
    n = C.c_int()
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"not a state file" * 8)
    assert r(str(bad).encode(), 10, C.byref(n), None, None, None, *([None] * 7)) == 1
    s = nb.plummer(100, seed=1)
    p = str(tmp_path / "s.bin").encode()
    assert w(p, 100, 0.0, 0.0, 1e-4, *[_vp(s[k].ctypes.data) for k in nb.FIELDS]) == 0
    out = {k: np.empty(100) for k in nb.FIELDS}
    ptrs = [_vp(out[k].ctypes.data) for k in nb.FIELDS]
    assert r(p, 50, C.byref(n), None, None, None, *ptrs) == 1          # buffers too small
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-8])
    assert r(p, 100, C.byref(n), None, None, None, *ptrs) == 1         # truncated
    assert r(b"/nonexistent/x.bin", 100, C.byref(n), None, None, None, *ptrs) == 1
