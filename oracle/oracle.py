"""ORACLE - test infrastructure only.

ctypes access to
  * ``liboracle.so`` - the serial C++ restatement of the reference's FP64 CPU
    Hermite-4 path with a runtime softening (oracle/nbody_oracle.cpp), and
  * ``_ref/libnbody_ref.so`` / ``_ref/libnbody_ref_f32.so`` - the unmodified
    reference CPU sources (src/nbody.cpp, src/utils.cpp, src/kernel.cpp)
    compiled with a one-rank MPI stub and wrapped by oracle/ref_harness.cpp.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs import this module, and only as the checker or the timed CPU baseline.
The product (``n-body-code_b200``) never imports it.

Array convention: SoA float64 numpy arrays of length n (x, y, z, m, vx, vy,
vz), derivatives returned as a (6, n) array (ax, ay, az, jx, jy, jz).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libnbody_ref.so")
_REF_F32 = os.path.join(HERE, "_ref", "libnbody_ref_f32.so")
REF_APP = os.path.join(HERE, "_ref", "nbody_app")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

_lib = None
_ref = {}


def build(ref_tree: str | None = None) -> None:
    """Compile the restatement (always) and, given the reference tree
    (`ref_tree`, else the NBODY_REFERENCE_TREE environment variable; there is
    no default location), the reference build in oracle/_ref."""
    ref_tree = ref_tree or os.environ.get("NBODY_REFERENCE_TREE")
    targets = ["oracle"]
    if ref_tree and os.path.isdir(ref_tree):
        targets.append("ref")
        # the reference's own driver linked against the engine library
        if os.path.exists(os.path.join(HERE, "..", "n-body-code_b200", "lib", "libnbody_cuda.so")):
            targets.append("ref_gpu")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={ref_tree or ''}", *targets], check=True,
                   stdout=subprocess.DEVNULL)


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        for name in ("orc_force_fp64", "orc_force_f32"):
            getattr(L, name).argtypes = [C.c_int, C.c_double] + [_dp] * 13
            getattr(L, name).restype = None
        L.orc_force_rows_fp64.argtypes = [C.c_int, C.c_double] + [_dp] * 7 + [C.c_int, _ip, _dp]
        L.orc_force_rows_f32.argtypes = [C.c_int, C.c_double] + [_dp] * 7 + [C.c_int, _ip, _dp]
        L.orc_potential_rows.argtypes = [C.c_int, C.c_double] + [_dp] * 4 + [C.c_int, _ip, _dp]
        L.orc_invsqrt2d.argtypes = [C.c_double]
        L.orc_invsqrt2d.restype = C.c_double
        L.orc_predict.argtypes = [C.c_int, C.c_double] + [_dp] * 12
        L.orc_snapcrackle.argtypes = [C.c_int, C.c_double] + [_dp] * 6
        L.orc_correct.argtypes = [C.c_int, C.c_double] + [_dp] * 4
        L.orc_updatedt.argtypes = [C.c_int, C.c_double] + [_dp] * 4
        L.orc_updatedt.restype = C.c_double
        L.orc_initialdt.argtypes = [C.c_int, C.c_double] + [_dp] * 2
        L.orc_initialdt.restype = C.c_double
        L.orc_eta.restype = C.c_double
        L.orc_eta0.restype = C.c_double
        L.orc_kinetic.argtypes = [C.c_int] + [_dp] * 4
        L.orc_kinetic.restype = C.c_double
        L.orc_potential.argtypes = [C.c_int, C.c_double, C.c_int] + [_dp] * 4
        L.orc_potential.restype = C.c_double
        L.orc_initialize.argtypes = [C.c_int] + [C.c_double] * 5 + [_dp] * 7
        L.orc_hermite_fixed.argtypes = ([C.c_int, C.c_double, C.c_double, C.c_int, C.c_int]
                                        + [_dp] * 8 + [_dp])
        L.orc_force_jvp.argtypes = [C.c_int, C.c_double] + [_dp] * 8
        L.orc_hermite_tlm.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int] + [_dp] * 6
        L.orc_plummer.argtypes = [C.c_int, C.c_uint64] + [_dp] * 7
        L.orc_plummer.restype = None
        _lib = L
    return _lib


def have_reference(f32: bool = False) -> bool:
    return os.path.exists(_REF_F32 if f32 else _REF)


def ref(f32: bool = False):
    """The compiled, unmodified reference (FP64 build or the _F32 build)."""
    key = "f32" if f32 else "fp64"
    if key not in _ref:
        path = _REF_F32 if f32 else _REF
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build with `make -C oracle ref`")
        L = C.CDLL(path)
        L.ref_eps2.restype = C.c_double
        L.ref_max_threads.restype = C.c_int
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_initialize.argtypes = [C.c_int] + [_dp] * 7
        L.ref_force.argtypes = [C.c_int] + [_dp] * 13
        L.ref_kinetic.argtypes = [C.c_int] + [_dp] * 4
        L.ref_kinetic.restype = C.c_double
        L.ref_potential.argtypes = [C.c_int] + [_dp] * 4
        L.ref_potential.restype = C.c_double
        L.ref_hermite_fixed.argtypes = [C.c_int, C.c_double, C.c_int] + [_dp] * 13 + [_dp]
        L.ref_cycle.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp]
        L.ref_initialdt.argtypes = [C.c_int] + [_dp] * 6
        L.ref_initialdt.restype = C.c_double
        L.ref_bench_create.argtypes = [C.c_int, C.c_double, C.c_int] + [_dp] * 7
        L.ref_bench_create.restype = C.c_void_p
        L.ref_bench_step.argtypes = [C.c_void_p, _dp]
        L.ref_bench_destroy.argtypes = [C.c_void_p]
        L.orc_plummer.argtypes = [C.c_int, C.c_uint64] + [_dp] * 7
        L.orc_plummer.restype = None
        _ref[key] = L
    return _ref[key]


# ----------------------------------------------------------------------------
# restatement
# ----------------------------------------------------------------------------

def _state(s):
    return [np.ascontiguousarray(s[k], dtype=np.float64) for k in
            ("x", "y", "z", "m", "vx", "vy", "vz")]


def force(state: dict, eps2: float, precision: str = "fp64") -> np.ndarray:
    x, y, z, m, vx, vy, vz = _state(state)
    n = x.size
    out = np.zeros((6, n))
    f = lib().orc_force_f32 if precision == "f32" else lib().orc_force_fp64
    f(n, eps2, *map(_p, (x, y, z, m, vx, vy, vz)), *[_p(out[k]) for k in range(6)])
    return out


def force_rows(state: dict, eps2: float, rows, precision: str = "fp64") -> np.ndarray:
    """Direct sums for the given i-rows; precision "f32" uses the reference's
    _F32 pair arithmetic (the accuracy floor of the mixed kernels)."""
    x, y, z, m, vx, vy, vz = _state(state)
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    out = np.zeros((6, rows.size))
    f = lib().orc_force_rows_f32 if precision == "f32" else lib().orc_force_rows_fp64
    f(x.size, eps2, *map(_p, (x, y, z, m, vx, vy, vz)), rows.size, rows.ctypes.data_as(_ip), _p(out))
    return out


def potential_rows(state: dict, eps2: float, rows) -> np.ndarray:
    x, y, z, m = _state(state)[:4]
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    out = np.zeros(rows.size)
    lib().orc_potential_rows(x.size, eps2, _p(x), _p(y), _p(z), _p(m), rows.size,
                             rows.ctypes.data_as(_ip), _p(out))
    return out


def invsqrt2d(x: float) -> float:
    return lib().orc_invsqrt2d(x)


def kinetic(state: dict) -> float:
    x, y, z, m, vx, vy, vz = _state(state)
    return lib().orc_kinetic(x.size, _p(m), _p(vx), _p(vy), _p(vz))


def potential(state: dict, eps2: float, compat: bool = False) -> float:
    x, y, z, m = _state(state)[:4]
    return lib().orc_potential(x.size, eps2, int(compat), _p(x), _p(y), _p(z), _p(m))


def plummer(n: int, seed: int, from_reference_build: bool = False) -> dict:
    """The benchmark's Plummer bodies (oracle/plummer.cpp), value for value
    the engine's nbody_plummer; from the library in oracle/_ref when
    `from_reference_build`, so that a CPU leg loads no other library."""
    arrs = [np.zeros(n) for _ in range(7)]
    L = ref() if from_reference_build else lib()
    L.orc_plummer(int(n), int(seed), *map(_p, arrs))
    return dict(zip(("x", "y", "z", "m", "vx", "vy", "vz"), arrs))


def initialize(n: int, eps2: float = 1e-7) -> dict:
    arrs = [np.zeros(n) for _ in range(7)]
    lib().orc_initialize(n, 1.0, 1.0, 0.01, 1.0, eps2, *map(_p, arrs))
    return dict(zip(("x", "y", "z", "m", "vx", "vy", "vz"), arrs))


def hermite_fixed(state: dict, eps2: float, dt: float, nsteps: int, precision: str = "fp64"):
    """Returns (state_after, derivs (6, n), dt_criterion_of_last_step)."""
    x, y, z, m, vx, vy, vz = [a.copy() for a in _state(state)]
    n = x.size
    d = np.zeros((6, n))
    dtn = C.c_double(0.0)
    lib().orc_hermite_fixed(n, eps2, dt, nsteps, 1 if precision == "f32" else 0,
                            *map(_p, (x, y, z, m, vx, vy, vz)), _p(d), C.byref(dtn))
    return dict(x=x, y=y, z=z, m=m, vx=vx, vy=vy, vz=vz), d, dtn.value


def predict(state: dict, derivs: np.ndarray, dt: float) -> dict:
    x, y, z, m, vx, vy, vz = [a.copy() for a in _state(state)]
    d = np.ascontiguousarray(derivs)
    lib().orc_predict(x.size, dt, *map(_p, (x, y, z, vx, vy, vz)), *[_p(d[k]) for k in range(6)])
    return dict(x=x, y=y, z=z, m=m, vx=vx, vy=vy, vz=vz)


def snapcrackle(d0: np.ndarray, d1: np.ndarray, dt: float):
    n = d0.shape[1]
    a = np.ascontiguousarray(d0[:3]); j = np.ascontiguousarray(d0[3:])
    a1 = np.ascontiguousarray(d1[:3]); j1 = np.ascontiguousarray(d1[3:])
    a2 = np.zeros((3, n)); a3 = np.zeros((3, n))
    lib().orc_snapcrackle(n, dt, _p(a), _p(j), _p(a1), _p(j1), _p(a2), _p(a3))
    return a2, a3


def updatedt(d0: np.ndarray, a2: np.ndarray, a3: np.ndarray, eta: float | None = None) -> float:
    n = d0.shape[1]
    a = np.ascontiguousarray(d0[:3]); j = np.ascontiguousarray(d0[3:])
    eta = lib().orc_eta() if eta is None else eta
    return lib().orc_updatedt(n, eta, _p(a), _p(j), _p(np.ascontiguousarray(a2)),
                              _p(np.ascontiguousarray(a3)))


def initialdt(d0: np.ndarray, eta0: float | None = None) -> float:
    n = d0.shape[1]
    a = np.ascontiguousarray(d0[:3]); j = np.ascontiguousarray(d0[3:])
    eta0 = lib().orc_eta0() if eta0 is None else eta0
    return lib().orc_initialdt(n, eta0, _p(a), _p(j))


# ----------------------------------------------------------------------------
# the compiled reference
# ----------------------------------------------------------------------------

def ref_initialize(n: int) -> dict:
    arrs = [np.zeros(n) for _ in range(7)]
    ref().ref_initialize(n, *map(_p, arrs))
    return dict(zip(("x", "y", "z", "m", "vx", "vy", "vz"), arrs))


def ref_force(state: dict, f32: bool = False) -> np.ndarray:
    x, y, z, m, vx, vy, vz = _state(state)
    out = np.zeros((6, x.size))
    ref(f32).ref_force(x.size, *map(_p, (x, y, z, m, vx, vy, vz)), *[_p(out[k]) for k in range(6)])
    return out


def ref_hermite_fixed(state: dict, dt: float, nsteps: int, f32: bool = False):
    x, y, z, m, vx, vy, vz = [a.copy() for a in _state(state)]
    d = np.zeros((6, x.size))
    dtn = C.c_double(0.0)
    ref(f32).ref_hermite_fixed(x.size, dt, nsteps, *map(_p, (x, y, z, m, vx, vy, vz)),
                               *[_p(d[k]) for k in range(6)], C.byref(dtn))
    return dict(x=x, y=y, z=z, m=m, vx=vx, vy=vy, vz=vz), d, dtn.value


def _blk(s, keys):
    return np.ascontiguousarray(np.stack([np.asarray(s[k], dtype=np.float64) for k in keys]))


def force_jvp(state: dict, eps2: float, dx, dv, dm):
    """Tangent of (acc, jerk) along (dx (3,n), dv (3,n), dm (n,)); returns (da, dj)."""
    X = _blk(state, ("x", "y", "z")); V = _blk(state, ("vx", "vy", "vz"))
    m = np.ascontiguousarray(state["m"], dtype=np.float64)
    dx = np.ascontiguousarray(dx, dtype=np.float64); dv = np.ascontiguousarray(dv, dtype=np.float64)
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    n = m.size
    da = np.zeros((3, n)); dj = np.zeros((3, n))
    lib().orc_force_jvp(n, eps2, _p(X), _p(V), _p(m), _p(dx), _p(dv), _p(dm), _p(da), _p(dj))
    return da, dj


def hermite_tlm(state: dict, eps2: float, dt: float, nsteps: int, dx, dv, dm):
    """Fixed-dt FP64 run and its tangent: returns (X1 (3,n), V1 (3,n), DX1, DV1)."""
    X = _blk(state, ("x", "y", "z")); V = _blk(state, ("vx", "vy", "vz"))
    m = np.ascontiguousarray(state["m"], dtype=np.float64)
    DX = np.array(dx, dtype=np.float64, copy=True, order="C")
    DV = np.array(dv, dtype=np.float64, copy=True, order="C")
    dm = np.ascontiguousarray(dm, dtype=np.float64)
    lib().orc_hermite_tlm(m.size, eps2, dt, nsteps, _p(X), _p(V), _p(m), _p(DX), _p(DV), _p(dm))
    return X, V, DX, DV
