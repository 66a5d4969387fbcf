"""Batched ensembles over the C-ABI (nbody_ensemble_*): many independent
systems of uneven size advanced by one persistent pair launch per step."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check
from .engine import FIELDS, PRECISIONS, _ptr, plummer


class EnsembleConfig(C.Structure):
    _fields_ = [("nclusters", C.c_int), ("n", C.POINTER(C.c_int)), ("eps2", C.POINTER(C.c_double)),
                ("dt", C.POINTER(C.c_double)), ("precision", C.c_int), ("device", C.c_int),
                ("tiles_per_item", C.c_int), ("tune", C.c_int), ("pair_variant", C.c_int),
                ("sort_every", C.c_int)]


class EnsembleInfo(C.Structure):
    _fields_ = [("nclusters", C.c_int), ("padded_rows", C.c_int), ("items", C.c_int),
                ("tiles_per_item", C.c_int), ("grid", C.c_int), ("threads", C.c_int),
                ("j_tile", C.c_int), ("interactions_per_step", C.c_double), ("steps", C.c_longlong),
                ("last_step_ms", C.c_double), ("record_format", C.c_int), ("step_kernels", C.c_int),
                ("reorders", C.c_longlong), ("order_kernels", C.c_int)]


_vp = C.c_void_p
_SIGS = {
    "nbody_ensemble_create": [C.POINTER(_vp), C.POINTER(EnsembleConfig)],
    "nbody_ensemble_destroy": [_vp],
    "nbody_ensemble_set_state": [_vp] + [_vp] * 7,
    "nbody_ensemble_get_state": [_vp] + [_vp] * 6,
    "nbody_ensemble_get_derivs": [_vp] + [_vp] * 6,
    "nbody_ensemble_acc_jerk": [_vp],
    "nbody_ensemble_step": [_vp, C.c_int],
    "nbody_ensemble_synchronize": [_vp],
    "nbody_ensemble_energy": [_vp, _vp, _vp],
    "nbody_ensemble_info": [_vp, C.POINTER(EnsembleInfo)],
    "nbody_ensemble_get_stream": [_vp, C.POINTER(_vp)],
}


def _f(name):
    return _lib.bind(name, _SIGS[name])


class Ensemble:
    """Clusters of sizes n[c] with softening eps2[c] and fixed step dt[c].

    Mixed precision: pair_variant 0 (default) and 3 use the packed hi/lo
    kernel; 4 the near/far tile-relative kernel, each cluster kept in Hilbert
    order within its own segment (states and derivatives come back in the
    caller's order); 5 the tile-relative kernel with every tile taken as far."""

    def __init__(self, n, eps2, dt, precision: str = "mixed", device: int = 0,
                 tiles_per_item: int = 0, tune: bool = False, pair_variant: int = 0,
                 sort_every: int = 0):
        self.n = np.ascontiguousarray(n, dtype=np.int32)
        C_ = self.n.size
        self.eps2 = np.ascontiguousarray(np.broadcast_to(eps2, (C_,)), dtype=np.float64)
        self.dt = np.ascontiguousarray(np.broadcast_to(dt, (C_,)), dtype=np.float64)
        cfg = EnsembleConfig(C_, self.n.ctypes.data_as(C.POINTER(C.c_int)),
                             self.eps2.ctypes.data_as(C.POINTER(C.c_double)),
                             self.dt.ctypes.data_as(C.POINTER(C.c_double)),
                             PRECISIONS[precision], device, tiles_per_item, int(tune),
                             pair_variant, sort_every)
        h = _vp()
        check(_f("nbody_ensemble_create")(C.byref(h), C.byref(cfg)), "nbody_ensemble_create")
        self._h = h
        self.total = int(self.n.sum())
        self.offsets = np.concatenate([[0], np.cumsum(self.n)]).astype(np.int64)
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            _f("nbody_ensemble_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_state(self, state: dict):
        arrs = [np.ascontiguousarray(state[k], dtype=np.float64) for k in FIELDS]
        assert all(a.size == self.total for a in arrs)
        check(_f("nbody_ensemble_set_state")(self._h, *map(_ptr, arrs)), "nbody_ensemble_set_state")

    def get_state(self) -> dict:
        out = {k: np.empty(self.total) for k in ("x", "y", "z", "vx", "vy", "vz")}
        check(_f("nbody_ensemble_get_state")(self._h, *[_ptr(out[k]) for k in out]),
              "nbody_ensemble_get_state")
        return out

    def get_derivs(self) -> np.ndarray:
        d = np.empty((6, self.total))
        check(_f("nbody_ensemble_get_derivs")(self._h, *[_ptr(d[k]) for k in range(6)]),
              "nbody_ensemble_get_derivs")
        return d

    def force_calculation(self):
        check(_f("nbody_ensemble_acc_jerk")(self._h), "nbody_ensemble_acc_jerk")

    def timestepping(self, nsteps: int = 1):
        check(_f("nbody_ensemble_step")(self._h, int(nsteps)), "nbody_ensemble_step")

    def synchronize(self):
        check(_f("nbody_ensemble_synchronize")(self._h), "nbody_ensemble_synchronize")

    def energy(self):
        T = np.empty(self.n.size)
        U = np.empty(self.n.size)
        check(_f("nbody_ensemble_energy")(self._h, _ptr(T), _ptr(U)), "nbody_ensemble_energy")
        return T, U

    def info(self) -> dict:
        i = EnsembleInfo()
        check(_f("nbody_ensemble_info")(self._h, C.byref(i)), "nbody_ensemble_info")
        return {name: getattr(i, name) for name, _ in EnsembleInfo._fields_}

    @property
    def stream(self) -> int:
        s = _vp()
        check(_f("nbody_ensemble_get_stream")(self._h, C.byref(s)), "nbody_ensemble_get_stream")
        return s.value or 0


def plummer_ensemble(nclusters: int, seed: int, nmin: int = 256, nmax: int = 8192):
    """Cluster sizes log-uniform in [nmin, nmax] (seeded), each a Plummer
    sphere in Henon units with its own derived seed; softening eps = 4/N.
    Returns (sizes, eps2, concatenated state)."""
    rng = np.random.default_rng(seed)
    sizes = np.rint(np.exp(rng.uniform(math.log(nmin), math.log(nmax), nclusters))).astype(np.int32)
    parts = [plummer(int(n), seed * 1_000_003 + c) for c, n in enumerate(sizes)]
    state = {k: np.concatenate([p[k] for p in parts]) for k in FIELDS}
    eps2 = (4.0 / sizes.astype(np.float64)) ** 2
    return sizes, eps2, state
