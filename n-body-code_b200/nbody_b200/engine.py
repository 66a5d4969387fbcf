"""Python face of the engine: the reference's NBody surface over the C-ABI.

Method names follow the reference's NBody (include/nbody.h:24-51):
``initialdt`` / ``prediction`` / ``force_calculation`` / ``correction`` /
``timestepping`` / ``cycle`` map onto the engine's device kernels; state is
exchanged as SoA float64 numpy arrays (x, y, z, m, vx, vy, vz) and
derivatives as a (6, n) array (ax, ay, az, jx, jy, jz).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import NBODY_FP64, NBODY_MIXED, NBodyConfig, NBodyPeaks, NBodyTimers, check

FIELDS = ("x", "y", "z", "m", "vx", "vy", "vz")
PRECISIONS = {"fp64": NBODY_FP64, "mixed": NBODY_MIXED}


def _arr(a, n=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.shape != (n,):
        raise ValueError(f"expected shape ({n},), got {a.shape}")
    return a


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class Engine:
    """One system of n bodies on one GPU (wraps nbody_create/nbody_destroy).

    precision "mixed" takes pair_variant (nbody_config.pair_variant): 0 picks
    the near/far tile-relative kernel (4) from 16384 bodies and the packed
    hi/lo kernel (3) below; 1 and 2 are the other hi/lo forms; 5 is the
    tile-relative kernel with every tile taken as far (a comparison).  The
    tile-relative engines keep their bodies in Hilbert order on the device;
    get_state and get_derivs return them in the caller's order.  sort_every
    sets how often they re-order (0 = every 16 steps).  eps2 must be >= 1e-24
    in mixed precision."""

    def __init__(self, n: int, eps2: float = 1e-7, precision: str = "fp64", device: int = 0,
                 dt: float | None = None, eta: float = 1e-2, eta0: float = 1e-4,
                 tune: bool = False, threads: int = 0, i_per_thread: int = 0, j_tile: int = 0,
                 split_j: int = 0, pair_variant: int = 0, sort_every: int = 0,
                 j_cluster: int = 0):
        L = _lib.load()
        cfg = NBodyConfig()
        check(L.nbody_config_init(C.byref(cfg)), "nbody_config_init")
        cfg.n = int(n)
        cfg.eps2 = float(eps2)
        cfg.precision = PRECISIONS[precision]
        cfg.device = int(device)
        cfg.dt = float(dt) if dt is not None else 0.0
        cfg.eta = float(eta)
        cfg.eta0 = float(eta0)
        cfg.tune = int(bool(tune))
        cfg.threads, cfg.i_per_thread, cfg.j_tile, cfg.split_j = threads, i_per_thread, j_tile, split_j
        cfg.pair_variant = pair_variant
        cfg.sort_every = sort_every
        cfg.j_cluster = j_cluster
        h = C.c_void_p()
        check(L.nbody_create(C.byref(h), C.byref(cfg)), "nbody_create")
        self._h = h
        self._L = L
        self.n = int(n)
        self.eps2 = float(eps2)
        self.precision = precision
        self.device = int(device)
        self.fixed_dt = dt

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.nbody_destroy(self._h)
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

    @property
    def handle(self):
        return self._h

    # -- state --------------------------------------------------------------
    def set_state(self, state: dict) -> None:
        arrs = [_arr(state[k], self.n) for k in FIELDS]
        check(self._L.nbody_set_state(self._h, *map(_ptr, arrs)), "nbody_set_state")

    def get_state(self) -> dict:
        out = {k: np.empty(self.n) for k in ("x", "y", "z", "vx", "vy", "vz")}
        check(self._L.nbody_get_state(self._h, *[_ptr(out[k]) for k in ("x", "y", "z", "vx", "vy", "vz")]),
              "nbody_get_state")
        return out

    def get_derivs(self) -> np.ndarray:
        d = np.empty((6, self.n))
        check(self._L.nbody_get_derivs(self._h, *[_ptr(d[k]) for k in range(6)]), "nbody_get_derivs")
        return d

    # -- the reference's NBody phases -----------------------------------------
    def force_calculation(self) -> None:
        """acc + jerk of the current state (and initialdt in adaptive mode)."""
        check(self._L.nbody_acc_jerk(self._h), "nbody_acc_jerk")

    def prediction(self) -> None:
        check(self._L.nbody_predict(self._h), "nbody_predict")

    def eval_predicted(self) -> None:
        check(self._L.nbody_eval_predicted(self._h), "nbody_eval_predicted")

    def correction(self) -> None:
        """snapandcrackle + correction + derivative swap (+ updatedt)."""
        check(self._L.nbody_correct(self._h), "nbody_correct")

    def timestepping(self, nsteps: int = 1) -> None:
        """nsteps full Hermite steps from the captured step graph (async)."""
        check(self._L.nbody_step(self._h, int(nsteps)), "nbody_step")

    def synchronize(self) -> None:
        check(self._L.nbody_synchronize(self._h), "nbody_synchronize")

    def cycle(self, state: dict, ncycle: int, ref_compat: bool = False) -> dict:
        """The reference's run (NBody::cycle, src/nbody.cpp:291-380): upload
        the bodies, first force evaluation (and initial dt when adaptive),
        E0, ncycle steps with per-phase timers, final energy; returns the
        reference's reported quantities (initE, finE, Q, Err and the per-cycle
        PRED / EVAL / CORR seconds)."""
        self.set_state(state)
        self.force_calculation()
        T0, U0 = self.energy(ref_compat)
        pred, ev, corr = [], [], []
        for _ in range(int(ncycle)):
            self.timestepping(1)
            t = self.timers()
            pred.append(t["pred_ms"] * 1e-3)
            ev.append(t["eval_ms"] * 1e-3)
            corr.append(t["corr_ms"] * 1e-3)
        T1, U1 = self.energy(ref_compat)
        e0, e1 = T0 + U0, T1 + U1
        return {"initE": e0, "finE": e1, "Q": -2.0 * T1 / U1, "Err": abs(e1 - e0) / abs(e0),
                "t_predv": pred, "t_evalv": ev, "t_corrv": corr,
                "t_eval_init": self.timers()["eval_init_ms"] * 1e-3}

    def energy(self, ref_compat: bool = False) -> tuple[float, float]:
        T, U = C.c_double(), C.c_double()
        check(self._L.nbody_energy(self._h, int(ref_compat), C.byref(T), C.byref(U)), "nbody_energy")
        return T.value, U.value

    def timers(self) -> dict:
        t = NBodyTimers()
        check(self._L.nbody_get_timers(self._h, C.byref(t)), "nbody_get_timers")
        return {name: getattr(t, name) for name, _ in NBodyTimers._fields_}

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(self._L.nbody_get_stream(self._h, C.byref(s)), "nbody_get_stream")
        return s.value or 0

    def acc_jerk_device(self, x, y, z, m, vx, vy, vz, out6, stream: int = 0) -> None:
        """Device-pointer entry: inputs/outputs are CUDA float64 tensors (or
        raw device addresses); ordered on `stream` (0 = engine stream)."""
        def p(t):
            return C.c_void_p(t if isinstance(t, int) else t.data_ptr())
        n = x.numel() if hasattr(x, "numel") else self.n
        check(self._L.nbody_acc_jerk_device(self._h, int(n), *map(p, (x, y, z, m, vx, vy, vz)),
                                            *map(p, out6), C.c_void_p(stream)),
              "nbody_acc_jerk_device")


def force_calculation(state: dict, eps2: float = 1e-7, precision: str = "fp64", i_begin: int = 0,
                      i_end: int | None = None) -> np.ndarray:
    """The drop-in for the reference's force_calculation (include/kernel.h:15-19):
    host arrays in, (6, n) acc/jerk out, rows outside [i_begin, i_end) zero."""
    L = _lib.load()
    arrs = [_arr(state[k]) for k in FIELDS]
    n = arrs[0].size
    i_end = n if i_end is None else i_end
    out = np.empty((6, n))
    check(L.nbody_force_calculation(n, float(eps2), PRECISIONS[precision], int(i_begin), int(i_end),
                                    *map(_ptr, arrs), *[_ptr(out[k]) for k in range(6)]),
          "nbody_force_calculation")
    return out


def force_calculation_tune(state: dict, eps2: float = 1e-7, precision: str = "fp64") -> None:
    """Autotune the drop-in's tiling for full-row calls on these bodies
    (nbody_force_calculation_tune); later force_calculation calls of this size
    and precision on this thread's device use it."""
    L = _lib.load()
    arrs = [_arr(state[k]) for k in FIELDS]
    check(L.nbody_force_calculation_tune(arrs[0].size, float(eps2), PRECISIONS[precision],
                                         *map(_ptr, arrs)), "nbody_force_calculation_tune")


def release_force_cache() -> None:
    check(_lib.load().nbody_force_calculation_release(), "nbody_force_calculation_release")


def plummer(n: int, seed: int) -> dict:
    """Plummer sphere in Henon units (G = M = 1, E = -1/4), masses 1/n."""
    out = {k: np.empty(n) for k in FIELDS}
    check(_lib.load().nbody_plummer(int(n), int(seed), *[_ptr(out[k]) for k in FIELDS]), "nbody_plummer")
    return out


def reference_ic(n: int, eps2: float = 1e-7) -> dict:
    """The reference's own initial conditions (src/nbody.cpp:69-114)."""
    out = {k: np.empty(n) for k in FIELDS}
    check(_lib.load().nbody_reference_ic(int(n), float(eps2), *[_ptr(out[k]) for k in FIELDS]),
          "nbody_reference_ic")
    return out


def measure_peaks(device: int = 0) -> dict:
    p = NBodyPeaks()
    check(_lib.load().nbody_measure_peaks(int(device), C.byref(p)), "nbody_measure_peaks")
    return {name: getattr(p, name) for name, _ in NBodyPeaks._fields_}
