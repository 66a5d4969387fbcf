"""ctypes view of libnbody_cuda.so (include/nbody_cuda.h).

The library is built in-tree by ``n-body-code_b200/build.py``.  There is no
fallback: if the library is missing, loading raises, so no caller can end up
on a CPU path by accident.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)                      # n-body-code_b200/
REPO_DIR = os.path.dirname(ROOT_DIR)
LIB_PATH = os.path.join(ROOT_DIR, "lib", "libnbody_cuda.so")
HEADER = os.path.join(REPO_DIR, "include", "nbody_cuda.h")

NBODY_FP64 = 0
NBODY_MIXED = 1

STATUS = {
    0: "NBODY_OK",
    1: "NBODY_ERR_INVALID_ARG",
    2: "NBODY_ERR_OOM",
    3: "NBODY_ERR_CUDA",
    4: "NBODY_ERR_TIMEOUT",
    5: "NBODY_ERR_NONFINITE",
    6: "NBODY_ERR_NO_DEVICE",
    7: "NBODY_ERR_STATE",
}


class NBodyConfig(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("eps2", C.c_double),
        ("precision", C.c_int),
        ("device", C.c_int),
        ("dt", C.c_double),
        ("eta", C.c_double),
        ("eta0", C.c_double),
        ("tune", C.c_int),
        ("threads", C.c_int),
        ("i_per_thread", C.c_int),
        ("j_tile", C.c_int),
        ("split_j", C.c_int),
        ("pair_variant", C.c_int),
        ("sort_every", C.c_int),
        ("j_cluster", C.c_int),
    ]


class NBodyTimers(C.Structure):
    _fields_ = [
        ("pred_ms", C.c_double),
        ("eval_ms", C.c_double),
        ("corr_ms", C.c_double),
        ("eval_init_ms", C.c_double),
        ("num_sms", C.c_int),
        ("threads", C.c_int),
        ("i_per_thread", C.c_int),
        ("j_tile", C.c_int),
        ("split_j", C.c_int),
        ("steps", C.c_longlong),
        ("t", C.c_double),
        ("dt", C.c_double),
        ("record_format", C.c_int),
        ("step_kernels", C.c_int),
        ("reorders", C.c_longlong),
        ("order_kernels", C.c_int),
        ("dt_crit", C.c_double),
        ("tiling_source", C.c_int),
        ("near_tile_fraction", C.c_double),
        ("j_cluster", C.c_int),
    ]


class NBodyPeaks(C.Structure):
    _fields_ = [
        ("fp64_tflops", C.c_double),
        ("fp32_tflops", C.c_double),
        ("fp32x2_tflops", C.c_double),
        ("mufu_rsqrt_gops", C.c_double),
        ("sm_clock_mhz", C.c_double),
    ]


_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
_eng = C.c_void_p

# name -> (argtypes); every function returns nbody_status (int) unless listed in _RESTYPE
_SIGS = {
    "nbody_config_init": [C.POINTER(NBodyConfig)],
    "nbody_create": [C.POINTER(_eng), C.POINTER(NBodyConfig)],
    "nbody_destroy": [_eng],
    "nbody_set_state": [_eng] + [_vp] * 7,
    "nbody_get_state": [_eng] + [_vp] * 6,
    "nbody_get_derivs": [_eng] + [_vp] * 6,
    "nbody_acc_jerk": [_eng],
    "nbody_predict": [_eng],
    "nbody_eval_predicted": [_eng],
    "nbody_correct": [_eng],
    "nbody_step": [_eng, C.c_int],
    "nbody_synchronize": [_eng],
    "nbody_energy": [_eng, C.c_int, _dp, _dp],
    "nbody_get_timers": [_eng, C.POINTER(NBodyTimers)],
    "nbody_get_stream": [_eng, C.POINTER(_vp)],
    "nbody_last_error": [],
    "nbody_status_string": [C.c_int],
    "nbody_force_calculation": [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int] + [_vp] * 13,
    "nbody_force_calculation_release": [],
    "nbody_force_calculation_tune": [C.c_int, C.c_double, C.c_int] + [_vp] * 7,
    "nbody_acc_jerk_device": [_eng, C.c_int] + [_vp] * 13 + [_vp],
    "nbody_plummer": [C.c_int, C.c_uint64] + [_vp] * 7,
    "nbody_reference_ic": [C.c_int, C.c_double] + [_vp] * 7,
    "nbody_measure_peaks": [C.c_int, C.POINTER(NBodyPeaks)],
}
_RESTYPE = {"nbody_last_error": C.c_char_p, "nbody_status_string": C.c_char_p}
# Entry points declared in the header beyond the ones above are bound by
# their own modules (ensemble, adjoint) through `bind`.

_lib = None


def header_functions() -> list[str]:
    """Function names declared in include/nbody_cuda.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(nbody_[a-z0-9_]+)\s*\(", txt)))


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is not built; run `python n-body-code_b200/build.py` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, C.c_int)
        _lib = L
    return _lib


def bind(name: str, argtypes, restype=C.c_int):
    f = getattr(load(), name)
    f.argtypes = argtypes
    f.restype = restype
    return f


class NBodyError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        self.name = STATUS.get(status, str(status))
        msg = load().nbody_last_error().decode(errors="replace")
        super().__init__(f"{where}: {self.name}: {msg}")


def check(status: int, where: str) -> None:
    if status != 0:
        raise NBodyError(status, where)
