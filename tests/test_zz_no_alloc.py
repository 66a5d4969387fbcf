"""nbody_acc_jerk_noalloc: the entry point for callers that must not allocate
device memory (an application that keeps the whole device memory budget in
its own pool, a real-time loop where cudaMalloc/cudaFree would stall the
device).  It must give the same acc and jerk as nbody_acc_jerk_device, the
existing device-pointer entry point, without an engine and without any
allocation: its scratch is a fixed 16 MiB static array in the library, so it
serves at most 32768 bodies.

The file name sorts last so that a run that stops at the first failure has
run every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

import nbody_b200 as nb
from nbody_b200 import _lib
from _util import derivs_rel

MAX_BODIES = 32768
TOL = 1e-12  # the FP64 per-body tolerance of the parity tests


def _noalloc():
    return _lib.bind("nbody_acc_jerk_noalloc",
                     [C.c_int, C.c_double, C.c_int] + [C.c_void_p] * 13 + [C.c_void_p])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    f = _noalloc()
    z = C.c_void_p(16)  # never dereferenced: the size check comes first
    assert f(MAX_BODIES + 1, 1e-4, 0, *([z] * 13), None) == 1  # NBODY_ERR_INVALID_ARG
    msg = nb.load().nbody_last_error().decode()
    assert "32768" in msg and "scratch" in msg
    assert f(0, 1e-4, 0, *([z] * 13), None) == 1
    # mixed precision: the float self-pair factor m eps2^-1.5 must stay finite
    assert f(100, 1e-26, 1, *([z] * 13), None) == 1
    assert "mixed" in nb.load().nbody_last_error().decode()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_device_entry_on_two_calls(precision):
    import torch
    f = _noalloc()
    prec = 0 if precision == "fp64" else 1
    eps2 = 1e-4
    stream = torch.cuda.current_stream()
    # two calls in a row on different systems: the second must not see the
    # first one's leftovers in the shared scratch
    for n, seed in ((5000, 21), (MAX_BODIES, 22)):
        s = nb.plummer(n, seed)
        t = [torch.tensor(s[k], dtype=torch.float64, device="cuda") for k in nb.FIELDS]
        ref = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(6)]
        out = [torch.full((n,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(6)]
        # the no-alloc mixed path runs the packed hi/lo kernel with register
        # accumulators: compare with the engine on that kernel (pair_variant 2)
        with nb.Engine(n, eps2=eps2, precision=precision, dt=1.0,
                       pair_variant=2 if precision == "mixed" else 0) as e:
            e.acc_jerk_device(*t, ref, stream=stream.cuda_stream)
            torch.cuda.synchronize()
        st = f(n, eps2, prec, *[C.c_void_p(x.data_ptr()) for x in t],
               *[C.c_void_p(x.data_ptr()) for x in out], C.c_void_p(stream.cuda_stream))
        assert st == 0, nb.load().nbody_last_error()
        torch.cuda.synchronize()
        got = torch.stack(out).cpu().numpy()
        want = torch.stack(ref).cpu().numpy()
        assert np.all(np.isfinite(got))
        ea, ej = derivs_rel(got, want)
        assert ea <= TOL and ej <= TOL, (n, precision, ea, ej)
