"""The ctypes mirrors of the C-ABI structures match include/nbody_cuda.h:
a small C program built from the header (host compiler, no GPU) prints
every structure's size and each field's offset, and the Python side must
agree.  A field added on one side only shows up here, not as silent
corruption in a GPU run."""
import ctypes as C
import os
import subprocess

import pytest

from nbody_b200 import _lib
from nbody_b200.adjoint import AdjointConfig
from nbody_b200.ensemble import EnsembleConfig, EnsembleInfo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "_build")

MIRRORS = {
    "nbody_config": _lib.NBodyConfig,
    "nbody_timers": _lib.NBodyTimers,
    "nbody_peaks": _lib.NBodyPeaks,
    "nbody_ensemble_config": EnsembleConfig,
    "nbody_ensemble_info_t": EnsembleInfo,
    "nbody_adjoint_config": AdjointConfig,
}


@pytest.fixture(scope="module")
def c_layout():
    lines = ["#include <stddef.h>", "#include <stdio.h>", "#include <stdint.h>",
             '#include "nbody_cuda.h"', "int main(void) {"]
    for cname, py in MIRRORS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    os.makedirs(BUILD, exist_ok=True)
    src, exe = os.path.join(BUILD, "abi_layout.c"), os.path.join(BUILD, "abi_layout")
    with open(src, "w") as f:
        f.write("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", exe, src],
                   check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        cname, key, value = line.split()
        layout[(cname, key)] = int(value)
    return layout


@pytest.mark.parametrize("cname", list(MIRRORS))
def test_ctypes_mirror_matches_header(c_layout, cname):
    py = MIRRORS[cname]
    assert C.sizeof(py) == c_layout[(cname, "sizeof")], cname
    for field, _ in py._fields_:
        assert getattr(py, field).offset == c_layout[(cname, field)], (cname, field)
