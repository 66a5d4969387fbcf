"""The C++ driver nbody_app (the reference's --N / --Ncycle CLI) on the GPU."""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APP = os.path.join(ROOT, "n-body-code_b200", "lib", "nbody_app")
REF_APP = os.path.join(ROOT, "oracle", "_ref", "nbody_app")


def run(*args):
    out = subprocess.run([APP, *map(str, args)], capture_output=True, text=True, timeout=300,
                         check=True).stdout
    vals = {}
    for key in ("Initial Energy", "Final Energy", "Q", "Err"):
        vals[key] = float(re.search(rf"^{key}\s*[:=]\s*(\S+)", out, re.M).group(1))
    rows = [line.split() for line in out.splitlines() if re.match(r"^\s+\d+\s+1\s+\d", line)]
    return vals, rows, out


def test_reference_run_known_answer():
    """nbody_app --N 1024 --Ncycle 10 prints the reference's E0 (a known
    answer of the stock CPU build) and an energy error of the same size (the
    adaptive dt is noise-seeded, so runs agree only in scale)."""
    vals, rows, out = run("--N", 1024, "--Ncycle", 10)
    assert vals["Initial Energy"] == -637.954412621
    assert len(rows) == 10 and all(float(r[3]) > 0 for r in rows)
    assert 1e-4 < vals["Err"] < 1e-2
    if os.path.exists(REF_APP):
        ref = subprocess.run([REF_APP, "--N", "1024", "--Ncycle", "10"], capture_output=True,
                             text=True, timeout=300, check=True,
                             env=dict(os.environ, OMP_NUM_THREADS="1")).stdout
        err_ref = float(re.search(r"^Err\s*=\s*(\S+)", ref, re.M).group(1))
        assert 0.5 < vals["Err"] / err_ref < 2.0


def test_fixed_dt_plummer_and_state_files(tmp_path):
    """Fixed-dt Plummer run; --dump writes a state file that --load resumes."""
    a = tmp_path / "a.bin"
    b = tmp_path / "b.bin"
    vals, _, _ = run("--N", 4096, "--Ncycle", 32, "--ic", "plummer", "--seed", 4, "--eps", 0.01,
                     "--dt", 1 / 1024, "--precision", "mixed", "--dump", a)
    assert abs(vals["Initial Energy"] + 0.25) < 0.02       # Henon units
    assert vals["Err"] < 1e-6
    vals2, _, _ = run("--N", 4096, "--Ncycle", 4, "--eps", 0.01, "--dt", 1 / 1024, "--load", a,
                      "--dump", b, "--energy", "physical")
    assert abs(vals2["Initial Energy"] - vals["Final Energy"]) <= 1e-12 * abs(vals["Final Energy"])
    import sys
    sys.path.insert(0, os.path.join(ROOT, "n-body-code_b200"))
    hdr = np.fromfile(b, dtype=np.float64, count=8)
    assert abs(hdr[2] - 36 / 1024) < 1e-12   # model time continued across the restart


@pytest.mark.parametrize("variant", [3, 4])
def test_mixed_kernel_choice_from_the_cli(variant):
    """--pair-variant selects the mixed kernel (3 packed hi/lo, 4 tile-relative):
    both keep the fixed-dt energy error of a short Plummer run small."""
    vals, rows, _ = run("--N", 8192, "--Ncycle", 8, "--ic", "plummer", "--seed", 2, "--eps", 0.01,
                        "--dt", 1 / 1024, "--precision", "mixed", "--pair-variant", variant,
                        "--energy", "physical")
    assert len(rows) == 8
    assert vals["Err"] < 1e-7, vals
