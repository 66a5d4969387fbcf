"""The reference's own driver and integrator on the engine's force back end.

oracle/_ref/nbody_app_gpu is the reference's src/main.cpp + src/nbody.cpp +
src/utils.cpp linked with n-body-code_b200/host/force_calculation_shim.cpp
instead of src/kernel.cpp (oracle/Makefile target ref_gpu).  Its stock run
(reference initial conditions, adaptive dt, 10 cycles) must print the same
initial energy as the CPU build and an energy error of the same size: the
adaptive dt is seeded by rounding noise (a2/a3 are finite differences over
dt0 ~ 4e-8), so individual trajectories agree only at that noise level.
"""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APP_GPU = os.path.join(ROOT, "oracle", "_ref", "nbody_app_gpu")
APP_CPU = os.path.join(ROOT, "oracle", "_ref", "nbody_app")


def run(app, n, ncycle):
    out = subprocess.run([app, "--N", str(n), "--Ncycle", str(ncycle)], capture_output=True,
                         text=True, timeout=300, check=True,
                         env=dict(os.environ, OMP_NUM_THREADS="1")).stdout
    def grab(key):
        return float(re.search(rf"{key}\s*[:=]\s*(\S+)", out).group(1))
    return grab("Initial Energy"), grab("Final Energy"), grab("Err")


@pytest.mark.skipif(not (os.path.exists(APP_GPU) and os.path.exists(APP_CPU)),
                    reason="reference builds (make -C oracle ref ref_gpu) not present")
def test_reference_driver_on_gpu_backend():
    e0g, efg, errg = run(APP_GPU, 1024, 10)
    e0c, efc, errc = run(APP_CPU, 1024, 10)
    assert e0g == e0c == -637.954412621
    assert abs(efg - efc) <= 1e-3 * abs(efc)
    assert 0.5 < errg / errc < 2.0
