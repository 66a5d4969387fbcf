"""Generates the golden fixtures in tests/golden/ from the UNMODIFIED reference.

The reference has no tests or fixtures of its own, so every golden vector
here is an output of the reference's own CPU code, compiled from its sources
by oracle/Makefile into oracle/_ref/ (FP64 build and the -D_F32 build) and
driven through oracle/ref_harness.cpp.  Run in a container that has the
reference tree:

    make -C oracle all REF=<reference tree> && OMP_NUM_THREADS=1 python tests/golden/make_golden.py

One thread makes the reference's OpenMP reductions sum in index order, so
the fixtures are reproducible bit for bit.

Per N in SIZES, ``ref_ic_n{N}.npz`` holds
    x y z m vx vy vz     NBody::initialize() bodies (src/nbody.cpp:69-114)
    force_fp64 (6, N)    force_calculation, FP64 build (src/kernel.cpp:1164-1224)
    force_f32  (6, N)    force_calculation, _F32 build (src/kernel.cpp:1101-1163)
    h_x ... h_vz, h_derivs (6, N), h_dtcrit
                         10 fixed-dt Hermite steps (dt = DT) through the
                         reference's prediction / force / snapandcrackle /
                         correction / swap (src/nbody.cpp:152-196, 224-289)
    T, U_ref             compute_kinetic and compute_potential (src/utils.cpp:125-153)
and ``kat.json`` records the stock nbody_app's printed initial energy for
--N 1024 --Ncycle 10 (src/main.cpp:118-124).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

SIZES = (1, 2, 33, 127, 1024)
DT = 3.8e-5      # the reference's own post-first-step dt scale at N = 1024
NSTEPS = 10


def main() -> None:
    assert os.environ.get("OMP_NUM_THREADS") == "1", "run with OMP_NUM_THREADS=1"
    assert O.have_reference() and O.have_reference(f32=True), "build oracle/_ref first"
    assert O.ref().ref_eps2() == 1e-7
    for n in SIZES:
        s = O.ref_initialize(n)
        f64 = O.ref_force(s)
        f32 = O.ref_force(s, f32=True)
        hs, hd, hdt = O.ref_hermite_fixed(s, DT, NSTEPS)
        args = dict(s)
        args.update(force_fp64=f64, force_f32=f32, h_derivs=hd, h_dtcrit=np.float64(hdt))
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            args["h_" + k] = hs[k]
        lib = O.ref()
        P = O._p
        args["T"] = np.float64(lib.ref_kinetic(n, P(s["m"]), P(s["vx"]), P(s["vy"]), P(s["vz"])))
        args["U_ref"] = np.float64(lib.ref_potential(n, P(s["x"]), P(s["y"]), P(s["z"]), P(s["m"])))
        args["dt"] = np.float64(DT)
        args["nsteps"] = np.int64(NSTEPS)
        np.savez_compressed(os.path.join(HERE, f"ref_ic_n{n}.npz"), **args)
        print("wrote", n)
    out = subprocess.run([O.REF_APP, "--N", "1024", "--Ncycle", "10"], capture_output=True,
                         text=True, check=True, env=dict(os.environ, OMP_NUM_THREADS="1")).stdout
    e0 = next(float(line.split(":")[1]) for line in out.splitlines()
              if line.startswith("Initial Energy"))
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump({"nbody_app --N 1024 --Ncycle 10": {"initial_energy": e0,
                                                      "printed_digits": 9}}, f, indent=1)
    print("E0", e0)


if __name__ == "__main__":
    main()
