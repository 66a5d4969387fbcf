"""The oracle against the reference (CPU only).

Pins the C++ restatement (oracle/nbody_oracle.cpp) to the reference's own
outputs: bit-for-bit against the committed golden fixtures (generated from
the unmodified reference build by tests/golden/make_golden.py) and, where the
reference build exists in this checkout (oracle/_ref), against fresh
reference calls on inputs the fixtures do not cover.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from _util import GOLDEN, GOLDEN_SIZES, golden, state_of

EPS2_REF = 1e-7  # the reference's compile-time EPS2 (include/kernel.h:13)


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


@pytest.mark.parametrize("n", GOLDEN_SIZES)
def test_initialize_matches_reference(n):
    g = golden(n)
    s = O.initialize(n, EPS2_REF)
    for k in ("x", "y", "z", "m", "vx", "vy", "vz"):
        assert same(s[k], g[k]), k


@pytest.mark.parametrize("n", GOLDEN_SIZES)
def test_force_fp64_bitwise(n):
    g = golden(n)
    assert same(O.force(state_of(g), EPS2_REF), g["force_fp64"])


@pytest.mark.parametrize("n", GOLDEN_SIZES)
def test_force_f32_bitwise(n):
    g = golden(n)
    assert same(O.force(state_of(g), EPS2_REF, "f32"), g["force_f32"])


@pytest.mark.parametrize("n", GOLDEN_SIZES)
def test_hermite_fixed_bitwise(n):
    g = golden(n)
    s, d, dtc = O.hermite_fixed(state_of(g), EPS2_REF, float(g["dt"]), int(g["nsteps"]))
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert same(s[k], g["h_" + k]), k
    assert same(d, g["h_derivs"])
    assert same(dtc, g["h_dtcrit"])


@pytest.mark.parametrize("n", GOLDEN_SIZES)
def test_energies_bitwise(n):
    g = golden(n)
    s = state_of(g)
    assert same(O.kinetic(s), g["T"])
    assert same(O.potential(s, EPS2_REF, compat=True), g["U_ref"])


def test_initial_energy_known_answer():
    """E0 printed by the stock nbody_app --N 1024 --Ncycle 10 (src/main.cpp:120)
    equals T + U of the initial bodies after the first force evaluation."""
    with open(os.path.join(GOLDEN, "kat.json")) as f:
        e0 = json.load(f)["nbody_app --N 1024 --Ncycle 10"]["initial_energy"]
    s = state_of(golden(1024))
    e = O.kinetic(s) + O.potential(s, EPS2_REF, compat=True)
    assert abs(e - e0) < 5e-10  # printed with 9 decimals


def test_invsqrt2d_accuracy():
    x = np.geomspace(1e-12, 1e12, 2001)
    y = np.array([O.invsqrt2d(v) for v in x])
    assert np.max(np.abs(y * np.sqrt(x) - 1.0)) < 4e-16


def test_rows_and_symmetric_loop_agree():
    """The direct row sum (large-N checker) vs the symmetric loop."""
    g = golden(1024)
    s = state_of(g)
    rows = np.arange(0, 1024, 7)
    d = O.force_rows(s, EPS2_REF, rows)
    ref = g["force_fp64"][:, rows]
    for blk in (slice(0, 3), slice(3, 6)):
        num = np.sqrt(((d[blk] - ref[blk]) ** 2).sum(0))
        den = np.sqrt((ref[blk] ** 2).sum(0))
        assert (num / den).max() < 1e-12


def test_potential_rows_consistent():
    g = golden(127)
    s = state_of(g)
    phi = O.potential_rows(s, EPS2_REF, np.arange(127))
    u = 0.5 * np.sum(s["m"] * phi)
    assert abs(u - O.potential(s, EPS2_REF, compat=False)) < 1e-12 * abs(u)


def test_updatedt_initialdt_match_hermite():
    g = golden(33)
    s = state_of(g)
    d0 = O.force(s, EPS2_REF)
    dt = float(g["dt"])
    p = O.predict(s, d0, dt)
    d1 = O.force(p, EPS2_REF)
    a2, a3 = O.snapcrackle(d0, d1, dt)
    _, _, dtc = O.hermite_fixed(s, EPS2_REF, dt, 1)
    assert O.updatedt(d0, a2, a3) == dtc
    assert O.initialdt(d0) > 0


@pytest.mark.skipif(not O.have_reference(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("n", (3, 64, 300))
def test_restatement_vs_reference_build(n, monkeypatch):
    """Fresh reference calls on other sizes (one thread: index-order sums)."""
    O.ref().ref_set_threads(1)
    O.ref(f32=True).ref_set_threads(1)
    s = O.ref_initialize(n)
    assert same(O.force(s, EPS2_REF), O.ref_force(s))
    assert same(O.force(s, EPS2_REF, "f32"), O.ref_force(s, f32=True))
    rs, rd, rdt = O.ref_hermite_fixed(s, 2.5e-5, 3)
    os_, od, odt = O.hermite_fixed(s, EPS2_REF, 2.5e-5, 3)
    assert all(same(rs[k], os_[k]) for k in rs) and same(rd, od) and rdt == odt


@pytest.mark.parametrize("n,seed", [(1, 1), (1000, 2), (65536, 1)])
def test_oracle_plummer_equals_engine_plummer(n, seed):
    """The CPU legs of the benchmark build their Plummer bodies with the
    oracle's own sampler (oracle/plummer.cpp) so that they load no product
    library; it must give the engine's nbody_plummer bodies value for value
    (the library's host-side generator needs no GPU)."""
    import nbody_b200 as nb
    want = nb.plummer(n, seed)
    got = O.plummer(n, seed)
    for k in ("x", "y", "z", "m", "vx", "vy", "vz"):
        assert same(got[k], want[k]), k
    if O.have_reference():
        got = O.plummer(n, seed, from_reference_build=True)
        for k in ("x", "y", "z", "m", "vx", "vy", "vz"):
            assert same(got[k], want[k]), k


@pytest.mark.parametrize("n", (33, 1024))
def test_f32_rows_equal_symmetric_f32_loop(n):
    """The row-wise _F32 sum (large-N accuracy floor) gives the symmetric
    _F32 loop's result up to the order of its double accumulation."""
    g = golden(n)
    s = state_of(g)
    rows = np.arange(n)
    d = O.force_rows(s, EPS2_REF, rows, "f32")
    ref = g["force_f32"]
    for blk in (slice(0, 3), slice(3, 6)):
        num = np.sqrt(((d[blk] - ref[blk]) ** 2).sum(0))
        den = np.sqrt((ref[blk] ** 2).sum(0))
        assert (num / den).max() < 1e-13
