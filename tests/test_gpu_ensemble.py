"""Batched ensembles: every cluster of one persistent launch must equal the
same cluster run alone (the single-system engine and the oracle)."""
import numpy as np
import pytest

import nbody_b200 as nb
import oracle as O
from _util import derivs_rel, pos_of, vec_rel, vel_of

pytestmark = pytest.mark.gpu


def split(state, offsets, c):
    a, b = offsets[c], offsets[c + 1]
    return {k: np.ascontiguousarray(state[k][a:b]) for k in state}


@pytest.fixture(scope="module")
def small_ensemble():
    sizes = np.array([1, 256, 300, 37, 1024, 513, 2000, 257], dtype=np.int32)
    parts = [nb.plummer(int(n), 100 + c) for c, n in enumerate(sizes)]
    state = {k: np.concatenate([p[k] for p in parts]) for k in nb.FIELDS}
    eps2 = (4.0 / sizes.astype(float)) ** 2
    return sizes, eps2, state


@pytest.mark.parametrize("tpi", [1, 2, 8, 64])
def test_ensemble_fp64_forces_vs_oracle(small_ensemble, tpi):
    sizes, eps2, state = small_ensemble
    with nb.Ensemble(sizes, eps2, 1 / 512, precision="fp64", tiles_per_item=tpi) as e:
        e.set_state(state)
        e.force_calculation()
        d = e.get_derivs()
        off = e.offsets
    for c, n in enumerate(sizes):
        got = d[:, off[c]:off[c + 1]]
        ref = O.force(split(state, off, c), eps2[c])
        if n == 1:
            assert np.all(got == 0)
            continue
        ea, ej = derivs_rel(got, ref)
        assert ea <= 1e-12 and ej <= 1e-12, (c, n, ea, ej)


def test_ensemble_mixed_matches_single_engine(small_ensemble):
    """Packed hi/lo kernels (pair_variant 3): the same pair arithmetic as the
    single-system engine's, so agreement to the reordering of split sums."""
    sizes, eps2, state = small_ensemble
    with nb.Ensemble(sizes, eps2, 1 / 512, precision="mixed", tiles_per_item=4, pair_variant=3) as e:
        e.set_state(state)
        e.force_calculation()
        d = e.get_derivs()
        off = e.offsets
    for c, n in enumerate(sizes):
        if n == 1:
            continue
        s = split(state, off, c)
        with nb.Engine(int(n), eps2=eps2[c], precision="mixed", dt=1.0, pair_variant=3) as single:
            single.set_state(s)
            single.force_calculation()
            ref = single.get_derivs()
        ea, ej = derivs_rel(d[:, off[c]:off[c + 1]], ref)
        assert ea <= 1e-9 and ej <= 1e-9, (c, n, ea, ej)   # same pair arithmetic, split sums reordered


def test_ensemble_hermite_steps_vs_single_engines(small_ensemble):
    sizes, eps2, state = small_ensemble
    steps = 16
    with nb.Ensemble(sizes, eps2, 1 / 512, precision="fp64") as e:
        e.set_state(state)
        e.timestepping(steps)
        got = e.get_state()
        T, U = e.energy()
        info = e.info()
        off = e.offsets
    assert info["steps"] == steps and info["items"] > 0
    for c, n in enumerate(sizes):
        s = split(state, off, c)
        ref_s, _, _ = O.hermite_fixed(s, eps2[c], 1 / 512, steps)
        g = {k: got[k][off[c]:off[c + 1]] for k in got}
        assert vec_rel(pos_of(g), pos_of(ref_s)).max() <= 1e-10, c
        assert vec_rel(vel_of(g), vel_of(ref_s)).max() <= 1e-9, c
        Uref = O.potential(ref_s | {"m": s["m"]}, eps2[c]) if n > 1 else 0.0
        Tref = O.kinetic(ref_s | {"m": s["m"]})
        assert abs(T[c] - Tref) <= 1e-12 * max(abs(Tref), 1e-300) + 1e-300
        assert abs(U[c] - Uref) <= 1e-11 * max(abs(Uref), 1e-300) + 1e-300


@pytest.mark.parametrize("variant", [0, 4])
def test_ensemble_deterministic(small_ensemble, variant):
    sizes, eps2, state = small_ensemble
    outs = []
    for _ in range(2):
        with nb.Ensemble(sizes, eps2, 1 / 512, precision="mixed", pair_variant=variant) as e:
            e.set_state(state)
            e.timestepping(4)
            outs.append(e.get_state())
            assert e.info()["record_format"] == (3 if variant == 4 else 2)
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_plummer_ensemble_config():
    """Plummer clusters with N log-uniform in [256, 8192]: the mixed path's energy error stays within 2x
    of the FP64 path's on the same run (at eps = 4/N and dt = 1/512 the
    integration error itself is large for the biggest clusters)."""
    sizes, eps2, state = nb.plummer_ensemble(64, seed=3)
    assert sizes.min() >= 256 and sizes.max() <= 8192
    assert state["x"].size == sizes.sum()
    de = {}
    for prec in ("fp64", "mixed"):
        with nb.Ensemble(sizes, eps2, 1 / 512, precision=prec, tune=(prec == "mixed")) as e:
            e.set_state(state)
            T0, U0 = e.energy()
            e.timestepping(8)
            T1, U1 = e.energy()
            info = e.info()
        de[prec] = np.abs((T1 + U1) - (T0 + U0)) / np.abs(T0 + U0)
    assert np.all(np.isfinite(de["mixed"]))
    assert np.all(de["mixed"] <= 2.0 * de["fp64"] + 1e-9), np.max(de["mixed"] / (de["fp64"] + 1e-12))
    assert info["tiles_per_item"] * info["j_tile"] in (256, 512, 1024, 2048, 4096, 8192)


@pytest.mark.parametrize("tpi", [1, 4, 64])
def test_ensemble_tile_relative_vs_oracle(small_ensemble, tpi):
    """Near/far tile-relative ensemble (pair_variant 4): per cluster against
    the FP64 oracle within the mixed bounds, and within 3x of the hi/lo
    ensemble's median and worst error (near tiles form separations in
    double-single)."""
    sizes, eps2, state = small_ensemble
    d = {}
    for name, kw in (("rel", dict(pair_variant=4)), ("hilo", {})):
        with nb.Ensemble(sizes, eps2, 1 / 512, precision="mixed", tiles_per_item=tpi, **kw) as e:
            e.set_state(state)
            e.force_calculation()
            d[name] = e.get_derivs()
            off = e.offsets
            info = e.info()
            if name == "rel":
                assert info["record_format"] == 3
    for c, n in enumerate(sizes):
        rel = d["rel"][:, off[c]:off[c + 1]]
        assert np.all(np.isfinite(rel))
        if n == 1:
            assert np.all(rel == 0)
            continue
        ref = O.force(split(state, off, c), eps2[c])
        er = vec_rel(rel[:3], ref[:3])
        eh = vec_rel(d["hilo"][:3, off[c]:off[c + 1]], ref[:3])
        assert np.median(er) <= 2e-6 and er.max() <= 2e-4, (c, n, np.median(er), er.max())
        assert np.median(er) <= 3 * np.median(eh) + 1e-8, (c, n, np.median(er), np.median(eh))
        assert er.max() <= 3 * eh.max() + 1e-8, (c, n, er.max(), eh.max())


def test_ensemble_tile_relative_steps_vs_fp64(small_ensemble):
    """16 steps with the order refreshed every step and every 16 steps: every
    cluster stays within mixed-precision distance of the FP64 ensemble."""
    sizes, eps2, state = small_ensemble
    runs = {}
    for name, prec, kw in (("fp64", "fp64", {}), ("rel1", "mixed", dict(sort_every=1, pair_variant=4)),
                           ("rel", "mixed", dict(pair_variant=4))):
        with nb.Ensemble(sizes, eps2, 1 / 512, precision=prec, **kw) as e:
            e.set_state(state)
            e.timestepping(16)
            runs[name] = e.get_state()
            info = e.info()
            if name == "rel1":
                # the first step uses the order made with the initial forces
                assert info["reorders"] == 15 and info["order_kernels"] >= 3
    for name in ("rel1", "rel"):
        dx = max(np.abs(runs[name][k] - runs["fp64"][k]).max() for k in ("x", "y", "z"))
        assert dx <= 1e-7, (name, dx)
