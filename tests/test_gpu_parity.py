"""GPU parity: the sm_100a engine, called through its C-ABI, against the
reference's own outputs (golden fixtures) and the oracle.

Tolerances (per body, vector norms |a - a_ref| / |a_ref|):
  FP64 acc and jerk                 <= 1e-12
  FP64 positions after 10 steps     <= 1e-10  (velocities <= 1e-9)
  mixed acc                         median <= 2e-6, max <= 2e-4, and against
                                    the reference's own _F32 arithmetic on the
                                    same bodies: hi/lo within 4x (median, p99)
                                    and 12x (max), near/far tile-relative
                                    within 6x (median, p99) and 8x (max)
"""
import numpy as np
import pytest

import nbody_b200 as nb
import oracle as O
from _util import derivs_rel, golden, pos_of, state_of, vec_rel, vel_of

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_POS = 1e-10
TOL_VEL = 1e-9


def engine_derivs(state, eps2, precision="fp64", **kw):
    n = state["x"].size
    with nb.Engine(n, eps2=eps2, precision=precision, dt=1.0, **kw) as e:
        e.set_state(state)
        e.force_calculation()
        return e.get_derivs()


@pytest.mark.parametrize("n", (2, 33, 127, 1024))
def test_fp64_force_vs_reference_golden(n):
    g = golden(n)
    d = engine_derivs(state_of(g), 1e-7)
    ea, ej = derivs_rel(d, g["force_fp64"])
    assert ea <= TOL_FP64 and ej <= TOL_FP64, (ea, ej)


@pytest.mark.parametrize("n", (2, 33, 1024))
def test_dropin_force_calculation_vs_reference_golden(n):
    g = golden(n)
    d = nb.force_calculation(state_of(g), eps2=1e-7)
    ea, ej = derivs_rel(d, g["force_fp64"])
    assert ea <= TOL_FP64 and ej <= TOL_FP64, (ea, ej)


@pytest.mark.parametrize("n", (1, 31, 255, 257, 1023, 4096))
def test_fp64_force_vs_oracle_plummer(n):
    s = nb.plummer(n, seed=11)
    eps2 = 1e-4
    d = engine_derivs(s, eps2)
    ref = O.force(s, eps2)
    if n == 1:
        assert np.all(d == 0.0)  # a lone body feels nothing (self term is exactly zero)
        return
    ea, ej = derivs_rel(d, ref)
    assert ea <= TOL_FP64 and ej <= TOL_FP64, (ea, ej)


@pytest.mark.parametrize("tiling", [dict(threads=128, i_per_thread=1, j_tile=128, split_j=1),
                                    dict(threads=128, i_per_thread=4, j_tile=128, split_j=7),
                                    dict(threads=256, i_per_thread=2, j_tile=128, split_j=3),
                                    dict(threads=64, i_per_thread=2, j_tile=128, split_j=64),
                                    dict(threads=128, i_per_thread=2, j_tile=256, split_j=5)])
def test_fp64_every_tiling_agrees(tiling):
    s = nb.plummer(3000, seed=5)
    d = engine_derivs(s, 1e-4, **tiling)
    ea, ej = derivs_rel(d, O.force(s, 1e-4))
    assert ea <= TOL_FP64 and ej <= TOL_FP64, (tiling, ea, ej)


@pytest.mark.parametrize("tiling", [
    # packed hi/lo, FP64 accumulators in shared memory (variant 3)
    dict(threads=128, i_per_thread=4, j_tile=128, split_j=1, pair_variant=3),
    dict(threads=128, i_per_thread=2, j_tile=128, split_j=5, pair_variant=3),
    dict(threads=256, i_per_thread=2, j_tile=128, split_j=2, pair_variant=2),
    dict(threads=64, i_per_thread=4, j_tile=128, split_j=64, pair_variant=3),
    dict(threads=128, i_per_thread=4, j_tile=64, split_j=3, pair_variant=3),
    dict(threads=256, i_per_thread=4, j_tile=128, split_j=4, pair_variant=3),
    dict(threads=128, i_per_thread=2, j_tile=128, split_j=11, pair_variant=3),
    # scalar hi/lo (1), packed hi/lo with register accumulators (2)
    dict(threads=128, i_per_thread=4, j_tile=128, split_j=2, pair_variant=1),
    dict(threads=128, i_per_thread=4, j_tile=256, split_j=1, pair_variant=1),
    dict(threads=128, i_per_thread=4, j_tile=128, split_j=9, pair_variant=2),
    # tile-relative (4; the automatic choice from 16384 bodies)
    dict(threads=128, i_per_thread=4, j_tile=128, split_j=1, pair_variant=4),
    dict(threads=128, i_per_thread=2, j_tile=128, split_j=7, pair_variant=4),
    dict(threads=64, i_per_thread=4, j_tile=128, split_j=64, pair_variant=4),
    dict(threads=256, i_per_thread=2, j_tile=128, split_j=3, pair_variant=4),
    dict(threads=256, i_per_thread=4, j_tile=128, split_j=2, pair_variant=4),
    dict(threads=128, i_per_thread=2, j_tile=64, split_j=5, pair_variant=4),
    dict(threads=128, i_per_thread=4, j_tile=64, split_j=2, pair_variant=4),
    dict(threads=128, i_per_thread=2, j_tile=256, split_j=2, pair_variant=4),
    # automatic (0): packed hi/lo at this size
    dict(),
    dict(split_j=3)])
def test_mixed_every_kernel_agrees(tiling):
    """Tile-relative, packed hi/lo and scalar mixed kernels, every shape:
    same accuracy class."""
    s = nb.plummer(3000, seed=5)
    ref = O.force(s, 1e-4)
    d = engine_derivs(s, 1e-4, precision="mixed", **tiling)
    ea = vec_rel(d[:3], ref[:3])
    ej = vec_rel(d[3:], ref[3:])
    assert np.median(ea) <= 2e-6 and ea.max() <= 2e-4, (tiling, np.median(ea), ea.max())
    assert np.median(ej) <= 1e-5, (tiling, np.median(ej))


def test_dropin_row_range():
    s = nb.plummer(2000, seed=3)
    full = nb.force_calculation(s, eps2=1e-4)
    part = nb.force_calculation(s, eps2=1e-4, i_begin=300, i_end=1100)
    assert np.all(part[:, :300] == 0) and np.all(part[:, 1100:] == 0)
    ea, ej = derivs_rel(part[:, 300:1100], full[:, 300:1100])
    assert ea <= 1e-13 and ej <= 1e-13
    empty = nb.force_calculation(s, eps2=1e-4, i_begin=700, i_end=700)
    assert np.all(empty == 0)


@pytest.mark.parametrize("n", [3000, 40000])
def test_dropin_row_range_mixed(n):
    """Mixed drop-in: a row range gives the full call's rows.  At 3000 bodies
    both calls run the packed hi/lo kernel (only the split of the j-sum may
    differ); at 40000 the full call runs the near/far kernel on the bodies in
    Hilbert order and the row range the hi/lo kernel, so the two agree to the
    mixed kernels' accuracy, and both match the FP64 direct sums."""
    s = nb.plummer(n, seed=4)
    full = nb.force_calculation(s, eps2=1e-4, precision="mixed")
    part = nb.force_calculation(s, eps2=1e-4, precision="mixed", i_begin=1000, i_end=2100)
    assert np.all(part[:, :1000] == 0) and np.all(part[:, 2100:] == 0)
    ea, ej = derivs_rel(part[:, 1000:2100], full[:, 1000:2100])
    assert ea <= 2e-6 and ej <= 2e-5, (ea, ej)
    rows = np.arange(0, n, max(1, n // 300))
    ref = O.force_rows(s, 1e-4, rows)
    assert vec_rel(full[:3, rows], ref[:3]).max() <= 2e-6
    sub = rows[(rows >= 1000) & (rows < 2100)]
    assert vec_rel(part[:3, sub], O.force_rows(s, 1e-4, sub)[:3]).max() <= 2e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dropin_tune_keeps_results(precision):
    """nbody_force_calculation_tune: after the drop-in's autotuner has run for
    this size, full-row calls (tuned tiling) and row ranges keep the accuracy
    of the heuristic tiling against the oracle's direct sums."""
    n = 40000 if precision == "mixed" else 5000
    eps2 = 1e-4
    tol, tol_j = (TOL_FP64, TOL_FP64) if precision == "fp64" else (2e-6, 5e-5)
    s = nb.plummer(n, seed=6)
    rows = np.arange(0, n, max(1, n // 300))
    ref = O.force_rows(s, eps2, rows)
    nb.release_force_cache()
    try:
        before = nb.force_calculation(s, eps2=eps2, precision=precision)
        nb.force_calculation_tune(s, eps2=eps2, precision=precision)
        after = nb.force_calculation(s, eps2=eps2, precision=precision)
        part = nb.force_calculation(s, eps2=eps2, precision=precision, i_begin=100, i_end=900)
    finally:
        nb.release_force_cache()
    for d in (before, after):
        ea, ej = derivs_rel(d[:, rows], ref)
        assert ea <= tol and ej <= tol_j, (precision, ea, ej)
    assert np.all(part[:, :100] == 0) and np.all(part[:, 900:] == 0)
    ea, _ = derivs_rel(part[:, 100:900], after[:, 100:900])
    assert ea <= tol, ea


def test_fp64_deterministic():
    s = nb.plummer(5000, seed=9)
    a = engine_derivs(s, 1e-4)
    b = engine_derivs(s, 1e-4)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("n", (2, 33, 127, 1024))
def test_hermite_10_steps_vs_reference_golden(n):
    g = golden(n)
    dt, steps = float(g["dt"]), int(g["nsteps"])
    with nb.Engine(n, eps2=1e-7, dt=dt) as e:
        e.set_state(state_of(g))
        e.timestepping(steps)
        s = e.get_state()
        d = e.get_derivs()
        tm = e.timers()
    ref = {k: g["h_" + k] for k in ("x", "y", "z", "vx", "vy", "vz")}
    ep = vec_rel(pos_of(s), pos_of(ref)).max()
    ev = vec_rel(vel_of(s), vel_of(ref)).max()
    assert ep <= TOL_POS and ev <= TOL_VEL, (ep, ev)
    ea, ej = derivs_rel(d, g["h_derivs"])
    assert ea <= 1e-9 and ej <= 1e-8, (ea, ej)
    assert tm["steps"] == steps and abs(tm["t"] - steps * dt) < 1e-15


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("mixed", 3), ("mixed", 4)])
def test_phase_calls_equal_graph_steps(precision, variant):
    """prediction / eval / correction one at a time == the captured step graph
    (tile-relative: re-ordered every 2 steps on both paths)."""
    s = nb.plummer(1500, seed=4)
    kw = dict(eps2=1e-4, dt=1 / 1024, precision=precision, sort_every=2, pair_variant=variant)
    with nb.Engine(1500, **kw) as a, nb.Engine(1500, **kw) as b:
        a.set_state(s)
        b.set_state(s)
        a.timestepping(5)
        b.force_calculation()
        for _ in range(5):
            b.prediction()
            b.eval_predicted()
            b.correction()
        sa, sb = a.get_state(), b.get_state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k


def test_hermite_plummer_vs_oracle():
    s = nb.plummer(512, seed=1)
    eps2, dt, steps = 1e-4, 1 / 1024, 20
    ref_s, ref_d, _ = O.hermite_fixed(s, eps2, dt, steps)
    with nb.Engine(512, eps2=eps2, dt=dt) as e:
        e.set_state(s)
        e.timestepping(steps)
        got = e.get_state()
    assert vec_rel(pos_of(got), pos_of(ref_s)).max() <= TOL_POS
    assert vec_rel(vel_of(got), vel_of(ref_s)).max() <= TOL_VEL


def test_adaptive_dt_matches_reference_criteria():
    g = golden(1024)
    s = state_of(g)
    d0 = O.force(s, 1e-7)
    dt0 = O.initialdt(d0)
    with nb.Engine(1024, eps2=1e-7, dt=None) as e:
        e.set_state(s)
        e.force_calculation()
        t0 = e.timers()
        assert abs(t0["dt"] - dt0) <= 1e-10 * dt0
        e.timestepping(3)
        t3 = e.timers()
        st = e.get_state()
    assert t3["steps"] == 3 and t3["dt"] > 0 and np.isfinite(t3["t"])
    assert all(np.all(np.isfinite(st[k])) for k in st)
    # the step-1 criterion is driven by rounding noise in the reference too
    # (a2/a3 are finite differences over dt0 ~ 4e-8), so only its scale is checked
    _, _, crit1 = O.hermite_fixed(s, 1e-7, dt0, 1)
    with nb.Engine(1024, eps2=1e-7, dt=None) as e:
        e.set_state(s)
        e.timestepping(1)
        dt1 = e.timers()["dt"]
    assert 0.3 < dt1 / crit1 < 3.0, (dt1, crit1)


def _crit_sensitivity(s, eps2, dt, steps, trials=4):
    """Largest relative change of the oracle's last-step Aarseth criterion when
    every input value is perturbed by about one ulp: the criterion is built from
    finite differences of acc and jerk over dt (snap and crackle,
    src/nbody.cpp:165-179), so rounding-level differences in the force sums are
    amplified by the conditioning of that difference, which depends on the
    system and dt."""
    _, _, c0 = O.hermite_fixed(s, eps2, dt, steps)
    rng = np.random.default_rng(0)
    worst = 0.0
    for _ in range(trials):
        p = {k: v * (1 + 2.2e-16 * rng.standard_normal(v.shape)) for k, v in s.items()}
        _, _, c1 = O.hermite_fixed(p, eps2, dt, steps)
        worst = max(worst, abs(c1 - c0) / c0)
    return worst


@pytest.mark.parametrize("n", (33, 127, 1024))
def test_updatedt_vs_reference_golden(n):
    """The GPU Aarseth criterion (src/nbody.cpp:198-222), computed by the
    corrector from the pre-step acc and jerk, against the reference build's own
    updatedt() after 10 fixed steps of its default bodies.  At the reference's
    dt = 3.8e-5 the criterion's finite differences are ill-conditioned for
    small systems (a one-ulp input change moves it by 3e-7 relative at n = 33,
    3e-9 at 127, 5e-12 at 1024), so the bound is 100x that measured
    sensitivity, and never looser than it needs to be: 1e-12 where the
    criterion is well-conditioned."""
    g = golden(n)
    dt, steps = float(g["dt"]), int(g["nsteps"])
    with nb.Engine(n, eps2=1e-7, dt=dt) as e:
        e.set_state(state_of(g))
        e.timestepping(steps)
        got = e.timers()["dt_crit"]
    want = float(g["h_dtcrit"])
    tol = max(1e-12, 100 * _crit_sensitivity(state_of(g), 1e-7, dt, steps))
    err = abs(got - want) / want
    print(f"n={n}: dt_crit {got!r} reference {want!r} rel {err:.2e} (bound {tol:.1e})")
    assert err <= tol, (n, got, want, err, tol)


@pytest.mark.parametrize("n,steps", [(1024, 1), (1024, 10), (2048, 10)])
def test_updatedt_vs_oracle_well_conditioned(n, steps):
    """Plummer bodies at dt = 1/256, where the criterion's finite differences
    are well-conditioned (one-ulp input changes move it by ~1e-14): the GPU
    criterion equals the oracle's to 1e-12 relative."""
    eps2, dt = 1e-4, 1.0 / 256
    s = nb.plummer(n, seed=5)
    _, _, want = O.hermite_fixed(s, eps2, dt, steps)
    with nb.Engine(n, eps2=eps2, dt=dt) as e:
        e.set_state(s)
        e.timestepping(steps)
        got = e.timers()["dt_crit"]
    assert abs(got - want) <= 1e-12 * want, (got, want)


@pytest.mark.parametrize("n", (33, 1024))
def test_energy_vs_reference(n):
    g = golden(n)
    s = state_of(g)
    with nb.Engine(n, eps2=1e-7, dt=1.0) as e:
        e.set_state(s)
        T, U = e.energy()
        Tc, Uc = e.energy(ref_compat=True)
    assert abs(T - float(g["T"])) <= 1e-13 * abs(float(g["T"]))
    assert abs(Uc - float(g["U_ref"])) <= 1e-12 * abs(float(g["U_ref"]))
    Up = O.potential(s, 1e-7, compat=False)
    assert abs(U - Up) <= 1e-12 * abs(Up)


def test_mixed_precision_accuracy():
    n, eps2 = 4096, 1e-4
    s = nb.plummer(n, seed=2)
    ref = O.force(s, eps2)
    mixed = engine_derivs(s, eps2, precision="mixed")
    f32ref = O.force(s, eps2, "f32")  # the reference's own _F32 arithmetic
    em = vec_rel(mixed[:3], ref[:3])
    ef = vec_rel(f32ref[:3], ref[:3])
    print(f"mixed acc err: median {np.median(em):.3e} max {em.max():.3e}; "
          f"reference _F32: median {np.median(ef):.3e} max {ef.max():.3e}")
    assert np.median(em) <= 2e-6 and em.max() <= 2e-4
    assert np.median(em) <= 4 * np.median(ef) + 1e-7
    ej = vec_rel(mixed[3:], ref[3:])
    assert np.median(ej) <= 1e-5


def test_large_n_sampled_rows_and_momentum():
    """N = 65536 Plummer: sampled rows vs the oracle's direct sums, plus
    Newton's third law on the whole system (sum_i m_i a_i = 0)."""
    n, eps2 = 65536, 1e-4
    s = nb.plummer(n, seed=1)
    d = engine_derivs(s, eps2)
    rows = np.linspace(0, n - 1, 48).astype(np.int64)
    ref = O.force_rows(s, eps2, rows)
    ea, ej = derivs_rel(d[:, rows], ref)
    assert ea <= TOL_FP64 and ej <= TOL_FP64, (ea, ej)
    m = s["m"]
    for blk in (slice(0, 3), slice(3, 6)):
        net = np.abs((m * d[blk]).sum(1)).max()
        scale = (m * np.sqrt((d[blk] ** 2).sum(0))).sum()
        assert net <= 1e-11 * scale


def test_device_pointer_entry_matches_engine():
    import torch
    n, eps2 = 3000, 1e-4
    s = nb.plummer(n, seed=8)
    ref = engine_derivs(s, eps2)
    t = {k: torch.tensor(s[k], dtype=torch.float64, device="cuda") for k in nb.FIELDS}
    out = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(6)]
    with nb.Engine(n, eps2=eps2, dt=1.0) as e:
        stream = torch.cuda.current_stream().cuda_stream
        e.acc_jerk_device(*[t[k] for k in nb.FIELDS], out, stream=stream)
        torch.cuda.synchronize()
    got = torch.stack(out).cpu().numpy()
    ea, ej = derivs_rel(got, ref)
    assert ea <= 1e-13 and ej <= 1e-13


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_max_size_sampled_rows(precision):
    """N = 2^20: indexing at scale (padded arrays of ~10^6 rows, 64-bit
    partial offsets); sampled rows against the oracle's direct sums."""
    n, eps2 = 1 << 20, 1e-4
    s = nb.plummer(n, seed=6)
    d = engine_derivs(s, eps2, precision=precision)
    rows = np.array([0, 1, 12345, n // 2, n - 2, n - 1])
    ref = O.force_rows(s, eps2, rows)
    ea, ej = derivs_rel(d[:, rows], ref)
    tol = TOL_FP64 if precision == "fp64" else 1e-5
    assert ea <= tol and ej <= 10 * tol, (precision, ea, ej)


# ---------------------------------------------------------------------------
# Tile-relative mixed kernel (pair_variant 4; the automatic choice from 16384
# bodies): j-bodies in Hilbert-ordered tiles, positions as float offsets from
# the tile centre.
# ---------------------------------------------------------------------------
REL = dict(pair_variant=4)
HILO = dict(pair_variant=3)


@pytest.mark.parametrize("case", ["plummer", "far_from_origin", "two_clusters", "offset_1e6",
                                  "flat_disk", "coincident_pairs", "lattice"])
def test_tile_relative_accuracy_vs_hilo(case):
    """Tile-relative separations stay in the hi/lo kernel's accuracy class:
    per-body acc error against the FP64 oracle within 3x of the hi/lo
    kernel's (median) and within the mixed bounds, wherever the system sits
    and whatever its shape: a degenerate bounding box (a flat disk), tied
    Hilbert keys (coincident bodies, a regular lattice) and a system 1e6 units
    from the origin, where the float hi parts have an ulp of 1/16."""
    n, eps2 = 4096, 1e-4
    s = nb.plummer(n, seed=2)
    if case == "far_from_origin":      # float hi parts alone would lose ~10 bits here
        for k in ("x", "y", "z"):
            s[k] = s[k] + 1000.0
    elif case == "offset_1e6":
        for k in ("x", "y", "z"):
            s[k] = s[k] + 1.0e6
    elif case == "two_clusters":       # a tight cluster 50 units from a wide one
        t = nb.plummer(n, seed=3)
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            s[k] = np.where(np.arange(n) % 2 == 0, s[k], 0.05 * t[k] + (50.0 if k == "x" else 0.0))
    elif case == "flat_disk":          # every z and vz zero: a box of zero height
        s["z"], s["vz"] = np.zeros(n), np.zeros(n)
    elif case == "coincident_pairs":   # body 2k+1 sits on body 2k (softened r = 0 pairs)
        for k in ("x", "y", "z"):
            s[k] = np.repeat(s[k][::2], 2)
    elif case == "lattice":            # 16^3 grid: many equal coordinates
        g = (np.arange(16) + 0.5) / 16.0
        X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
        s["x"], s["y"], s["z"] = X.ravel(), Y.ravel(), Z.ravel()
    ref = O.force(s, eps2)
    rel = engine_derivs(s, eps2, precision="mixed", **REL)
    hilo = engine_derivs(s, eps2, precision="mixed", **HILO)
    er, eh = vec_rel(rel[:3], ref[:3]), vec_rel(hilo[:3], ref[:3])
    jr, jh = vec_rel(rel[3:], ref[3:]), vec_rel(hilo[3:], ref[3:])
    print(f"{case}: acc median rel {np.median(er):.3e} hilo {np.median(eh):.3e}; "
          f"max rel {er.max():.3e} hilo {eh.max():.3e}; jerk median rel {np.median(jr):.3e} "
          f"hilo {np.median(jh):.3e}")
    assert np.median(er) <= 2e-6 and er.max() <= 2e-4
    assert np.median(er) <= 3 * np.median(eh) + 1e-8
    assert np.median(jr) <= 3 * np.median(jh) + 1e-7


def _acc_term_scale(s, eps2, block=256):
    """sum_j m_j |r_ij| / s_ij^1.5 per body (FP64): the size of the terms an
    acceleration sums, the scale its rounding errors are relative to."""
    P = np.stack([s["x"], s["y"], s["z"]])
    out = np.empty(P.shape[1])
    for i0 in range(0, P.shape[1], block):
        d = P[:, None, :] - P[:, i0:i0 + block, None]
        r2 = (d ** 2).sum(0)
        out[i0:i0 + block] = (s["m"][None, :] * np.sqrt(r2) / (r2 + eps2) ** 1.5).sum(1)
    return out


def test_tile_relative_on_a_line():
    """Bodies on one axis: the pulls from both sides cancel, so |a| is far
    below the terms it sums and every float kernel's error relative to |a|
    grows on the bodies where they cancel (measured worst 3e-4 for hi/lo, 3e-3
    for near/far).  Relative to the size of the terms, the near/far error
    stays within 12x the hi/lo kernel's, as the far tiles' separation bound
    (9 ulp of |r| against about 1) allows, and below 1e-6 (measured median /
    max 4.3e-8 / 5.7e-7, hi/lo 1.1e-8 / 2.9e-7)."""
    n, eps2 = 4096, 1e-4
    s = nb.plummer(n, seed=2)
    for k in ("y", "z", "vy", "vz"):
        s[k] = np.zeros(n)
    ref = O.force(s, eps2)
    scale = _acc_term_scale(s, eps2)
    err = {}
    for name, kw in (("rel", REL), ("hilo", HILO)):
        d = engine_derivs(s, eps2, precision="mixed", **kw)
        err[name] = np.sqrt(((d[:3] - ref[:3]) ** 2).sum(0)) / scale
    print(f"line: acc error / term scale median rel {np.median(err['rel']):.3e} hilo "
          f"{np.median(err['hilo']):.3e}; max rel {err['rel'].max():.3e} hilo {err['hilo'].max():.3e}")
    assert err["rel"].max() <= 1e-6
    assert err["rel"].max() <= 12 * err["hilo"].max() + 1e-9
    assert np.median(err["rel"]) <= 12 * np.median(err["hilo"]) + 1e-10


@pytest.mark.parametrize("n", (1, 2, 33, 255, 257, 1000))
def test_tile_relative_small_and_ragged(n):
    """Padding slots and partly filled tiles (n not a multiple of the tile)."""
    eps2 = 1e-4
    s = nb.plummer(max(n, 2), seed=11)
    s = {k: v[:n].copy() for k, v in s.items()}
    d = engine_derivs(s, eps2, precision="mixed", **REL)
    assert np.all(np.isfinite(d))
    if n == 1:
        assert np.all(d == 0)
        return
    ref = O.force(s, eps2)
    ea = vec_rel(d[:3], ref[:3])
    assert ea.max() <= 2e-4, ea.max()


@pytest.mark.parametrize("cl", [2, 4, 8])
def test_near_far_on_thread_block_clusters(cl):
    """pair_variant 4 on clusters of cl CTAs along j (j_cluster): the CTAs of
    a cluster sum their split partials through distributed shared memory
    before one partial per cluster is written.  Same terms as the one-CTA
    kernel with the split sums associated differently, so the two agree to
    FP64 rounding; a split count that is not a multiple of cl is rounded up;
    Hermite steps (graph-captured) follow the one-CTA engine."""
    n, eps2 = 20000, 1e-4
    s = nb.plummer(n, seed=12)
    shape = dict(pair_variant=4, threads=128, i_per_thread=4, j_tile=128)
    base = engine_derivs(s, eps2, precision="mixed", split_j=16, **shape)
    for split in (16, 10):
        d = engine_derivs(s, eps2, precision="mixed", split_j=split, j_cluster=cl, **shape)
        ea, ej = derivs_rel(d, base)
        assert ea <= 1e-10 and ej <= 1e-10, (cl, split, ea, ej)
    rows = np.arange(0, n, 97)
    ea, _ = derivs_rel(d[:, rows], O.force_rows(s, eps2, rows))
    assert ea <= 2e-6, ea
    runs = {}
    for name, kw in (("one", {}), ("cluster", dict(j_cluster=cl))):
        with nb.Engine(n, eps2=eps2, precision="mixed", dt=1.0 / 1024, split_j=16, **shape, **kw) as e:
            e.set_state(s)
            e.force_calculation()
            e.timestepping(8)
            runs[name] = e.get_state()
            tm = e.timers()
    assert tm["split_j"] == 16
    dx = max(np.abs(runs["cluster"][k] - runs["one"][k]).max() for k in ("x", "y", "z"))
    assert dx <= 1e-12, dx


def test_tile_relative_deterministic_and_order_free():
    """Bitwise reproducible (stable sort, fixed reduction order); the result
    does not depend on the order the bodies are given in."""
    n, eps2 = 5000, 1e-4
    s = nb.plummer(n, seed=9)
    a = engine_derivs(s, eps2, precision="mixed", **REL)
    b = engine_derivs(s, eps2, precision="mixed", **REL)
    assert np.array_equal(a, b)
    perm = np.random.default_rng(0).permutation(n)
    c = engine_derivs({k: v[perm] for k, v in s.items()}, eps2, precision="mixed", **REL)
    ea, ej = derivs_rel(c, a[:, perm])
    assert ea <= 1e-5 and ej <= 1e-4, (ea, ej)


def test_tile_relative_device_entry_and_steps():
    """Caller-owned device arrays (n below the engine's size), then Hermite
    runs against the FP64 engine with the Hilbert order refreshed every step
    and every 16 steps."""
    import torch
    n, eps2 = 3000, 1e-4
    s = nb.plummer(n, seed=8)
    m = n - 100
    sub = {k: v[:m] for k, v in s.items()}
    t = {k: torch.tensor(sub[k], dtype=torch.float64, device="cuda") for k in nb.FIELDS}
    out = [torch.empty(m, dtype=torch.float64, device="cuda") for _ in range(6)]
    with nb.Engine(n, eps2=eps2, precision="mixed", dt=1.0, **REL) as e:
        e.acc_jerk_device(*[t[k] for k in nb.FIELDS], out, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = torch.stack(out).cpu().numpy()
        # the engine's own system after a foreign call: its order is rebuilt
        e.set_state(s)
        e.force_calculation()
        own = e.get_derivs()
    ref = O.force(sub, eps2)
    assert vec_rel(got[:3], ref[:3]).max() <= 2e-4
    assert vec_rel(own[:3], O.force(s, eps2)[:3]).max() <= 2e-4
    runs = {}
    for name, prec, kw in (("fp64", "fp64", {}), ("rel1", "mixed", dict(REL, sort_every=1)),
                           ("rel16", "mixed", REL)):
        with nb.Engine(n, eps2=eps2, precision=prec, dt=1.0 / 1024, **kw) as e:
            e.set_state(s)
            e.force_calculation()
            e.timestepping(40)
            runs[name] = e.get_state()
    for name in ("rel1", "rel16"):
        dx = max(np.abs(runs[name][k] - runs["fp64"][k]).max() for k in ("x", "y", "z"))
        assert dx <= 1e-8, (name, dx)


def test_mixed_rejects_softening_too_small_for_float():
    """m eps2^-1.5 overflows float below eps2 ~ 1e-25 (the self pair would
    give 0 x inf = NaN): mixed engines refuse eps2 < 1e-24, FP64 accepts it."""
    with pytest.raises(nb.NBodyError, match="mixed"):
        nb.Engine(64, eps2=1e-26, precision="mixed", dt=1.0)
    s = nb.plummer(64, seed=1)
    d = engine_derivs(s, 1e-26)
    assert np.all(np.isfinite(d))
    with nb.Engine(64, eps2=1e-24, precision="mixed", dt=1.0) as e:
        e.set_state(s)
        e.force_calculation()
        assert np.all(np.isfinite(e.get_derivs()))


# ---------------------------------------------------------------------------
# Autotuner (nbody_config.tune): tilings chosen per system size by timing the
# registered kernel shapes, then reused by later engines of the same size.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n,precision", [(4096, "fp64"), (4096, "mixed"), (65536, "fp64"),
                                         (65536, "mixed")])
def test_autotuned_engine_parity_and_reuse(n, precision):
    eps2 = 1e-4
    s = nb.plummer(n, seed=13)
    runs = []
    for _ in range(2):
        with nb.Engine(n, eps2=eps2, precision=precision, dt=1.0, tune=True) as e:
            e.set_state(s)
            e.force_calculation()
            runs.append((e.get_derivs(), e.timers()))
    (d, t1), (d2, t2) = runs
    keys = ("threads", "i_per_thread", "j_tile", "split_j", "j_cluster", "record_format")
    print(f"n={n} {precision}: tuned tiling {[t1[k] for k in keys]} (source {t1['tiling_source']})")
    assert t1["tiling_source"] in (2, 3)      # timed here, or by an earlier engine of this size
    assert t2["tiling_source"] == 3           # the second engine reuses the cached choice
    assert all(t1[k] == t2[k] for k in keys)
    assert np.array_equal(d, d2)              # same kernel, same split: bitwise equal
    rows = np.arange(n) if n <= 4096 else np.linspace(0, n - 1, 64).astype(np.int64)
    ref = O.force_rows(s, eps2, rows)
    if precision == "fp64":
        ea, ej = derivs_rel(d[:, rows], ref)
        assert ea <= TOL_FP64 and ej <= TOL_FP64, (ea, ej)
    else:
        ea = vec_rel(d[:3, rows], ref[:3])
        assert np.median(ea) <= 2e-6 and ea.max() <= 2e-4, (np.median(ea), ea.max())


def test_heuristic_tiling_reports_its_source():
    with nb.Engine(3000, eps2=1e-4, dt=1.0) as e:
        assert e.timers()["tiling_source"] == 0   # nothing chosen before the first evaluation
        e.set_state(nb.plummer(3000, seed=1))
        e.force_calculation()
        assert e.timers()["tiling_source"] == 1


# ---------------------------------------------------------------------------
# Mixed kernels against the reference's own _F32 arithmetic
# (src/kernel.cpp:1101-1163: separations rounded to float, float pair math,
# double accumulation): per-body acceleration errors against FP64 direct sums,
# compared with the _F32 arithmetic's own errors on the same bodies.
# ---------------------------------------------------------------------------
def _err_stats(e):
    return np.median(e), np.quantile(e, 0.99), e.max()


@pytest.mark.parametrize("variant", [3, 4])
@pytest.mark.parametrize("n", [4096, 65536])
def test_mixed_accuracy_vs_reference_f32(variant, n):
    eps2 = 1e-4
    s = nb.plummer(n, seed=2 if n == 4096 else 1)
    rows = np.arange(n) if n <= 4096 else np.linspace(0, n - 1, 2048).astype(np.int64)
    d64 = O.force_rows(s, eps2, rows)
    f32 = O.force_rows(s, eps2, rows, "f32")
    dm = engine_derivs(s, eps2, precision="mixed", pair_variant=variant)[:, rows]
    em, ef = vec_rel(dm[:3], d64[:3]), vec_rel(f32[:3], d64[:3])
    jm, jf = vec_rel(dm[3:], d64[3:]), vec_rel(f32[3:], d64[3:])
    sm, sf = _err_stats(em), _err_stats(ef)
    print(f"variant {variant} n={n}: acc err median/p99/max {sm[0]:.2e}/{sm[1]:.2e}/{sm[2]:.2e}; "
          f"reference _F32 {sf[0]:.2e}/{sf[1]:.2e}/{sf[2]:.2e}; ratios "
          f"{sm[0] / sf[0]:.2f}/{sm[1] / sf[1]:.2f}/{sm[2] / sf[2]:.2f}; jerk median "
          f"{np.median(jm):.2e} vs _F32 {np.median(jf):.2e}")
    # Both form every separation to float accuracy relative to |r| (hi/lo: one
    # rounding; near/far: double-single for near tiles, <= 9 ulp for far
    # ones); the rest of their gap to _F32 is the MUFU rsqrt/rcp and the float
    # sums over each j-tile.  Measured ratios to _F32 (median/p99/max):
    # near/far 4.6/3.9/4.1 at n = 4096 and 4.7/4.0/5.7 at n = 65536; hi/lo
    # 2.9/2.1/3.5 and 2.7/1.4/1.6.
    bound = {3: (4, 4, 12), 4: (6, 6, 8)}[variant]
    assert sm[0] <= bound[0] * sf[0] and sm[1] <= bound[1] * sf[1] and sm[2] <= bound[2] * sf[2]
    assert np.median(jm) <= 4 * np.median(jf)


@pytest.mark.parametrize("n", [4096, 65536])
def test_near_tiles_keep_close_pairs_accurate(n):
    """The near/far kernel against the same kernel with every tile taken as
    far (pair_variant 5): plain tile-relative offsets lose the close pairs of
    tiles whose offsets are large (measured worst error 2.7e-2 at n = 4096 and
    7.5e-4 at 65536), the near tiles' double-single separations keep them."""
    eps2 = 1e-4
    s = nb.plummer(n, seed=2 if n == 4096 else 1)
    rows = np.arange(n) if n <= 4096 else np.linspace(0, n - 1, 2048).astype(np.int64)
    d64 = O.force_rows(s, eps2, rows)
    e4 = vec_rel(engine_derivs(s, eps2, precision="mixed", pair_variant=4)[:3, rows], d64[:3])
    e5 = vec_rel(engine_derivs(s, eps2, precision="mixed", pair_variant=5)[:3, rows], d64[:3])
    print(f"n={n}: max acc error near/far {e4.max():.2e}, all far {e5.max():.2e}")
    assert e5.max() >= 30 * e4.max() and e4.max() <= 2e-6


def test_near_far_kernel_reports_its_near_share_and_keeps_caller_order():
    """The near/far engine keeps its bodies in Hilbert order: its energy equals
    the FP64 engine's on the same bodies (order-independent sums), its state
    comes back in the caller's order, and a Plummer sphere of 65536 bodies
    sends a minority of (warp, tile) pairs down the double-single path."""
    n, eps2 = 65536, 1e-4
    s = nb.plummer(n, seed=1)
    with nb.Engine(n, eps2=eps2, precision="mixed", dt=1 / 1024, pair_variant=4) as e, \
            nb.Engine(n, eps2=eps2, precision="fp64", dt=1 / 1024) as f:
        e.set_state(s)
        f.set_state(s)
        e.force_calculation()
        T, U = e.energy()
        T64, U64 = f.energy()
        near = e.timers()["near_tile_fraction"]
        st = e.get_state()
        d = e.get_derivs()
    assert abs(T - T64) <= 1e-12 * abs(T64) and abs(U - U64) <= 1e-12 * abs(U64)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(st[k], s[k]), k
    rows = np.linspace(0, n - 1, 64).astype(np.int64)
    ref = O.force_rows(s, eps2, rows)
    assert vec_rel(d[:3, rows], ref[:3]).max() <= 2e-6
    print(f"near share {near:.3f}")
    assert 0.02 < near < 0.5, near
    with nb.Engine(n, eps2=eps2, precision="mixed", dt=1 / 1024, pair_variant=5) as e:
        e.set_state(s)
        e.force_calculation()
        assert e.timers()["near_tile_fraction"] == 0.0
