"""CPU model of the tile-relative separations of the mixed pair kernel.

The one-add tile-relative form (the far tiles of pair.cuh RowsMixedNF, and
every tile with pair_variant 5) stores each body of a tile as -D(x) with
D(x) = fl(fl(c - x_hi) - x_lo) for the tile centre c (a float); an i-row forms
D(x_i) with the same float operations and r_ij = D(x_i) + (-D(x_j)).  This file
restates that arithmetic in numpy float32 (one rounding per operation, like
the kernel's sub.rn / add.rn) and checks the properties the design relies on:

* the self pair cancels exactly, whatever the tile centre;
* the separation error stays at about one float ulp of |x - c| per side, so
  with tiles of spatially ordered bodies the accelerations stay in the mixed
  accuracy class, and without an order (tiles of arbitrary bodies) close
  pairs far from their tiles' centres lose accuracy;
* the near/far kernel (bodies in Hilbert order, double-single separations on
  near tiles, reltiles.cuh rel_tile_nf_kernel) keeps the hi/lo kernel's
  accuracy, bounds the far tiles' separation error, and sends a small share
  of the work down the double-single path.
"""
import numpy as np

import nbody_b200 as nb
import oracle as O
from _util import vec_rel

F32 = np.float32


def _spread16(v):
    x = v.astype(np.uint64) & np.uint64(0xFFFF)
    for sh, m in ((32, 0x1F00000000FFFF), (16, 0x1F0000FF0000FF), (8, 0x100F00F00F00F00F),
                  (4, 0x10C30C30C30C30C3), (2, 0x1249249249249249)):
        x = (x | (x << np.uint64(sh))) & np.uint64(m)
    return x


def morton_order(P):
    """Stable order of 48-bit Morton keys (16 bits per axis) over the bounding box."""
    lo, hi = P.min(1), P.max(1)
    q = np.clip((P - lo[:, None]) * (65535.0 / (hi - lo))[:, None], 0, 65535).astype(np.uint64)
    key = _spread16(q[0]) | (_spread16(q[1]) << np.uint64(1)) | (_spread16(q[2]) << np.uint64(2))
    return np.argsort(key, kind="stable")


def hi_lo(P):
    h = P.astype(F32)
    return h, (P - h.astype(np.float64)).astype(F32)


def D(c, h, l):
    """fl(fl(c - x_hi) - x_lo), one float rounding per operation."""
    return (F32(c) - h).astype(F32) - l


def tile_centres(P, idx):
    """Median of up to 32 evenly spaced samples per axis, rounded to float."""
    nv = len(idx)
    ns = min(32, nv)
    smp = (np.arange(ns) * nv) // 32 if ns == 32 else np.arange(ns)
    return np.array([np.sort(P[k, idx[smp]])[ns // 2] for k in range(3)]).astype(F32)


def model_acc(s, eps2, TJ=128, ordered=True):
    """Accelerations from the kernel's float separations (the rest in FP64,
    so the comparison isolates the separation arithmetic)."""
    P = np.stack([s["x"], s["y"], s["z"]])
    n = P.shape[1]
    order = morton_order(P) if ordered else np.arange(n)
    h, l = hi_lo(P)
    acc = np.zeros((3, n))
    for t0 in range(0, n, TJ):
        idx = order[t0:t0 + TJ]
        c = tile_centres(P, idx)
        Di = np.stack([D(c[k], h[k], l[k]) for k in range(3)])      # rows: D(x_i)
        rec = -Di[:, idx]                                           # records: -D(x_j)
        r = (rec[:, None, :] + Di[:, :, None]).astype(F32).astype(np.float64)
        s2 = (r ** 2).sum(0) + eps2
        acc += (s["m"][idx][None, None, :] * r / s2[None] ** 1.5).sum(2)
    return acc


def test_self_pair_cancels_exactly():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.normal(0, 1, 500), rng.normal(0, 30, 500), [1e-30, -7.25, 1000.0]])
    h, l = hi_lo(x[None])
    for c in (0.0, 0.5, -3.25, 17.0, 1000.0, float(np.float32(0.1))):
        d = D(c, h[0], l[0])
        assert np.all((-d) + d == 0)


def test_separation_error_is_one_ulp_of_the_offsets():
    rng = np.random.default_rng(2)
    c = F32(2.5)
    xi = 2.5 + rng.normal(0, 0.05, 2000)
    xj = xi + rng.normal(0, 1e-3, 2000)
    hi_, li = hi_lo(xi[None])
    hj, lj = hi_lo(xj[None])
    r = (D(c, hi_[0], li[0]) - D(c, hj[0], lj[0])).astype(np.float64)
    err = np.abs(r - (xj - xi))
    bound = 2.0 ** -23 * (np.abs(xi - 2.5) + np.abs(xj - 2.5) + np.abs(xj - xi))
    assert np.all(err <= 1.5 * bound)


def _two_clusters(n):
    """A wide Plummer sphere at the origin and a tight one 50 units away."""
    s, t = nb.plummer(n, seed=2), nb.plummer(n, seed=3)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        s[k] = np.where(np.arange(n) % 2 == 0, s[k], 0.05 * t[k] + (50.0 if k == "x" else 0.0))
    return s


def test_morton_tiles_keep_the_mixed_accuracy_class():
    n, eps2 = 3000, 1e-4
    for s in (nb.plummer(n, seed=5), _two_clusters(n)):
        ref = O.force(s, eps2)[:3]
        e = vec_rel(model_acc(s, eps2, ordered=True), ref)
        assert np.median(e) <= 1e-7 and e.max() <= 2e-5, (np.median(e), e.max())


def test_ordering_is_what_keeps_offsets_small():
    """With tiles of arbitrary bodies the tight cluster's offsets are ~50
    units, and its close pairs lose ~10 bits; Morton tiles keep them local."""
    n, eps2 = 3000, 1e-4
    s = _two_clusters(n)
    ref = O.force(s, eps2)[:3]
    e_tiles = vec_rel(model_acc(s, eps2, ordered=True), ref)
    e_plain = vec_rel(model_acc(s, eps2, ordered=False), ref)
    assert np.percentile(e_plain, 99) >= 30 * np.percentile(e_tiles, 99)


# ---------------------------------------------------------------------------
# Near/far tile-relative kernel (pair.cuh RowsMixedNF, reltiles.cuh
# rel_tile_nf_kernel): bodies in Hilbert order, warps of consecutive positions,
# and per (warp rows, tile) either the one-add form on float offsets (far:
# boxes apart by d > 0 with d >= R/2) or double-single offsets (near).
# ---------------------------------------------------------------------------
U = 2.0 ** -24


def hilbert_keys(q):
    """48-bit Hilbert indices of 16-bit cells q (3, n): Skilling's transpose
    algorithm, as the engine's hilbert_key48 (reltiles.cuh) computes them."""
    X = [q[k].astype(np.uint64).copy() for k in range(3)]
    Q = np.uint64(1 << 15)
    while Q > 1:
        Pm = Q - np.uint64(1)
        for i in range(3):
            m = (X[i] & Q) != 0
            X[0] = np.where(m, X[0] ^ Pm, X[0])
            t = np.where(m, np.uint64(0), (X[0] ^ X[i]) & Pm)
            X[0] ^= t
            X[i] ^= t
        Q >>= np.uint64(1)
    X[1] ^= X[0]
    X[2] ^= X[1]
    t = np.zeros_like(X[0])
    Q = np.uint64(1 << 15)
    while Q > 1:
        t = np.where((X[2] & Q) != 0, t ^ (Q - np.uint64(1)), t)
        Q >>= np.uint64(1)
    return (_spread16(X[0] ^ t) << np.uint64(2)) | (_spread16(X[1] ^ t) << np.uint64(1)) | _spread16(X[2] ^ t)


def hilbert_order(P):
    """Stable order of the Hilbert indices of bodies P (3, n) over their
    bounding box (2^16 cells per axis), as order_key_kernel sorts them."""
    lo, hi = P.min(1), P.max(1)
    q = np.clip((P - lo[:, None]) * (65535.0 / (hi - lo))[:, None], 0, 65535).astype(np.uint64)
    return np.argsort(hilbert_keys(q), kind="stable")


def test_hilbert_keys_trace_a_continuous_curve():
    """Consecutive Hilbert indices are face-neighbouring cells: the 8^3 cells
    of the top three levels (multiples of 2^13), sorted by key, step by
    exactly one cell every time, and the keys are distinct."""
    g = np.stack(np.meshgrid(*[np.arange(8)] * 3, indexing="ij")).reshape(3, -1)
    keys = hilbert_keys((g * 8192).astype(np.uint64))
    assert np.unique(keys).size == keys.size
    o = np.argsort(keys)
    steps = np.abs(np.diff(g[:, o], axis=1)).sum(0)
    assert np.all(steps == 1)


def ds_offset(c, xh, xl):
    """(hi, lo) = c - (xh + xl) in double-single: TwoSum of c - xh, the low
    part folded in, renormalised by a second TwoSum; float32 rounding per
    operation as in the kernel."""
    c, xh, xl = F32(c), np.asarray(xh, F32), np.asarray(xl, F32)
    s = c - xh
    bb = s - c
    e = (c - (s - bb)) - (xh + bb)
    t = e - xl
    hi = s + t
    b2 = hi - s
    lo = (s - (hi - b2)) + (t - b2)
    return hi, lo


def test_ds_offset_is_double_single_accurate():
    rng = np.random.default_rng(3)
    for scale in (1e-3, 1.0, 40.0):
        x = rng.normal(0, scale, 5000)
        h, l = hi_lo(x[None])
        for c in (F32(0.0), F32(scale * 0.37), F32(-scale * 1.9)):
            hi, lo = ds_offset(c, h[0], l[0])
            exact = float(c) - (h[0].astype(np.float64) + l[0].astype(np.float64))
            got = hi.astype(np.float64) + lo.astype(np.float64)
            assert np.all(np.abs(got - exact) <= 2.0 ** -44 * np.abs(exact) + 1e-300)


def model_acc_near_far(s, eps2, TJ=128, ROWS=128, kappa=0.5):
    """Accelerations from the near/far kernel's separations (the rest of the
    pair math in FP64) and the share of (warp rows, tile) pairs taken as near:
    tiles of TJ and warps of ROWS consecutive Morton positions, tile centre =
    the midpoint of its bounding box, far iff the boxes are apart by
    d > 0 with d >= kappa R."""
    P = np.stack([s["x"], s["y"], s["z"]])
    n = P.shape[1]
    order = hilbert_order(P)
    Q = P[:, order]                       # engine positions (Morton order)
    m = s["m"][order]
    h, l = hi_lo(Q)
    acc = np.zeros((3, n))
    near = total = 0
    for t0 in range(0, n, TJ):
        j = np.arange(t0, min(n, t0 + TJ))
        c = (0.5 * Q[:, j].min(1) + 0.5 * Q[:, j].max(1)).astype(F32)
        R = np.sqrt(((Q[:, j] - c[:, None].astype(np.float64)) ** 2).sum(0)).max()
        tlo, thi = Q[:, j].min(1), Q[:, j].max(1)
        Dj = [ds_offset(c[k], h[k, j], l[k, j]) for k in range(3)]
        for r0 in range(0, n, ROWS):
            i = np.arange(r0, min(n, r0 + ROWS))
            blo, bhi = Q[:, i].min(1), Q[:, i].max(1)
            gap = np.maximum(0, np.maximum(blo - thi, tlo - bhi))
            d2 = (gap ** 2).sum()
            far = d2 > 0 and d2 >= (kappa * R) ** 2
            total += 1
            near += 0 if far else 1
            r = np.empty((3, i.size, j.size))
            for k in range(3):
                if far:
                    Di = (F32(c[k]) - h[k, i]) - l[k, i]
                    r[k] = (Di[:, None] + (-Dj[k][0])[None, :]).astype(np.float64)
                else:
                    Dih, Dil = ds_offset(c[k], h[k, i], l[k, i])
                    r[k] = ((Dih[:, None] + (-Dj[k][0])[None, :]) +
                            (Dil[:, None] + (-Dj[k][1])[None, :])).astype(np.float64)
            s2 = (r ** 2).sum(0) + eps2
            acc[:, i] += (m[j][None, None, :] * r / s2[None] ** 1.5).sum(2)
    out = np.zeros_like(acc)
    out[:, order] = acc
    return out, near / total


def model_acc_hilo(s, eps2):
    """Accelerations from the hi/lo kernel's separations (rest in FP64)."""
    P = np.stack([s["x"], s["y"], s["z"]])
    h, l = hi_lo(P)
    r = np.stack([((h[k][None, :] - h[k][:, None]) + (l[k][None, :] - l[k][:, None])).astype(np.float64)
                  for k in range(3)])
    s2 = (r ** 2).sum(0) + eps2
    return (s["m"][None, None, :] * r / s2[None] ** 1.5).sum(2)


def near_fraction(P, TJ=128, ROWS=128, kappa=0.5):
    """Share of (warp rows, tile) pairs the near/far kernel takes as near, for
    bodies P (3, n) with n a multiple of TJ and ROWS (vectorised classifier)."""
    Q = P[:, hilbert_order(P)]
    n = Q.shape[1]
    T = Q.reshape(3, n // TJ, TJ)
    tlo, thi = T.min(2), T.max(2)
    c = (0.5 * tlo + 0.5 * thi).astype(F32).astype(np.float64)
    R = np.sqrt(((T - c[:, :, None]) ** 2).sum(0)).max(1)
    B = Q.reshape(3, n // ROWS, ROWS)
    blo, bhi = B.min(2), B.max(2)
    near = 0
    for b0 in range(0, blo.shape[1], 64):
        gap = np.maximum(0, np.maximum(blo[:, b0:b0 + 64, None] - thi[:, None, :],
                                       tlo[:, None, :] - bhi[:, b0:b0 + 64, None]))
        d2 = (gap ** 2).sum(0)
        near += (~((d2 > 0) & (d2 >= (kappa * R[None, :]) ** 2))).sum()
    return near / (blo.shape[1] * T.shape[1])


def test_near_far_separations_keep_the_hilo_accuracy():
    """Far tiles (one add) and near tiles (double-single) together: per-body
    accelerations as accurate as the hi/lo kernel's (max and p99 within 1.5x),
    where plain tile-relative offsets lose more than an order of magnitude on
    the worst bodies (64-body tiles and warps so that far tiles occur at this
    size)."""
    n, eps2 = 8192, 1e-4
    for s in (nb.plummer(n, seed=5), _two_clusters(n)):
        ref = O.force(s, eps2)[:3]
        a, frac = model_acc_near_far(s, eps2, TJ=64, ROWS=64)
        e_nf = vec_rel(a, ref)
        e_hl = vec_rel(model_acc_hilo(s, eps2), ref)
        assert 0.2 < frac < 0.8, frac
        assert e_nf.max() <= 1.5 * e_hl.max(), (e_nf.max(), e_hl.max())
        assert np.quantile(e_nf, 0.99) <= 1.5 * np.quantile(e_hl, 0.99)


def test_near_share_falls_with_system_size():
    """The near (three-add) share of the work at the kernel's default shape
    (128-body tiles, warps of 128 rows): about an eighth at N = 65536 with
    Hilbert order (Morton order, whose jumps make wide tiles: a quarter)."""
    fr = {n: near_fraction(np.stack([nb.plummer(n, seed=1)[k] for k in ("x", "y", "z")]))
          for n in (16384, 65536)}
    assert fr[65536] < 0.2 and fr[65536] < fr[16384], fr


def test_far_tiles_bound_the_separation_error():
    """A far pair's separation from float offsets has error <= 9u |r| (u =
    2^-24): about u (3 |r| + 3 R) with |x_i - c| <= |r| + R and |r| >= d >= R/2."""
    rng = np.random.default_rng(4)
    c = F32(0.75)
    R = 0.01
    xj = 0.75 + rng.uniform(-R, R, (3000, 3)) / np.sqrt(3)
    dirs = rng.normal(size=(3000, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    xi = xj + dirs * rng.uniform(0.5 * R + 2 * R, 50 * R, (3000, 1))   # d >= R/2 from the tile's box
    hi_, li = hi_lo(xi.T)
    hj, lj = hi_lo(xj.T)
    r = np.stack([((c - hi_[k]) - li[k]) + (-((c - hj[k]) - lj[k])) for k in range(3)]).astype(np.float64)
    exact = (hj.astype(np.float64) + lj) - (hi_.astype(np.float64) + li)
    err = np.linalg.norm(r - exact, axis=0)
    assert np.all(err <= 9 * U * np.linalg.norm(exact, axis=0))
