"""CPU model of the tile-relative separations of the mixed pair kernel.

The kernel (pair.cuh RowsMixedRel, reltiles.cuh rel_tile_kernel) orders the
j-bodies along a Morton curve, cuts them into tiles, and stores each body as
-D(x) with D(x) = fl(fl(c - x_hi) - x_lo) for the tile centre c (a float);
an i-row forms D(x_i) with the same float operations and r_ij = D(x_i) +
(-D(x_j)).  This file restates that arithmetic in numpy float32 (one
rounding per operation, like the kernel's sub.rn / add.rn) and checks the
properties the design relies on:

* the self pair cancels exactly, whatever the tile centre;
* the separation error stays at about one float ulp of |x - c| per side,
  so with Morton tiles the accelerations keep the mixed accuracy class
  against the FP64 oracle;
* without the Morton order (tiles of arbitrary bodies) the same arithmetic
  loses accuracy wherever close pairs sit far from the tiles' centres (a
  tight cluster beside a wide one) - the ordering keeps the offsets local.
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
