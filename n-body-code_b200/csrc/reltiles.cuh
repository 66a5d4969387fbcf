// Hilbert ordering and the j-records of the near/far tile-relative mixed
// kernel (JBodyNF, pair.cuh).
//
// Bodies are ordered along a Hilbert curve of their positions; the
// engine keeps its state in that order (re-ordered every sort_every steps),
// so each j-tile of TJ consecutive positions covers a compact region and
// stores its bodies as offsets from the tile's centre.
//
//   bbox_partial_kernel   per-CTA min/max of x, y, z          (O(N) read, 24 B/body)
//   order_key_kernel      48-bit Hilbert key (16 bits per axis) + index (O(N), 24 B in, 12 B out)
//   (stable radix sort of (key, index) pairs: cub::DeviceRadixSort)
//   gather_rows_kernel    the state (13 arrays) or a caller's input into that order
//   scatter_rows_kernel   back to the caller's order (downloads, outputs)
//   rel_tile_nf_kernel<TJ> tile box, centre and radius; hi/lo offsets per body
//                         (O(N), 56 B read coalesced, 96 B written per body,
//                         one bulk copy per tile from shared memory)
//
// Every step is deterministic: the bounding box reduces in a fixed order and
// the sort is stable, so the records (and the pair sums) are reproducible.
#pragma once
#include <cstdint>

#include "hermite.cuh"
#include "pair.cuh"

namespace nbody {

constexpr int kBBoxThreads = 256;

// Interleaves the low 21 bits of v with two zero bits between each.
__device__ __forceinline__ uint64_t spread21(uint32_t v) {
  uint64_t x = v & 0x1fffffull;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// 48-bit Hilbert index of a point given its 16-bit cell coordinates, by
// Skilling's transpose algorithm (J. Skilling, "Programming the Hilbert
// curve", AIP Conf. Proc. 707, 2004): the axes are turned into the curve's
// transposed index by inverting and exchanging low bits level by level, Gray
// decoding follows, and the three 16-bit words are interleaved, axis 0 most
// significant.  Consecutive indices are neighbouring cells (no jumps, unlike
// a Morton curve), so runs of consecutive bodies cover compact regions.
__device__ __forceinline__ uint64_t hilbert_key48(uint32_t a0, uint32_t a1, uint32_t a2) {
  uint32_t X[3] = {a0, a1, a2};
  for (uint32_t Q = 1u << 15; Q > 1u; Q >>= 1) {
    const uint32_t P = Q - 1u;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];
  X[2] ^= X[1];
  uint32_t t = 0;
  for (uint32_t Q = 1u << 15; Q > 1u; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1u;
  return (spread21(X[0] ^ t) << 2) | (spread21(X[1] ^ t) << 1) |
         spread21(X[2] ^ t);
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide min (k < 3) / max (k >= 3) of six values; every thread gets the
// result.  sh holds 6 * 32 doubles.
__device__ __forceinline__ void block_minmax6(double v[6], double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = k < 3 ? warp_min(v[k]) : warp_max(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 6; ++k) sh[k * 32 + warp] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double w = k < 3 ? INFINITY : -INFINITY;
    for (int q = 0; q < nw; ++q) w = k < 3 ? fmin(w, sh[k * 32 + q]) : fmax(w, sh[k * 32 + q]);
    v[k] = w;
  }
  __syncthreads();
}

// part[b*6 + k]: min x, y, z (k < 3) and max x, y, z of the bodies CTA b visits.
static __global__ void __launch_bounds__(kBBoxThreads) bbox_partial_kernel(int n, SoA7 in,
                                                                          double* __restrict__ part) {
  __shared__ double sh[6 * 32];
  double v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = in.x[i], y = in.y[i], z = in.z[i];
    v[0] = fmin(v[0], x); v[1] = fmin(v[1], y); v[2] = fmin(v[2], z);
    v[3] = fmax(v[3], x); v[4] = fmax(v[4], y); v[5] = fmax(v[5], z);
  }
  block_minmax6(v, sh);
#pragma unroll
  for (int k = 0; k < 6; ++k)
    if (threadIdx.x == k) part[blockIdx.x * 6 + k] = v[k];
}

// keys[i] = Hilbert index of body i's cell (2^16 cells per axis) in the box
// of the nparts partial boxes; vals[i] = i.  Non-finite coordinates map to
// cell 0.
static __global__ void __launch_bounds__(kBBoxThreads) order_key_kernel(
    int n, SoA7 in, const double* __restrict__ part, int nparts, uint64_t* __restrict__ keys,
    int* __restrict__ vals) {
  __shared__ double sh[6 * 32];
  double v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (int b = threadIdx.x; b < nparts; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < 6; ++k)
      v[k] = k < 3 ? fmin(v[k], part[b * 6 + k]) : fmax(v[k], part[b * 6 + k]);
  block_minmax6(v, sh);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  constexpr double kCells = 65535.0;  // 2^16 - 1 cells per axis: a 48-bit key
  const double p[3] = {in.x[i], in.y[i], in.z[i]};
  uint32_t cell[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double w = v[k + 3] - v[k];
    double q = w > 0.0 ? (p[k] - v[k]) * (kCells / w) : 0.0;
    q = fmin(fmax(q, 0.0), kCells);  // NaN -> 0
    cell[k] = static_cast<uint32_t>(q);
  }
  keys[i] = hilbert_key48(cell[0], cell[1], cell[2]);
  vals[i] = i;
}


// Records of the near/far kernel from bodies already in Hilbert order: tile t
// (CTA t, TJ threads) = header + the bodies at positions t*TJ + k, k < TJ, read
// straight (coalesced) from `in`; positions >= n are zero-mass padding at the
// centre.  Centre: the midpoint of the tile's bounding box, rounded to float
// (it keeps R, the largest offset, near the box's half-diagonal, which decides
// how many row blocks may take the tile as far; how close pairs are formed
// does not depend on the centre).  Header: the centre, the bounding box
// rounded outward to float, and R = max |x - c| rounded up.  Body records:
// -D_hi, -D_lo with (D_hi, D_lo) = ds_offset(c, x_hi, x_lo) (pair.cuh).
// With cid (ensembles), slots whose cid is negative are padding as well.
static_assert(sizeof(JBodyNF) == 96, "tile records are 96 bytes: a tile starts 16-byte aligned");
template <int TJ>
__global__ void __launch_bounds__(TJ) rel_tile_nf_kernel(int n, SoA7 in, JBodyNF* __restrict__ out,
                                                         const int* __restrict__ cid = nullptr) {
  __shared__ double box[6][TJ / 32];
  __shared__ float rmax[TJ / 32];
  __shared__ __align__(128) JBodyNF stage[TJ + 1];  // the tile, written out in one bulk copy
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int slot = blockIdx.x * TJ + tid;
  const bool valid = slot < n && (!cid || cid[slot] >= 0);
  double p[3] = {0.0, 0.0, 0.0}, m = 0, vx = 0, vy = 0, vz = 0;
  if (valid) {
    p[0] = in.x[slot]; p[1] = in.y[slot]; p[2] = in.z[slot]; m = in.m[slot];
    vx = in.vx[slot]; vy = in.vy[slot]; vz = in.vz[slot];
  }
  // bounding box in double (empty tile: +inf/-inf)
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double w = k < 3 ? (valid ? p[k] : INFINITY) : (valid ? p[k - 3] : -INFINITY);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double u = __shfl_xor_sync(0xffffffffu, w, o);
      w = k < 3 ? fmin(w, u) : fmax(w, u);
    }
    if (lane == 0) box[k][warp] = w;
  }
  __syncthreads();
  double lo[3], hi[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    lo[k] = box[k][0];
    hi[k] = box[3 + k][0];
    for (int q = 1; q < TJ / 32; ++q) {
      lo[k] = fmin(lo[k], box[k][q]);
      hi[k] = fmax(hi[k], box[3 + k][q]);
    }
  }
  float c[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double mid = 0.5 * lo[k] + 0.5 * hi[k];
    c[k] = isfinite(mid) ? static_cast<float>(mid) : 0.0f;
  }
  // largest offset from the (float) centre, rounded up
  double r2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double d = p[k] - static_cast<double>(c[k]);
    r2 += valid ? d * d : 0.0;
  }
  float R = __double2float_ru(sqrt(r2));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) R = fmaxf(R, __shfl_xor_sync(0xffffffffu, R, o));
  if (lane == 0) rmax[warp] = R;
  __syncthreads();
  JBodyNF* tile = out + static_cast<size_t>(blockIdx.x) * (TJ + 1);
  if (tid == 0) {
    for (int q = 1; q < TJ / 32; ++q) R = fmaxf(R, rmax[q]);
    JBodyNF h;
    h.x = make_float2(c[0], c[0]); h.y = make_float2(c[1], c[1]); h.z = make_float2(c[2], c[2]);
    h.m = make_float2(__double2float_rd(lo[0]), __double2float_rd(lo[1]));
    h.vx = make_float2(__double2float_rd(lo[2]), __double2float_ru(hi[0]));
    h.vy = make_float2(__double2float_ru(hi[1]), __double2float_ru(hi[2]));
    h.vz = make_float2(R, 0.f);
    h.pad = h.xl = h.yl = h.zl = h.pad2 = make_float2(0.f, 0.f);
    stage[0] = h;
  }
  float oh[3], ol[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float hv = static_cast<float>(p[k]);
    const float lv = static_cast<float>(p[k] - static_cast<double>(hv));
    float dh = 0.f, dl = 0.f;
    if (valid) ds_offset(c[k], hv, lv, dh, dl);
    oh[k] = -dh;
    ol[k] = -dl;
  }
  const float fm = static_cast<float>(m), fu = static_cast<float>(vx);
  const float fv = static_cast<float>(vy), fw = static_cast<float>(vz);
  JBodyNF r;
  r.x = make_float2(oh[0], oh[0]); r.y = make_float2(oh[1], oh[1]); r.z = make_float2(oh[2], oh[2]);
  r.m = make_float2(fm, fm);
  r.vx = make_float2(fu, fu); r.vy = make_float2(fv, fv); r.vz = make_float2(fw, fw);
  r.pad = make_float2(0.f, 0.f);
  r.xl = make_float2(ol[0], ol[0]); r.yl = make_float2(ol[1], ol[1]); r.zl = make_float2(ol[2], ol[2]);
  r.pad2 = make_float2(0.f, 0.f);
  stage[1 + tid] = r;
  // (TJ + 1) * 96 bytes from a 96-byte multiple: both 16-byte aligned
  bulk_store_fence();
  __syncthreads();
  if (tid == 0) bulk_store(tile, stage, static_cast<uint32_t>(sizeof(JBodyNF) * (TJ + 1)));
}

// Gathers rows [0, n) of up to kMaxGather float64 arrays through a position
// map: dst[a][q] = src[a][ord[q]] (and, with perm_out, perm_out[q] =
// perm[ord[q]], or ord[q] without perm).  Re-orders an engine's state into
// Hilbert order, or a caller's input.
constexpr int kMaxGather = 13;
struct GatherArgs {
  const double* src[kMaxGather];
  double* dst[kMaxGather];
  int arrays;
};
static __global__ void gather_rows_kernel(int n, const int* __restrict__ ord, GatherArgs g,
                                          const int* __restrict__ perm, int* __restrict__ perm_out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int src = ord[q];
#pragma unroll
  for (int a = 0; a < kMaxGather; ++a)
    if (a < g.arrays) g.dst[a][q] = g.src[a][src];
  if (perm_out) perm_out[q] = perm ? perm[src] : src;
}

// The inverse: dst[a][perm[p]] = src[a][p] for rows [0, n) (back to the
// caller's body order).
static __global__ void scatter_rows_kernel(int n, const int* __restrict__ perm, GatherArgs g) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int dst = perm[p];
#pragma unroll
  for (int a = 0; a < kMaxGather; ++a)
    if (a < g.arrays) g.dst[a][dst] = g.src[a][p];
}

static __global__ void iota_kernel(int n, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = i;
}

}  // namespace nbody
