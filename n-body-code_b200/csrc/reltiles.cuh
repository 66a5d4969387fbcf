// j-records of the tile-relative mixed kernel (JBodyRel, pair.cuh).
//
// Bodies are ordered along a Morton (Z-order) curve of their positions so
// that each j-tile of TJ consecutive records covers a compact region; every
// tile then stores its bodies as float offsets from the tile's centre.
//
//   bbox_partial_kernel   per-CTA min/max of x, y, z          (O(N) read, 24 B/body)
//   morton_key_kernel     48-bit key (16 bits per axis) + index (O(N), 24 B in, 12 B out)
//   (stable radix sort of (key, index) pairs: cub::DeviceRadixSort)
//   rel_tile_kernel<TJ>   gather by sorted index, median tile centre, records
//                         (O(N), 56 B gathered, 64 B written per body)
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
__device__ __forceinline__ uint64_t morton_spread21(uint32_t v) {
  uint64_t x = v & 0x1fffffull;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
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

// keys[i] = Morton code of body i in the box of the nparts partial boxes;
// vals[i] = i.  Non-finite coordinates map to cell 0.
static __global__ void __launch_bounds__(kBBoxThreads) morton_key_kernel(
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
  uint64_t key = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double w = v[k + 3] - v[k];
    double q = w > 0.0 ? (p[k] - v[k]) * (kCells / w) : 0.0;
    q = fmin(fmax(q, 0.0), kCells);  // NaN -> 0
    key |= morton_spread21(static_cast<uint32_t>(q)) << k;
  }
  keys[i] = key;
  vals[i] = i;
}

// Tile t (CTA t, TJ threads) = header + the bodies order[t*TJ + k], k < TJ
// (slots >= n, and rows with cid[row] < 0 when cid is given, are zero-mass
// padding at the centre).
//
// Centre c = the per-axis median of up to 32 evenly spaced bodies of the
// tile, rounded to float (a tile that straddles a jump of the Morton curve
// keeps its centre with the majority of its bodies).  The valid slots of a
// tile are a prefix (padding sorts last), so the samples are slots
// floor(j * nv / 32); warp 0 ranks them with shuffles.  A body's stored offset is -D, with
// D = fl(fl(c - x_hi) - x_lo) the very float operations the pair kernel
// applies to an i-row (x_hi = fl(x), x_lo = fl(x - x_hi)); the self pair
// therefore cancels exactly (r_ii = -D + D = 0), whatever the rounding.
template <int TJ>
__global__ void __launch_bounds__(TJ) rel_tile_kernel(int n, SoA7 in, const int* __restrict__ order,
                                                      JBodyRel* __restrict__ out,
                                                      const int* __restrict__ cid) {
  __shared__ double med[3];
  const int tid = threadIdx.x;
  const int slot = blockIdx.x * TJ + tid;
  int b = slot < n ? order[slot] : -1;
  if (b >= 0 && cid && cid[b] < 0) b = -1;
  double p[3] = {0.0, 0.0, 0.0}, m = 0, vx = 0, vy = 0, vz = 0;
  if (b >= 0) {
    p[0] = in.x[b]; p[1] = in.y[b]; p[2] = in.z[b]; m = in.m[b];
    vx = in.vx[b]; vy = in.vy[b]; vz = in.vz[b];
  }
  if (tid < 3) med[tid] = 0.0;
  const int nv = __syncthreads_count(b >= 0);
  if (tid < 32 && nv > 0) {
    const int ns = min(32, nv);
    // sample `tid` = slot tid * nv / 32 (all distinct when nv >= 32)
    const int q = ns == 32 ? static_cast<int>((static_cast<long long>(tid) * nv) >> 5) : tid;
    const int bq = q < ns || ns == 32 ? order[blockIdx.x * TJ + q] : -1;
    double s[3] = {0.0, 0.0, 0.0};
    if (tid < ns) {
      s[0] = in.x[bq]; s[1] = in.y[bq]; s[2] = in.z[bq];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {  // rank among the ns samples (ties by lane)
      int r = 0;
      for (int l = 0; l < ns; ++l) {
        const double w = __shfl_sync(0xffffffffu, s[k], l);
        r += (w < s[k] || (w == s[k] && l < tid)) ? 1 : 0;
      }
      if (tid < ns && r == ns / 2) med[k] = s[k];
    }
  }
  __syncthreads();
  float c[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) c[k] = isfinite(med[k]) ? static_cast<float>(med[k]) : 0.0f;
  JBodyRel* tile = out + static_cast<size_t>(blockIdx.x) * (TJ + 1);
  if (tid == 0) {
    JBodyRel h;
    h.x = make_float2(c[0], c[0]); h.y = make_float2(c[1], c[1]); h.z = make_float2(c[2], c[2]);
    h.m = h.vx = h.vy = h.vz = h.pad = make_float2(0.f, 0.f);
    tile[0] = h;
  }
  float o[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float hi = static_cast<float>(p[k]);
    const float lo = static_cast<float>(p[k] - static_cast<double>(hi));
    o[k] = b >= 0 ? -__fsub_rn(__fsub_rn(c[k], hi), lo) : 0.0f;
  }
  const float fm = static_cast<float>(m), fu = static_cast<float>(vx);
  const float fv = static_cast<float>(vy), fw = static_cast<float>(vz);
  JBodyRel r;
  r.x = make_float2(o[0], o[0]); r.y = make_float2(o[1], o[1]); r.z = make_float2(o[2], o[2]);
  r.m = make_float2(fm, fm);
  r.vx = make_float2(fu, fu); r.vy = make_float2(fv, fv); r.vz = make_float2(fw, fw);
  r.pad = make_float2(0.f, 0.f);
  tile[1 + tid] = r;
}

}  // namespace nbody
