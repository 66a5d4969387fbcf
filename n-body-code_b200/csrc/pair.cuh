// O(N^2) pair acc + jerk kernels (the hot path).
//
// Physics (src/kernel.cpp:1187-1221 in the reference, restated): for every
// i-row, a_i = sum_j m_j q r_ij and jerk_i = sum_j m_j q (v_ij + c r_ij) with
// r_ij = x_j - x_i, v_ij = v_j - v_i, s = r^2 + eps2, q = s^(-3/2),
// c = -3 (r.v)/s.  The reference walks j < i and applies Newton's third law;
// here every row sums over all j (the self term is exactly zero since r = 0,
// v = 0 and s = eps2 > 0), which removes the scattered j-side updates and
// makes each row independent.
//
// Work decomposition: a CTA owns NT*IPT consecutive i-rows (IPT rows per
// thread held in registers, rows k*NT + tid so global loads and stores
// coalesce) and one contiguous range of j-tiles (split-j: blockIdx.y).  Each
// j-tile of TJ bodies is one contiguous AoS record block, moved into shared
// memory by a single bulk copy issued by thread 0 and double-buffered on two
// mbarriers; all threads read every record as a shared-memory broadcast.
// Partial sums of split s go to out + s*6*stride ([6][stride] doubles per
// split, rows indexed absolutely); a later pass adds the splits in a fixed
// order, so results are bitwise reproducible.
//
// Precision variants
//   FP64:  the whole pair computation in double.  1/sqrt(s) is seeded by the
//          MUFU single-precision rsqrt on (float)s and refined by one
//          third-order Householder step y(1 + r/2 + 3r^2/8), r = 1 - s y^2,
//          which takes the ~2^-22 seed error below double rounding.
//   Mixed: positions as float hi/lo pairs (hi = fl(x), lo = fl(x - hi)), the
//          separation formed as (xj_hi - xi_hi) + (xj_lo - xi_lo) (the hi
//          difference is exact for nearby bodies, so dx keeps float relative
//          accuracy however close two bodies are), velocities and the rest
//          of the pair math in float with the MUFU rsqrt, float partial sums
//          over one j-tile flushed into double accumulators after each tile.
#pragma once
#include <cstdint>

#include "tma.cuh"

namespace nbody {

// j-record, FP64 path: 64 bytes.
struct __align__(16) JBody64 {
  double x, y, z, m, vx, vy, vz, pad;
};

// j-record, mixed path: 48 bytes.
struct __align__(16) JBody32 {
  float xh, yh, zh, m;
  float xl, yl, zl, pad0;
  float vx, vy, vz, pad1;
};

// j-record, packed-pair mixed path: every field stored twice so that one
// 64-bit shared-memory word is a ready (value, value) operand of the f32x2
// instructions; 96 bytes.
struct __align__(16) JBodyX2 {
  float2 xh, yh, zh, m;
  float2 xl, yl, zl, vx;
  float2 vy, vz, pad0, pad1;
};

// Packed single precision (sm_100+): one instruction performs the operation
// on both halves of a 64-bit register pair.  Same FP32-pipe throughput per
// lane-op as scalar FMA, half the issue slots.
__device__ __forceinline__ uint64_t f2_add(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_sub(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ uint64_t f2_pack(float lo, float hi) {
  uint64_t d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
  return d;
}
__device__ __forceinline__ void f2_unpack(uint64_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

__device__ __forceinline__ float rcp_mufu(float s) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(s));
  return y;
}

__device__ __forceinline__ float rsqrt_mufu(float s) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(s));
  return y;
}

// 1/sqrt(s) in double: MUFU seed + one third-order Householder step
// (relative error ~1 ulp for s in the normal float range).
__device__ __forceinline__ double rsqrt_f64(double s) {
  const double y = static_cast<double>(rsqrt_mufu(__double2float_rn(s)));
  const double r = fma(-s, y * y, 1.0);
  const double p = fma(r, 0.375, 0.5);
  return fma(y * r, p, y);
}

// Bulk-copy pipeline over j-tiles [t_begin, t_begin + nt): calls
// consume(tile) for each tile with all threads; false if a wait timed out
// (status already reported, copies in flight drained).
template <class JB, int TJ, class Consume>
__device__ __forceinline__ bool run_j_tiles(const JB* __restrict__ jb, int t_begin, int nt,
                                            JB* buf, uint64_t* full, int* status,
                                            Consume&& consume) {
  constexpr uint32_t kBytes = TJ * sizeof(JB);
  static_assert(kBytes % 16 == 0, "bulk copies move multiples of 16 bytes");
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (tid == 0) {
    for (int b = 0; b < 2 && b < nt; ++b) {
      mbar_arrive_expect_tx(&full[b], kBytes);
      bulk_load(buf + b * TJ, jb + static_cast<size_t>(t_begin + b) * TJ, kBytes, &full[b]);
    }
  }
  for (int t = 0; t < nt; ++t) {
    const int b = t & 1;
    const uint32_t parity = (t >> 1) & 1;
    const bool ok = mbar_wait(&full[b], parity);
    if (ok) consume(buf + b * TJ);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        report_status(status, kKernelTimeout);
        (void)mbar_wait(&full[b], parity);
        if (t + 1 < nt) (void)mbar_wait(&full[b ^ 1], ((t + 1) >> 1) & 1);
      }
      return false;
    }
    if (tid == 0 && t + 2 < nt) {
      mbar_arrive_expect_tx(&full[b], kBytes);
      bulk_load(buf + b * TJ, jb + static_cast<size_t>(t_begin + t + 2) * TJ, kBytes, &full[b]);
    }
  }
  return true;
}

// Rows handled by this CTA and the j-tile range of its split.
struct PairArgs {
  int i_begin, i_end;      // rows [i_begin, i_end) are stored
  int n_rows_pad;          // rows are read (clamped) below this bound
  int n_tiles;             // j-tiles of TJ bodies in the (padded) system
  int tiles_per_split;
  double eps2;
  double* out;             // split s, field c, row i at out[(s*6 + c)*stride + i]
  size_t stride;
  int* status;
};

template <int NT, int IPT, int TJ, int JU = 2>
__global__ void __launch_bounds__(NT) pair_fp64_kernel(const JBody64* __restrict__ jb,
                                                       PairArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  JBody64* buf = reinterpret_cast<JBody64*>(smem_raw);
  __shared__ uint64_t full[2];

  const int tid = threadIdx.x;
  const int row0 = a.i_begin + blockIdx.x * (NT * IPT) + tid;
  const int split = blockIdx.y;
  const int t_begin = split * a.tiles_per_split;
  const int nt = max(0, min(a.tiles_per_split, a.n_tiles - t_begin));

  double xi[IPT], yi[IPT], zi[IPT], ui[IPT], vi[IPT], wi[IPT];
  double ax[IPT], ay[IPT], az[IPT], jx[IPT], jy[IPT], jz[IPT];
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const int i = min(row0 + k * NT, a.n_rows_pad - 1);
    const double2* r = reinterpret_cast<const double2*>(jb + i);
    const double2 p0 = r[0], p1 = r[1], p2 = r[2], p3 = r[3];
    xi[k] = p0.x; yi[k] = p0.y; zi[k] = p1.x;
    ui[k] = p2.x; vi[k] = p2.y; wi[k] = p3.x;
    ax[k] = ay[k] = az[k] = 0.0;
    jx[k] = jy[k] = jz[k] = 0.0;
  }
  const double eps2 = a.eps2;

  const bool ok = run_j_tiles<JBody64, TJ>(
      jb, t_begin, nt, buf, full, a.status, [&](const JBody64* tile) {
#pragma unroll JU
        for (int j = 0; j < TJ; ++j) {
          const double2* r = reinterpret_cast<const double2*>(tile + j);
          const double2 p0 = r[0], p1 = r[1], p2 = r[2], p3 = r[3];
          const double xj = p0.x, yj = p0.y, zj = p1.x, mj = p1.y;
          const double uj = p2.x, vj = p2.y, wj = p3.x;
#pragma unroll
          for (int k = 0; k < IPT; ++k) {
            const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
            const double du = uj - ui[k], dv = vj - vi[k], dw = wj - wi[k];
            const double s = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
            const double rv = fma(dx, du, fma(dy, dv, dz * dw));
            const double y = rsqrt_f64(s);
            const double y2 = y * y;
            const double q = mj * (y * y2);
            const double c = rv * (-3.0 * y2);
            ax[k] = fma(q, dx, ax[k]);
            ay[k] = fma(q, dy, ay[k]);
            az[k] = fma(q, dz, az[k]);
            jx[k] = fma(q, fma(c, dx, du), jx[k]);
            jy[k] = fma(q, fma(c, dy, dv), jy[k]);
            jz[k] = fma(q, fma(c, dz, dw), jz[k]);
          }
        }
      });
  if (!ok) return;

  double* out = a.out + static_cast<size_t>(split) * 6 * a.stride;
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const int i = row0 + k * NT;
    if (i < a.i_end) {
      out[0 * a.stride + i] = ax[k];
      out[1 * a.stride + i] = ay[k];
      out[2 * a.stride + i] = az[k];
      out[3 * a.stride + i] = jx[k];
      out[4 * a.stride + i] = jy[k];
      out[5 * a.stride + i] = jz[k];
    }
  }
}

template <int NT, int IPT, int TJ>
__global__ void __launch_bounds__(NT) pair_mixed_kernel(const JBody32* __restrict__ jb,
                                                        PairArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  JBody32* buf = reinterpret_cast<JBody32*>(smem_raw);
  __shared__ uint64_t full[2];

  const int tid = threadIdx.x;
  const int row0 = a.i_begin + blockIdx.x * (NT * IPT) + tid;
  const int split = blockIdx.y;
  const int t_begin = split * a.tiles_per_split;
  const int nt = max(0, min(a.tiles_per_split, a.n_tiles - t_begin));

  float xh[IPT], yh[IPT], zh[IPT], xl[IPT], yl[IPT], zl[IPT], ui[IPT], vi[IPT], wi[IPT];
  float fax[IPT], fay[IPT], faz[IPT], fjx[IPT], fjy[IPT], fjz[IPT];
  double ax[IPT], ay[IPT], az[IPT], jx[IPT], jy[IPT], jz[IPT];
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const int i = min(row0 + k * NT, a.n_rows_pad - 1);
    const float4* r = reinterpret_cast<const float4*>(jb + i);
    const float4 p0 = r[0], p1 = r[1], p2 = r[2];
    xh[k] = p0.x; yh[k] = p0.y; zh[k] = p0.z;
    xl[k] = p1.x; yl[k] = p1.y; zl[k] = p1.z;
    ui[k] = p2.x; vi[k] = p2.y; wi[k] = p2.z;
    ax[k] = ay[k] = az[k] = 0.0;
    jx[k] = jy[k] = jz[k] = 0.0;
  }
  const float eps2 = static_cast<float>(a.eps2);

  const bool ok = run_j_tiles<JBody32, TJ>(
      jb, t_begin, nt, buf, full, a.status, [&](const JBody32* tile) {
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
          fax[k] = fay[k] = faz[k] = 0.f;
          fjx[k] = fjy[k] = fjz[k] = 0.f;
        }
#pragma unroll 4
        for (int j = 0; j < TJ; ++j) {
          const float4* r = reinterpret_cast<const float4*>(tile + j);
          const float4 p0 = r[0], p1 = r[1], p2 = r[2];
#pragma unroll
          for (int k = 0; k < IPT; ++k) {
            const float dx = (p0.x - xh[k]) + (p1.x - xl[k]);
            const float dy = (p0.y - yh[k]) + (p1.y - yl[k]);
            const float dz = (p0.z - zh[k]) + (p1.z - zl[k]);
            const float du = p2.x - ui[k], dv = p2.y - vi[k], dw = p2.z - wi[k];
            const float s = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
            const float rv = fmaf(dx, du, fmaf(dy, dv, dz * dw));
            const float y = rsqrt_mufu(s);
            const float y2 = y * y;
            const float q = p0.w * (y * y2);
            const float c = rv * (-3.0f * y2);
            fax[k] = fmaf(q, dx, fax[k]);
            fay[k] = fmaf(q, dy, fay[k]);
            faz[k] = fmaf(q, dz, faz[k]);
            fjx[k] = fmaf(q, fmaf(c, dx, du), fjx[k]);
            fjy[k] = fmaf(q, fmaf(c, dy, dv), fjy[k]);
            fjz[k] = fmaf(q, fmaf(c, dz, dw), fjz[k]);
          }
        }
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
          ax[k] += fax[k]; ay[k] += fay[k]; az[k] += faz[k];
          jx[k] += fjx[k]; jy[k] += fjy[k]; jz[k] += fjz[k];
        }
      });
  if (!ok) return;

  double* out = a.out + static_cast<size_t>(split) * 6 * a.stride;
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const int i = row0 + k * NT;
    if (i < a.i_end) {
      out[0 * a.stride + i] = ax[k];
      out[1 * a.stride + i] = ay[k];
      out[2 * a.stride + i] = az[k];
      out[3 * a.stride + i] = jx[k];
      out[4 * a.stride + i] = jy[k];
      out[5 * a.stride + i] = jz[k];
    }
  }
}

// Mixed precision on packed pairs: i-rows (2p, 2p+1) of a thread share one
// 64-bit register per quantity, so each f32x2 instruction advances two
// interactions.  Same arithmetic as pair_mixed_kernel except that 1/s comes
// from the MUFU reciprocal (one FP32-pipe multiply fewer per interaction):
// y = rsqrt(s), y2 = rcp(s), q = m_j y y2, c = -3 (r.v) y2.
// ACC_SMEM = 1 keeps the per-row FP64 accumulators in shared memory
// ([6*IPT][NT] doubles, one column per thread) instead of registers, which
// frees 12 registers per row for more rows per thread; JU unrolls the j loop.
template <int NT, int IPT, int TJ, int ACC_SMEM = 0, int JU = 2>
__global__ void __launch_bounds__(NT) pair_mixed_x2_kernel(const JBodyX2* __restrict__ jb,
                                                           PairArgs a) {
  static_assert(IPT % 2 == 0, "rows are processed in pairs");
  constexpr int NP = IPT / 2;
  constexpr int NACC = ACC_SMEM ? 1 : IPT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  JBodyX2* buf = reinterpret_cast<JBodyX2*>(smem_raw);
  double* acc_sm = reinterpret_cast<double*>(smem_raw + 2 * TJ * sizeof(JBodyX2));
  __shared__ uint64_t full[2];

  const int tid = threadIdx.x;
  const int row0 = a.i_begin + blockIdx.x * (NT * IPT) + tid;
  const int split = blockIdx.y;
  const int t_begin = split * a.tiles_per_split;
  const int nt = max(0, min(a.tiles_per_split, a.n_tiles - t_begin));

  uint64_t xh[NP], yh[NP], zh[NP], xl[NP], yl[NP], zl[NP], ui[NP], vi[NP], wi[NP];
  uint64_t fax[NP], fay[NP], faz[NP], fjx[NP], fjy[NP], fjz[NP];
  double ax[NACC], ay[NACC], az[NACC], jx[NACC], jy[NACC], jz[NACC];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    const JBodyX2 b0 = jb[min(row0 + (2 * p) * NT, a.n_rows_pad - 1)];
    const JBodyX2 b1 = jb[min(row0 + (2 * p + 1) * NT, a.n_rows_pad - 1)];
    xh[p] = f2_pack(b0.xh.x, b1.xh.x); yh[p] = f2_pack(b0.yh.x, b1.yh.x); zh[p] = f2_pack(b0.zh.x, b1.zh.x);
    xl[p] = f2_pack(b0.xl.x, b1.xl.x); yl[p] = f2_pack(b0.yl.x, b1.yl.x); zl[p] = f2_pack(b0.zl.x, b1.zl.x);
    ui[p] = f2_pack(b0.vx.x, b1.vx.x); vi[p] = f2_pack(b0.vy.x, b1.vy.x); wi[p] = f2_pack(b0.vz.x, b1.vz.x);
  }
#pragma unroll
  for (int k = 0; k < NACC; ++k) {
    ax[k] = ay[k] = az[k] = 0.0;
    jx[k] = jy[k] = jz[k] = 0.0;
  }
  if (ACC_SMEM) {
#pragma unroll
    for (int r = 0; r < 6 * IPT; ++r) acc_sm[r * NT + tid] = 0.0;
  }
  const float e2f = static_cast<float>(a.eps2);
  const uint64_t eps2 = f2_pack(e2f, e2f);
  const uint64_t m3 = f2_pack(-3.0f, -3.0f);

  // adds the float pair (lo, hi) of field c, pair p into the FP64 accumulators
  auto flush = [&](int c, int p, uint64_t v) {
    float lo, hi;
    f2_unpack(v, lo, hi);
    if (ACC_SMEM) {
      acc_sm[(c * IPT + 2 * p) * NT + tid] += lo;
      acc_sm[(c * IPT + 2 * p + 1) * NT + tid] += hi;
    } else {
      double* f = c == 0 ? ax : c == 1 ? ay : c == 2 ? az : c == 3 ? jx : c == 4 ? jy : jz;
      f[(2 * p) % NACC] += lo;
      f[(2 * p + 1) % NACC] += hi;
    }
  };

  const bool ok = run_j_tiles<JBodyX2, TJ>(
      jb, t_begin, nt, buf, full, a.status, [&](const JBodyX2* tile) {
#pragma unroll
        for (int p = 0; p < NP; ++p) fax[p] = fay[p] = faz[p] = fjx[p] = fjy[p] = fjz[p] = 0ull;
#pragma unroll JU
        for (int j = 0; j < TJ; ++j) {
          const ulonglong2* r = reinterpret_cast<const ulonglong2*>(tile + j);
          const ulonglong2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4];
          // r0 = (xh, yh) r1 = (zh, m) r2 = (xl, yl) r3 = (zl, vx) r4 = (vy, vz)
#pragma unroll
          for (int p = 0; p < NP; ++p) {
            const uint64_t dx = f2_add(f2_sub(r0.x, xh[p]), f2_sub(r2.x, xl[p]));
            const uint64_t dy = f2_add(f2_sub(r0.y, yh[p]), f2_sub(r2.y, yl[p]));
            const uint64_t dz = f2_add(f2_sub(r1.x, zh[p]), f2_sub(r3.x, zl[p]));
            const uint64_t du = f2_sub(r3.y, ui[p]);
            const uint64_t dv = f2_sub(r4.x, vi[p]);
            const uint64_t dw = f2_sub(r4.y, wi[p]);
            const uint64_t s = f2_fma(dx, dx, f2_fma(dy, dy, f2_fma(dz, dz, eps2)));
            const uint64_t rv = f2_fma(dx, du, f2_fma(dy, dv, f2_mul(dz, dw)));
            float s0, s1;
            f2_unpack(s, s0, s1);
            const uint64_t y = f2_pack(rsqrt_mufu(s0), rsqrt_mufu(s1));
            const uint64_t y2 = f2_pack(rcp_mufu(s0), rcp_mufu(s1));
            const uint64_t q = f2_mul(r1.y, f2_mul(y, y2));
            const uint64_t c = f2_mul(rv, f2_mul(y2, m3));
            fax[p] = f2_fma(q, dx, fax[p]);
            fay[p] = f2_fma(q, dy, fay[p]);
            faz[p] = f2_fma(q, dz, faz[p]);
            fjx[p] = f2_fma(q, f2_fma(c, dx, du), fjx[p]);
            fjy[p] = f2_fma(q, f2_fma(c, dy, dv), fjy[p]);
            fjz[p] = f2_fma(q, f2_fma(c, dz, dw), fjz[p]);
          }
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          flush(0, p, fax[p]); flush(1, p, fay[p]); flush(2, p, faz[p]);
          flush(3, p, fjx[p]); flush(4, p, fjy[p]); flush(5, p, fjz[p]);
        }
      });
  if (!ok) return;

  double* out = a.out + static_cast<size_t>(split) * 6 * a.stride;
#pragma unroll
  for (int k = 0; k < IPT; ++k) {
    const int i = row0 + k * NT;
    if (i < a.i_end) {
      if (ACC_SMEM) {
#pragma unroll
        for (int c = 0; c < 6; ++c) out[c * a.stride + i] = acc_sm[(c * IPT + k) * NT + tid];
      } else {
        out[0 * a.stride + i] = ax[k % NACC];
        out[1 * a.stride + i] = ay[k % NACC];
        out[2 * a.stride + i] = az[k % NACC];
        out[3 * a.stride + i] = jx[k % NACC];
        out[4 * a.stride + i] = jy[k % NACC];
        out[5 * a.stride + i] = jz[k % NACC];
      }
    }
  }
}

}  // namespace nbody
