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
//          hardware rsqrt.approx.f64 and refined by one third-order
//          Householder step y(1 + r/2 + 3r^2/8), r = 1 - s y^2, which takes
//          the ~2^-20 seed error below double rounding.
//   Mixed: positions as float hi/lo pairs (hi = fl(x), lo = fl(x - hi)), the
//          separation formed as (xj_hi - xi_hi) + (xj_lo - xi_lo) (the hi
//          difference is exact for nearby bodies, so dx keeps float relative
//          accuracy however close two bodies are), velocities and the rest
//          of the pair math in float with the MUFU rsqrt, float partial sums
//          over one j-tile flushed into double accumulators after each tile.
//   Mixed, near/far tile-relative (default for large systems): bodies in
//          Hilbert order, j-tiles of float offsets from each tile's centre;
//          the separation costs one add per component for tiles far from a
//          warp's rows and is formed in double-single for near tiles
//          (RowsMixedNF below), so close pairs keep the hi/lo accuracy.
#pragma once
#include <cooperative_groups.h>
#include <cstdint>

#include "tma.cuh"

namespace nbody {

// Smallest softening the FP32 pair math accepts: every row's self pair is
// evaluated (r = 0, s = eps2) and its factor m s^(-3/2) must stay finite in
// float (1e36 x m here; 3.4e38 is the float limit), else 0 x inf = NaN.
constexpr double kMinEps2Mixed = 1e-24;

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

// j-record of the near/far tile-relative kernel: 96 bytes, every field twice.
// Record 0 of a tile is its header: x, y, z = the tile centre c; m = (lo_x,
// lo_y), vx = (lo_z, hi_x), vy = (hi_y, hi_z) = the tile's bounding box
// (rounded outward to float); vz = (R, 0) with R >= max |x_j - c| over the
// tile's bodies.  A body record holds x, y, z = -D_hi and xl, yl, zl = -D_lo,
// where (D_hi, D_lo) = ds_offset(c, x_hi, x_lo) is the double-single value of
// c - x, and its mass and velocity.
struct __align__(16) JBodyNF {
  float2 x, y, z, m;
  float2 vx, vy, vz, pad;
  float2 xl, yl, zl, pad2;
};

// FP64 source of the i-rows of the tile-relative kernels.
struct RowSrc {
  const double *x, *y, *z, *vx, *vy, *vz;
};

// (hi, lo) with hi + lo = c - (xh + xl) to about 2^-48 relative: the exact
// difference c - xh as a float sum s + e (Knuth's TwoSum), the low part xl
// folded into e, and the result renormalised by a second TwoSum.  Every
// operation rounds to nearest and none is contracted, so the records
// (rel_tile_nf_kernel) and the i-rows (RowsMixedNF) get bit-identical
// offsets for the same body and a pair's self term cancels exactly.
__device__ __forceinline__ void ds_offset(float c, float xh, float xl, float& hi, float& lo) {
  const float s = __fsub_rn(c, xh);
  const float bb = __fsub_rn(s, c);
  const float e = __fsub_rn(__fsub_rn(c, __fsub_rn(s, bb)), __fadd_rn(xh, bb));
  const float t = __fsub_rn(e, xl);
  hi = __fadd_rn(s, t);
  const float b2 = __fsub_rn(hi, s);
  lo = __fadd_rn(__fsub_rn(s, __fsub_rn(hi, b2)), __fsub_rn(t, b2));
}

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

// 1/sqrt(s) in double: the hardware approximation rsqrt.approx.f64 (measured
// max relative error 9.2e-7 on B200) refined by one third-order Householder
// step y (1 + r/2 + 3r^2/8), r = 1 - s y^2, whose error 5r^3/16 is below
// double rounding: measured <= 1 ulp for s in 2^[-99, 99].
__device__ __forceinline__ double rsqrt_f64(double s) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(s));
  const double r = fma(-s, y * y, 1.0);
  const double p = fma(r, 0.375, 0.5);
  return fma(y * r, p, y);
}

// ---------------------------------------------------------------------------
// j-tile pipeline
// ---------------------------------------------------------------------------
// Bulk copies of j-tiles into two shared-memory buffers, each tracked by an
// mbarrier transaction count.  `seq` counts tiles over the pipeline's whole
// life, so a persistent CTA can run it over many work items: tile g lands in
// buffer g & 1 and completes phase (g >> 1) & 1 of that buffer's barrier.
template <class JB, int TJ>
struct TilePipe {
  JB* buf;
  uint64_t* full;
  uint32_t seq;

  __device__ __forceinline__ void init(JB* b, uint64_t* f) {
    buf = b;
    full = f;
    seq = 0;
    if (threadIdx.x == 0) {
      mbar_init(&full[0], 1);
      mbar_init(&full[1], 1);
      mbar_init_fence();
    }
    __syncthreads();
  }

  // Streams tiles src[t*TJ ...] for t < nt through shared memory and calls
  // consume(tile) with all threads; false if a wait timed out (status
  // reported, copies in flight drained).
  template <class Consume>
  __device__ __forceinline__ bool run(const JB* __restrict__ src, int nt, int* status,
                                      Consume&& consume) {
    constexpr uint32_t kBytes = TJ * sizeof(JB);
    static_assert(kBytes % 16 == 0, "bulk copies move multiples of 16 bytes");
    const int tid = threadIdx.x;
    if (tid == 0)
      for (int t = 0; t < 2 && t < nt; ++t) {
        const uint32_t b = (seq + t) & 1u;
        mbar_arrive_expect_tx(&full[b], kBytes);
        bulk_load(buf + b * TJ, src + static_cast<size_t>(t) * TJ, kBytes, &full[b]);
      }
    for (int t = 0; t < nt; ++t) {
      const uint32_t g = seq + t;
      const uint32_t b = g & 1u, parity = (g >> 1) & 1u;
      const bool ok = mbar_wait(&full[b], parity);
      if (ok) consume(buf + b * TJ);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          report_status(status, kKernelTimeout);
          (void)mbar_wait(&full[b], parity);
          if (t + 1 < nt) (void)mbar_wait(&full[b ^ 1u], ((g + 1) >> 1) & 1u);
        }
        return false;
      }
      if (tid == 0 && t + 2 < nt) {
        mbar_arrive_expect_tx(&full[b], kBytes);
        bulk_load(buf + b * TJ, src + static_cast<size_t>(t + 2) * TJ, kBytes, &full[b]);
      }
    }
    seq += nt;
    return true;
  }
};

// ---------------------------------------------------------------------------
// Row blocks: the i-rows one CTA evaluates.  begin() loads the thread's rows
// (rows row, row + NT, ...; clamped to row_max for reading), consume() adds
// one j-tile, store() writes out[c*stride + i] for rows i < row_end.
// extra points at the kernel's shared memory past the two tile buffers.
// ---------------------------------------------------------------------------
template <int NT_, int IPT, int TJ_, int JU>
struct RowsFP64 {
  static constexpr int NT = NT_, ROWS = NT_ * IPT, TJ = TJ_;
  using JB = JBody64;
  static constexpr size_t kExtraSmem = 0;
  double xi[IPT], yi[IPT], zi[IPT], ui[IPT], vi[IPT], wi[IPT];
  double ax[IPT], ay[IPT], az[IPT], jx[IPT], jy[IPT], jz[IPT];
  double eps2;

  __device__ __forceinline__ void begin(const JB* __restrict__ jb, int row, int row_max, double e2,
                                        unsigned char*) {
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int i = min(row + k * NT, row_max);
      const double2* r = reinterpret_cast<const double2*>(jb + i);
      const double2 p0 = r[0], p1 = r[1], p2 = r[2], p3 = r[3];
      xi[k] = p0.x; yi[k] = p0.y; zi[k] = p1.x;
      ui[k] = p2.x; vi[k] = p2.y; wi[k] = p3.x;
      ax[k] = ay[k] = az[k] = 0.0;
      jx[k] = jy[k] = jz[k] = 0.0;
    }
    eps2 = e2;
  }

  __device__ __forceinline__ void consume(const JB* tile) {
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
  }

  __device__ __forceinline__ void store(double* out, size_t stride, int row, int row_end) const {
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int i = row + k * NT;
      if (i < row_end) {
        out[0 * stride + i] = ax[k];
        out[1 * stride + i] = ay[k];
        out[2 * stride + i] = az[k];
        out[3 * stride + i] = jx[k];
        out[4 * stride + i] = jy[k];
        out[5 * stride + i] = jz[k];
      }
    }
  }
};

template <int NT_, int IPT, int TJ_>
struct RowsMixed {
  static constexpr int NT = NT_, ROWS = NT_ * IPT, TJ = TJ_;
  using JB = JBody32;
  static constexpr size_t kExtraSmem = 0;
  float xh[IPT], yh[IPT], zh[IPT], xl[IPT], yl[IPT], zl[IPT], ui[IPT], vi[IPT], wi[IPT];
  double ax[IPT], ay[IPT], az[IPT], jx[IPT], jy[IPT], jz[IPT];
  float eps2;

  __device__ __forceinline__ void begin(const JB* __restrict__ jb, int row, int row_max, double e2,
                                        unsigned char*) {
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int i = min(row + k * NT, row_max);
      const float4* r = reinterpret_cast<const float4*>(jb + i);
      const float4 p0 = r[0], p1 = r[1], p2 = r[2];
      xh[k] = p0.x; yh[k] = p0.y; zh[k] = p0.z;
      xl[k] = p1.x; yl[k] = p1.y; zl[k] = p1.z;
      ui[k] = p2.x; vi[k] = p2.y; wi[k] = p2.z;
      ax[k] = ay[k] = az[k] = 0.0;
      jx[k] = jy[k] = jz[k] = 0.0;
    }
    eps2 = static_cast<float>(e2);
  }

  __device__ __forceinline__ void consume(const JB* tile) {
    float fax[IPT], fay[IPT], faz[IPT], fjx[IPT], fjy[IPT], fjz[IPT];
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
  }

  __device__ __forceinline__ void store(double* out, size_t stride, int row, int row_end) const {
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int i = row + k * NT;
      if (i < row_end) {
        out[0 * stride + i] = ax[k];
        out[1 * stride + i] = ay[k];
        out[2 * stride + i] = az[k];
        out[3 * stride + i] = jx[k];
        out[4 * stride + i] = jy[k];
        out[5 * stride + i] = jz[k];
      }
    }
  }
};

// Packed pairs: rows (2p, 2p+1) of a thread share one 64-bit register per
// quantity, so each f32x2 instruction advances two interactions.  Same
// arithmetic as RowsMixed except that 1/s comes from the MUFU reciprocal (one
// FP32-pipe multiply fewer per interaction): y = rsqrt(s), y2 = rcp(s),
// q = m_j y y2, c = -3 (r.v) y2.  ACC_SMEM = 1 keeps the FP64 accumulators in
// shared memory ([6*IPT][NT] doubles, one column per thread) instead of
// registers, which frees 12 registers per row; JU unrolls the j loop.
template <int NT_, int IPT, int TJ_, int ACC_SMEM, int JU>
struct RowsMixedX2 {
  static_assert(IPT % 2 == 0, "rows are processed in pairs");
  static constexpr int NT = NT_, ROWS = NT_ * IPT, TJ = TJ_, NP = IPT / 2;
  static constexpr int NACC = ACC_SMEM ? 1 : IPT;
  using JB = JBodyX2;
  static constexpr size_t kExtraSmem = ACC_SMEM ? sizeof(double) * 6 * IPT * NT_ : 0;
  uint64_t xh[NP], yh[NP], zh[NP], xl[NP], yl[NP], zl[NP], ui[NP], vi[NP], wi[NP];
  double ax[NACC], ay[NACC], az[NACC], jx[NACC], jy[NACC], jz[NACC];
  double* acc_sm;
  uint64_t eps2, m3;

  __device__ __forceinline__ void begin(const JB* __restrict__ jb, int row, int row_max, double e2,
                                        unsigned char* extra) {
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const JBodyX2 b0 = jb[min(row + (2 * p) * NT, row_max)];
      const JBodyX2 b1 = jb[min(row + (2 * p + 1) * NT, row_max)];
      xh[p] = f2_pack(b0.xh.x, b1.xh.x); yh[p] = f2_pack(b0.yh.x, b1.yh.x); zh[p] = f2_pack(b0.zh.x, b1.zh.x);
      xl[p] = f2_pack(b0.xl.x, b1.xl.x); yl[p] = f2_pack(b0.yl.x, b1.yl.x); zl[p] = f2_pack(b0.zl.x, b1.zl.x);
      ui[p] = f2_pack(b0.vx.x, b1.vx.x); vi[p] = f2_pack(b0.vy.x, b1.vy.x); wi[p] = f2_pack(b0.vz.x, b1.vz.x);
    }
    init_acc(e2, extra);
  }

  __device__ __forceinline__ void init_acc(double e2, unsigned char* extra) {
#pragma unroll
    for (int k = 0; k < NACC; ++k) {
      ax[k] = ay[k] = az[k] = 0.0;
      jx[k] = jy[k] = jz[k] = 0.0;
    }
    acc_sm = reinterpret_cast<double*>(extra);
    if (ACC_SMEM) {
#pragma unroll
      for (int r = 0; r < 6 * IPT; ++r) acc_sm[r * NT + threadIdx.x] = 0.0;
    }
    const float e2f = static_cast<float>(e2);
    eps2 = f2_pack(e2f, e2f);
    m3 = f2_pack(-3.0f, -3.0f);
  }

  // adds the float pair (lo, hi) of field c, pair p into the FP64 accumulators
  __device__ __forceinline__ void flush(int c, int p, uint64_t v) {
    float lo, hi;
    f2_unpack(v, lo, hi);
    if (ACC_SMEM) {
      acc_sm[(c * IPT + 2 * p) * NT + threadIdx.x] += lo;
      acc_sm[(c * IPT + 2 * p + 1) * NT + threadIdx.x] += hi;
    } else {
      double* f = c == 0 ? ax : c == 1 ? ay : c == 2 ? az : c == 3 ? jx : c == 4 ? jy : jz;
      f[(2 * p) % NACC] += lo;
      f[(2 * p + 1) % NACC] += hi;
    }
  }

  __device__ __forceinline__ void consume(const JB* tile) {
    uint64_t fax[NP], fay[NP], faz[NP], fjx[NP], fjy[NP], fjz[NP];
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
  }

  __device__ __forceinline__ void store(double* out, size_t stride, int row, int row_end) const {
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int i = row + k * NT;
      if (i < row_end) {
        if (ACC_SMEM) {
#pragma unroll
          for (int c = 0; c < 6; ++c) out[c * stride + i] = acc_sm[(c * IPT + k) * NT + threadIdx.x];
        } else {
          out[0 * stride + i] = ax[k % NACC];
          out[1 * stride + i] = ay[k % NACC];
          out[2 * stride + i] = az[k % NACC];
          out[3 * stride + i] = jx[k % NACC];
          out[4 * stride + i] = jy[k % NACC];
          out[5 * stride + i] = jz[k % NACC];
        }
      }
    }
  }
};

// The pair terms shared by the packed mixed kernels once the separation
// (dx, dy, dz) of rows (2p, 2p+1) is formed: mj = (m_j, m_j), the j-body's
// velocity, and the accumulators of this tile.
template <int NP>
__device__ __forceinline__ void pair_terms_x2(int p, uint64_t dx, uint64_t dy, uint64_t dz,
                                              uint64_t mj, uint64_t vxj, uint64_t vyj,
                                              uint64_t vzj, const uint64_t* ui, const uint64_t* vi,
                                              const uint64_t* wi, uint64_t eps2, uint64_t m3,
                                              uint64_t* fax, uint64_t* fay, uint64_t* faz,
                                              uint64_t* fjx, uint64_t* fjy, uint64_t* fjz) {
  const uint64_t du = f2_sub(vxj, ui[p]);
  const uint64_t dv = f2_sub(vyj, vi[p]);
  const uint64_t dw = f2_sub(vzj, wi[p]);
  const uint64_t s = f2_fma(dx, dx, f2_fma(dy, dy, f2_fma(dz, dz, eps2)));
  const uint64_t rv = f2_fma(dx, du, f2_fma(dy, dv, f2_mul(dz, dw)));
  float s0, s1;
  f2_unpack(s, s0, s1);
  const uint64_t y = f2_pack(rsqrt_mufu(s0), rsqrt_mufu(s1));
  const uint64_t y2 = f2_pack(rcp_mufu(s0), rcp_mufu(s1));
  const uint64_t q = f2_mul(mj, f2_mul(y, y2));
  const uint64_t c = f2_mul(rv, f2_mul(y2, m3));
  fax[p] = f2_fma(q, dx, fax[p]);
  fay[p] = f2_fma(q, dy, fay[p]);
  faz[p] = f2_fma(q, dz, faz[p]);
  fjx[p] = f2_fma(q, f2_fma(c, dx, du), fjx[p]);
  fjy[p] = f2_fma(q, f2_fma(c, dy, dv), fjy[p]);
  fjz[p] = f2_fma(q, f2_fma(c, dz, dw), fjz[p]);
}

// Near/far tile-relative rows (the default mixed kernel for large systems).
// The engine keeps its bodies in Hilbert order, and each warp takes 32 * IPT
// consecutive positions (row k of lane l is warp_row0 + 32 k + l), so a
// warp's rows occupy a compact region, whose bounding box begin_rows records.
// Each j-tile is then classified per warp (a warp-uniform branch):
//   far  - the boxes are separated by d > 0 with d >= R / 2 (R: the tile's
//          largest offset from its centre).  r_ij = D(x_i) + (-D_hi(x_j)) with
//          D(x_i) = fl(fl(c - x_hi) - x_lo): one add per component.  Its error
//          is at most about 2^-24 (3 |r| + 3 R) <= 9 * 2^-24 |r|, float
//          accuracy of the separation itself.
//   near - everything else (the warp's own tiles, its neighbours, and tiles
//          whose boxes are wide for their body count): the separation in
//          double-single, r = (D_hi(x_i) - D_hi(x_j)) + (D_lo(x_i) - D_lo(x_j))
//          with (D_hi, D_lo) = ds_offset(c, x_hi, x_lo), three adds per
//          component like the hi/lo kernel, so close pairs keep float
//          relative accuracy however close they are, and the self pair
//          cancels exactly.
// NEAR = 0 takes the far form for every tile (the plain tile-relative
// kernel, kept as a measured comparison); NEAR >= 1 is the near/far kernel
// with its near loop unrolled NEAR times.
template <int NT_, int IPT, int TJ_, int ACC_SMEM, int JU, int NEAR>
struct RowsMixedNF : RowsMixedX2<NT_, IPT, TJ_, ACC_SMEM, JU> {
  using Base = RowsMixedX2<NT_, IPT, TJ_, ACC_SMEM, JU>;
  using JB = JBodyNF;
  static constexpr int NP = Base::NP, NT = NT_, TJ = TJ_, kNear = NEAR;
  static constexpr size_t kExtraSmem = Base::kExtraSmem;
  float blo[3], bhi[3];  // bounding box of the warp's rows (same in every lane)
  int warp_row0;         // first row of this warp
  int near_tiles;

  __device__ __forceinline__ int row_of(int k) const { return warp_row0 + 32 * k + (threadIdx.x & 31); }

  // Rows of the CTA starting at cta_row0, read (clamped to row_max) from the
  // FP64 source; rows >= row_end are padding and stay out of the box.
  __device__ __forceinline__ void begin_rows(const RowSrc& src, int cta_row0, int row_max,
                                             int row_end, double e2, unsigned char* extra) {
    auto hl = [](double v, float& h, float& l) {
      h = static_cast<float>(v);
      l = static_cast<float>(v - static_cast<double>(h));
    };
    warp_row0 = cta_row0 + (threadIdx.x >> 5) * 32 * IPT;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int r0 = row_of(2 * p), r1 = row_of(2 * p + 1);
      const int i0 = min(r0, row_max), i1 = min(r1, row_max);
      const double x0[3] = {src.x[i0], src.y[i0], src.z[i0]};
      const double x1[3] = {src.x[i1], src.y[i1], src.z[i1]};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (r0 < row_end) { lo[k] = fmin(lo[k], x0[k]); hi[k] = fmax(hi[k], x0[k]); }
        if (r1 < row_end) { lo[k] = fmin(lo[k], x1[k]); hi[k] = fmax(hi[k], x1[k]); }
      }
      float h0, l0, h1, l1;
      hl(x0[0], h0, l0); hl(x1[0], h1, l1);
      this->xh[p] = f2_pack(h0, h1); this->xl[p] = f2_pack(l0, l1);
      hl(x0[1], h0, l0); hl(x1[1], h1, l1);
      this->yh[p] = f2_pack(h0, h1); this->yl[p] = f2_pack(l0, l1);
      hl(x0[2], h0, l0); hl(x1[2], h1, l1);
      this->zh[p] = f2_pack(h0, h1); this->zl[p] = f2_pack(l0, l1);
      this->ui[p] = f2_pack(static_cast<float>(src.vx[i0]), static_cast<float>(src.vx[i1]));
      this->vi[p] = f2_pack(static_cast<float>(src.vy[i0]), static_cast<float>(src.vy[i1]));
      this->wi[p] = f2_pack(static_cast<float>(src.vz[i0]), static_cast<float>(src.vz[i1]));
    }
    // the warp's box, rounded outward to float (no valid row: +inf/-inf,
    // which every tile is far from)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float l = __double2float_rd(lo[k]), h = __double2float_ru(hi[k]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        l = fminf(l, __shfl_xor_sync(0xffffffffu, l, o));
        h = fmaxf(h, __shfl_xor_sync(0xffffffffu, h, o));
      }
      blo[k] = l;
      bhi[k] = h;
    }
    near_tiles = 0;
    this->init_acc(e2, extra);
  }

  // Far: the boxes are apart by d > 0 with d^2 >= R^2 / 4.  The gaps are
  // computed from float boxes rounded outward, so d never exceeds the true
  // distance between any row and any body of the tile.
  __device__ __forceinline__ bool is_far(const JBodyNF& h) const {
    const float tlo[3] = {h.m.x, h.m.y, h.vx.x}, thi[3] = {h.vx.y, h.vy.x, h.vy.y};
    float d2 = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float g = fmaxf(0.f, fmaxf(__fsub_rd(blo[k], thi[k]), __fsub_rd(tlo[k], bhi[k])));
      d2 = __fmaf_rd(g, g, d2);
    }
    const float R = h.vz.x;
    return d2 > 0.f && d2 >= __fmul_ru(0.25f, __fmul_ru(R, R));
  }

  __device__ __forceinline__ void consume(const JB* tile) {
    const JBodyNF& h = tile[0];
    if (!NEAR || is_far(h)) {
      consume_far(tile, h);
    } else {
      ++near_tiles;
      consume_near(tile, h);
    }
  }

  __device__ __forceinline__ void consume_far(const JB* tile, const JBodyNF& h) {
    const uint64_t cx = f2_pack(h.x.x, h.x.x), cy = f2_pack(h.y.x, h.y.x), cz = f2_pack(h.z.x, h.z.x);
    uint64_t ox[NP], oy[NP], oz[NP];  // D(x_i) to float accuracy: fl(fl(c - x_hi) - x_lo)
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      ox[p] = f2_sub(f2_sub(cx, this->xh[p]), this->xl[p]);
      oy[p] = f2_sub(f2_sub(cy, this->yh[p]), this->yl[p]);
      oz[p] = f2_sub(f2_sub(cz, this->zh[p]), this->zl[p]);
    }
    uint64_t fax[NP], fay[NP], faz[NP], fjx[NP], fjy[NP], fjz[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) fax[p] = fay[p] = faz[p] = fjx[p] = fjy[p] = fjz[p] = 0ull;
    const uint64_t eps2 = this->eps2, m3 = this->m3;
#pragma unroll JU
    for (int j = 1; j <= TJ; ++j) {
      const ulonglong2* r = reinterpret_cast<const ulonglong2*>(tile + j);
      const ulonglong2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3];
      // r0 = (-Dx, -Dy) r1 = (-Dz, m) r2 = (vx, vy) r3 = (vz, pad)
#pragma unroll
      for (int p = 0; p < NP; ++p)
        pair_terms_x2<NP>(p, f2_add(r0.x, ox[p]), f2_add(r0.y, oy[p]), f2_add(r1.x, oz[p]), r1.y,
                          r2.x, r2.y, r3.x, this->ui, this->vi, this->wi, eps2, m3, fax, fay, faz,
                          fjx, fjy, fjz);
    }
    flush_all(fax, fay, faz, fjx, fjy, fjz);
  }

  __device__ __forceinline__ void consume_near(const JB* tile, const JBodyNF& h) {
    const float c[3] = {h.x.x, h.y.x, h.z.x};
    uint64_t oh[3][NP], ol[3][NP];  // (D_hi, D_lo)(x_i), bit-identical to the records'
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const uint64_t xs[3] = {this->xh[p], this->yh[p], this->zh[p]};
      const uint64_t ls[3] = {this->xl[p], this->yl[p], this->zl[p]};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        float h0, h1, l0, l1, dh0, dl0, dh1, dl1;
        f2_unpack(xs[k], h0, h1);
        f2_unpack(ls[k], l0, l1);
        ds_offset(c[k], h0, l0, dh0, dl0);
        ds_offset(c[k], h1, l1, dh1, dl1);
        oh[k][p] = f2_pack(dh0, dh1);
        ol[k][p] = f2_pack(dl0, dl1);
      }
    }
    uint64_t fax[NP], fay[NP], faz[NP], fjx[NP], fjy[NP], fjz[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) fax[p] = fay[p] = faz[p] = fjx[p] = fjy[p] = fjz[p] = 0ull;
    const uint64_t eps2 = this->eps2, m3 = this->m3;
#pragma unroll(NEAR > 1 ? NEAR : 1)
    for (int j = 1; j <= TJ; ++j) {
      const ulonglong2* r = reinterpret_cast<const ulonglong2*>(tile + j);
      const ulonglong2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4], r5 = r[5];
      // r4 = (-Dx_lo, -Dy_lo) r5 = (-Dz_lo, pad)
#pragma unroll
      for (int p = 0; p < NP; ++p)
        pair_terms_x2<NP>(p, f2_add(f2_add(r0.x, oh[0][p]), f2_add(r4.x, ol[0][p])),
                          f2_add(f2_add(r0.y, oh[1][p]), f2_add(r4.y, ol[1][p])),
                          f2_add(f2_add(r1.x, oh[2][p]), f2_add(r5.x, ol[2][p])), r1.y, r2.x, r2.y,
                          r3.x, this->ui, this->vi, this->wi, eps2, m3, fax, fay, faz, fjx, fjy,
                          fjz);
    }
    flush_all(fax, fay, faz, fjx, fjy, fjz);
  }

  __device__ __forceinline__ void flush_all(const uint64_t* fax, const uint64_t* fay,
                                            const uint64_t* faz, const uint64_t* fjx,
                                            const uint64_t* fjy, const uint64_t* fjz) {
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      this->flush(0, p, fax[p]); this->flush(1, p, fay[p]); this->flush(2, p, faz[p]);
      this->flush(3, p, fjx[p]); this->flush(4, p, fjy[p]); this->flush(5, p, fjz[p]);
    }
  }

  // out[c*stride + i] for this thread's rows i = row_of(k) < row_end.
  __device__ __forceinline__ void store(double* out, size_t stride, int row_end) const {
    constexpr int NACC = Base::NACC;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int i = row_of(k);
      if (i < row_end) {
        if (ACC_SMEM) {
#pragma unroll
          for (int c = 0; c < 6; ++c) out[c * stride + i] = this->acc_sm[(c * IPT + k) * NT + threadIdx.x];
        } else {
          out[0 * stride + i] = this->ax[k % NACC];
          out[1 * stride + i] = this->ay[k % NACC];
          out[2 * stride + i] = this->az[k % NACC];
          out[3 * stride + i] = this->jx[k % NACC];
          out[4 * stride + i] = this->jy[k % NACC];
          out[5 * stride + i] = this->jz[k % NACC];
        }
      }
    }
  }
};

// Dynamic shared memory of a row-block kernel: two tile buffers + extras.
template <class R>
constexpr size_t pair_smem_bytes() {
  return 2 * R::TJ * sizeof(typename R::JB) + R::kExtraSmem;
}

// ---------------------------------------------------------------------------
// One system: CTA (blockIdx.x, blockIdx.y) = (row block, j split).
// ---------------------------------------------------------------------------
struct PairArgs {
  int i_begin, i_end;      // rows [i_begin, i_end) are stored
  int n_rows_pad;          // rows are read (clamped) below this bound
  int n_tiles;             // j-tiles of TJ bodies in the (padded) system
  int tiles_per_split;
  double eps2;
  double* out;             // split s, field c, row i at out[(s*6 + c)*stride + i]
  size_t stride;
  int* status;
  RowSrc rows;             // i-row source of the tile-relative kernel (else unused)
  unsigned long long* near_count = nullptr;  // near/far kernel: += near tiles (nullable)
};

template <class R>
__device__ __forceinline__ void pair_system(const typename R::JB* __restrict__ jb,
                                            const PairArgs& a, unsigned char* smem,
                                            uint64_t* full) {
  using JB = typename R::JB;
  TilePipe<JB, R::TJ> pipe;
  pipe.init(reinterpret_cast<JB*>(smem), full);
  const int row = a.i_begin + blockIdx.x * R::ROWS + threadIdx.x;
  const int split = blockIdx.y;
  const int t_begin = split * a.tiles_per_split;
  const int nt = max(0, min(a.tiles_per_split, a.n_tiles - t_begin));
  R r;
  r.begin(jb, row, a.n_rows_pad - 1, a.eps2, smem + 2 * R::TJ * sizeof(JB));
  if (!pipe.run(jb + static_cast<size_t>(t_begin) * R::TJ, nt, a.status,
                [&](const JB* tile) { r.consume(tile); }))
    return;
  r.store(a.out + static_cast<size_t>(split) * 6 * a.stride, a.stride, row, a.i_end);
}

// MINB: minimum resident CTAs per SM requested from the register allocator.
template <int NT, int IPT, int TJ, int JU = 2, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) pair_fp64_kernel(const JBody64* __restrict__ jb,
                                                             PairArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[2];
  pair_system<RowsFP64<NT, IPT, TJ, JU>>(jb, a, smem_raw, full);
}

template <int NT, int IPT, int TJ>
__global__ void __launch_bounds__(NT) pair_mixed_kernel(const JBody32* __restrict__ jb,
                                                        PairArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[2];
  pair_system<RowsMixed<NT, IPT, TJ>>(jb, a, smem_raw, full);
}

template <int NT, int IPT, int TJ, int ACC_SMEM = 0, int JU = 2, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) pair_mixed_x2_kernel(const JBodyX2* __restrict__ jb,
                                                                 PairArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[2];
  pair_system<RowsMixedX2<NT, IPT, TJ, ACC_SMEM, JU>>(jb, a, smem_raw, full);
}

// Near/far tile-relative mixed kernel: tile t is TJ + 1 records at
// jt + t*(TJ + 1) (header first); i-rows (engine positions, Hilbert order) come
// from a.rows, clamped below a.n_rows_pad; rows >= a.i_end are not stored and
// stay out of the warps' bounding boxes.
template <int NT, int IPT, int TJ, int ACC_SMEM = 1, int JU = 1, int MINB = 1, int NEAR = 1>
__global__ void __launch_bounds__(NT, MINB) pair_mixed_nf_kernel(const JBodyNF* __restrict__ jt,
                                                                 PairArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[2];
  using R = RowsMixedNF<NT, IPT, TJ, ACC_SMEM, JU, NEAR>;
  constexpr int kRecs = TJ + 1;
  TilePipe<JBodyNF, kRecs> pipe;
  pipe.init(reinterpret_cast<JBodyNF*>(smem_raw), full);
  const int row0 = a.i_begin + blockIdx.x * R::ROWS;
  const int t_begin = blockIdx.y * a.tiles_per_split;
  const int nt = max(0, min(a.tiles_per_split, a.n_tiles - t_begin));
  R r;
  r.begin_rows(a.rows, row0, a.n_rows_pad - 1, a.i_end, a.eps2,
               smem_raw + 2 * kRecs * sizeof(JBodyNF));
  if (!pipe.run(jt + static_cast<size_t>(t_begin) * kRecs, nt, a.status,
                [&](const JBodyNF* tile) { r.consume(tile); }))
    return;
  r.store(a.out + static_cast<size_t>(blockIdx.y) * 6 * a.stride, a.stride, a.i_end);
  // near tiles of this launch, counted per warp (the unit that classifies)
  if (NEAR && a.near_count && (threadIdx.x & 31) == 0 && r.near_tiles)
    atomicAdd(a.near_count, static_cast<unsigned long long>(r.near_tiles));
}

// The near/far kernel on thread-block clusters of CL CTAs along the j-split
// dimension: the CTAs of a cluster share a row block and take consecutive
// j-ranges, then sum their FP64 accumulators (shared memory) through
// distributed shared memory, in rank order, and write one split partial per
// cluster (split index blockIdx.y / CL).  The corrector then reads S / CL
// partials instead of S.  Each CTA sums a 1/CL slice of the entries.  Every
// CTA reaches both cluster barriers: a timed-out tile wait sets the status
// word and ends only the tile loop, so no CTA leaves the others waiting.
template <int NT, int IPT, int TJ, int JU, int MINB, int NEAR, int CL>
__global__ void __cluster_dims__(1, CL, 1) __launch_bounds__(NT, MINB)
    pair_mixed_nf_cluster_kernel(const JBodyNF* __restrict__ jt, PairArgs a) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[2];
  using R = RowsMixedNF<NT, IPT, TJ, 1, JU, NEAR>;
  constexpr int kRecs = TJ + 1;
  TilePipe<JBodyNF, kRecs> pipe;
  pipe.init(reinterpret_cast<JBodyNF*>(smem_raw), full);
  const int row0 = a.i_begin + blockIdx.x * R::ROWS;
  const int t_begin = blockIdx.y * a.tiles_per_split;
  const int nt = max(0, min(a.tiles_per_split, a.n_tiles - t_begin));
  R r;
  r.begin_rows(a.rows, row0, a.n_rows_pad - 1, a.i_end, a.eps2,
               smem_raw + 2 * kRecs * sizeof(JBodyNF));
  const bool ok = pipe.run(jt + static_cast<size_t>(t_begin) * kRecs, nt, a.status,
                           [&](const JBodyNF* tile) { r.consume(tile); });
  cg::cluster_group cluster = cg::this_cluster();
  cluster.sync();  // every CTA's accumulators are final and visible to the cluster
  const unsigned q = cluster.block_rank();
  const double* acc[CL];
#pragma unroll
  for (int p = 0; p < CL; ++p) acc[p] = cluster.map_shared_rank(r.acc_sm, p);
  double* out = a.out + static_cast<size_t>(blockIdx.y / CL) * 6 * a.stride;
  constexpr int kEntries = 6 * IPT * NT;  // acc_sm[(c * IPT + k) * NT + thread]
  for (int e = static_cast<int>(q) * NT + threadIdx.x; e < kEntries; e += CL * NT) {
    double s = 0.0;
#pragma unroll
    for (int p = 0; p < CL; ++p) s += acc[p][e];
    const int c = e / (IPT * NT), k = (e / NT) % IPT, t = e % NT;
    const int i = row0 + (t >> 5) * 32 * IPT + 32 * k + (t & 31);  // RowsMixedNF::row_of
    if (i < a.i_end) out[static_cast<size_t>(c) * a.stride + i] = s;
  }
  cluster.sync();  // peers keep their shared memory until every slice is read
  if (NEAR && ok && a.near_count && (threadIdx.x & 31) == 0 && r.near_tiles)
    atomicAdd(a.near_count, static_cast<unsigned long long>(r.near_tiles));
}

// ---------------------------------------------------------------------------
// Ensemble: one persistent launch over a work list of (cluster, row block,
// j-tile range) items; CTAs take items from an atomic counter (zeroed before
// each launch) until the list is exhausted.
// ---------------------------------------------------------------------------
struct EnsItem {
  int jrow0;          // first padded row of the cluster (its j-records and rows)
  int row0;           // first i-row of the item, cluster-relative
  int rows_end;       // the cluster's bodies: rows >= rows_end are not stored
  int ld;             // padded rows of the cluster = stride of its partials
  int t_begin, nt;    // j-tile range, cluster-relative
  long long out_off;  // doubles from the partial-sum base to this split's [6][ld] block
  double eps2;
};

template <class R>
__device__ __forceinline__ void pair_ensemble(const typename R::JB* __restrict__ jb,
                                              const EnsItem* __restrict__ items, int n_items,
                                              unsigned int* counter, double* P, int* status,
                                              unsigned char* smem, uint64_t* full, int* s_item) {
  using JB = typename R::JB;
  TilePipe<JB, R::TJ> pipe;
  pipe.init(reinterpret_cast<JB*>(smem), full);
  for (;;) {
    if (threadIdx.x == 0) *s_item = static_cast<int>(atomicAdd(counter, 1u));
    __syncthreads();
    const int k = *s_item;
    __syncthreads();
    if (k >= n_items) return;
    const EnsItem it = items[k];
    const JB* cj = jb + it.jrow0;
    const int row = it.row0 + threadIdx.x;
    R r;
    r.begin(cj, row, it.ld - 1, it.eps2, smem + 2 * R::TJ * sizeof(JB));
    if (!pipe.run(cj + static_cast<size_t>(it.t_begin) * R::TJ, it.nt, status,
                  [&](const JB* tile) { r.consume(tile); }))
      return;
    r.store(P + it.out_off, static_cast<size_t>(it.ld), row, it.rows_end);
  }
}

// Near/far tile-relative ensemble: tiles of TJ + 1 records over the whole
// padded array (cluster segments are multiples of 256 rows, so a tile never
// spans two clusters); i-rows from the FP64 state `rows`, whose bodies each
// cluster keeps in Hilbert order within its segment.  R is a RowsMixedNF.
template <class R, int MINB = 1>
__global__ void __launch_bounds__(R::NT, MINB) ensemble_pair_nf_kernel(
    const JBodyNF* __restrict__ jt, const EnsItem* __restrict__ items, int n_items,
    unsigned int* counter, double* P, int* status, RowSrc rows) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[2];
  __shared__ int s_item;
  constexpr int kRecs = R::TJ + 1;
  TilePipe<JBodyNF, kRecs> pipe;
  pipe.init(reinterpret_cast<JBodyNF*>(smem_raw), full);
  for (;;) {
    if (threadIdx.x == 0) s_item = static_cast<int>(atomicAdd(counter, 1u));
    __syncthreads();
    const int k = s_item;
    __syncthreads();
    if (k >= n_items) return;
    const EnsItem it = items[k];
    const RowSrc src{rows.x + it.jrow0, rows.y + it.jrow0, rows.z + it.jrow0,
                     rows.vx + it.jrow0, rows.vy + it.jrow0, rows.vz + it.jrow0};
    R r;
    r.begin_rows(src, it.row0, it.ld - 1, it.rows_end, it.eps2,
                 smem_raw + 2 * kRecs * sizeof(JBodyNF));
    const JBodyNF* ct = jt + static_cast<size_t>(it.jrow0 / R::TJ + it.t_begin) * kRecs;
    if (!pipe.run(ct, it.nt, status, [&](const JBodyNF* tile) { r.consume(tile); })) return;
    r.store(P + it.out_off, static_cast<size_t>(it.ld), it.rows_end);
  }
}

template <class R>
__global__ void __launch_bounds__(R::NT) ensemble_pair_kernel(const typename R::JB* __restrict__ jb,
                                                              const EnsItem* __restrict__ items,
                                                              int n_items, unsigned int* counter,
                                                              double* P, int* status) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[2];
  __shared__ int s_item;
  pair_ensemble<R>(jb, items, n_items, counter, P, status, smem_raw, full, &s_item);
}

}  // namespace nbody
