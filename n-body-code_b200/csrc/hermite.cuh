// O(N) Hermite-4 kernels (HBM-bound) and the FP64 energy diagnostic.
//
// Device state is SoA float64 with a padded row stride `ld` (a multiple of
// 256): X = [3][ld] positions, V = [3][ld] velocities, M = [ld] masses,
// D = [6][ld] current acc (0..2) and jerk (3..5).  Padding rows hold zero
// mass at the origin and are never integrated.
//
// Reference formulas (restated, src/nbody.cpp):
//   prediction      152-163  x += v dt + a dt^2/2 + j dt^3/6;  v += a dt + j dt^2/2
//   snapandcrackle  165-179  a2 = 2/dt^2 [-3(a - a1) - (2j + j1) dt]
//                            a3 = 6/dt^3 [ 2(a - a1) + (j + j1) dt]
//   correction      181-196  x += a2 dt^4/24 + a3 dt^5/120;  v += a2 dt^3/6 + a3 dt^4/24
//   updatedt        198-222  min_i sqrt(eta (|a||a2| + |j|^2) / (|j||a3| + |a2|^2)),
//                            with the pre-step a, j
//   initialdt       131-150  min_i eta0 |a| / |j|
#pragma once
#include <cstdint>

#include "pair.cuh"

namespace nbody {

// Step control block in device memory; updated by the last CTA of the
// corrector so that a captured step graph needs no host round trip.
struct StepCtl {
  double dt;                       // shared step in use
  double t;                        // model time
  double dt_crit;                  // last Aarseth / initial criterion
  unsigned long long crit_bits;    // atomicMin accumulator (+inf when idle)
  unsigned int blocks_done;        // last-block detection counter
  int adaptive;                    // 1: adopt dt_crit as the next dt
  long long steps;                 // completed steps
};

constexpr unsigned long long kPosInfBits = 0x7FF0000000000000ull;

// Deterministic block reductions for a fixed blockDim (multiple of 32, <= 1024).
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sh[k];
  __syncthreads();
  return r;  // valid in thread 0
}

__device__ __forceinline__ double block_min(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = __longlong_as_double(static_cast<long long>(kPosInfBits));
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = fmin(r, sh[k]);
  __syncthreads();
  return r;  // valid in thread 0
}

// Folds this CTA's criterion into ctl->crit_bits; the last CTA to finish
// publishes it and, for a step, advances t / steps (and dt when adaptive).
__device__ __forceinline__ void finish_criterion(StepCtl* ctl, double local, bool is_step,
                                                 double* sh) {
  __shared__ bool last;
  const double bmin = block_min(local, sh);
  if (threadIdx.x == 0) {
    // positive doubles order like their bit patterns; NaN (bits above +inf) never wins
    if (bmin >= 0.0) atomicMin(&ctl->crit_bits, static_cast<unsigned long long>(__double_as_longlong(bmin)));
    __threadfence();
    const unsigned prev = atomicAdd(&ctl->blocks_done, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const unsigned long long bits = atomicExch(&ctl->crit_bits, kPosInfBits);
    const double crit = __longlong_as_double(static_cast<long long>(bits));
    ctl->dt_crit = crit;
    if (is_step) {
      ctl->t += ctl->dt;
      ctl->steps += 1;
    }
    if (ctl->adaptive && bits < kPosInfBits) ctl->dt = crit;
    ctl->blocks_done = 0;
  }
}

__device__ __forceinline__ void split_hilo(double x, float& hi, float& lo) {
  hi = __double2float_rn(x);
  lo = __double2float_rn(x - static_cast<double>(hi));
}

__device__ __forceinline__ JBody32 make_jb32(double x, double y, double z, double m, double vx,
                                             double vy, double vz) {
  JBody32 b;
  split_hilo(x, b.xh, b.xl);
  split_hilo(y, b.yh, b.yl);
  split_hilo(z, b.zh, b.zl);
  b.m = __double2float_rn(m);
  b.vx = __double2float_rn(vx);
  b.vy = __double2float_rn(vy);
  b.vz = __double2float_rn(vz);
  b.pad0 = b.pad1 = 0.f;
  return b;
}

__device__ __forceinline__ JBodyX2 make_jbx2(double x, double y, double z, double m, double vx,
                                             double vy, double vz) {
  const JBody32 b = make_jb32(x, y, z, m, vx, vy, vz);
  JBodyX2 d;
  d.xh = make_float2(b.xh, b.xh); d.yh = make_float2(b.yh, b.yh); d.zh = make_float2(b.zh, b.zh);
  d.m = make_float2(b.m, b.m);
  d.xl = make_float2(b.xl, b.xl); d.yl = make_float2(b.yl, b.yl); d.zl = make_float2(b.zl, b.zl);
  d.vx = make_float2(b.vx, b.vx); d.vy = make_float2(b.vy, b.vy); d.vz = make_float2(b.vz, b.vz);
  d.pad0 = d.pad1 = make_float2(0.f, 0.f);
  return d;
}

// j-record formats of the pair kernels.
enum RecordFormat { kRecF64 = 0, kRecF32 = 1, kRecX2 = 2, kRecRel = 3 };

// Seven SoA input arrays (caller's or the engine's own).
struct SoA7 {
  const double *x, *y, *z, *m, *vx, *vy, *vz;
};
// Six SoA output arrays.
struct SoA6 {
  double *ax, *ay, *az, *jx, *jy, *jz;
};

// Writes j-records for rows [0, ld): rows < n from `in`, the rest as
// zero-mass bodies at rest at the origin (they contribute exactly zero).
static __global__ void pack_kernel(int n, int ld, SoA7 in, JBody64* __restrict__ jb64,
                            JBody32* __restrict__ jb32, JBodyX2* __restrict__ jbx2 = nullptr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ld) return;
  double x = 0, y = 0, z = 0, m = 0, vx = 0, vy = 0, vz = 0;
  if (i < n) {
    x = in.x[i]; y = in.y[i]; z = in.z[i]; m = in.m[i];
    vx = in.vx[i]; vy = in.vy[i]; vz = in.vz[i];
  }
  if (jb64) {
    JBody64 b;
    b.x = x; b.y = y; b.z = z; b.m = m;
    b.vx = vx; b.vy = vy; b.vz = vz; b.pad = 0.0;
    jb64[i] = b;
  }
  if (jb32) jb32[i] = make_jb32(x, y, z, m, vx, vy, vz);
  if (jbx2) jbx2[i] = make_jbx2(x, y, z, m, vx, vy, vz);
}

// Predictor: in place on X, V (rows < n) and writes the j-records of the
// predicted state (jb64 or jb32, whichever is non-null).
static __global__ void predict_kernel(int n, int ld, const StepCtl* __restrict__ ctl, double* __restrict__ X,
                               double* __restrict__ V, const double* __restrict__ M,
                               const double* __restrict__ D, JBody64* __restrict__ jb64,
                               JBody32* __restrict__ jb32, JBodyX2* __restrict__ jbx2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double dt = ctl->dt;
  const double h2 = 0.5 * dt * dt;
  const double h3 = dt * dt * dt * (1.0 / 6.0);
  double p[3], u[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double x = X[c * ld + i], v = V[c * ld + i];
    const double a = D[c * ld + i], j = D[(3 + c) * ld + i];
    p[c] = x + (v * dt + (a * h2 + j * h3));
    u[c] = v + (a * dt + j * h2);
    X[c * ld + i] = p[c];
    V[c * ld + i] = u[c];
  }
  const double m = M[i];
  if (jb64) {
    JBody64 b;
    b.x = p[0]; b.y = p[1]; b.z = p[2]; b.m = m;
    b.vx = u[0]; b.vy = u[1]; b.vz = u[2]; b.pad = 0.0;
    jb64[i] = b;
  }
  if (jb32) jb32[i] = make_jb32(p[0], p[1], p[2], m, u[0], u[1], u[2]);
  if (jbx2) jbx2[i] = make_jbx2(p[0], p[1], p[2], m, u[0], u[1], u[2]);
}

// sum[c] = sum over splits s = 0, 1, ..., S-1 (in that order) of
// P[s][c][i], for the six fields at once: one pass over the splits with
// several loads in flight, so a small system (few CTAs) is not bound by
// one load latency per split.
__device__ __forceinline__ void split_sums(const double* __restrict__ P, int ld, int S, int i,
                                           double sum[6]) {
#pragma unroll
  for (int c = 0; c < 6; ++c) sum[c] = 0.0;
#pragma unroll 4
  for (int s = 0; s < S; ++s) {
    const double* p = P + static_cast<size_t>(s) * 6 * ld + i;
#pragma unroll
    for (int c = 0; c < 6; ++c) sum[c] += p[static_cast<size_t>(c) * ld];
  }
}

// Corrector fused with the split-j reduction and the Aarseth criterion:
// a1/j1 = sum over S splits of P; snap/crackle; correct X, V; D <- a1/j1.
static __global__ void correct_kernel(int n, int ld, int S, const double* __restrict__ P,
                               double* __restrict__ X, double* __restrict__ V,
                               double* __restrict__ D, StepCtl* __restrict__ ctl, double eta) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double crit = __longlong_as_double(static_cast<long long>(kPosInfBits));
  if (i < n) {
    const double dt = ctl->dt;
    const double idt2 = 1.0 / (dt * dt);
    const double idt3 = idt2 / dt;
    const double dt3 = dt * dt * dt, dt4 = dt3 * dt, dt5 = dt4 * dt;
    double A2 = 0, J2 = 0, S2 = 0, C2 = 0;
    double sum[6];
    split_sums(P, ld, S, i, sum);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double a1 = sum[c], j1 = sum[3 + c];
      const double a = D[c * ld + i], j = D[(3 + c) * ld + i];
      const double da = a - a1;
      const double a2 = 2.0 * idt2 * (-3.0 * da - (2.0 * j + j1) * dt);
      const double a3 = 6.0 * idt3 * (2.0 * da + (j + j1) * dt);
      X[c * ld + i] += a2 * dt4 * (1.0 / 24.0) + a3 * dt5 * (1.0 / 120.0);
      V[c * ld + i] += a2 * dt3 * (1.0 / 6.0) + a3 * dt4 * (1.0 / 24.0);
      D[c * ld + i] = a1;
      D[(3 + c) * ld + i] = j1;
      A2 += a * a; J2 += j * j; S2 += a2 * a2; C2 += a3 * a3;
    }
    const double num = sqrt(A2) * sqrt(S2) + J2;
    const double den = sqrt(J2) * sqrt(C2) + S2;
    crit = sqrt(eta * num / den);
  }
  finish_criterion(ctl, crit, true, sh);
}

// out[c][i] = sum_s P[s][c][i] for rows [i_begin, i_end), splits in order.
// With a status word (callers that cannot read it back before using the
// outputs), a non-zero word - a pair kernel gave up a bounded wait - makes
// every output NaN instead.  With an index map, row i is written to
// out[c][index[i]] (partials kept in Hilbert order, outputs in the caller's
// body order).
static __global__ void reduce_splits_kernel(int i_begin, int i_end, int ld, int S,
                                     const double* __restrict__ P, SoA6 out,
                                     const int* __restrict__ status = nullptr,
                                     const int* __restrict__ index = nullptr) {
  const int i = i_begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= i_end) return;
  double* dst[6] = {out.ax, out.ay, out.az, out.jx, out.jy, out.jz};
  const int o = index ? index[i] : i;
  if (status && *status != 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c) dst[c][o] = __longlong_as_double(0x7FF8000000000000ll);
    return;
  }
  double sum[6];
  split_sums(P, ld, S, i, sum);
#pragma unroll
  for (int c = 0; c < 6; ++c) dst[c][o] = sum[c];
}

// One field of reduce_splits_kernel: out[index ? index[i] : i] = sum over
// the S splits of P[(s*6 + c)*ld + i], for the field c whose [ld] block of
// split 0 is Pc.  Same summation order as split_sums, so the same bits.
// Lets a caller copy each finished field to the host while the next one
// reduces.
static __global__ void reduce_split_field_kernel(int i_begin, int i_end, int ld, int S,
                                                 const double* __restrict__ Pc,
                                                 double* __restrict__ out,
                                                 const int* __restrict__ index = nullptr) {
  const int i = i_begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= i_end) return;
  double sum = 0.0;
#pragma unroll 8
  for (int s = 0; s < S; ++s) sum += Pc[static_cast<size_t>(s) * 6 * ld + i];
  out[index ? index[i] : i] = sum;
}

// Initial step criterion min_i eta0 |a| / |j| (published via ctl).
static __global__ void initialdt_kernel(int n, int ld, const double* __restrict__ D, StepCtl* ctl,
                                 double eta0) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double crit = __longlong_as_double(static_cast<long long>(kPosInfBits));
  if (i < n) {
    const double a0 = D[i], a1 = D[ld + i], a2 = D[2 * ld + i];
    const double j0 = D[3 * ld + i], j1 = D[4 * ld + i], j2 = D[5 * ld + i];
    crit = eta0 * sqrt(a0 * a0 + a1 * a1 + a2 * a2) / sqrt(j0 * j0 + j1 * j1 + j2 * j2);
  }
  finish_criterion(ctl, crit, false, sh);
}

// Per-CTA partial of 0.5 m v^2.
static __global__ void kinetic_kernel(int n, int ld, const double* __restrict__ V,
                               const double* __restrict__ M, double* __restrict__ partial) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (i < n) {
    const double u = V[i], v = V[ld + i], w = V[2 * ld + i];
    e = 0.5 * M[i] * (u * u + v * v + w * w);
  }
  const double b = block_sum(e, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// Potential: per row i, phi_i = sum_{j != i} m_j / sqrt(r^2 + eps2)
// (mode 0; CTA partial of m_i phi_i) or psi_i = sum_{j < i} 1/sqrt(.)
// (mode 1, the reference's printed potential sum_i sum_{j>i} m_j^2/r_ij
// regrouped by j; CTA partial of m_i^2 psi_i).  FP64, j-tiles staged
// through shared memory by the CTA's threads.  The j-range is split over
// gridDim.y (CTA (x, y) takes tiles [y*tps, (y+1)*tps)), so a system of few
// row blocks still fills the GPU; partial[y*gridDim.x + x] holds each CTA's
// sum and sum_partials_kernel adds them in that fixed order.
template <int NT>
static __global__ void __launch_bounds__(NT) potential_kernel(int n, int ld, double eps2, int mode,
                                                       const JBody64* __restrict__ jb,
                                                       double* __restrict__ partial) {
  __shared__ double4 tile[NT];
  __shared__ double sh[32];
  const int i = blockIdx.x * NT + threadIdx.x;
  const JBody64 bi = jb[min(i, ld - 1)];
  const int tiles = ld / NT, tps = (tiles + gridDim.y - 1) / gridDim.y;
  const int jb0 = blockIdx.y * tps * NT, jb1 = min(ld, (blockIdx.y + 1) * tps * NT);
  // four accumulators (partner k adds into acc[k % 4]), combined in a fixed
  // order: four independent add chains instead of one
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int j0 = jb0; j0 < jb1; j0 += NT) {
    const JBody64 bj = jb[j0 + threadIdx.x];
    tile[threadIdx.x] = make_double4(bj.x, bj.y, bj.z, bj.m);
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < NT; ++k) {
      const double4 p = tile[k];
      const int j = j0 + k;
      const double dx = p.x - bi.x, dy = p.y - bi.y, dz = p.z - bi.z;
      const double y = rsqrt_f64(fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2))));
      const bool take = mode == 0 ? (j != i) : (j < i);
      acc[k & 3] += take ? (mode == 0 ? p.w * y : y) : 0.0;
    }
    __syncthreads();
  }
  const double phi = (acc[0] + acc[1]) + (acc[2] + acc[3]);
  double e = 0.0;
  if (i < n) e = mode == 0 ? bi.m * phi : bi.m * bi.m * phi;
  const double b = block_sum(e, sh);
  if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = b;
}

// Sums `count` partials in a fixed order (one CTA).
static __global__ void sum_partials_kernel(int count, const double* __restrict__ partial,
                                    double* __restrict__ out) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int k = threadIdx.x; k < count; k += blockDim.x) v += partial[k];
  const double b = block_sum(v, sh);
  if (threadIdx.x == 0) *out = b;
}

}  // namespace nbody
