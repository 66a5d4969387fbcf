// Reverse-mode gradients of a fixed-dt Hermite-4 trajectory.
//
// Step map (shared step h), per body, with the corrector written out:
//   predict   xp = x0 + h v0 + h^2/2 a0 + h^3/6 j0,   vp = v0 + h a0 + h^2/2 j0
//   evaluate  (a1, j1) = F(xp, vp, m)                      (the pair acc + jerk)
//   correct   x1 = xp - 0.15 h^2 (a0 - a1) - h^3 (7/60 j0 + 1/30 j1)
//             v1 = vp - 0.5  h   (a0 - a1) - h^2 (5/12 j0 + 1/12 j1)
// (the last two lines are a2 h^4/24 + a3 h^5/120 and a2 h^3/6 + a3 h^4/24
// with the reference's snap/crackle, src/nbody.cpp:165-196, expanded).  The
// state carried between steps is (x, v, a, j); the initial (a0, j0) is
// F(x_init, v_init, m).
//
// Backward: adjoints (xb, vb, ab, jb) of a step's outputs give those of its
// inputs through
//   pre   ab1 = 0.15 h^2 xb1 + 0.5 h vb1 + ab_out,  jb1 = -(h^3/30) xb1 - (h^2/12) vb1 + jb_out
//         ab0 = -0.15 h^2 xb1 - 0.5 h vb1,          jb0 = -(7 h^3/60) xb1 - (5 h^2/12) vb1
//   VJP   (xbp, vbp, mb) += F^T (ab1, jb1) at (xp, vp, m);  xbp, vbp start at xb1, vb1
//   post  xb0 = xbp, vb0 = h xbp + vbp,  ab0 += h^2/2 xbp + h vbp,  jb0 += h^3/6 xbp + h^2/2 vbp
// The forward keeps the state every `checkpoint_every` steps; the backward
// restores each segment's checkpoint, recomputes its steps keeping the
// predicted (xp, vp), and runs the reverse steps.  The pair VJP is FP64 for
// both precisions (for a mixed-precision forward it is the FP64 adjoint of
// the same trajectory).
//
// Pair VJP (gather form, no atomics).  For rows k, partners p, with
// r = x_p - x_k, u = v_p - v_k, s = r^2 + eps2, y2 = 1/s, q = s^(-3/2),
// w = r.u, c = -3 w y2, and the term T = m q (a.r + b.u + c b.r) that row k's
// acc/jerk adjoint (a, b) = (ab_k, jb_k) sees from partner p:
//   dT/dr = m q [a + c b - 3 y2 B u + (6 w y2^2 B - 3 y2 G) r],  dT/du = m q (b - 3 y2 B r),
//   dT/dm = q G,  with B = b.r, G = a.r + b.u + c B.
// Row k collects -dT_kp/dr (its own term, m = m_p) and +dT_pk/dr' (the
// partner's term, r' = -r, m = m_k), and dT_pk/dm_k for its mass.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "../../include/nbody_cuda.h"
#include "errors.h"
#include "hermite.cuh"
#include "pair.cuh"
#include "trace.h"

using namespace nbody;

namespace {

constexpr int kPad = 256;
constexpr int kBlock = 256;
constexpr int kTile = 128;

// j-record of the pair VJP: position, mass, velocity and the acc/jerk adjoints.
struct __align__(16) JAdj {
  double x, y, z, m, vx, vy, vz, ax, ay, az, bx, by, bz, pad0, pad1, pad2;
};

constexpr int kVjpNT = 128, kVjpTile = 64;

// Row block of the pair VJP: one row per thread.
struct RowsVJP {
  static constexpr int TJ = kVjpTile;
  using JB = JAdj;
  double x, y, z, m, u, v, w, ax, ay, az, bx, by, bz;
  double rpk[3], upk[3], rkp[3], ukp[3], mb;
  double eps2;
  int row;

  __device__ __forceinline__ void begin(const JB* __restrict__ jb, int r, int row_max, double e2,
                                        unsigned char*) {
    row = r;
    const JAdj o = jb[min(r, row_max)];
    x = o.x; y = o.y; z = o.z; m = o.m; u = o.vx; v = o.vy; w = o.vz;
    ax = o.ax; ay = o.ay; az = o.az; bx = o.bx; by = o.by; bz = o.bz;
    for (int c = 0; c < 3; ++c) rpk[c] = upk[c] = rkp[c] = ukp[c] = 0.0;
    mb = 0.0;
    eps2 = e2;
  }

  __device__ __forceinline__ void consume(const JB* tile, int tile_row0) {
    // Two partners per iteration.  The self pair (r = u = 0, s = eps2) has
    // finite terms; q = 0 removes them without a branch, which lets the
    // compiler interleave the two pairs (measured 6 % faster backward).
#pragma unroll 2
    for (int t = 0; t < TJ; ++t) {
      const JAdj p = tile[t];
      const bool self = tile_row0 + t == row;
      const double r0 = p.x - x, r1 = p.y - y, r2 = p.z - z;
      const double u0 = p.vx - u, u1 = p.vy - v, u2 = p.vz - w;
      const double s = fma(r0, r0, fma(r1, r1, fma(r2, r2, eps2)));
      const double yy = rsqrt_f64(s);
      const double y2 = yy * yy;
      const double q = self ? 0.0 : yy * y2;
      const double wr = fma(r0, u0, fma(r1, u1, r2 * u2));
      const double c = -3.0 * wr * y2;
      // own term (adjoints of row k, partner mass m_p)
      {
        const double B = bx * r0 + by * r1 + bz * r2;
        const double G = (ax * r0 + ay * r1 + az * r2) + (bx * u0 + by * u1 + bz * u2) + c * B;
        const double kr = 6.0 * wr * y2 * y2 * B - 3.0 * y2 * G;
        const double mq = p.m * q;
        rkp[0] += mq * (ax + c * bx - 3.0 * y2 * B * u0 + kr * r0);
        rkp[1] += mq * (ay + c * by - 3.0 * y2 * B * u1 + kr * r1);
        rkp[2] += mq * (az + c * bz - 3.0 * y2 * B * u2 + kr * r2);
        ukp[0] += mq * (bx - 3.0 * y2 * B * r0);
        ukp[1] += mq * (by - 3.0 * y2 * B * r1);
        ukp[2] += mq * (bz - 3.0 * y2 * B * r2);
      }
      // partner's term (adjoints of p, mass m_k applied at the end)
      {
        const double B = p.bx * r0 + p.by * r1 + p.bz * r2;
        const double G = -((p.ax * r0 + p.ay * r1 + p.az * r2) + (p.bx * u0 + p.by * u1 + p.bz * u2) + c * B);
        const double kr = 6.0 * wr * y2 * y2 * B + 3.0 * y2 * G;
        rpk[0] += q * (p.ax + c * p.bx - 3.0 * y2 * B * u0 + kr * r0);
        rpk[1] += q * (p.ay + c * p.by - 3.0 * y2 * B * u1 + kr * r1);
        rpk[2] += q * (p.az + c * p.bz - 3.0 * y2 * B * u2 + kr * r2);
        upk[0] += q * (p.bx - 3.0 * y2 * B * r0);
        upk[1] += q * (p.by - 3.0 * y2 * B * r1);
        upk[2] += q * (p.bz - 3.0 * y2 * B * r2);
        mb += q * G;
      }
    }
  }

  // out: [7][stride] = d(xbar) (3), d(vbar) (3), d(mbar)
  __device__ __forceinline__ void store(double* out, size_t stride, int row_end) const {
    if (row >= row_end) return;
    for (int c = 0; c < 3; ++c) {
      out[c * stride + row] = m * rpk[c] - rkp[c];
      out[(3 + c) * stride + row] = m * upk[c] - ukp[c];
    }
    out[6 * stride + row] = mb;
  }
};

__global__ void __launch_bounds__(kVjpNT) vjp_pair_kernel(const JAdj* __restrict__ jb, int n, int ld,
                                                          int tiles_per_split, double eps2,
                                                          double* __restrict__ P, int* status) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[2];
  TilePipe<JAdj, kVjpTile> pipe;
  pipe.init(reinterpret_cast<JAdj*>(smem_raw), full);
  const int n_tiles = ld / kVjpTile;
  const int split = blockIdx.y;
  const int t_begin = split * tiles_per_split;
  const int nt = max(0, min(tiles_per_split, n_tiles - t_begin));
  RowsVJP r;
  r.begin(jb, blockIdx.x * kVjpNT + threadIdx.x, ld - 1, eps2, nullptr);
  int tile_row0 = t_begin * kVjpTile;
  if (!pipe.run(jb + static_cast<size_t>(t_begin) * kVjpTile, nt, status, [&](const JAdj* tile) {
        r.consume(tile, tile_row0);
        tile_row0 += kVjpTile;
      }))
    return;
  r.store(P + static_cast<size_t>(split) * 7 * ld, ld, n);
}

// Packs the VJP records from a predicted state and the acc/jerk adjoints;
// rows >= n are zero (zero mass and zero adjoints contribute nothing).
__global__ void vjp_pack_kernel(int n, int ld, const double* __restrict__ XV, const double* __restrict__ M,
                                const double* __restrict__ AB, JAdj* __restrict__ jb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ld) return;
  JAdj o;
  const bool real = i < n;
  o.x = real ? XV[i] : 0; o.y = real ? XV[ld + i] : 0; o.z = real ? XV[2 * ld + i] : 0;
  o.vx = real ? XV[3 * ld + i] : 0; o.vy = real ? XV[4 * ld + i] : 0; o.vz = real ? XV[5 * ld + i] : 0;
  o.m = real ? M[i] : 0;
  o.ax = real ? AB[i] : 0; o.ay = real ? AB[ld + i] : 0; o.az = real ? AB[2 * ld + i] : 0;
  o.bx = real ? AB[3 * ld + i] : 0; o.by = real ? AB[4 * ld + i] : 0; o.bz = real ? AB[5 * ld + i] : 0;
  o.pad0 = o.pad1 = o.pad2 = 0;
  jb[i] = o;
}

// Adds the VJP split partials into xb/vb ([6][ld]) and mb.
__global__ void vjp_reduce_kernel(int n, int ld, int S, const double* __restrict__ P,
                                  double* __restrict__ XVB, double* __restrict__ MB) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < 7; ++c) {
    double v = 0.0;
    for (int s = 0; s < S; ++s) v += P[(static_cast<size_t>(s) * 7 + c) * ld + i];
    if (c < 6) XVB[c * ld + i] += v;
    else MB[i] += v;
  }
}

// Reverse corrector: ADJ = [xb(3) vb(3) ab(3) jb(3)] holds the adjoint of the
// step's outputs; writes ab1/jb1 into AB1 and the corrector part of ab0/jb0
// into ADJ's ab/jb slots (xb, vb stay as xbp, vbp).
__global__ void adj_pre_kernel(int n, int ld, double h, double* __restrict__ ADJ,
                               double* __restrict__ AB1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double h2 = h * h, h3 = h2 * h;
  for (int c = 0; c < 3; ++c) {
    const double xb = ADJ[c * ld + i], vb = ADJ[(3 + c) * ld + i];
    const double ab_out = ADJ[(6 + c) * ld + i], jb_out = ADJ[(9 + c) * ld + i];
    AB1[c * ld + i] = 0.15 * h2 * xb + 0.5 * h * vb + ab_out;
    AB1[(3 + c) * ld + i] = -(h3 / 30.0) * xb - (h2 / 12.0) * vb + jb_out;
    ADJ[(6 + c) * ld + i] = -0.15 * h2 * xb - 0.5 * h * vb;
    ADJ[(9 + c) * ld + i] = -(7.0 * h3 / 60.0) * xb - (5.0 * h2 / 12.0) * vb;
  }
}

// Reverse predictor: (xbp, vbp) -> (xb0, vb0), ab0/jb0 completed.
__global__ void adj_post_kernel(int n, int ld, double h, double* __restrict__ ADJ) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double h2 = h * h, h3 = h2 * h;
  for (int c = 0; c < 3; ++c) {
    const double xbp = ADJ[c * ld + i], vbp = ADJ[(3 + c) * ld + i];
    ADJ[(3 + c) * ld + i] = h * xbp + vbp;
    ADJ[(6 + c) * ld + i] += 0.5 * h2 * xbp + h * vbp;
    ADJ[(9 + c) * ld + i] += (h3 / 6.0) * xbp + 0.5 * h2 * vbp;
  }
}

#define AD_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return nbody_set_error(e_ == cudaErrorMemoryAllocation ? NBODY_ERR_OOM : NBODY_ERR_CUDA, \
                             "%s failed: %s", #call, cudaGetErrorString(e_));              \
  } while (0)
#define AD_TRY(expr)               \
  do {                             \
    nbody_status s_ = (expr);      \
    if (s_ != NBODY_OK) return s_; \
  } while (0)

using FwdFP64 = RowsFP64<128, 2, kTile, 1>;
using FwdFP64Small = RowsFP64<128, 1, kTile, 2>;  // n < kSmallN: twice the row blocks
constexpr int kSmallN = 32768;
using FwdMixed = RowsMixedX2<128, 4, kTile, 1, 1>;

template <class R>
__global__ void __launch_bounds__(R::NT) adj_pair_kernel(const typename R::JB* __restrict__ jb, PairArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[2];
  pair_system<R>(jb, a, smem_raw, full);
}

int splits_for(int sms, int row_blocks, int n_tiles, int ctas_per_sm) {
  const int target = sms * ctas_per_sm;
  return std::max(1, std::min(n_tiles, (target + row_blocks - 1) / row_blocks));
}

}  // namespace

struct nbody_adjoint {
  nbody_adjoint_config cfg{};
  int n = 0, ld = 0, sms = 0, nseg = 0;
  double* state = nullptr;  // [13][ld]: X V M D
  double *X = nullptr, *V = nullptr, *M = nullptr, *D = nullptr;
  double* ckpt = nullptr;   // [nseg][13][ld]
  double* segxv = nullptr;  // [checkpoint_every][6][ld] predicted states of a segment
  double* adj = nullptr;    // [12][ld] xb vb ab jb
  double* ab1 = nullptr;    // [6][ld]
  double* mb = nullptr;     // [ld]
  double* P = nullptr;      // forward partials [S][6][ld]
  double* Pv = nullptr;     // VJP partials [Sv][7][ld]
  JBody64* jb64 = nullptr;
  JBodyX2* jbx = nullptr;
  JAdj* jadj = nullptr;
  StepCtl* ctl = nullptr;
  int* status = nullptr;
  int S = 1, Sv = 1;
  bool have_forward = false;
};

namespace {

nbody_status fwd_eval(nbody_adjoint* a, cudaStream_t st) {
  const bool fp64 = a->cfg.precision == NBODY_FP64;
  const size_t ld = a->ld;
  PairArgs pa;
  pa.i_begin = 0;
  pa.i_end = a->n;
  pa.n_rows_pad = a->ld;
  pa.n_tiles = a->ld / kTile;
  pa.tiles_per_split = (pa.n_tiles + a->S - 1) / a->S;
  pa.eps2 = a->cfg.eps2;
  pa.out = a->P;
  pa.stride = ld;
  pa.status = a->status;
  if (fp64 && a->n < kSmallN) {
    const dim3 grid((a->n + FwdFP64Small::ROWS - 1) / FwdFP64Small::ROWS, a->S);
    adj_pair_kernel<FwdFP64Small><<<grid, FwdFP64Small::NT, pair_smem_bytes<FwdFP64Small>(), st>>>(
        a->jb64, pa);
  } else if (fp64) {
    const dim3 grid((a->n + FwdFP64::ROWS - 1) / FwdFP64::ROWS, a->S);
    adj_pair_kernel<FwdFP64><<<grid, FwdFP64::NT, pair_smem_bytes<FwdFP64>(), st>>>(a->jb64, pa);
  } else {
    const dim3 grid((a->n + FwdMixed::ROWS - 1) / FwdMixed::ROWS, a->S);
    adj_pair_kernel<FwdMixed><<<grid, FwdMixed::NT, pair_smem_bytes<FwdMixed>(), st>>>(a->jbx, pa);
  }
  AD_CUDA(cudaGetLastError());
  return NBODY_OK;
}

nbody_status fwd_initial(nbody_adjoint* a, cudaStream_t st) {
  const bool fp64 = a->cfg.precision == NBODY_FP64;
  const size_t ld = a->ld;
  SoA7 in{a->X, a->X + ld, a->X + 2 * ld, a->M, a->V, a->V + ld, a->V + 2 * ld};
  pack_kernel<<<(a->ld + kBlock - 1) / kBlock, kBlock, 0, st>>>(a->n, a->ld, in, fp64 ? a->jb64 : nullptr,
                                                               nullptr, fp64 ? nullptr : a->jbx);
  AD_TRY(fwd_eval(a, st));
  double* D = a->D;
  reduce_splits_kernel<<<(a->n + kBlock - 1) / kBlock, kBlock, 0, st>>>(
      0, a->n, a->ld, a->S, a->P, SoA6{D, D + ld, D + 2 * ld, D + 3 * ld, D + 4 * ld, D + 5 * ld});
  AD_CUDA(cudaGetLastError());
  return NBODY_OK;
}

// One Hermite step; if xp_out, the predicted X/V ([6][ld]) are copied there.
nbody_status fwd_step(nbody_adjoint* a, cudaStream_t st, double* xp_out) {
  const bool fp64 = a->cfg.precision == NBODY_FP64;
  predict_kernel<<<(a->n + kBlock - 1) / kBlock, kBlock, 0, st>>>(
      a->n, a->ld, a->ctl, a->X, a->V, a->M, a->D, fp64 ? a->jb64 : nullptr, nullptr,
      fp64 ? nullptr : a->jbx);
  if (xp_out)
    AD_CUDA(cudaMemcpyAsync(xp_out, a->X, sizeof(double) * 6 * a->ld, cudaMemcpyDeviceToDevice, st));
  AD_TRY(fwd_eval(a, st));
  correct_kernel<<<(a->n + kBlock - 1) / kBlock, kBlock, 0, st>>>(a->n, a->ld, a->S, a->P, a->X, a->V,
                                                                 a->D, a->ctl, 1.0);
  AD_CUDA(cudaGetLastError());
  return NBODY_OK;
}

// (xb, vb, mb) += VJP of the pair acc/jerk at state XV ([6][ld]) with
// acc/jerk adjoints AB ([6][ld]).
nbody_status vjp(nbody_adjoint* a, cudaStream_t st, const double* XV, const double* AB) {
  vjp_pack_kernel<<<(a->ld + kBlock - 1) / kBlock, kBlock, 0, st>>>(a->n, a->ld, XV, a->M, AB, a->jadj);
  const int n_tiles = a->ld / kVjpTile;
  const int tps = (n_tiles + a->Sv - 1) / a->Sv;
  const dim3 grid((a->n + kVjpNT - 1) / kVjpNT, a->Sv);
  vjp_pair_kernel<<<grid, kVjpNT, 2 * kVjpTile * sizeof(JAdj), st>>>(a->jadj, a->n, a->ld, tps,
                                                                    a->cfg.eps2, a->Pv, a->status);
  vjp_reduce_kernel<<<(a->n + kBlock - 1) / kBlock, kBlock, 0, st>>>(a->n, a->ld, a->Sv, a->Pv, a->adj, a->mb);
  AD_CUDA(cudaGetLastError());
  return NBODY_OK;
}

nbody_status set_ctl(nbody_adjoint* a, cudaStream_t st) {
  StepCtl c{};
  c.dt = a->cfg.dt;
  c.crit_bits = kPosInfBits;
  c.adaptive = 0;
  AD_CUDA(cudaMemcpyAsync(a->ctl, &c, sizeof c, cudaMemcpyHostToDevice, st));
  return NBODY_OK;
}

nbody_status check_status(nbody_adjoint* a, cudaStream_t st) {
  int h = 0;
  AD_CUDA(cudaMemcpyAsync(&h, a->status, sizeof h, cudaMemcpyDeviceToHost, st));
  AD_CUDA(cudaStreamSynchronize(st));
  if (h) {
    cudaMemsetAsync(a->status, 0, sizeof(int), st);
    return nbody_set_error(NBODY_ERR_TIMEOUT, "an adjoint pair-kernel wait exceeded its limit");
  }
  return NBODY_OK;
}

}  // namespace

extern "C" {

nbody_status nbody_adjoint_destroy(nbody_adjoint* a) {
  if (!a) return NBODY_OK;
  cudaSetDevice(a->cfg.device);
  cudaDeviceSynchronize();
  void* bufs[] = {a->state, a->ckpt, a->segxv, a->adj, a->ab1, a->mb, a->P, a->Pv,
                  a->jb64, a->jbx, a->jadj, a->ctl, a->status};
  for (void* p : bufs) cudaFree(p);
  delete a;
  return NBODY_OK;
}

nbody_status nbody_adjoint_create(nbody_adjoint** out, const nbody_adjoint_config* cfg) {
  if (!out || !cfg) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (cfg->n < 1 || cfg->n > (1 << 22)) return nbody_set_error(NBODY_ERR_INVALID_ARG, "n = %d", cfg->n);
  if (!(cfg->eps2 >= 1e-30 && cfg->eps2 <= 1e30)) return nbody_set_error(NBODY_ERR_INVALID_ARG, "eps2 = %g", cfg->eps2);
  if (!(cfg->dt > 0)) return nbody_set_error(NBODY_ERR_INVALID_ARG, "dt must be > 0 (fixed step)");
  if (cfg->nsteps < 0 || cfg->checkpoint_every < 1)
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "nsteps = %d, checkpoint_every = %d", cfg->nsteps, cfg->checkpoint_every);
  if (cfg->precision != NBODY_FP64 && cfg->precision != NBODY_MIXED)
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "precision = %d", cfg->precision);
  if (cfg->precision == NBODY_MIXED && cfg->eps2 < kMinEps2Mixed)
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "eps2 = %g below %g (mixed precision)", cfg->eps2,
                           kMinEps2Mixed);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return nbody_set_error(NBODY_ERR_NO_DEVICE, "no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev) return nbody_set_error(NBODY_ERR_INVALID_ARG, "device %d", cfg->device);
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, cfg->device);
  if (major != 10) return nbody_set_error(NBODY_ERR_NO_DEVICE, "device %d is not sm_100", cfg->device);
  AD_CUDA(cudaSetDevice(cfg->device));
  std::unique_ptr<nbody_adjoint> a(new nbody_adjoint);
  a->cfg = *cfg;
  a->n = cfg->n;
  a->ld = (cfg->n + kPad - 1) / kPad * kPad;
  a->nseg = std::max(1, (cfg->nsteps + cfg->checkpoint_every - 1) / cfg->checkpoint_every);
  cudaDeviceGetAttribute(&a->sms, cudaDevAttrMultiProcessorCount, cfg->device);
  const int rows_fwd = cfg->precision == NBODY_FP64
                           ? (cfg->n < kSmallN ? FwdFP64Small::ROWS : FwdFP64::ROWS)
                           : FwdMixed::ROWS;
  // forward: small systems take as many j-splits as the wave allows (the
  // pair pass is latency-bound there); VJP: about 4 CTAs per SM
  a->S = splits_for(a->sms, (a->n + rows_fwd - 1) / rows_fwd, a->ld / kTile, 8);
  a->Sv = splits_for(a->sms, (a->n + kVjpNT - 1) / kVjpNT, a->ld / kVjpTile, 4);
  nbody_adjoint* r = a.get();
  auto body = [&]() -> nbody_status {
    const size_t ld = r->ld;
    AD_CUDA(cudaMalloc(&r->state, sizeof(double) * 13 * ld));
    AD_CUDA(cudaMemset(r->state, 0, sizeof(double) * 13 * ld));
    r->X = r->state;
    r->V = r->state + 3 * ld;
    r->M = r->state + 6 * ld;
    r->D = r->state + 7 * ld;
    AD_CUDA(cudaMalloc(&r->ckpt, sizeof(double) * 13 * ld * r->nseg));
    AD_CUDA(cudaMalloc(&r->segxv, sizeof(double) * 6 * ld * cfg->checkpoint_every));
    AD_CUDA(cudaMalloc(&r->adj, sizeof(double) * 12 * ld));
    AD_CUDA(cudaMalloc(&r->ab1, sizeof(double) * 6 * ld));
    AD_CUDA(cudaMalloc(&r->mb, sizeof(double) * ld));
    AD_CUDA(cudaMalloc(&r->P, sizeof(double) * 6 * ld * r->S));
    AD_CUDA(cudaMalloc(&r->Pv, sizeof(double) * 7 * ld * r->Sv));
    AD_CUDA(cudaMalloc(&r->jb64, sizeof(JBody64) * ld));
    AD_CUDA(cudaMalloc(&r->jbx, sizeof(JBodyX2) * ld));
    AD_CUDA(cudaMalloc(&r->jadj, sizeof(JAdj) * ld));
    AD_CUDA(cudaMalloc(&r->ctl, sizeof(StepCtl)));
    AD_CUDA(cudaMalloc(&r->status, sizeof(int)));
    AD_CUDA(cudaMemset(r->status, 0, sizeof(int)));
    AD_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(&adj_pair_kernel<FwdMixed>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(pair_smem_bytes<FwdMixed>())));
    AD_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(&adj_pair_kernel<FwdFP64>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(pair_smem_bytes<FwdFP64>())));
    AD_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(&adj_pair_kernel<FwdFP64Small>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(pair_smem_bytes<FwdFP64Small>())));
    AD_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(&vjp_pair_kernel),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(2 * kVjpTile * sizeof(JAdj))));
    return NBODY_OK;
  };
  nbody_status s = body();
  if (s != NBODY_OK) {
    nbody_adjoint_destroy(a.release());
    return s;
  }
  *out = a.release();
  return NBODY_OK;
}

nbody_status nbody_adjoint_forward(nbody_adjoint* a, const double* x, const double* y, const double* z,
                                   const double* m, const double* vx, const double* vy,
                                   const double* vz, double* x1, double* y1, double* z1, double* vx1,
                                   double* vy1, double* vz1, void* stream) {
  TraceRange trace_("nbody_adjoint_forward");
  if (!a) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null adjoint");
  const void* ptrs[13] = {x, y, z, m, vx, vy, vz, x1, y1, z1, vx1, vy1, vz1};
  for (auto p : ptrs)
    if (!p) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null device array");
  AD_CUDA(cudaSetDevice(a->cfg.device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t ld = a->ld, b = sizeof(double) * a->n;
  AD_CUDA(cudaMemsetAsync(a->state, 0, sizeof(double) * 13 * ld, st));
  const double* src[7] = {x, y, z, vx, vy, vz, m};
  double* dst[7] = {a->X, a->X + ld, a->X + 2 * ld, a->V, a->V + ld, a->V + 2 * ld, a->M};
  for (int k = 0; k < 7; ++k) AD_CUDA(cudaMemcpyAsync(dst[k], src[k], b, cudaMemcpyDeviceToDevice, st));
  AD_TRY(set_ctl(a, st));
  AD_TRY(fwd_initial(a, st));
  const int K = a->cfg.checkpoint_every;
  for (int s = 0; s < a->cfg.nsteps; ++s) {
    if (s % K == 0)
      AD_CUDA(cudaMemcpyAsync(a->ckpt + static_cast<size_t>(s / K) * 13 * ld, a->state,
                              sizeof(double) * 13 * ld, cudaMemcpyDeviceToDevice, st));
    AD_TRY(fwd_step(a, st, nullptr));
  }
  if (a->cfg.nsteps == 0)
    AD_CUDA(cudaMemcpyAsync(a->ckpt, a->state, sizeof(double) * 13 * ld, cudaMemcpyDeviceToDevice, st));
  double* outs[6] = {x1, y1, z1, vx1, vy1, vz1};
  const double* res[6] = {a->X, a->X + ld, a->X + 2 * ld, a->V, a->V + ld, a->V + 2 * ld};
  for (int k = 0; k < 6; ++k) AD_CUDA(cudaMemcpyAsync(outs[k], res[k], b, cudaMemcpyDeviceToDevice, st));
  a->have_forward = true;
  return check_status(a, st);
}

nbody_status nbody_adjoint_backward(nbody_adjoint* a, const double* gx, const double* gy,
                                    const double* gz, const double* gvx, const double* gvy,
                                    const double* gvz, double* gx0, double* gy0, double* gz0,
                                    double* gvx0, double* gvy0, double* gvz0, double* gm,
                                    void* stream) {
  TraceRange trace_("nbody_adjoint_backward");
  if (!a) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null adjoint");
  if (!a->have_forward) return nbody_set_error(NBODY_ERR_STATE, "backward before forward");
  const void* ptrs[13] = {gx, gy, gz, gvx, gvy, gvz, gx0, gy0, gz0, gvx0, gvy0, gvz0, gm};
  for (auto p : ptrs)
    if (!p) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null device array");
  AD_CUDA(cudaSetDevice(a->cfg.device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t ld = a->ld, b = sizeof(double) * a->n;
  const double h = a->cfg.dt;
  const int K = a->cfg.checkpoint_every, NS = a->cfg.nsteps;
  AD_CUDA(cudaMemsetAsync(a->adj, 0, sizeof(double) * 12 * ld, st));
  AD_CUDA(cudaMemsetAsync(a->mb, 0, sizeof(double) * ld, st));
  const double* g[6] = {gx, gy, gz, gvx, gvy, gvz};
  for (int k = 0; k < 6; ++k) AD_CUDA(cudaMemcpyAsync(a->adj + k * ld, g[k], b, cudaMemcpyDeviceToDevice, st));
  AD_TRY(set_ctl(a, st));
  const int nb = (a->n + kBlock - 1) / kBlock;
  for (int seg = a->nseg - 1; seg >= 0; --seg) {
    const int s0 = seg * K, s1 = std::min(NS, s0 + K);
    if (s1 <= s0) continue;
    AD_CUDA(cudaMemcpyAsync(a->state, a->ckpt + static_cast<size_t>(seg) * 13 * ld,
                            sizeof(double) * 13 * ld, cudaMemcpyDeviceToDevice, st));
    for (int s = s0; s < s1; ++s) AD_TRY(fwd_step(a, st, a->segxv + static_cast<size_t>(s - s0) * 6 * ld));
    for (int s = s1 - 1; s >= s0; --s) {
      adj_pre_kernel<<<nb, kBlock, 0, st>>>(a->n, a->ld, h, a->adj, a->ab1);
      AD_TRY(vjp(a, st, a->segxv + static_cast<size_t>(s - s0) * 6 * ld, a->ab1));
      adj_post_kernel<<<nb, kBlock, 0, st>>>(a->n, a->ld, h, a->adj);
      AD_CUDA(cudaGetLastError());
    }
  }
  // the initial acc/jerk: (a0, j0) = F(x_init, v_init, m), x_init in checkpoint 0
  AD_TRY(vjp(a, st, a->ckpt, a->adj + 6 * ld));
  double* outs[7] = {gx0, gy0, gz0, gvx0, gvy0, gvz0, gm};
  for (int k = 0; k < 6; ++k) AD_CUDA(cudaMemcpyAsync(outs[k], a->adj + k * ld, b, cudaMemcpyDeviceToDevice, st));
  AD_CUDA(cudaMemcpyAsync(gm, a->mb, b, cudaMemcpyDeviceToDevice, st));
  return check_status(a, st);
}

nbody_status nbody_adjoint_vjp_acc_jerk(nbody_adjoint* a, const double* x, const double* y,
                                        const double* z, const double* m, const double* vx,
                                        const double* vy, const double* vz, const double* abx,
                                        const double* aby, const double* abz, const double* jbx,
                                        const double* jby, const double* jbz, double* gx,
                                        double* gy, double* gz, double* gvx, double* gvy,
                                        double* gvz, double* gm, void* stream) {
  if (!a) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null adjoint");
  const void* ptrs[20] = {x, y, z, m, vx, vy, vz, abx, aby, abz, jbx, jby, jbz, gx, gy, gz, gvx, gvy, gvz, gm};
  for (auto p : ptrs)
    if (!p) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null device array");
  AD_CUDA(cudaSetDevice(a->cfg.device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t ld = a->ld, b = sizeof(double) * a->n;
  // inputs go to the segment buffer (state) and ab1 (adjoints); outputs via adj/mb
  AD_CUDA(cudaMemsetAsync(a->segxv, 0, sizeof(double) * 6 * ld, st));
  AD_CUDA(cudaMemsetAsync(a->ab1, 0, sizeof(double) * 6 * ld, st));
  AD_CUDA(cudaMemsetAsync(a->adj, 0, sizeof(double) * 6 * ld, st));
  AD_CUDA(cudaMemsetAsync(a->mb, 0, sizeof(double) * ld, st));
  AD_CUDA(cudaMemsetAsync(a->M, 0, sizeof(double) * ld, st));
  const double* xv[6] = {x, y, z, vx, vy, vz};
  const double* ab[6] = {abx, aby, abz, jbx, jby, jbz};
  for (int k = 0; k < 6; ++k) {
    AD_CUDA(cudaMemcpyAsync(a->segxv + k * ld, xv[k], b, cudaMemcpyDeviceToDevice, st));
    AD_CUDA(cudaMemcpyAsync(a->ab1 + k * ld, ab[k], b, cudaMemcpyDeviceToDevice, st));
  }
  AD_CUDA(cudaMemcpyAsync(a->M, m, b, cudaMemcpyDeviceToDevice, st));
  AD_TRY(vjp(a, st, a->segxv, a->ab1));
  double* outs[6] = {gx, gy, gz, gvx, gvy, gvz};
  for (int k = 0; k < 6; ++k) AD_CUDA(cudaMemcpyAsync(outs[k], a->adj + k * ld, b, cudaMemcpyDeviceToDevice, st));
  AD_CUDA(cudaMemcpyAsync(gm, a->mb, b, cudaMemcpyDeviceToDevice, st));
  a->have_forward = false;  // the state buffers now hold this call's inputs
  return check_status(a, st);
}

}  // extern "C"
