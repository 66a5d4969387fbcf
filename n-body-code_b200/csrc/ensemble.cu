// Batched ensembles: many independent systems ("clusters") of uneven size
// advanced together, one persistent pair launch per Hermite step.
//
// Layout: cluster c owns padded rows [row0_c, row0_c + ld_c) of every
// ensemble array (ld_c = n_c rounded up to 256), so j-tiles never straddle
// clusters and padding rows are zero-mass bodies that add nothing.  A row's
// cluster comes from cid[row] (-1 on padding rows).
//
// Work list: item = (cluster, 256-row block, j-tile range of at most
// `tiles_per_item` tiles).  Items are sorted by cost (longest first) and a
// fixed grid of SMs x resident CTAs takes them from an atomic counter, so a
// 256-body cluster and an 8192-body cluster share one launch without the
// small one idling the GPU.  Split partial sums of cluster c live at
// P + p_off_c ([S_c][6][ld_c]) and are added in a fixed order by the
// corrector, so results are bitwise reproducible.
//
// A step is memset(counter) -> predict -> persistent pair -> correct,
// captured once into a CUDA graph.  Mixed ensembles use the near/far
// tile-relative kernel (pair.cuh RowsMixedNF): each cluster keeps its bodies
// in Hilbert order within its own padded segment (every sort_every steps a
// second captured graph sorts (cluster, Hilbert code) keys over all rows and
// gathers the state into that order; perm maps positions back to the
// caller's rows), and the j-tile records are rebuilt right after predict.
// Each cluster has its own softening and fixed shared step (the adaptive
// criterion is per system in the reference, src/nbody.cpp:198-222; ensembles
// here run fixed steps).
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include "../../include/nbody_cuda.h"
#include "errors.h"
#include "hermite.cuh"
#include "pair.cuh"
#include "reltiles.cuh"
#include "trace.h"

using namespace nbody;

namespace {

constexpr int kPadRows = 256;  // cluster padding = rows per work item
constexpr int kBlock = 256;

struct ClusterDev {
  int row0, n, ld, S;
  long long p_off;
  double eps2, dt;
};

#define EN_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return nbody_set_error(e_ == cudaErrorMemoryAllocation ? NBODY_ERR_OOM : NBODY_ERR_CUDA, \
                             "%s failed: %s", #call, cudaGetErrorString(e_));              \
  } while (0)
#define EN_TRY(expr)               \
  do {                             \
    nbody_status s_ = (expr);      \
    if (s_ != NBODY_OK) return s_; \
  } while (0)

// ---- kernels ----------------------------------------------------------------

__global__ void ens_pack_kernel(int L, const int* __restrict__ cid, const double* __restrict__ X,
                                const double* __restrict__ V, const double* __restrict__ M,
                                JBody64* __restrict__ jb64, JBodyX2* __restrict__ jbx) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= L) return;
  const bool real = cid[r] >= 0;
  const double x = real ? X[r] : 0, y = real ? X[L + r] : 0, z = real ? X[2 * L + r] : 0;
  const double m = real ? M[r] : 0;
  const double u = real ? V[r] : 0, v = real ? V[L + r] : 0, w = real ? V[2 * L + r] : 0;
  if (jb64) {
    JBody64 b;
    b.x = x; b.y = y; b.z = z; b.m = m; b.vx = u; b.vy = v; b.vz = w; b.pad = 0;
    jb64[r] = b;
  }
  if (jbx) jbx[r] = make_jbx2(x, y, z, m, u, v, w);
}

__global__ void ens_predict_kernel(int L, const int* __restrict__ cid,
                                   const ClusterDev* __restrict__ cl, double* __restrict__ X,
                                   double* __restrict__ V, const double* __restrict__ M,
                                   const double* __restrict__ D, JBody64* __restrict__ jb64,
                                   JBodyX2* __restrict__ jbx) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= L) return;
  const int c = cid[r];
  if (c < 0) return;
  const double dt = cl[c].dt;
  const double h2 = 0.5 * dt * dt;
  const double h3 = dt * dt * dt * (1.0 / 6.0);
  double p[3], u[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double x = X[k * L + r], v = V[k * L + r];
    const double a = D[k * L + r], j = D[(3 + k) * L + r];
    p[k] = x + (v * dt + (a * h2 + j * h3));
    u[k] = v + (a * dt + j * h2);
    X[k * L + r] = p[k];
    V[k * L + r] = u[k];
  }
  const double m = M[r];
  if (jb64) {
    JBody64 b;
    b.x = p[0]; b.y = p[1]; b.z = p[2]; b.m = m; b.vx = u[0]; b.vy = u[1]; b.vz = u[2]; b.pad = 0;
    jb64[r] = b;
  }
  if (jbx) jbx[r] = make_jbx2(p[0], p[1], p[2], m, u[0], u[1], u[2]);
}

// bbox[c*6 + k]: min (k < 3) / max of cluster c's positions (one CTA each).
__global__ void __launch_bounds__(kBlock) ens_bbox_kernel(const ClusterDev* __restrict__ cl,
                                                         const double* __restrict__ X, int L,
                                                         double* __restrict__ bbox) {
  __shared__ double sh[6 * 32];
  const ClusterDev k = cl[blockIdx.x];
  double v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (int i = threadIdx.x; i < k.n; i += blockDim.x) {
    const int r = k.row0 + i;
    const double x = X[r], y = X[L + r], z = X[2 * L + r];
    v[0] = fmin(v[0], x); v[1] = fmin(v[1], y); v[2] = fmin(v[2], z);
    v[3] = fmax(v[3], x); v[4] = fmax(v[4], y); v[5] = fmax(v[5], z);
  }
  block_minmax6(v, sh);
#pragma unroll
  for (int q = 0; q < 6; ++q)
    if (threadIdx.x == q) bbox[blockIdx.x * 6 + q] = v[q];
}

// keys[r] = (segment cluster << 48) | 48-bit Hilbert index (16 bits per axis)
// in the cluster's box; padding rows take the segment's largest key, so the
// sorted rows of cluster c fill exactly its padded segment, bodies first.
__global__ void ens_key_kernel(int L, const int* __restrict__ cid, const int* __restrict__ seg,
                               const double* __restrict__ X, const double* __restrict__ bbox,
                               uint64_t* __restrict__ keys, int* __restrict__ vals) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= L) return;
  const int c = seg[r];
  uint64_t key = static_cast<uint64_t>(c) << 48;
  if (cid[r] < 0) {
    key |= 0xffffffffffffull;
  } else {
    constexpr double kCells = 65535.0;
    uint32_t cell[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double lo = bbox[c * 6 + k], w = bbox[c * 6 + 3 + k] - lo;
      double q = w > 0.0 ? (X[k * L + r] - lo) * (kCells / w) : 0.0;
      q = fmin(fmax(q, 0.0), kCells);  // NaN -> 0
      cell[k] = static_cast<uint32_t>(q);
    }
    key |= hilbert_key48(cell[0], cell[1], cell[2]);
  }
  keys[r] = key;
  vals[r] = r;
}

__global__ void ens_correct_kernel(int L, const int* __restrict__ cid,
                                   const ClusterDev* __restrict__ cl, const double* __restrict__ P,
                                   double* __restrict__ X, double* __restrict__ V,
                                   double* __restrict__ D) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= L) return;
  const int c = cid[r];
  if (c < 0) return;
  const ClusterDev k = cl[c];
  const int i = r - k.row0;
  const double dt = k.dt;
  const double idt2 = 1.0 / (dt * dt), idt3 = idt2 / dt;
  const double dt3 = dt * dt * dt, dt4 = dt3 * dt, dt5 = dt4 * dt;
  double sum[6];
  split_sums(P + k.p_off, k.ld, k.S, i, sum);  // cluster partials: [S_c][6][ld_c]
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double a1 = sum[q], j1 = sum[3 + q];
    const double a = D[q * L + r], j = D[(3 + q) * L + r];
    const double da = a - a1;
    const double a2 = 2.0 * idt2 * (-3.0 * da - (2.0 * j + j1) * dt);
    const double a3 = 6.0 * idt3 * (2.0 * da + (j + j1) * dt);
    X[q * L + r] += a2 * dt4 * (1.0 / 24.0) + a3 * dt5 * (1.0 / 120.0);
    V[q * L + r] += a2 * dt3 * (1.0 / 6.0) + a3 * dt4 * (1.0 / 24.0);
    D[q * L + r] = a1;
    D[(3 + q) * L + r] = j1;
  }
}

__global__ void ens_reduce_kernel(int L, const int* __restrict__ cid,
                                  const ClusterDev* __restrict__ cl, const double* __restrict__ P,
                                  double* __restrict__ D) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= L) return;
  const int c = cid[r];
  if (c < 0) return;
  const ClusterDev k = cl[c];
  double sum[6];
  split_sums(P + k.p_off, k.ld, k.S, r - k.row0, sum);
  for (int f = 0; f < 6; ++f) D[f * L + r] = sum[f];
}

// phi[r] = sum over the same cluster's j != r of m_j / sqrt(r^2 + eps2_c);
// one CTA per 256-row block, blocks listed in `blk` as cluster ids.
__global__ void __launch_bounds__(kBlock) ens_phi_kernel(const int* __restrict__ blk_cluster,
                                                         const int* __restrict__ blk_row,
                                                         const ClusterDev* __restrict__ cl,
                                                         const JBody64* __restrict__ jb,
                                                         double* __restrict__ phi) {
  __shared__ double4 tile[kBlock];
  const ClusterDev k = cl[blk_cluster[blockIdx.x]];
  const int i = blk_row[blockIdx.x] + threadIdx.x;  // cluster-relative row
  const JBody64 bi = jb[k.row0 + i];
  double acc = 0.0;
  for (int j0 = 0; j0 < k.ld; j0 += kBlock) {
    const JBody64 bj = jb[k.row0 + j0 + threadIdx.x];
    tile[threadIdx.x] = make_double4(bj.x, bj.y, bj.z, bj.m);
    __syncthreads();
#pragma unroll 4
    for (int t = 0; t < kBlock; ++t) {
      const double4 p = tile[t];
      const double dx = p.x - bi.x, dy = p.y - bi.y, dz = p.z - bi.z;
      const double y = rsqrt_f64(fma(dx, dx, fma(dy, dy, fma(dz, dz, k.eps2))));
      acc += (j0 + t != i) ? p.w * y : 0.0;
    }
    __syncthreads();
  }
  phi[k.row0 + i] = acc;
}

// Per cluster (one CTA each): T = sum 0.5 m v^2, U = -0.5 sum m phi.
__global__ void ens_energy_sum_kernel(const ClusterDev* __restrict__ cl, const double* __restrict__ V,
                                      const double* __restrict__ M, const double* __restrict__ phi,
                                      int L, double* __restrict__ T, double* __restrict__ U) {
  __shared__ double sh[32];
  const ClusterDev k = cl[blockIdx.x];
  double t = 0.0, u = 0.0;
  for (int i = threadIdx.x; i < k.n; i += blockDim.x) {
    const int r = k.row0 + i;
    const double a = V[r], b = V[L + r], c = V[2 * L + r];
    t += 0.5 * M[r] * (a * a + b * b + c * c);
    u += M[r] * phi[r];
  }
  const double bt = block_sum(t, sh);
  const double bu = block_sum(u, sh);
  if (threadIdx.x == 0) {
    T[blockIdx.x] = bt;
    U[blockIdx.x] = -0.5 * bu;
  }
}

// Persistent-kernel shapes (all with 256-row items = one padding unit); the
// first of each precision is the default, the autotuner times all of them.
struct EnsKernel {
  int precision, nt, tile;
  int fmt;  // RecordFormat of its j-records
  const void* fn;
  size_t smem;
  int near = 0;  // tile-relative: 1 = near tiles in double-single, 0 = every tile far
};

template <class R>
EnsKernel ens_kernel(int precision) {
  static_assert(R::ROWS == kPadRows, "an item's row block is one padding unit");
  return {precision, R::NT, R::TJ, precision == NBODY_FP64 ? kRecF64 : kRecX2,
          reinterpret_cast<const void*>(&ensemble_pair_kernel<R>), pair_smem_bytes<R>()};
}

template <class R, int MINB = 1>
EnsKernel ens_kernel_nf() {
  static_assert(R::ROWS == kPadRows, "an item's row block is one padding unit");
  return {NBODY_MIXED, R::NT, R::TJ, kRecRel,
          reinterpret_cast<const void*>(&ensemble_pair_nf_kernel<R, MINB>),
          2 * (R::TJ + 1) * sizeof(JBodyNF) + R::kExtraSmem, R::kNear ? 1 : 0};
}

// The first entry of each (precision, record format, near) is its default.
const std::vector<EnsKernel>& ens_registry() {
  static const std::vector<EnsKernel> r = {
      ens_kernel<RowsFP64<128, 2, 128, 1>>(NBODY_FP64),
      ens_kernel<RowsFP64<256, 1, 128, 4>>(NBODY_FP64),
      ens_kernel_nf<RowsMixedNF<64, 4, 64, 1, 1, 1>>(),
      ens_kernel_nf<RowsMixedNF<64, 4, 128, 1, 1, 1>>(),
      ens_kernel_nf<RowsMixedNF<128, 2, 128, 1, 1, 1>>(),
      ens_kernel_nf<RowsMixedNF<128, 2, 64, 1, 1, 1>>(),
      ens_kernel_nf<RowsMixedNF<64, 4, 64, 1, 2, 1>>(),
      ens_kernel_nf<RowsMixedNF<128, 2, 128, 1, 2, 1>>(),
      ens_kernel_nf<RowsMixedNF<64, 4, 128, 1, 2, 1>>(),
      ens_kernel_nf<RowsMixedNF<64, 4, 64, 1, 1, 2>>(),
      // 64 threads capped at 128 registers: 8 CTAs (16 warps) per SM
      ens_kernel_nf<RowsMixedNF<64, 4, 64, 1, 1, 1>, 8>(),
      ens_kernel_nf<RowsMixedNF<64, 4, 64, 1, 2, 1>, 8>(),
      ens_kernel_nf<RowsMixedNF<64, 4, 64, 1, 1, 2>, 8>(),
      ens_kernel_nf<RowsMixedNF<64, 4, 128, 1, 1, 1>, 8>(),
      ens_kernel_nf<RowsMixedNF<64, 4, 64, 1, 1, 0>>(),
      ens_kernel_nf<RowsMixedNF<128, 2, 128, 1, 1, 0>>(),
      ens_kernel<RowsMixedX2<64, 4, 128, 1, 1>>(NBODY_MIXED),
      ens_kernel<RowsMixedX2<128, 2, 128, 1, 1>>(NBODY_MIXED),
      ens_kernel<RowsMixedX2<64, 4, 64, 1, 1>>(NBODY_MIXED),
      ens_kernel<RowsMixedX2<64, 4, 64, 1, 2>>(NBODY_MIXED),
      ens_kernel<RowsMixedX2<128, 2, 64, 1, 1>>(NBODY_MIXED),
      ens_kernel<RowsMixedX2<128, 2, 64, 1, 2>>(NBODY_MIXED),
      ens_kernel<RowsMixedX2<64, 4, 64, 0, 2>>(NBODY_MIXED),
  };
  return r;
}

}  // namespace

struct nbody_ensemble {
  int C = 0, L = 0, dev = 0, sms = 0, precision = 0;
  int fmt = kRecF64;  // record format of the pair kernels in use
  int tiles_per_item = 8;
  const EnsKernel* kern = nullptr;  // persistent pair kernel in use
  int grid = 0;
  long long interactions = 0;  // sum of n_c^2 per step
  cudaStream_t stream = nullptr;
  std::vector<int> n, row0, ld;
  std::vector<double> eps2, dt;
  double* state = nullptr;  // [13][L]
  double *X = nullptr, *V = nullptr, *M = nullptr, *D = nullptr;
  double* P = nullptr;
  size_t p_doubles = 0;
  JBody64* jb64 = nullptr;
  JBodyX2* jbx = nullptr;
  int* cid = nullptr;
  ClusterDev* cl = nullptr;
  EnsItem* items = nullptr;
  int n_items = 0;
  unsigned int* counter = nullptr;
  int* status = nullptr;
  int *blk_cluster = nullptr, *blk_row = nullptr;
  int n_blk = 0;
  double *phi = nullptr, *Tc = nullptr, *Uc = nullptr;
  cudaGraphExec_t graph = nullptr;
  int step_kernels = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool have_derivs = false;
  long long steps = 0;
  // Hilbert ordering (mixed, tile-relative variants): each cluster keeps its
  // bodies in Hilbert order within its segment; position r holds the body of
  // padded row perm[r] (the caller's order).
  int near = 1;                   // near/far kernel (variant 4) or every tile far (5)
  int* perm = nullptr;            // [2][L]
  double* scratch = nullptr;      // [13][L]
  bool sorted = false, permuted = false;
  int* seg = nullptr;             // [L] cluster owning each padded row
  double* bbox = nullptr;         // [C][6]
  uint64_t* sort_keys = nullptr;  // [2][L]
  int* sort_idx = nullptr;        // [2][L]; second half = order
  void* sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;
  int sort_bits = 49, sort_every = 16, since_sort = 0;
  cudaGraphExec_t order_graph = nullptr;
  int order_kernels = 0;
  long long reorders = 0;
};

namespace {

nbody_status ens_status(nbody_ensemble* e) {
  int h = 0;
  EN_CUDA(cudaMemcpyAsync(&h, e->status, sizeof h, cudaMemcpyDeviceToHost, e->stream));
  EN_CUDA(cudaStreamSynchronize(e->stream));
  if (h) {
    cudaMemsetAsync(e->status, 0, sizeof(int), e->stream);
    return nbody_set_error(NBODY_ERR_TIMEOUT, "an ensemble pair-kernel wait exceeded its limit");
  }
  return NBODY_OK;
}

// (Re)builds the work list and partial-sum layout for `tpi` tiles per item.
nbody_status build_items(nbody_ensemble* e, int tpi) {
  std::vector<ClusterDev> cl(e->C);
  std::vector<EnsItem> items;
  long long p_off = 0;
  for (int c = 0; c < e->C; ++c) {
    // j-tiles that hold bodies: the padding rows of a segment come last (in
    // the tile-relative order too), so whole padding tiles are skipped
    const int tiles = (e->n[c] + e->kern->tile - 1) / e->kern->tile;
    const int S = (tiles + tpi - 1) / tpi;
    cl[c] = ClusterDev{e->row0[c], e->n[c], e->ld[c], S, p_off, e->eps2[c], e->dt[c]};
    for (int rb = 0; rb < e->ld[c] / kPadRows; ++rb)
      for (int s = 0; s < S; ++s) {
        EnsItem it;
        it.jrow0 = e->row0[c];
        it.row0 = rb * kPadRows;
        it.rows_end = e->n[c];
        it.ld = e->ld[c];
        it.t_begin = s * tpi;
        it.nt = std::min(tpi, tiles - it.t_begin);
        it.out_off = p_off + static_cast<long long>(s) * 6 * e->ld[c];
        it.eps2 = e->eps2[c];
        items.push_back(it);
      }
    p_off += static_cast<long long>(S) * 6 * e->ld[c];
  }
  // longest items first, then by cluster so neighbours share L2 lines
  std::stable_sort(items.begin(), items.end(),
                   [](const EnsItem& a, const EnsItem& b) { return a.nt > b.nt; });
  if (e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  EN_CUDA(cudaStreamSynchronize(e->stream));
  cudaFree(e->P);
  cudaFree(e->items);
  e->P = nullptr;
  e->items = nullptr;
  e->p_doubles = static_cast<size_t>(p_off);
  EN_CUDA(cudaMalloc(&e->P, sizeof(double) * e->p_doubles));
  EN_CUDA(cudaMalloc(&e->items, sizeof(EnsItem) * items.size()));
  EN_CUDA(cudaMemcpy(e->items, items.data(), sizeof(EnsItem) * items.size(), cudaMemcpyHostToDevice));
  EN_CUDA(cudaMemcpy(e->cl, cl.data(), sizeof(ClusterDev) * e->C, cudaMemcpyHostToDevice));
  e->n_items = static_cast<int>(items.size());
  e->tiles_per_item = tpi;
  return NBODY_OK;
}

nbody_status launch_ens_pair(nbody_ensemble* e) {
  EN_CUDA(cudaMemsetAsync(e->counter, 0, sizeof(unsigned int), e->stream));
  const bool fp64 = e->precision == NBODY_FP64;
  const void* jb = fp64 ? static_cast<const void*>(e->jb64) : static_cast<const void*>(e->jbx);
  const size_t L = e->L;
  RowSrc rows{e->X, e->X + L, e->X + 2 * L, e->V, e->V + L, e->V + 2 * L};
  void* args[] = {const_cast<void*>(static_cast<const void*>(&jb)), &e->items, &e->n_items,
                  &e->counter, &e->P, &e->status, &rows};
  EN_CUDA(cudaLaunchKernel(e->kern->fn, dim3(e->grid), dim3(e->kern->nt), args, e->kern->smem,
                           e->stream));
  return NBODY_OK;
}

// Hilbert order of every cluster's bodies within its padded segment.
nbody_status ens_order(nbody_ensemble* e, cudaStream_t st) {
  ens_bbox_kernel<<<e->C, kBlock, 0, st>>>(e->cl, e->X, e->L, e->bbox);
  ens_key_kernel<<<(e->L + kBlock - 1) / kBlock, kBlock, 0, st>>>(e->L, e->cid, e->seg, e->X,
                                                                  e->bbox, e->sort_keys, e->sort_idx);
  EN_CUDA(cudaGetLastError());
  const size_t L = e->L;
  size_t bytes = e->sort_tmp_bytes;
  EN_CUDA(cub::DeviceRadixSort::SortPairs(e->sort_tmp, bytes, e->sort_keys, e->sort_keys + L,
                                          e->sort_idx, e->sort_idx + L, e->L, 0, e->sort_bits, st));
  return NBODY_OK;
}

// Puts every cluster's bodies into Hilbert order within its segment: the
// order of ens_order, a gather of all 13 state arrays (and of perm) into
// scratch, and a copy back.  Capturable (the re-ordering graph).
nbody_status ens_reorder_state(nbody_ensemble* e, cudaStream_t st) {
  const size_t L = e->L;
  EN_TRY(ens_order(e, st));
  GatherArgs g;
  g.arrays = 13;
  for (int a = 0; a < 13; ++a) {
    g.src[a] = e->state + a * L;
    g.dst[a] = e->scratch + a * L;
  }
  gather_rows_kernel<<<(e->L + kBlock - 1) / kBlock, kBlock, 0, st>>>(e->L, e->sort_idx + L, g,
                                                                     e->perm, e->perm + L);
  EN_CUDA(cudaGetLastError());
  EN_CUDA(cudaMemcpyAsync(e->state, e->scratch, sizeof(double) * 13 * L, cudaMemcpyDeviceToDevice, st));
  EN_CUDA(cudaMemcpyAsync(e->perm, e->perm + L, sizeof(int) * L, cudaMemcpyDeviceToDevice, st));
  e->sorted = e->permuted = true;
  e->since_sort = 0;
  return NBODY_OK;
}

// Near/far tile records (tiles of the kernel's TJ) of the state, which is in
// Hilbert order within each cluster segment.
nbody_status ens_tiles(nbody_ensemble* e, cudaStream_t st) {
  const size_t L = e->L;
  const SoA7 in{e->X, e->X + L, e->X + 2 * L, e->M, e->V, e->V + L, e->V + 2 * L};
  JBodyNF* out = reinterpret_cast<JBodyNF*>(e->jbx);
  const int tiles = e->L / e->kern->tile;
  switch (e->kern->tile) {
    case 64: rel_tile_nf_kernel<64><<<tiles, 64, 0, st>>>(e->L, in, out, e->cid); break;
    case 128: rel_tile_nf_kernel<128><<<tiles, 128, 0, st>>>(e->L, in, out, e->cid); break;
    default: return nbody_set_error(NBODY_ERR_INVALID_ARG, "no record builder for tile %d", e->kern->tile);
  }
  EN_CUDA(cudaGetLastError());
  return NBODY_OK;
}

// Copies `count` [L] arrays starting at src to the caller's concatenated
// arrays (cluster c's n_c bodies in turn), through scratch when permuted.
nbody_status ens_download(nbody_ensemble* e, const double* src, double* const* dst, int count) {
  const size_t L = e->L;
  const double* from = src;
  if (e->permuted) {
    GatherArgs g;
    g.arrays = count;
    for (int a = 0; a < count; ++a) {
      g.src[a] = src + a * L;
      g.dst[a] = e->scratch + a * L;
    }
    scatter_rows_kernel<<<(e->L + kBlock - 1) / kBlock, kBlock, 0, e->stream>>>(e->L, e->perm, g);
    EN_CUDA(cudaGetLastError());
    from = e->scratch;
  }
  long long off = 0;
  for (int c = 0; c < e->C; ++c) {
    for (int k = 0; k < count; ++k)
      if (dst[k])
        EN_CUDA(cudaMemcpyAsync(dst[k] + off, from + k * L + e->row0[c], sizeof(double) * e->n[c],
                                cudaMemcpyDeviceToHost, e->stream));
    off += e->n[c];
  }
  EN_CUDA(cudaStreamSynchronize(e->stream));
  return NBODY_OK;
}

// Selects a persistent kernel: opts in to its shared memory and sizes the
// grid to the SMs x resident CTAs it reaches.
nbody_status use_kernel(nbody_ensemble* e, const EnsKernel* k) {
  EN_CUDA(cudaFuncSetAttribute(k->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(k->smem)));
  int occ = 0;
  EN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k->fn, k->nt, k->smem));
  e->kern = k;
  e->grid = e->sms * std::max(occ, 1);
  return NBODY_OK;
}

nbody_status launch_ens_pack(nbody_ensemble* e) {
  if (e->fmt == kRecRel && !e->sorted)  // tile-relative: bodies into Hilbert order first
    EN_TRY(ens_reorder_state(e, e->stream));
  ens_pack_kernel<<<(e->L + kBlock - 1) / kBlock, kBlock, 0, e->stream>>>(
      e->L, e->cid, e->X, e->V, e->M, e->jb64, e->fmt == kRecX2 ? e->jbx : nullptr);
  EN_CUDA(cudaGetLastError());
  if (e->fmt == kRecRel) EN_TRY(ens_tiles(e, e->stream));
  return NBODY_OK;
}

int count_graph_kernels(cudaGraph_t g) {
  size_t nodes = 0;
  int kernels = 0;
  if (cudaGraphGetNodes(g, nullptr, &nodes) == cudaSuccess && nodes > 0) {
    std::vector<cudaGraphNode_t> v(nodes);
    if (cudaGraphGetNodes(g, v.data(), &nodes) == cudaSuccess)
      for (size_t k = 0; k < nodes; ++k) {
        cudaGraphNodeType ty;
        if (cudaGraphNodeGetType(v[k], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel)
          ++kernels;
      }
  }
  return kernels;
}

nbody_status ens_eval_current(nbody_ensemble* e) {
  EN_TRY(launch_ens_pack(e));
  EN_TRY(launch_ens_pair(e));
  ens_reduce_kernel<<<(e->L + kBlock - 1) / kBlock, kBlock, 0, e->stream>>>(e->L, e->cid, e->cl,
                                                                          e->P, e->D);
  EN_CUDA(cudaGetLastError());
  e->have_derivs = true;
  return NBODY_OK;
}

nbody_status ens_build_graph(nbody_ensemble* e) {
  if (e->graph) return NBODY_OK;
  const bool fp64 = e->precision == NBODY_FP64;
  cudaGraph_t g = nullptr;
  EN_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  nbody_status s = NBODY_OK;
  if (cudaEventRecordWithFlags(e->ev[0], e->stream, cudaEventRecordExternal) != cudaSuccess)
    s = nbody_set_error(NBODY_ERR_CUDA, "event record during capture failed");
  ens_predict_kernel<<<(e->L + kBlock - 1) / kBlock, kBlock, 0, e->stream>>>(
      e->L, e->cid, e->cl, e->X, e->V, e->M, e->D, fp64 ? e->jb64 : nullptr,
      e->fmt == kRecX2 ? e->jbx : nullptr);
  if (s == NBODY_OK && e->fmt == kRecRel) s = ens_tiles(e, e->stream);
  if (s == NBODY_OK) s = launch_ens_pair(e);
  ens_correct_kernel<<<(e->L + kBlock - 1) / kBlock, kBlock, 0, e->stream>>>(e->L, e->cid, e->cl,
                                                                           e->P, e->X, e->V, e->D);
  if (s == NBODY_OK && cudaEventRecordWithFlags(e->ev[1], e->stream, cudaEventRecordExternal) != cudaSuccess)
    s = nbody_set_error(NBODY_ERR_CUDA, "event record during capture failed");
  cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
  if (s != NBODY_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (ce != cudaSuccess) return nbody_set_error(NBODY_ERR_CUDA, "capture: %s", cudaGetErrorString(ce));
  e->step_kernels = count_graph_kernels(g);
  ce = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    e->graph = nullptr;
    return nbody_set_error(NBODY_ERR_CUDA, "instantiate: %s", cudaGetErrorString(ce));
  }
  if (e->fmt == kRecRel && !e->order_graph) {
    const bool sorted = e->sorted, permuted = e->permuted;
    const int since = e->since_sort;
    EN_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    s = ens_reorder_state(e, e->stream);
    g = nullptr;
    ce = cudaStreamEndCapture(e->stream, &g);
    e->sorted = sorted;  // capturing ran nothing
    e->permuted = permuted;
    e->since_sort = since;
    if (s != NBODY_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    if (ce != cudaSuccess) return nbody_set_error(NBODY_ERR_CUDA, "capture: %s", cudaGetErrorString(ce));
    e->order_kernels = count_graph_kernels(g);
    ce = cudaGraphInstantiate(&e->order_graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      e->order_graph = nullptr;
      return nbody_set_error(NBODY_ERR_CUDA, "instantiate: %s", cudaGetErrorString(ce));
    }
  }
  return NBODY_OK;
}

// Times the pair launch for every (kernel shape, item size) pair; keeps the
// fastest.  Items count j-tiles, so tiles_per_item x tile = j per item.
nbody_status ens_autotune(nbody_ensemble* e) {
  EN_TRY(launch_ens_pack(e));
  cudaEvent_t a, b;
  EN_CUDA(cudaEventCreate(&a));
  EN_CUDA(cudaEventCreate(&b));
  float best = 1e30f;
  const EnsKernel* best_k = e->kern;
  int best_tpi = 8;
  for (const EnsKernel& k : ens_registry()) {
    if (k.precision != e->precision || k.fmt != e->fmt || (k.fmt == kRecRel && k.near != e->near)) continue;
    EN_TRY(use_kernel(e, &k));
    if (e->fmt == kRecRel) EN_TRY(ens_tiles(e, e->stream));  // this kernel's tile size
    for (int j_per_item : {256, 512, 1024, 2048, 4096, 8192}) {
      const int tpi = std::max(1, j_per_item / k.tile);
      EN_TRY(build_items(e, tpi));
      EN_TRY(launch_ens_pair(e));
      EN_CUDA(cudaEventRecord(a, e->stream));
      for (int r = 0; r < 2; ++r) EN_TRY(launch_ens_pair(e));
      EN_CUDA(cudaEventRecord(b, e->stream));
      EN_CUDA(cudaEventSynchronize(b));
      float ms = 0;
      EN_CUDA(cudaEventElapsedTime(&ms, a, b));
      if (getenv("NBODY_TUNE_VERBOSE"))
        fprintf(stderr, "[nbody ens tune] nt=%d tile=%d tiles_per_item=%d  %.4f ms\n", k.nt, k.tile,
                tpi, ms / 2);
      if (ms < best) {
        best = ms;
        best_k = &k;
        best_tpi = tpi;
      }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  EN_TRY(ens_status(e));
  EN_TRY(use_kernel(e, best_k));
  if (e->fmt == kRecRel) EN_TRY(ens_tiles(e, e->stream));
  return build_items(e, best_tpi);
}

nbody_status ens_check(nbody_ensemble* e) {
  if (!e) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null ensemble");
  if (cudaSetDevice(e->dev) != cudaSuccess) return nbody_set_error(NBODY_ERR_CUDA, "cudaSetDevice failed");
  return NBODY_OK;
}

}  // namespace

extern "C" {

nbody_status nbody_ensemble_destroy(nbody_ensemble* e) {
  if (!e) return NBODY_OK;
  cudaSetDevice(e->dev);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->order_graph) cudaGraphExecDestroy(e->order_graph);
  for (auto ev : e->ev)
    if (ev) cudaEventDestroy(ev);
  void* bufs[] = {e->state, e->P, e->jb64, e->jbx, e->cid, e->cl, e->items, e->counter,
                  e->status, e->blk_cluster, e->blk_row, e->phi, e->Tc, e->Uc,
                  e->seg, e->bbox, e->sort_keys, e->sort_idx, e->sort_tmp, e->perm, e->scratch};
  for (void* p : bufs) cudaFree(p);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return NBODY_OK;
}

nbody_status nbody_ensemble_create(nbody_ensemble** out, const nbody_ensemble_config* cfg) {
  if (!out || !cfg || !cfg->n || !cfg->eps2 || !cfg->dt)
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "null ensemble argument");
  *out = nullptr;
  const int C = cfg->nclusters;
  if (C < 1) return nbody_set_error(NBODY_ERR_INVALID_ARG, "nclusters = %d", C);
  if (cfg->precision != NBODY_FP64 && cfg->precision != NBODY_MIXED)
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "precision = %d", cfg->precision);
  if (cfg->tiles_per_item < 0) return nbody_set_error(NBODY_ERR_INVALID_ARG, "tiles_per_item < 0");
  if (cfg->precision == NBODY_MIXED && cfg->pair_variant != 0 && cfg->pair_variant != 3 &&
      cfg->pair_variant != 4 && cfg->pair_variant != 5)
    return nbody_set_error(NBODY_ERR_INVALID_ARG,
                           "ensemble pair_variant = %d (0 automatic = packed hi/lo, 3 packed hi/lo, "
                           "4 near/far tile-relative, 5 plain tile-relative)", cfg->pair_variant);
  if (cfg->sort_every < 0) return nbody_set_error(NBODY_ERR_INVALID_ARG, "sort_every < 0");
  // Mixed default: packed hi/lo.  In clusters of 256-8192 bodies a 64-body
  // tile is rarely far from a warp's 128 rows (near share of a Plummer
  // sphere: 0.48 at 8192 bodies, 0.73 at 4096, 0.93 at 2048), so the
  // near/far kernel saves less than its tile building and re-ordering cost
  // (measured 855 vs 878 G interactions/s on 512 Plummer clusters of
  // 256-8192 bodies).
  const bool rel = cfg->precision == NBODY_MIXED && (cfg->pair_variant == 4 || cfg->pair_variant == 5);
  if (rel && C > 65536)
    return nbody_set_error(NBODY_ERR_INVALID_ARG,
                           "tile-relative ensembles hold at most 65536 clusters (use pair_variant 3)");
  long long L = 0;
  for (int c = 0; c < C; ++c) {
    if (cfg->n[c] < 1) return nbody_set_error(NBODY_ERR_INVALID_ARG, "cluster %d has n = %d", c, cfg->n[c]);
    if (!(cfg->eps2[c] >= 1e-30 && cfg->eps2[c] <= 1e30))
      return nbody_set_error(NBODY_ERR_INVALID_ARG, "cluster %d eps2 = %g", c, cfg->eps2[c]);
    if (cfg->precision == NBODY_MIXED && cfg->eps2[c] < kMinEps2Mixed)
      return nbody_set_error(NBODY_ERR_INVALID_ARG, "cluster %d eps2 = %g below %g (mixed precision)",
                             c, cfg->eps2[c], kMinEps2Mixed);
    if (!(cfg->dt[c] > 0)) return nbody_set_error(NBODY_ERR_INVALID_ARG, "cluster %d dt = %g (ensembles use fixed steps)", c, cfg->dt[c]);
    L += (cfg->n[c] + kPadRows - 1) / kPadRows * kPadRows;
  }
  if (L > (1LL << 28)) return nbody_set_error(NBODY_ERR_INVALID_ARG, "ensemble too large");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return nbody_set_error(NBODY_ERR_NO_DEVICE, "no CUDA device visible");
  if (cfg->device < 0 || cfg->device >= ndev)
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "device %d of %d", cfg->device, ndev);
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, cfg->device);
  if (major != 10) return nbody_set_error(NBODY_ERR_NO_DEVICE, "device %d is not sm_100", cfg->device);
  EN_CUDA(cudaSetDevice(cfg->device));

  std::unique_ptr<nbody_ensemble> e(new nbody_ensemble);
  e->C = C;
  e->L = static_cast<int>(L);
  e->dev = cfg->device;
  e->precision = cfg->precision;
  e->fmt = cfg->precision == NBODY_FP64 ? kRecF64 : (rel ? kRecRel : kRecX2);
  e->near = cfg->pair_variant == 4 ? 1 : 0;
  e->sort_every = cfg->sort_every > 0 ? cfg->sort_every : 16;
  while ((1LL << (e->sort_bits - 48)) < C) ++e->sort_bits;  // cluster id above the 48-bit code
  cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->dev);
  e->n.assign(cfg->n, cfg->n + C);
  e->eps2.assign(cfg->eps2, cfg->eps2 + C);
  e->dt.assign(cfg->dt, cfg->dt + C);
  std::vector<int> cid(e->L, -1), seg(e->L, 0), blk_cluster, blk_row;
  int r0 = 0;
  for (int c = 0; c < C; ++c) {
    const int ld = (e->n[c] + kPadRows - 1) / kPadRows * kPadRows;
    e->row0.push_back(r0);
    e->ld.push_back(ld);
    for (int i = 0; i < e->n[c]; ++i) cid[r0 + i] = c;
    for (int i = 0; i < ld; ++i) seg[r0 + i] = c;
    for (int b = 0; b < ld; b += kPadRows) {
      blk_cluster.push_back(c);
      blk_row.push_back(b);
    }
    e->interactions += static_cast<long long>(e->n[c]) * e->n[c];
    r0 += ld;
  }
  e->n_blk = static_cast<int>(blk_cluster.size());
  nbody_ensemble* raw = e.get();
  auto body = [&]() -> nbody_status {
    EN_CUDA(cudaStreamCreateWithFlags(&raw->stream, cudaStreamNonBlocking));
    const size_t Ls = raw->L;
    EN_CUDA(cudaMalloc(&raw->state, sizeof(double) * 13 * Ls));
    EN_CUDA(cudaMemset(raw->state, 0, sizeof(double) * 13 * Ls));
    raw->X = raw->state;
    raw->V = raw->state + 3 * Ls;
    raw->M = raw->state + 6 * Ls;
    raw->D = raw->state + 7 * Ls;
    EN_CUDA(cudaMalloc(&raw->jb64, sizeof(JBody64) * Ls));
    // JBodyX2 records, or tiles of TJ + 1 JBodyNF records (TJ >= 64)
    if (raw->precision == NBODY_MIXED) EN_CUDA(cudaMalloc(&raw->jbx, sizeof(JBodyNF) * (Ls / 64) * 65));
    EN_CUDA(cudaMalloc(&raw->cid, sizeof(int) * Ls));
    EN_CUDA(cudaMemcpy(raw->cid, cid.data(), sizeof(int) * Ls, cudaMemcpyHostToDevice));
    EN_CUDA(cudaMalloc(&raw->cl, sizeof(ClusterDev) * raw->C));
    EN_CUDA(cudaMalloc(&raw->counter, sizeof(unsigned int)));
    EN_CUDA(cudaMalloc(&raw->status, sizeof(int)));
    EN_CUDA(cudaMemset(raw->status, 0, sizeof(int)));
    EN_CUDA(cudaMalloc(&raw->blk_cluster, sizeof(int) * raw->n_blk));
    EN_CUDA(cudaMalloc(&raw->blk_row, sizeof(int) * raw->n_blk));
    EN_CUDA(cudaMemcpy(raw->blk_cluster, blk_cluster.data(), sizeof(int) * raw->n_blk, cudaMemcpyHostToDevice));
    EN_CUDA(cudaMemcpy(raw->blk_row, blk_row.data(), sizeof(int) * raw->n_blk, cudaMemcpyHostToDevice));
    EN_CUDA(cudaMalloc(&raw->phi, sizeof(double) * Ls));
    EN_CUDA(cudaMalloc(&raw->Tc, sizeof(double) * raw->C));
    EN_CUDA(cudaMalloc(&raw->Uc, sizeof(double) * raw->C));
    if (raw->fmt == kRecRel) {
      EN_CUDA(cudaMalloc(&raw->seg, sizeof(int) * Ls));
      EN_CUDA(cudaMemcpy(raw->seg, seg.data(), sizeof(int) * Ls, cudaMemcpyHostToDevice));
      EN_CUDA(cudaMalloc(&raw->bbox, sizeof(double) * 6 * raw->C));
      EN_CUDA(cudaMalloc(&raw->sort_keys, sizeof(uint64_t) * 2 * Ls));
      EN_CUDA(cudaMalloc(&raw->sort_idx, sizeof(int) * 2 * Ls));
      EN_CUDA(cudaMalloc(&raw->perm, sizeof(int) * 2 * Ls));
      iota_kernel<<<(raw->L + kBlock - 1) / kBlock, kBlock, 0, raw->stream>>>(raw->L, raw->perm);
      EN_CUDA(cudaGetLastError());
      EN_CUDA(cudaMalloc(&raw->scratch, sizeof(double) * 13 * Ls));
      EN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, raw->sort_tmp_bytes, raw->sort_keys,
                                              raw->sort_keys + Ls, raw->sort_idx,
                                              raw->sort_idx + Ls, raw->L, 0, raw->sort_bits,
                                              raw->stream));
      EN_CUDA(cudaMalloc(&raw->sort_tmp, std::max<size_t>(raw->sort_tmp_bytes, 16)));
    }
    for (auto& ev : raw->ev) EN_CUDA(cudaEventCreate(&ev));
    for (const EnsKernel& k : ens_registry())
      if (k.precision == raw->precision && k.fmt == raw->fmt && (k.fmt != kRecRel || k.near == raw->near)) {
        EN_TRY(use_kernel(raw, &k));
        break;
      }
    return build_items(raw, cfg->tiles_per_item > 0 ? cfg->tiles_per_item : 8);
  };
  nbody_status s = body();
  if (s != NBODY_OK) {
    nbody_ensemble_destroy(e.release());
    return s;
  }
  if (cfg->tune && cfg->tiles_per_item == 0) e->tiles_per_item = -1;  // tune at first state
  *out = e.release();
  return NBODY_OK;
}

nbody_status nbody_ensemble_set_state(nbody_ensemble* e, const double* x, const double* y,
                                      const double* z, const double* m, const double* vx,
                                      const double* vy, const double* vz) {
  EN_TRY(ens_check(e));
  const double* src[7] = {x, y, z, vx, vy, vz, m};
  for (auto p : src)
    if (!p) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null state array");
  const size_t L = e->L;
  double* dst[7] = {e->X, e->X + L, e->X + 2 * L, e->V, e->V + L, e->V + 2 * L, e->M};
  long long off = 0;
  for (int c = 0; c < e->C; ++c) {
    for (int k = 0; k < 7; ++k)
      EN_CUDA(cudaMemcpyAsync(dst[k] + e->row0[c], src[k] + off, sizeof(double) * e->n[c],
                              cudaMemcpyHostToDevice, e->stream));
    off += e->n[c];
  }
  EN_CUDA(cudaMemsetAsync(e->D, 0, sizeof(double) * 6 * L, e->stream));
  if (e->perm) {  // the caller's order again; re-ordered before the next evaluation
    iota_kernel<<<(e->L + kBlock - 1) / kBlock, kBlock, 0, e->stream>>>(e->L, e->perm);
    EN_CUDA(cudaGetLastError());
  }
  e->sorted = e->permuted = false;
  EN_TRY(launch_ens_pack(e));
  EN_CUDA(cudaStreamSynchronize(e->stream));
  e->have_derivs = false;
  e->steps = 0;
  if (e->tiles_per_item < 0) EN_TRY(ens_autotune(e));
  return NBODY_OK;
}

nbody_status nbody_ensemble_get_state(nbody_ensemble* e, double* x, double* y, double* z,
                                      double* vx, double* vy, double* vz) {
  EN_TRY(ens_check(e));
  double* dst[6] = {x, y, z, vx, vy, vz};
  EN_TRY(ens_download(e, e->X, dst, 6));  // X(3) and V(3) are consecutive state arrays
  return ens_status(e);
}

nbody_status nbody_ensemble_get_derivs(nbody_ensemble* e, double* ax, double* ay, double* az,
                                       double* jx, double* jy, double* jz) {
  EN_TRY(ens_check(e));
  if (!e->have_derivs) return nbody_set_error(NBODY_ERR_STATE, "no derivatives yet");
  double* dst[6] = {ax, ay, az, jx, jy, jz};
  EN_TRY(ens_download(e, e->D, dst, 6));
  return ens_status(e);
}

nbody_status nbody_ensemble_acc_jerk(nbody_ensemble* e) {
  EN_TRY(ens_check(e));
  return ens_eval_current(e);
}

nbody_status nbody_ensemble_step(nbody_ensemble* e, int nsteps) {
  TraceRange trace_("nbody_ensemble_step");
  EN_TRY(ens_check(e));
  if (nsteps < 0) return nbody_set_error(NBODY_ERR_INVALID_ARG, "nsteps < 0");
  if (!e->have_derivs) EN_TRY(ens_eval_current(e));
  EN_TRY(ens_build_graph(e));
  for (int k = 0; k < nsteps; ++k) {
    if (e->fmt == kRecRel && e->since_sort >= e->sort_every) {
      EN_CUDA(cudaGraphLaunch(e->order_graph, e->stream));
      e->since_sort = 0;
      ++e->reorders;
    }
    EN_CUDA(cudaGraphLaunch(e->graph, e->stream));
    ++e->since_sort;
  }
  e->steps += nsteps;
  return NBODY_OK;
}

nbody_status nbody_ensemble_synchronize(nbody_ensemble* e) {
  EN_TRY(ens_check(e));
  EN_CUDA(cudaStreamSynchronize(e->stream));
  return ens_status(e);
}

nbody_status nbody_ensemble_energy(nbody_ensemble* e, double* T, double* U) {
  EN_TRY(ens_check(e));
  if (!T || !U) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null energy arrays");
  ens_pack_kernel<<<(e->L + kBlock - 1) / kBlock, kBlock, 0, e->stream>>>(e->L, e->cid, e->X, e->V,
                                                                        e->M, e->jb64, nullptr);
  ens_phi_kernel<<<e->n_blk, kBlock, 0, e->stream>>>(e->blk_cluster, e->blk_row, e->cl, e->jb64, e->phi);
  ens_energy_sum_kernel<<<e->C, kBlock, 0, e->stream>>>(e->cl, e->V, e->M, e->phi, e->L, e->Tc, e->Uc);
  EN_CUDA(cudaGetLastError());
  EN_CUDA(cudaMemcpyAsync(T, e->Tc, sizeof(double) * e->C, cudaMemcpyDeviceToHost, e->stream));
  EN_CUDA(cudaMemcpyAsync(U, e->Uc, sizeof(double) * e->C, cudaMemcpyDeviceToHost, e->stream));
  EN_CUDA(cudaStreamSynchronize(e->stream));
  return NBODY_OK;
}

nbody_status nbody_ensemble_info(nbody_ensemble* e, nbody_ensemble_info_t* out) {
  EN_TRY(ens_check(e));
  if (!out) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null info");
  EN_CUDA(cudaStreamSynchronize(e->stream));
  memset(out, 0, sizeof *out);
  out->nclusters = e->C;
  out->padded_rows = e->L;
  out->items = e->n_items;
  out->tiles_per_item = e->tiles_per_item;
  out->j_tile = e->kern->tile;
  out->threads = e->kern->nt;
  out->grid = e->grid;
  out->interactions_per_step = static_cast<double>(e->interactions);
  out->steps = e->steps;
  float ms = 0;
  if (e->graph && cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]) == cudaSuccess) out->last_step_ms = ms;
  cudaGetLastError();
  out->record_format = e->fmt;
  out->step_kernels = e->step_kernels;
  out->reorders = e->reorders;
  out->order_kernels = e->order_kernels;
  return NBODY_OK;
}

nbody_status nbody_ensemble_get_stream(nbody_ensemble* e, void** stream) {
  EN_TRY(ens_check(e));
  if (!stream) return nbody_set_error(NBODY_ERR_INVALID_ARG, "null stream out");
  *stream = e->stream;
  return NBODY_OK;
}

}  // extern "C"
