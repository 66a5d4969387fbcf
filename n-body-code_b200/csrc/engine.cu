// libnbody_cuda: the engine behind include/nbody_cuda.h.
//
// One engine = one system of n bodies on one device, one CUDA stream, and
// device memory allocated once at creation:
//   state  [13][ld] float64  X(3) V(3) M(1) D(6)  (D = current acc, jerk)
//   P      [S][6][ld]        split-j partial sums of the pair kernel
//   jb64   [ld] JBody64      FP64 j-records (also used by the potential)
//   jb32   [ld] JBody32      mixed-precision j-records (mixed engines):
//                            JBody32, JBodyX2, or tiles of JBodyNF
//   sort   keys, indices, CUB scratch of the Hilbert ordering (mixed engines)
//   perm   [2][ld] int       position -> caller's body index (tile-relative
//                            engines keep their state in Hilbert order)
//   scratch [13][ld]         re-ordered state, gathered caller input, or
//                            output on its way back to the caller's order
//   ctl    StepCtl           dt, t, Aarseth criterion, step counter
// ld = n rounded up to a multiple of 256 (kPad).
//
// A Hermite step - predict (O(N), writes the j-records; the near/far
// tile-relative kernel's records come from rel_tile_nf_kernel right after),
// pair (O(N^2)), correct (O(N), fused split reduction + snap/crackle +
// correction + dt criterion) - is captured once into a CUDA graph and
// replayed.  The Hilbert re-ordering of a tile-relative engine's state is a
// second captured graph, replayed ahead of every sort_every-th step.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/nbody_cuda.h"
#include "errors.h"
#include "hermite.cuh"
#include "pair.cuh"
#include "reltiles.cuh"
#include "trace.h"

using namespace nbody;

namespace {

constexpr int kPad = 256;        // body padding granularity (multiple of every j-tile)
constexpr int kMaxSplit = 64;    // split-j upper bound
// Rate at which the corrector sums split partials (64 splits at N = 65536:
// 201 MB in 52 us), the autotuner's price for each partial a tiling leaves.
constexpr double kSplitSumBytesPerMs = 3.9e9;
constexpr int kBlockO1 = 256;    // threads per CTA of the O(N) kernels
constexpr int kMaxBBoxParts = 512;  // CTAs of the bounding-box pass
constexpr int kOrderBits = 48;     // Hilbert key width (order_key_kernel)
// The drop-in orders by the top 30 bits (1024 cells per axis, the curve's
// level-10 cells): four radix passes instead of six on every call.  Bodies
// that share a cell keep their input order, which moves no tile boundary
// beyond the cell.
constexpr int kDropInOrderLowBit = 18;
constexpr int kMaxPotSplit = 32;    // j-splits of the potential diagnostic

thread_local std::string g_last_error;

nbody_status fail(nbody_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

#define NB_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? NBODY_ERR_OOM : NBODY_ERR_CUDA,          \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#define NB_TRY(expr)                 \
  do {                               \
    nbody_status s_ = (expr);        \
    if (s_ != NBODY_OK) return s_;   \
  } while (0)

// ---------------------------------------------------------------------------
// Pair-kernel registry: every compiled (precision, NT, IPT, TJ) instantiation.
// ---------------------------------------------------------------------------
struct PairKernel {
  int precision, nt, ipt, tj;
  int fmt;      // RecordFormat of the j-records it reads
  const void* fn;
  size_t smem;  // dynamic shared memory: two j-tile buffers (+ FP64 accumulators)
  int acc_smem = 0, junroll = 2, minb = 1;
  int near = 0;  // tile-relative: 1 = near tiles in double-single (variant 4), 0 = all far (5)
  int cluster = 1;  // CTAs per thread-block cluster along j (splits summed in the cluster)
};

template <int NT, int IPT, int TJ, int JU = 2, int MINB = 1>
PairKernel make_fp64() {
  return {NBODY_FP64, NT, IPT, TJ, kRecF64,
          reinterpret_cast<const void*>(&pair_fp64_kernel<NT, IPT, TJ, JU, MINB>),
          2 * TJ * sizeof(JBody64), 0, JU, MINB};
}
template <int NT, int IPT, int TJ>
PairKernel make_mixed() {
  return {NBODY_MIXED, NT, IPT, TJ, kRecF32,
          reinterpret_cast<const void*>(&pair_mixed_kernel<NT, IPT, TJ>), 2 * TJ * sizeof(JBody32)};
}
template <int NT, int IPT, int TJ, int ACC = 0, int JU = 2, int MINB = 1>
PairKernel make_mixed_x2() {
  return {NBODY_MIXED, NT, IPT, TJ, kRecX2,
          reinterpret_cast<const void*>(&pair_mixed_x2_kernel<NT, IPT, TJ, ACC, JU, MINB>),
          2 * TJ * sizeof(JBodyX2) + (ACC ? sizeof(double) * 6 * IPT * NT : 0), ACC, JU, MINB};
}

template <int NT, int IPT, int TJ, int ACC = 1, int JU = 1, int MINB = 1, int NEAR = 1>
PairKernel make_mixed_nf() {
  return {NBODY_MIXED, NT, IPT, TJ, kRecRel,
          reinterpret_cast<const void*>(&pair_mixed_nf_kernel<NT, IPT, TJ, ACC, JU, MINB, NEAR>),
          2 * (TJ + 1) * sizeof(JBodyNF) + (ACC ? sizeof(double) * 6 * IPT * NT : 0), ACC, JU,
          MINB, NEAR ? 1 : 0};
}

// Near/far rows on clusters of CL CTAs along j: split count a multiple of CL,
// S / CL partials (pair_mixed_nf_cluster_kernel).
template <int NT, int IPT, int TJ, int JU, int MINB, int NEAR, int CL>
PairKernel make_mixed_nf_cl() {
  return {NBODY_MIXED, NT, IPT, TJ, kRecRel,
          reinterpret_cast<const void*>(&pair_mixed_nf_cluster_kernel<NT, IPT, TJ, JU, MINB, NEAR, CL>),
          2 * (TJ + 1) * sizeof(JBodyNF) + sizeof(double) * 6 * IPT * NT, 1, JU, MINB, 1, CL};
}

// The first entry of each shape/variant is the one explicit tilings select
// (never a cluster kernel); the autotuner times all of them.
const std::vector<PairKernel>& registry() {
  static const std::vector<PairKernel> r = {
      make_fp64<128, 2, 128, 1>(),  make_fp64<128, 2, 128, 2>(),  make_fp64<128, 1, 128, 4>(),
      make_fp64<128, 1, 128, 2>(),  make_fp64<128, 4, 128, 1>(),  make_fp64<256, 1, 128, 4>(),
      make_fp64<256, 2, 128, 1>(),  make_fp64<128, 2, 256, 1>(),  make_fp64<64, 2, 128, 1>(),
      make_fp64<128, 2, 128, 1, 6>(), make_fp64<128, 2, 64, 1, 6>(), make_fp64<128, 1, 128, 4, 8>(),
      // near/far tile-relative packed pairs (bodies in Hilbert order; default
      // mixed: 128 x 4 rows, j-unroll 2, 4 CTAs/SM = 128 registers, no spills)
      make_mixed_nf<128, 4, 128, 1, 2, 4>(), make_mixed_nf<64, 4, 128>(), make_mixed_nf<128, 2, 128>(),
      make_mixed_nf<256, 2, 128>(), make_mixed_nf<256, 4, 128>(), make_mixed_nf<128, 2, 64>(),
      make_mixed_nf<128, 4, 64>(),  make_mixed_nf<128, 2, 256>(), make_mixed_nf<128, 4, 128, 0, 2>(),
      make_mixed_nf<128, 4, 128>(), make_mixed_nf<128, 4, 128, 1, 1, 4>(),
      make_mixed_nf<64, 4, 128, 1, 1, 8>(),  make_mixed_nf<128, 6, 128, 1, 1>(),
      make_mixed_nf<64, 6, 128, 1, 1>(),     make_mixed_nf<128, 4, 128, 1, 2>(),
      make_mixed_nf<128, 4, 64, 1, 2, 4>(),  make_mixed_nf<128, 2, 64, 1, 2, 4>(),
      make_mixed_nf<128, 4, 128, 1, 2, 4, 2>(), make_mixed_nf<64, 4, 128, 1, 2, 8, 2>(),
      // the same kernel with every tile taken as far (plain tile-relative
      // separations; pair_variant 5, a measured comparison)
      make_mixed_nf<128, 4, 128, 1, 2, 4, 0>(), make_mixed_nf<128, 2, 128, 1, 1, 1, 0>(),
      // near/far on thread-block clusters along j (fewer split partials;
      // selected by nbody_config.j_cluster, not by the autotuner)
      make_mixed_nf_cl<128, 4, 128, 2, 4, 2, 8>(), make_mixed_nf_cl<128, 4, 128, 2, 4, 2, 4>(),
      make_mixed_nf_cl<128, 4, 128, 2, 4, 2, 2>(),
      // packed pairs, FP64 accumulators in shared memory (default)
      make_mixed_x2<128, 4, 128, 1, 1>(), make_mixed_x2<256, 4, 128, 1, 1>(),
      make_mixed_x2<128, 4, 128, 1, 2>(), make_mixed_x2<64, 4, 128, 1, 1>(),
      make_mixed_x2<128, 2, 128, 1, 1>(),
      make_mixed_x2<128, 4, 64, 1, 1, 5>(), make_mixed_x2<128, 4, 64, 1, 1, 6>(),
      make_mixed_x2<128, 4, 64, 1, 1>(),    make_mixed_x2<64, 4, 64, 1, 1, 10>(),
      // packed pairs, FP64 accumulators in registers
      make_mixed_x2<128, 4, 128, 0, 2>(), make_mixed_x2<128, 2, 128, 0, 2>(),
      make_mixed_x2<256, 2, 128, 0, 2>(), make_mixed_x2<64, 4, 128, 0, 2>(),
      make_mixed_x2<128, 4, 64, 0, 2>(),
      // scalar FP32
      make_mixed<128, 4, 128>(),    make_mixed<128, 2, 128>(),    make_mixed<256, 2, 128>(),
      make_mixed<128, 4, 256>(),    make_mixed<64, 4, 128>(),
  };
  return r;
}

// variant (mixed only, after resolving 0 = automatic): 1 = scalar FP32
// hi/lo, 2 = packed hi/lo pairs with register accumulators, 3 = packed
// hi/lo pairs with shared-memory FP64 accumulators (falling back to
// register accumulators where that shape has none), 4 = near/far
// tile-relative, 5 = tile-relative with every tile taken as far.
const PairKernel* find_kernel(int precision, int nt, int ipt, int tj, int variant,
                              int cluster = 1) {
  auto match = [&](int fmt, int acc, int near = 1) -> const PairKernel* {
    for (const auto& k : registry())
      if (k.precision == precision && k.nt == nt && k.ipt == ipt && k.tj == tj &&
          (fmt < 0 || k.fmt == fmt) && (acc < 0 || k.acc_smem == acc) &&
          (k.fmt != kRecRel || k.near == near) && k.cluster == cluster)
        return &k;
    return nullptr;
  };
  if (precision == NBODY_FP64) return match(kRecF64, -1);
  if (variant == 1) return match(kRecF32, -1);
  if (variant == 4) return match(kRecRel, -1, 1);
  if (variant == 5) return match(kRecRel, -1, 0);
  if (variant == 2) return match(kRecX2, 0);
  const PairKernel* k = match(kRecX2, 1);
  return k ? k : match(kRecX2, 0);
}


struct Tiling {
  const PairKernel* k = nullptr;
  int split = 1;   // CTAs along j
  int source = 0;  // nbody_timers.tiling_source: 1 heuristic/explicit, 2 timed, 3 cached
};

// Split partials a launch of tiling t leaves in P (cluster kernels sum their
// CL CTAs' partials into one).
int partial_count(const Tiling& t) { return t.split / t.k->cluster; }

// Autotune results shared by all engines of the process: (device, precision,
// record format, ld, rows) -> tiling.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, std::pair<int, int>> g_tuned;  // -> (kernel idx, split)

}  // namespace

nbody_status nbody_set_error(nbody_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

struct nbody_engine {
  nbody_config cfg{};
  int n = 0, ld = 0, dev = 0, num_sms = 0;
  cudaStream_t stream = nullptr;
  double* state = nullptr;  // [13][ld]
  double *X = nullptr, *V = nullptr, *M = nullptr, *D = nullptr;
  double* P = nullptr;
  int p_splits = 0;
  JBody64* jb64 = nullptr;
  void* jb32 = nullptr;  // mixed records: JBody32 or JBodyX2 (sized for the larger)
  JBody64* jbe = nullptr;  // records of the energy diagnostic (never a pair kernel's input)
  // Hilbert ordering (mixed engines).  A tile-relative engine keeps its state
  // in Hilbert order: position p holds the caller's body perm[p].
  uint64_t* sort_keys = nullptr;  // [2][ld]: keys, sorted keys
  int* sort_idx = nullptr;        // [2][ld]: positions, sorted positions (= order)
  double* bbox_part = nullptr;    // [kMaxBBoxParts][6]
  void* sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;
  int* perm = nullptr;            // [2][ld]: position -> body index, and its re-ordered copy
  double* scratch = nullptr;      // [13][ld]: re-ordered state / gathered caller input / un-permuted output
  unsigned long long* near_count = nullptr;  // near tiles of the last near/far pair launch
  bool sorted = false;            // the state is in (recent) Hilbert order
  bool permuted = false;          // perm is not the identity
  int since_sort = 0;             // steps since the last re-ordering
  StepCtl* ctl = nullptr;
  double* partial = nullptr;  // reduction scratch: ld / 256 + 1 doubles + 4 scalars
  int* status = nullptr;
  Tiling tiling;
  bool tiled = false;
  cudaGraphExec_t graph = nullptr;
  int graph_kernels = 0;  // kernel nodes of the captured step
  // automatic mixed kernel (pair_variant 0): near/far from this many bodies,
  // packed hi/lo below (measured Hermite steps, Plummer spheres: N = 8192
  // 0.136 vs 0.124 ms, N = 16384 0.352 vs 0.366 ms).  Engines re-order every
  // sort_every steps; the drop-in re-orders on every call and raises the
  // threshold.
  int rel_min_bodies = 16384;
  // drop-in engines: reuse a tiling the autotuner chose for the same
  // (device, precision, record format, size) in this process; never tune
  bool tune_lookup = false;
  cudaGraphExec_t order_graph = nullptr;  // captured Hilbert re-ordering (variant 0)
  cudaStream_t aux = nullptr;              // drop-in: uploads that overlap the ordering
  cudaEvent_t aux_ev[2] = {nullptr, nullptr};
  int order_kernels = 0;
  long long reorders = 0;  // re-orderings run before steps
  bool have_state = false, have_derivs = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev_init[2] = {nullptr, nullptr};
  bool step_events = false, init_events = false;
};

namespace {

int round_up(int a, int b) { return (a + b - 1) / b * b; }

// The mixed kernel family in use: pair_variant, with 0 (automatic)
// resolved by the system size.
int effective_variant(const nbody_engine* e) {
  const nbody_config& c = e->cfg;
  if (c.precision != NBODY_MIXED || c.pair_variant != 0) return c.pair_variant;
  return e->n >= e->rel_min_bodies ? 4 : 3;
}

// Record format of the autotuner's family (the automatic choice).
int default_format(const nbody_engine* e) {
  if (e->cfg.precision == NBODY_FP64) return kRecF64;
  return effective_variant(e) >= 4 ? kRecRel : kRecX2;
}

// The engine keeps its bodies in Hilbert order (positions != body indices).
bool curve_resident(const nbody_engine* e);

nbody_status check_status_word(nbody_engine* e) {
  int h = 0;
  NB_CUDA(cudaMemcpyAsync(&h, e->status, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  NB_CUDA(cudaStreamSynchronize(e->stream));
  if (h == kKernelTimeout) {
    cudaMemsetAsync(e->status, 0, sizeof(int), e->stream);
    return fail(NBODY_ERR_TIMEOUT, "a pair-kernel shared-memory wait exceeded its limit");
  }
  return NBODY_OK;
}

// Split count from a wave model: CTAs = i_blocks * S run in waves of
// (SMs x resident CTAs); each CTA costs its j-tiles plus a fixed overhead.
nbody_status prepare_kernel(const PairKernel& k);

int choose_split(const nbody_engine* e, const PairKernel& k, int rows) {
  prepare_kernel(k);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k.fn, k.nt, k.smem) != cudaSuccess ||
      occ < 1)
    occ = 1;
  const long slots = static_cast<long>(e->num_sms) * occ;
  const long i_blocks = (rows + k.nt * k.ipt - 1) / (k.nt * k.ipt);
  const int n_tiles = e->ld / k.tj;
  // A small system (a few tile-units of work per resident CTA slot) is
  // latency-bound: the most CTAs win (N = 4096: S = 32 measured 40 us,
  // S = 16 46 us, FP64 one row per thread).
  if (i_blocks * n_tiles <= 4 * slots) return std::min(n_tiles, kMaxSplit);
  double best = 1e300;
  int best_s = 1;
  for (int s = 1; s <= std::min(kMaxSplit, n_tiles); ++s) {
    const long ctas = i_blocks * s;
    const long waves = (ctas + slots - 1) / slots;
    const int tps = (n_tiles + s - 1) / s;
    const double cost = waves * (tps + 0.25) + 0.002 * s;  // last term: split reduction traffic
    if (cost < best - 1e-9) {
      best = cost;
      best_s = s;
    }
  }
  return best_s;
}

nbody_status ensure_partials(nbody_engine* e, int split) {
  if (split <= e->p_splits) return NBODY_OK;
  if (e->P) {
    NB_CUDA(cudaStreamSynchronize(e->stream));
    cudaFree(e->P);
  }
  if (e->graph) {  // the captured step refers to the old buffer
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  e->P = nullptr;
  e->p_splits = 0;
  NB_CUDA(cudaMalloc(&e->P, sizeof(double) * 6 * static_cast<size_t>(e->ld) * split));
  e->p_splits = split;
  return NBODY_OK;
}

// Every pair kernel opts in to its dynamic shared memory size once per
// device (static + dynamic above 48 KB needs the attribute).
std::mutex g_prep_mu;
std::set<std::pair<int, const void*>> g_prepared;

nbody_status prepare_kernel(const PairKernel& k) {
  int dev = 0;
  NB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(g_prep_mu);
  if (g_prepared.count({dev, k.fn})) return NBODY_OK;
  NB_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(k.smem)));
  g_prepared.insert({dev, k.fn});
  return NBODY_OK;
}

SoA7 own_inputs(nbody_engine* e);

// src / n_src: the inputs the records were built from (the tile-relative
// kernel reads its i-rows there); nullptr = the engine's own state.
nbody_status launch_pair(nbody_engine* e, const Tiling& t, int i_begin, int i_end,
                         cudaStream_t st, const SoA7* src = nullptr, int n_src = 0) {
  const PairKernel& k = *t.k;
  NB_TRY(prepare_kernel(k));
  PairArgs a;
  a.i_begin = i_begin;
  a.i_end = i_end;
  a.n_rows_pad = e->ld;
  if (k.fmt == kRecRel) {
    const SoA7 in = src ? *src : own_inputs(e);
    a.rows = RowSrc{in.x, in.y, in.z, in.vx, in.vy, in.vz};
    a.n_rows_pad = src ? n_src : e->n;
    if (k.near && i_end > i_begin) {  // count this launch's near tiles
      NB_CUDA(cudaMemsetAsync(e->near_count, 0, sizeof(unsigned long long), st));
      a.near_count = e->near_count;
    }
  }
  a.n_tiles = e->ld / k.tj;
  a.tiles_per_split = (a.n_tiles + t.split - 1) / t.split;
  a.eps2 = e->cfg.eps2;
  a.out = e->P;
  a.stride = static_cast<size_t>(e->ld);
  a.status = e->status;
  const int rows = i_end - i_begin;
  if (rows <= 0) return NBODY_OK;
  dim3 grid((rows + k.nt * k.ipt - 1) / (k.nt * k.ipt), t.split);
  const void* jb = k.fmt == kRecF64 ? static_cast<const void*>(e->jb64)
                                     : static_cast<const void*>(e->jb32);
  void* args[] = {const_cast<void*>(static_cast<const void*>(&jb)), static_cast<void*>(&a)};
  NB_CUDA(cudaLaunchKernel(k.fn, grid, dim3(k.nt), args, k.smem, st));
  return NBODY_OK;
}

nbody_status launch_pack(nbody_engine* e, int n, const SoA7& in, cudaStream_t st, int fmt,
                         int tj);
nbody_status enqueue_reorder_state(nbody_engine* e, cudaStream_t st);

// The tiling the autotuner cached for this engine's (device, precision,
// record format, ld, rows), if any.
bool tuned_lookup(const nbody_engine* e, int rows, Tiling* out) {
  const auto key = std::make_tuple(e->dev, e->cfg.precision, default_format(e), e->ld, rows);
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tuned.find(key);
  if (it == g_tuned.end()) return false;
  out->k = &registry()[it->second.first];
  out->split = it->second.second;
  out->source = 3;
  return true;
}

nbody_status autotune(nbody_engine* e, int rows, Tiling* out) {
  const auto key = std::make_tuple(e->dev, e->cfg.precision, default_format(e), e->ld, rows);
  if (tuned_lookup(e, rows, out)) return NBODY_OK;
  cudaEvent_t a, b;
  NB_CUDA(cudaEventCreate(&a));
  NB_CUDA(cudaEventCreate(&b));
  float best = 1e30f;
  int best_idx = -1, best_split = 1;
  const auto& reg = registry();
  // the near/far kernel's cost depends on the bodies being in Hilbert order
  if (default_format(e) == kRecRel && e->have_state && !e->sorted)
    NB_TRY(enqueue_reorder_state(e, e->stream));
  for (size_t idx = 0; idx < reg.size(); ++idx) {
    const PairKernel& k = reg[idx];
    if (k.precision != e->cfg.precision || k.fmt != default_format(e)) continue;
    if (k.fmt == kRecRel && !k.near) continue;  // the automatic choice keeps near tiles exact
    // cluster kernels save in the split sums what their pair pass loses
    // (N = 65536: 4.071 vs 4.071 ms with the sums priced in); not timed
    if (k.cluster > 1) continue;
    const int s0 = choose_split(e, k, rows);
    NB_TRY(launch_pack(e, e->n, own_inputs(e), e->stream, k.fmt, k.tj));
    for (int s : {std::max(1, s0 / 2), s0, std::min(kMaxSplit, s0 * 2)}) {
      s = std::min(kMaxSplit, (s + k.cluster - 1) / k.cluster * k.cluster);
      NB_TRY(ensure_partials(e, s));
      Tiling t{&k, s};
      NB_TRY(launch_pair(e, t, 0, rows, e->stream));  // warm-up
      NB_CUDA(cudaEventRecord(a, e->stream));
      for (int r = 0; r < 3; ++r) NB_TRY(launch_pair(e, t, 0, rows, e->stream));
      NB_CUDA(cudaEventRecord(b, e->stream));
      NB_CUDA(cudaEventSynchronize(b));
      float pair_ms = 0.f;
      NB_CUDA(cudaEventElapsedTime(&pair_ms, a, b));
      pair_ms /= 3;
      // the split partials are summed after every pass (corrector or
      // reduction): 48 bytes per row and partial at the measured 3.9 TB/s
      const float ms = pair_ms + static_cast<float>(48.0 * (s / k.cluster) * rows / kSplitSumBytesPerMs);
      if (getenv("NBODY_TUNE_VERBOSE"))
        fprintf(stderr, "[nbody tune] #%zu prec=%d rows=%d nt=%d ipt=%d tj=%d fmt=%d acc_smem=%d ju=%d minb=%d cluster=%d split=%d  %.4f ms (pair %.4f)\n",
                idx, k.precision, rows, k.nt, k.ipt, k.tj, k.fmt, k.acc_smem, k.junroll, k.minb,
                k.cluster, s, ms, pair_ms);
      if (ms < best) {
        best = ms;
        best_idx = static_cast<int>(idx);
        best_split = s;
      }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  NB_TRY(check_status_word(e));
  if (best_idx < 0) return fail(NBODY_ERR_STATE, "autotune found no kernel");
  out->k = &reg[best_idx];
  out->split = best_split;
  out->source = 2;
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tuned[key] = {best_idx, best_split};
  return NBODY_OK;
}

// Tiling for `rows` i-rows: explicit config, else tuned, else heuristic.
nbody_status get_tiling(nbody_engine* e, int rows, Tiling* out) {
  const nbody_config& c = e->cfg;
  // defaults: the best measured shape of each family (Plummer N = 65536);
  // small systems take half the rows per thread, which doubles their row
  // blocks (FP64 below 32768 rows: N = 4096 40 vs 48 us per launch;
  // tile-relative below 8192 rows)
  const int variant = effective_variant(e);
  const bool rel = c.precision == NBODY_MIXED && variant == 4;
  int nt = c.threads ? c.threads : 128;
  int ipt = c.i_per_thread ? c.i_per_thread
                           : rel ? (rows < 8192 ? 2 : 4)
                                 : (c.precision == NBODY_FP64 && rows < 32768 ? 1 : 2);
  int tj = c.j_tile ? c.j_tile : 128;
  const int cl = c.j_cluster > 1 ? c.j_cluster : 1;
  const PairKernel* k = find_kernel(c.precision, nt, ipt, tj, variant, cl);
  if (!k)
    return fail(NBODY_ERR_INVALID_ARG,
                "no compiled pair kernel for threads=%d i_per_thread=%d j_tile=%d variant=%d", nt,
                ipt, tj, variant);
  const bool automatic = !c.threads && !c.i_per_thread && !c.j_tile && !c.split_j &&
                         !c.pair_variant && !c.j_cluster;
  if (c.tune && automatic) return autotune(e, rows, out);
  if (e->tune_lookup && automatic && tuned_lookup(e, rows, out)) return NBODY_OK;
  out->k = k;
  out->split = c.split_j ? std::min(c.split_j, kMaxSplit) : choose_split(e, *k, rows);
  out->split = std::min(kMaxSplit, (out->split + cl - 1) / cl * cl);  // whole clusters
  out->source = 1;
  return NBODY_OK;
}

// The packed hi/lo kernel (pair_variant 3) for `rows` rows, heuristic split.
nbody_status hilo_tiling(nbody_engine* e, int rows, Tiling* out) {
  const PairKernel* k = find_kernel(NBODY_MIXED, 128, 2, 128, 3);
  if (!k) return fail(NBODY_ERR_STATE, "no packed hi/lo kernel compiled");
  out->k = k;
  out->split = choose_split(e, *k, rows);
  out->source = 1;
  return NBODY_OK;
}

nbody_status ensure_tiling(nbody_engine* e) {
  if (e->tiled) return NBODY_OK;
  NB_TRY(get_tiling(e, e->n, &e->tiling));
  NB_TRY(ensure_partials(e, e->tiling.split));
  e->tiled = true;
  return NBODY_OK;
}

SoA7 own_inputs(nbody_engine* e) {
  return SoA7{e->X, e->X + e->ld, e->X + 2 * e->ld, e->M, e->V, e->V + e->ld, e->V + 2 * e->ld};
}
SoA6 own_derivs(nbody_engine* e) {
  double* D = e->D;
  const size_t ld = e->ld;
  return SoA6{D, D + ld, D + 2 * ld, D + 3 * ld, D + 4 * ld, D + 5 * ld};
}

// Hilbert order of bodies [0, n) of `in` (bounding box, keys, stable sort):
// sort_idx + ld then holds, for each sorted position q, the index in `in` of
// the body that goes there.
nbody_status enqueue_curve_order(nbody_engine* e, int n, const SoA7& in, cudaStream_t st,
                                 int low_bit = 0) {
  const int parts = std::min(kMaxBBoxParts, (n + kBBoxThreads - 1) / kBBoxThreads);
  bbox_partial_kernel<<<parts, kBBoxThreads, 0, st>>>(n, in, e->bbox_part);
  NB_CUDA(cudaGetLastError());
  const size_t ld = e->ld;
  order_key_kernel<<<(n + kBBoxThreads - 1) / kBBoxThreads, kBBoxThreads, 0, st>>>(
      n, in, e->bbox_part, parts, e->sort_keys, e->sort_idx);
  NB_CUDA(cudaGetLastError());
  size_t bytes = e->sort_tmp_bytes;
  NB_CUDA(cub::DeviceRadixSort::SortPairs(e->sort_tmp, bytes, e->sort_keys, e->sort_keys + ld,
                                          e->sort_idx, e->sort_idx + ld, n, low_bit, kOrderBits,
                                          st));
  return NBODY_OK;
}

GatherArgs gather_args(const double* src, double* dst, size_t ld, int arrays) {
  GatherArgs g;
  g.arrays = arrays;
  for (int a = 0; a < kMaxGather; ++a) {
    g.src[a] = a < arrays && src ? src + a * ld : nullptr;
    g.dst[a] = a < arrays ? dst + a * ld : nullptr;
  }
  return g;
}

// Re-orders the engine's own state into the Hilbert order of its current
// positions: keys and sort, a gather of all 13 state arrays (and of perm)
// into scratch, and a copy back.  Capturable (the re-ordering graph).
nbody_status enqueue_reorder_state(nbody_engine* e, cudaStream_t st) {
  const size_t ld = e->ld;
  NB_TRY(enqueue_curve_order(e, e->n, own_inputs(e), st));
  gather_rows_kernel<<<(e->n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, st>>>(
      e->n, e->sort_idx + ld, gather_args(e->state, e->scratch, ld, 13), e->perm, e->perm + ld);
  NB_CUDA(cudaGetLastError());
  // scratch rows >= n are zero from creation and never written, so the padding stays zero
  NB_CUDA(cudaMemcpyAsync(e->state, e->scratch, sizeof(double) * 13 * ld, cudaMemcpyDeviceToDevice, st));
  NB_CUDA(cudaMemcpyAsync(e->perm, e->perm + ld, sizeof(int) * e->n, cudaMemcpyDeviceToDevice, st));
  e->sorted = true;
  e->permuted = true;
  e->since_sort = 0;
  return NBODY_OK;
}

// Near/far tile records of bodies [0, n) of `in`, which must already be in
// Hilbert order (positions).
nbody_status build_rel_tiles(nbody_engine* e, int n, const SoA7& in, cudaStream_t st, int tj) {
  JBodyNF* out = static_cast<JBodyNF*>(e->jb32);
  const int tiles = e->ld / tj;
  switch (tj) {
    case 64: rel_tile_nf_kernel<64><<<tiles, 64, 0, st>>>(n, in, out); break;
    case 128: rel_tile_nf_kernel<128><<<tiles, 128, 0, st>>>(n, in, out); break;
    case 256: rel_tile_nf_kernel<256><<<tiles, 256, 0, st>>>(n, in, out); break;
    default: return fail(NBODY_ERR_INVALID_ARG, "no tile-relative record builder for j_tile %d", tj);
  }
  NB_CUDA(cudaGetLastError());
  return NBODY_OK;
}

// Writes the j-records of a pair kernel's format: FP64 records (hi/lo
// kernels: also theirs), or tiles of tj near/far records of `in`, which must
// then be in Hilbert order.  (The energy diagnostic packs its own records.)
nbody_status launch_pack(nbody_engine* e, int n, const SoA7& in, cudaStream_t st, int fmt,
                         int tj) {
  if (fmt != kRecRel) {
    pack_kernel<<<(e->ld + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, st>>>(
        n, e->ld, in, e->jb64, fmt == kRecF32 ? static_cast<JBody32*>(e->jb32) : nullptr,
        fmt == kRecX2 ? static_cast<JBodyX2*>(e->jb32) : nullptr);
    NB_CUDA(cudaGetLastError());
  } else {
    NB_TRY(build_rel_tiles(e, n, in, st, tj));
  }
  return NBODY_OK;
}

// acc + jerk of n bodies given in any order (`in`, device arrays) with the
// near/far kernel, after enqueue_curve_order(in): a gather of `in` into
// scratch in that order, tiles, the pair pass, and the split reduction
// written back through the order into `out` (the caller's body order).
// Leaves the engine's own state alone.
nbody_status eval_foreign_rel(nbody_engine* e, const Tiling& t, int n, const SoA7& in,
                              const SoA6& out, cudaStream_t st, bool reduce = true) {
  const size_t ld = e->ld;
  const int* ord = e->sort_idx + ld;
  const double* srcs[7] = {in.x, in.y, in.z, in.m, in.vx, in.vy, in.vz};
  GatherArgs g = gather_args(nullptr, e->scratch, ld, 7);
  for (int a = 0; a < 7; ++a) g.src[a] = srcs[a];
  gather_rows_kernel<<<(n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, st>>>(n, ord, g, nullptr, nullptr);
  NB_CUDA(cudaGetLastError());
  const SoA7 sorted{g.dst[0], g.dst[1], g.dst[2], g.dst[3], g.dst[4], g.dst[5], g.dst[6]};
  NB_TRY(build_rel_tiles(e, n, sorted, st, t.k->tj));
  NB_TRY(launch_pair(e, t, 0, n, st, &sorted, n));
  if (!reduce) return NBODY_OK;  // the caller sums the splits (rows in sort_idx + ld order)
  reduce_splits_kernel<<<(n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, st>>>(
      0, n, e->ld, partial_count(t), e->P, out, nullptr, ord);
  NB_CUDA(cudaGetLastError());
  return NBODY_OK;
}

int tiling_fmt(const nbody_engine* e) { return e->tiled ? e->tiling.k->fmt : kRecF64; }
int tiling_tj(const nbody_engine* e) { return e->tiled ? e->tiling.k->tj : 0; }
int sort_period(const nbody_engine* e) { return e->cfg.sort_every > 0 ? e->cfg.sort_every : 16; }

bool curve_resident(const nbody_engine* e) { return tiling_fmt(e) == kRecRel; }

// Before a step of the engine's own state: re-order when the order is stale
// (never made since set_state, or sort_every steps old).
nbody_status maybe_reorder(nbody_engine* e, cudaStream_t st) {
  if (!curve_resident(e)) return NBODY_OK;
  if (!e->sorted || e->since_sort >= sort_period(e)) {
    if (e->order_graph && st == e->stream) {
      NB_CUDA(cudaGraphLaunch(e->order_graph, st));
      e->sorted = true;
      e->permuted = true;
      e->since_sort = 0;
    } else {
      NB_TRY(enqueue_reorder_state(e, st));
    }
    ++e->reorders;
  }
  ++e->since_sort;
  return NBODY_OK;
}

// acc + jerk of the engine's current X, V, M into D (rows [0, n)).
nbody_status eval_current(nbody_engine* e) {
  NB_TRY(ensure_tiling(e));
  if (curve_resident(e) && !e->sorted) NB_TRY(enqueue_reorder_state(e, e->stream));
  NB_TRY(launch_pack(e, e->n, own_inputs(e), e->stream, tiling_fmt(e), tiling_tj(e)));
  if (!e->init_events) {
    NB_CUDA(cudaEventCreate(&e->ev_init[0]));
    NB_CUDA(cudaEventCreate(&e->ev_init[1]));
    e->init_events = true;
  }
  NB_CUDA(cudaEventRecord(e->ev_init[0], e->stream));
  NB_TRY(launch_pair(e, e->tiling, 0, e->n, e->stream));
  reduce_splits_kernel<<<(e->n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, e->stream>>>(
      0, e->n, e->ld, partial_count(e->tiling), e->P, own_derivs(e));
  NB_CUDA(cudaGetLastError());
  NB_CUDA(cudaEventRecord(e->ev_init[1], e->stream));
  if (e->cfg.dt <= 0.0) {
    initialdt_kernel<<<(e->n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, e->stream>>>(
        e->n, e->ld, e->D, e->ctl, e->cfg.eta0);
    NB_CUDA(cudaGetLastError());
  }
  e->have_derivs = true;
  return NBODY_OK;
}

nbody_status enqueue_predict(nbody_engine* e, cudaStream_t st) {
  const int fmt = tiling_fmt(e);
  predict_kernel<<<(e->n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, st>>>(
      e->n, e->ld, e->ctl, e->X, e->V, e->M, e->D, fmt == kRecF64 ? e->jb64 : nullptr,
      fmt == kRecF32 ? static_cast<JBody32*>(e->jb32) : nullptr,
      fmt == kRecX2 ? static_cast<JBodyX2*>(e->jb32) : nullptr);
  NB_CUDA(cudaGetLastError());
  if (fmt == kRecRel) NB_TRY(build_rel_tiles(e, e->n, own_inputs(e), st, tiling_tj(e)));
  return NBODY_OK;
}

nbody_status enqueue_correct(nbody_engine* e, cudaStream_t st) {
  correct_kernel<<<(e->n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, st>>>(
      e->n, e->ld, partial_count(e->tiling), e->P, e->X, e->V, e->D, e->ctl, e->cfg.eta);
  NB_CUDA(cudaGetLastError());
  return NBODY_OK;
}

int count_kernel_nodes(cudaGraph_t g) {
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

nbody_status build_step_graph(nbody_engine* e) {
  if (e->graph) return NBODY_OK;
  NB_TRY(ensure_tiling(e));
  if (!e->step_events) {
    for (auto& ev : e->ev) NB_CUDA(cudaEventCreate(&ev));
    e->step_events = true;
  }
  cudaGraph_t g = nullptr;
  NB_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  nbody_status s = NBODY_OK;
  auto rec = [&](cudaEvent_t ev) {
    if (s == NBODY_OK && cudaEventRecordWithFlags(ev, e->stream, cudaEventRecordExternal) != cudaSuccess)
      s = fail(NBODY_ERR_CUDA, "event record during capture failed");
  };
  rec(e->ev[0]);
  if (s == NBODY_OK) s = enqueue_predict(e, e->stream);
  rec(e->ev[1]);
  if (s == NBODY_OK) s = launch_pair(e, e->tiling, 0, e->n, e->stream);
  rec(e->ev[2]);
  if (s == NBODY_OK) s = enqueue_correct(e, e->stream);
  rec(e->ev[3]);
  cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
  if (s != NBODY_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (ce != cudaSuccess) return fail(NBODY_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
  e->graph_kernels = count_kernel_nodes(g);
  ce = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    e->graph = nullptr;
    return fail(NBODY_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
  }
  if (tiling_fmt(e) == kRecRel && !e->order_graph) {
    // the Hilbert re-ordering of the engine's own state, replayed every
    // sort_every steps ahead of the step graph
    const bool sorted = e->sorted, permuted = e->permuted;
    const int since = e->since_sort;
    NB_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    s = enqueue_reorder_state(e, e->stream);
    g = nullptr;
    ce = cudaStreamEndCapture(e->stream, &g);
    e->sorted = sorted;  // capturing ran nothing
    e->permuted = permuted;
    e->since_sort = since;
    if (s != NBODY_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    if (ce != cudaSuccess) return fail(NBODY_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    e->order_kernels = count_kernel_nodes(g);
    ce = cudaGraphInstantiate(&e->order_graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      e->order_graph = nullptr;
      return fail(NBODY_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
    }
  }
  return NBODY_OK;
}

nbody_status check_engine(nbody_engine* e) {
  if (!e) return fail(NBODY_ERR_INVALID_ARG, "null engine");
  if (cudaSetDevice(e->dev) != cudaSuccess) return fail(NBODY_ERR_CUDA, "cudaSetDevice(%d) failed", e->dev);
  return NBODY_OK;
}

nbody_status need_state(nbody_engine* e) {
  NB_TRY(check_engine(e));
  if (!e->have_state) return fail(NBODY_ERR_STATE, "no state uploaded (call nbody_set_state)");
  return NBODY_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* nbody_last_error(void) { return g_last_error.c_str(); }

const char* nbody_status_string(nbody_status s) {
  switch (s) {
    case NBODY_OK: return "ok";
    case NBODY_ERR_INVALID_ARG: return "invalid argument";
    case NBODY_ERR_OOM: return "out of memory";
    case NBODY_ERR_CUDA: return "CUDA error";
    case NBODY_ERR_TIMEOUT: return "in-kernel wait timed out";
    case NBODY_ERR_NONFINITE: return "non-finite value";
    case NBODY_ERR_NO_DEVICE: return "no usable device";
    case NBODY_ERR_STATE: return "call order";
  }
  return "unknown status";
}

nbody_status nbody_config_init(nbody_config* c) {
  if (!c) return fail(NBODY_ERR_INVALID_ARG, "null config");
  memset(c, 0, sizeof *c);
  c->n = 0;
  c->eps2 = 1.0e-7;
  c->precision = NBODY_FP64;
  c->device = 0;
  c->dt = 0.0;
  c->eta = 1.0e-2;
  c->eta0 = 1.0e-4;
  return NBODY_OK;
}

nbody_status nbody_create(nbody_engine** out, const nbody_config* cfg) {
  if (!out || !cfg) return fail(NBODY_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (cfg->n < 1 || cfg->n > (1 << 28)) return fail(NBODY_ERR_INVALID_ARG, "n = %d out of range", cfg->n);
  if (!(cfg->eps2 >= 1e-30 && cfg->eps2 <= 1e30))
    return fail(NBODY_ERR_INVALID_ARG, "eps2 = %g outside [1e-30, 1e30]", cfg->eps2);
  if (cfg->precision == NBODY_MIXED && cfg->eps2 < kMinEps2Mixed)
    return fail(NBODY_ERR_INVALID_ARG,
                "eps2 = %g below %g: the mixed path's float self-pair factor would overflow",
                cfg->eps2, kMinEps2Mixed);
  if (cfg->precision != NBODY_FP64 && cfg->precision != NBODY_MIXED)
    return fail(NBODY_ERR_INVALID_ARG, "precision = %d", cfg->precision);
  if (!(cfg->eta > 0) || !(cfg->eta0 > 0)) return fail(NBODY_ERR_INVALID_ARG, "eta/eta0 must be > 0");
  if (cfg->split_j < 0 || cfg->threads < 0 || cfg->i_per_thread < 0 || cfg->j_tile < 0)
    return fail(NBODY_ERR_INVALID_ARG, "negative tiling parameter");
  if (cfg->pair_variant < 0 || cfg->pair_variant > 5)
    return fail(NBODY_ERR_INVALID_ARG, "pair_variant = %d", cfg->pair_variant);
  if (cfg->j_cluster != 0 && cfg->j_cluster != 1 && cfg->j_cluster != 2 && cfg->j_cluster != 4 &&
      cfg->j_cluster != 8)
    return fail(NBODY_ERR_INVALID_ARG, "j_cluster = %d (0, 1, 2, 4 or 8)", cfg->j_cluster);
  if (cfg->sort_every < 0) return fail(NBODY_ERR_INVALID_ARG, "sort_every = %d", cfg->sort_every);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(NBODY_ERR_NO_DEVICE, "no CUDA device visible");
  if (cfg->device < 0 || cfg->device >= ndev)
    return fail(NBODY_ERR_INVALID_ARG, "device %d of %d", cfg->device, ndev);
  cudaDeviceProp prop;
  NB_CUDA(cudaGetDeviceProperties(&prop, cfg->device));
  if (prop.major != 10)
    return fail(NBODY_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a",
                cfg->device, prop.major, prop.minor);
  NB_CUDA(cudaSetDevice(cfg->device));

  std::unique_ptr<nbody_engine> e(new nbody_engine);
  e->cfg = *cfg;
  e->n = cfg->n;
  e->ld = round_up(cfg->n, kPad);
  e->dev = cfg->device;
  e->num_sms = prop.multiProcessorCount;
  const size_t ld = e->ld;
  auto cleanup_on_fail = [&](nbody_status s) {
    nbody_destroy(e.release());
    return s;
  };
  nbody_status s = [&]() -> nbody_status {
    NB_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    NB_CUDA(cudaMalloc(&e->state, sizeof(double) * 13 * ld));
    NB_CUDA(cudaMemsetAsync(e->state, 0, sizeof(double) * 13 * ld, e->stream));
    e->X = e->state;
    e->V = e->state + 3 * ld;
    e->M = e->state + 6 * ld;
    e->D = e->state + 7 * ld;
    NB_CUDA(cudaMalloc(&e->jb64, sizeof(JBody64) * ld));
    NB_CUDA(cudaMalloc(&e->jbe, sizeof(JBody64) * ld));
    if (cfg->precision == NBODY_MIXED) {
      // JBodyX2 records, or tiles of TJ + 1 JBodyNF records (TJ >= 64)
      static_assert(sizeof(JBodyNF) >= sizeof(JBodyX2), "jb32 sized by the larger record");
      NB_CUDA(cudaMalloc(&e->jb32, sizeof(JBodyNF) * (ld / 64) * 65));
      NB_CUDA(cudaMalloc(&e->perm, sizeof(int) * 2 * ld));
      iota_kernel<<<(e->n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, e->stream>>>(e->n, e->perm);
      NB_CUDA(cudaGetLastError());
      NB_CUDA(cudaMalloc(&e->scratch, sizeof(double) * 13 * ld));
      NB_CUDA(cudaMemsetAsync(e->scratch, 0, sizeof(double) * 13 * ld, e->stream));
      NB_CUDA(cudaMalloc(&e->near_count, sizeof(unsigned long long)));
      NB_CUDA(cudaMemsetAsync(e->near_count, 0, sizeof(unsigned long long), e->stream));
      NB_CUDA(cudaMalloc(&e->sort_keys, sizeof(uint64_t) * 2 * ld));
      NB_CUDA(cudaMalloc(&e->sort_idx, sizeof(int) * 2 * ld));
      NB_CUDA(cudaMalloc(&e->bbox_part, sizeof(double) * 6 * kMaxBBoxParts));
      NB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, e->sort_tmp_bytes, e->sort_keys,
                                              e->sort_keys + ld, e->sort_idx, e->sort_idx + ld,
                                              static_cast<int>(ld), 0, kOrderBits, e->stream));
      NB_CUDA(cudaMalloc(&e->sort_tmp, std::max<size_t>(e->sort_tmp_bytes, 16)));
    }
    NB_CUDA(cudaMalloc(&e->ctl, sizeof(StepCtl)));
    NB_CUDA(cudaMalloc(&e->partial, sizeof(double) * (ld / kBlockO1 * kMaxPotSplit + 8)));
    NB_CUDA(cudaMalloc(&e->status, sizeof(int)));
    NB_CUDA(cudaMemsetAsync(e->status, 0, sizeof(int), e->stream));
    NB_CUDA(cudaStreamSynchronize(e->stream));
    return NBODY_OK;
  }();
  if (s != NBODY_OK) return cleanup_on_fail(s);
  *out = e.release();
  return NBODY_OK;
}

nbody_status nbody_destroy(nbody_engine* e) {
  if (!e) return NBODY_OK;
  cudaSetDevice(e->dev);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->order_graph) cudaGraphExecDestroy(e->order_graph);
  for (auto ev : e->aux_ev)
    if (ev) cudaEventDestroy(ev);
  if (e->aux) cudaStreamDestroy(e->aux);
  for (auto ev : e->ev)
    if (ev) cudaEventDestroy(ev);
  for (auto ev : e->ev_init)
    if (ev) cudaEventDestroy(ev);
  cudaFree(e->state);
  cudaFree(e->P);
  cudaFree(e->jb64);
  cudaFree(e->jb32);
  cudaFree(e->jbe);
  cudaFree(e->sort_keys);
  cudaFree(e->sort_idx);
  cudaFree(e->perm);
  cudaFree(e->scratch);
  cudaFree(e->near_count);
  cudaFree(e->bbox_part);
  cudaFree(e->sort_tmp);
  cudaFree(e->ctl);
  cudaFree(e->partial);
  cudaFree(e->status);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return NBODY_OK;
}

nbody_status nbody_set_state(nbody_engine* e, const double* x, const double* y, const double* z,
                             const double* m, const double* vx, const double* vy,
                             const double* vz) {
  TraceRange trace_("nbody_set_state");
  NB_TRY(check_engine(e));
  const double* src[7] = {x, y, z, vx, vy, vz, m};
  for (auto p : src)
    if (!p) return fail(NBODY_ERR_INVALID_ARG, "null state array");
  const size_t ld = e->ld, b = sizeof(double) * e->n;
  double* dst[7] = {e->X, e->X + ld, e->X + 2 * ld, e->V, e->V + ld, e->V + 2 * ld, e->M};
  for (int k = 0; k < 7; ++k)
    NB_CUDA(cudaMemcpyAsync(dst[k], src[k], b, cudaMemcpyHostToDevice, e->stream));
  StepCtl c{};
  c.dt = e->cfg.dt > 0 ? e->cfg.dt : 0.0;
  c.t = 0.0;
  c.dt_crit = 0.0;
  c.crit_bits = kPosInfBits;
  c.blocks_done = 0;
  c.adaptive = e->cfg.dt > 0 ? 0 : 1;
  c.steps = 0;
  NB_CUDA(cudaMemcpyAsync(e->ctl, &c, sizeof c, cudaMemcpyHostToDevice, e->stream));
  NB_CUDA(cudaMemsetAsync(e->D, 0, sizeof(double) * 6 * ld, e->stream));
  if (e->perm) {  // body order again; a tile-relative engine re-orders at its next evaluation
    iota_kernel<<<(e->n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, e->stream>>>(e->n, e->perm);
    NB_CUDA(cudaGetLastError());
  }
  e->sorted = e->permuted = false;
  if (!curve_resident(e))
    NB_TRY(launch_pack(e, e->n, own_inputs(e), e->stream, tiling_fmt(e), tiling_tj(e)));
  NB_CUDA(cudaStreamSynchronize(e->stream));
  e->have_state = true;
  e->have_derivs = false;
  return NBODY_OK;
}

namespace {
// Downloads `count` [ld] arrays starting at `src` (engine positions) to the
// caller's arrays in body order: through scratch when the state is permuted.
nbody_status download_rows(nbody_engine* e, const double* src, double* const* dst, int count) {
  const size_t ld = e->ld, b = sizeof(double) * e->n;
  const double* from = src;
  if (e->permuted) {
    scatter_rows_kernel<<<(e->n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, e->stream>>>(
        e->n, e->perm, gather_args(src, e->scratch, ld, count));
    NB_CUDA(cudaGetLastError());
    from = e->scratch;
  }
  for (int k = 0; k < count; ++k)
    if (dst[k]) NB_CUDA(cudaMemcpyAsync(dst[k], from + k * ld, b, cudaMemcpyDeviceToHost, e->stream));
  NB_CUDA(cudaStreamSynchronize(e->stream));
  return NBODY_OK;
}
}  // namespace

nbody_status nbody_get_state(nbody_engine* e, double* x, double* y, double* z, double* vx,
                             double* vy, double* vz) {
  TraceRange trace_("nbody_get_state");
  NB_TRY(need_state(e));
  double* dst[6] = {x, y, z, vx, vy, vz};
  NB_TRY(download_rows(e, e->X, dst, 6));  // X(3) and V(3) are consecutive state arrays
  return check_status_word(e);
}

nbody_status nbody_get_derivs(nbody_engine* e, double* ax, double* ay, double* az, double* jx,
                              double* jy, double* jz) {
  NB_TRY(need_state(e));
  if (!e->have_derivs) return fail(NBODY_ERR_STATE, "no derivatives yet (call nbody_acc_jerk)");
  double* dst[6] = {ax, ay, az, jx, jy, jz};
  NB_TRY(download_rows(e, e->D, dst, 6));
  return check_status_word(e);
}

nbody_status nbody_acc_jerk(nbody_engine* e) {
  TraceRange trace_("nbody_acc_jerk");
  NB_TRY(need_state(e));
  return eval_current(e);
}

nbody_status nbody_predict(nbody_engine* e) {
  NB_TRY(need_state(e));
  if (!e->have_derivs) NB_TRY(eval_current(e));
  NB_TRY(ensure_tiling(e));
  NB_TRY(maybe_reorder(e, e->stream));
  return enqueue_predict(e, e->stream);
}

nbody_status nbody_eval_predicted(nbody_engine* e) {
  NB_TRY(need_state(e));
  NB_TRY(ensure_tiling(e));
  return launch_pair(e, e->tiling, 0, e->n, e->stream);
}

nbody_status nbody_correct(nbody_engine* e) {
  NB_TRY(need_state(e));
  NB_TRY(ensure_tiling(e));
  return enqueue_correct(e, e->stream);
}

nbody_status nbody_step(nbody_engine* e, int nsteps) {
  TraceRange trace_("nbody_step");
  NB_TRY(need_state(e));
  if (nsteps < 0) return fail(NBODY_ERR_INVALID_ARG, "nsteps < 0");
  if (!e->have_derivs) NB_TRY(eval_current(e));
  NB_TRY(build_step_graph(e));
  for (int k = 0; k < nsteps; ++k) {
    NB_TRY(maybe_reorder(e, e->stream));
    NB_CUDA(cudaGraphLaunch(e->graph, e->stream));
  }
  return NBODY_OK;
}

nbody_status nbody_synchronize(nbody_engine* e) {
  NB_TRY(check_engine(e));
  NB_CUDA(cudaStreamSynchronize(e->stream));
  return check_status_word(e);
}

nbody_status nbody_energy(nbody_engine* e, int ref_compat, double* T, double* U) {
  TraceRange trace_("nbody_energy");
  NB_TRY(need_state(e));
  const int nb = e->ld / kBlockO1;
  // j-splits of the potential: about 8 CTAs per SM in all
  const int ps = std::max(1, std::min({kMaxPotSplit, nb, (8 * e->num_sms + nb - 1) / nb}));
  double* scal = e->partial + nb * kMaxPotSplit;  // two result slots after the partials
  kinetic_kernel<<<nb, kBlockO1, 0, e->stream>>>(e->n, e->ld, e->V, e->M, e->partial);
  sum_partials_kernel<<<1, 256, 0, e->stream>>>(nb, e->partial, scal);
  pack_kernel<<<nb, kBlockO1, 0, e->stream>>>(e->n, e->ld, own_inputs(e), e->jbe, nullptr, nullptr);
  potential_kernel<kBlockO1><<<dim3(nb, ps), kBlockO1, 0, e->stream>>>(
      e->n, e->ld, e->cfg.eps2, ref_compat ? 1 : 0, e->jbe, e->partial);
  sum_partials_kernel<<<1, 256, 0, e->stream>>>(nb * ps, e->partial, scal + 1);
  NB_CUDA(cudaGetLastError());
  double h[2];
  NB_CUDA(cudaMemcpyAsync(h, scal, sizeof h, cudaMemcpyDeviceToHost, e->stream));
  NB_CUDA(cudaStreamSynchronize(e->stream));
  const double t = h[0];
  const double u = ref_compat ? -h[1] : -0.5 * h[1];
  if (T) *T = t;
  if (U) *U = u;
  if (!std::isfinite(t) || !std::isfinite(u))
    return fail(NBODY_ERR_NONFINITE, "energy is not finite (T=%g U=%g)", t, u);
  return NBODY_OK;
}

nbody_status nbody_get_timers(nbody_engine* e, nbody_timers* out) {
  NB_TRY(check_engine(e));
  if (!out) return fail(NBODY_ERR_INVALID_ARG, "null timers");
  memset(out, 0, sizeof *out);
  NB_CUDA(cudaStreamSynchronize(e->stream));
  float ms = 0.f;
  if (e->step_events && e->graph) {
    if (cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]) == cudaSuccess) out->pred_ms = ms;
    if (cudaEventElapsedTime(&ms, e->ev[1], e->ev[2]) == cudaSuccess) out->eval_ms = ms;
    if (cudaEventElapsedTime(&ms, e->ev[2], e->ev[3]) == cudaSuccess) out->corr_ms = ms;
    cudaGetLastError();
  }
  if (e->init_events && cudaEventElapsedTime(&ms, e->ev_init[0], e->ev_init[1]) == cudaSuccess)
    out->eval_init_ms = ms;
  cudaGetLastError();
  out->num_sms = e->num_sms;
  if (e->tiled) {
    out->threads = e->tiling.k->nt;
    out->i_per_thread = e->tiling.k->ipt;
    out->j_tile = e->tiling.k->tj;
    out->split_j = e->tiling.split;
    out->j_cluster = e->tiling.k->cluster;
    out->record_format = e->tiling.k->fmt;
    out->tiling_source = e->tiling.source;
    const PairKernel& k = *e->tiling.k;
    if (k.fmt == kRecRel && k.near) {
      unsigned long long near = 0;
      NB_CUDA(cudaMemcpy(&near, e->near_count, sizeof near, cudaMemcpyDeviceToHost));
      // classified per (warp, tile): warps = row blocks x NT / 32
      const double pairs = static_cast<double>((e->n + k.nt * k.ipt - 1) / (k.nt * k.ipt)) *
                           (k.nt / 32) * static_cast<double>(e->ld / k.tj);
      out->near_tile_fraction = static_cast<double>(near) / pairs;
    }
  }
  out->step_kernels = e->graph_kernels;
  out->reorders = e->reorders;
  out->order_kernels = e->order_kernels;
  if (e->have_state) {
    StepCtl c;
    NB_CUDA(cudaMemcpy(&c, e->ctl, sizeof c, cudaMemcpyDeviceToHost));
    out->steps = c.steps;
    out->t = c.t;
    out->dt = c.dt;
    out->dt_crit = c.dt_crit;
  }
  return NBODY_OK;
}

nbody_status nbody_set_time(nbody_engine* e, double t, double dt) {
  NB_TRY(need_state(e));
  if (!std::isfinite(t)) return fail(NBODY_ERR_INVALID_ARG, "t is not finite");
  StepCtl c;
  NB_CUDA(cudaStreamSynchronize(e->stream));
  NB_CUDA(cudaMemcpy(&c, e->ctl, sizeof c, cudaMemcpyDeviceToHost));
  c.t = t;
  if (dt > 0) c.dt = dt;
  NB_CUDA(cudaMemcpy(e->ctl, &c, sizeof c, cudaMemcpyHostToDevice));
  return NBODY_OK;
}

nbody_status nbody_get_stream(nbody_engine* e, void** stream) {
  NB_TRY(check_engine(e));
  if (!stream) return fail(NBODY_ERR_INVALID_ARG, "null stream out");
  *stream = e->stream;
  return NBODY_OK;
}

nbody_status nbody_acc_jerk_device(nbody_engine* e, int n, const double* x, const double* y,
                                   const double* z, const double* m, const double* vx,
                                   const double* vy, const double* vz, double* ax, double* ay,
                                   double* az, double* jx, double* jy, double* jz, void* stream) {
  TraceRange trace_("nbody_acc_jerk_device");
  NB_TRY(check_engine(e));
  if (n < 1 || n > e->n) return fail(NBODY_ERR_INVALID_ARG, "n = %d outside [1, %d]", n, e->n);
  const void* ptrs[13] = {x, y, z, m, vx, vy, vz, ax, ay, az, jx, jy, jz};
  for (auto p : ptrs)
    if (!p) return fail(NBODY_ERR_INVALID_ARG, "null device array");
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : e->stream;
  Tiling t;
  NB_TRY(get_tiling(e, n, &t));
  NB_TRY(ensure_partials(e, t.split));
  const SoA7 in{x, y, z, m, vx, vy, vz};
  const SoA6 out{ax, ay, az, jx, jy, jz};
  if (t.k->fmt == kRecRel) {  // Hilbert order of the caller's bodies, gathered into scratch
    NB_TRY(enqueue_curve_order(e, n, in, st, kDropInOrderLowBit));
    return eval_foreign_rel(e, t, n, in, out, st);
  }
  NB_TRY(launch_pack(e, n, in, st, t.k->fmt, t.k->tj));
  NB_TRY(launch_pair(e, t, 0, n, st, &in, n));
  reduce_splits_kernel<<<(n + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, st>>>(
      0, n, e->ld, partial_count(t), e->P, out);
  NB_CUDA(cudaGetLastError());
  return NBODY_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Drop-in force_calculation: cached engines per (thread, device, precision).
// ---------------------------------------------------------------------------
namespace {

struct DropIn {
  nbody_engine* e = nullptr;
  int n = 0;
  double eps2 = 0;
};

struct DropInCache {
  std::map<std::pair<int, int>, DropIn> m;
  ~DropInCache() {
    for (auto& kv : m) nbody_destroy(kv.second.e);
  }
};
thread_local DropInCache g_dropin;

}  // namespace

namespace {

// The calling thread's cached drop-in engine for (device, precision), made
// (again) for n bodies and eps2 when those change.
nbody_status dropin_engine(int n, double eps2, int precision, nbody_engine** out) {
  int dev = 0;
  NB_CUDA(cudaGetDevice(&dev));
  DropIn& d = g_dropin.m[{dev, precision}];
  if (!d.e || d.n != n || d.eps2 != eps2) {
    nbody_destroy(d.e);
    d.e = nullptr;
    nbody_config c;
    nbody_config_init(&c);
    c.n = n;
    c.eps2 = eps2;
    c.precision = precision;
    c.device = dev;
    c.dt = 1.0;  // fixed: no initial-dt pass on the drop-in path
    NB_TRY(nbody_create(&d.e, &c));
    // every call re-orders: tile-relative pays off only above ~24k bodies
    // (measured per call: N = 16384 428 vs 357 us hi/lo; N = 65536 it wins)
    d.e->rel_min_bodies = 32768;
    d.e->tune_lookup = true;
    d.n = n;
    d.eps2 = eps2;
  }
  *out = d.e;
  return NBODY_OK;
}

}  // namespace

extern "C" nbody_status nbody_force_calculation_tune(int n, double eps2, int precision,
                                                     const double* x, const double* y,
                                                     const double* z, const double* m,
                                                     const double* vx, const double* vy,
                                                     const double* vz) {
  TraceRange trace_("nbody_force_calculation_tune");
  if (n < 1) return fail(NBODY_ERR_INVALID_ARG, "n = %d", n);
  const void* ptrs[7] = {x, y, z, m, vx, vy, vz};
  for (auto p : ptrs)
    if (!p) return fail(NBODY_ERR_INVALID_ARG, "null array");
  nbody_engine* e = nullptr;
  NB_TRY(dropin_engine(n, eps2, precision, &e));
  NB_TRY(nbody_set_state(e, x, y, z, m, vx, vy, vz));  // the bodies the trials run on
  // the autotuner times the full-row call's kernel family on these bodies
  // (in curve order for the near/far kernel) and caches its choice for the
  // process; drop-in calls of this size then look it up
  e->cfg.tune = 1;
  e->tiled = false;
  const nbody_status st = ensure_tiling(e);
  e->cfg.tune = 0;
  NB_TRY(st);
  NB_CUDA(cudaStreamSynchronize(e->stream));
  return check_status_word(e);
}

extern "C" nbody_status nbody_force_calculation(int n, double eps2, int precision, int i_begin,
                                                int i_end, const double* x, const double* y,
                                                const double* z, const double* m,
                                                const double* vx, const double* vy,
                                                const double* vz, double* ax, double* ay,
                                                double* az, double* jx, double* jy, double* jz) {
  TraceRange trace_("nbody_force_calculation");
  if (n < 1) return fail(NBODY_ERR_INVALID_ARG, "n = %d", n);
  if (i_begin < 0 || i_end > n || i_begin > i_end)
    return fail(NBODY_ERR_INVALID_ARG, "row range [%d, %d) outside [0, %d)", i_begin, i_end, n);
  const void* ptrs[13] = {x, y, z, m, vx, vy, vz, ax, ay, az, jx, jy, jz};
  for (auto p : ptrs)
    if (!p) return fail(NBODY_ERR_INVALID_ARG, "null array");
  nbody_engine* e = nullptr;
  NB_TRY(dropin_engine(n, eps2, precision, &e));
  const size_t ld = e->ld, b = sizeof(double) * n;
  const double* src[7] = {x, y, z, vx, vy, vz, m};
  double* dst[7] = {e->X, e->X + ld, e->X + 2 * ld, e->V, e->V + ld, e->V + 2 * ld, e->M};
  NB_TRY(ensure_tiling(e));
  Tiling t = e->tiling;
  const bool full = i_begin == 0 && i_end == n;
  if (!full) NB_TRY(get_tiling(e, i_end - i_begin, &t));
  // a row range: the packed hi/lo kernel, whose rows stay in the caller's
  // order (the near/far kernel evaluates all rows in Hilbert order)
  if (!full && t.k->fmt == kRecRel) NB_TRY(hilo_tiling(e, i_end - i_begin, &t));
  NB_TRY(ensure_partials(e, t.split));
  if (!e->aux) {
    NB_CUDA(cudaStreamCreateWithFlags(&e->aux, cudaStreamNonBlocking));
    for (auto& ev : e->aux_ev) NB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  const int* index = nullptr;  // row -> output position (the near/far rows are in Hilbert order)
  if (t.k->fmt == kRecRel) {
    // positions first: their Hilbert ordering runs while the masses and
    // velocities upload on a second stream
    NB_CUDA(cudaEventRecord(e->aux_ev[0], e->stream));
    NB_CUDA(cudaStreamWaitEvent(e->aux, e->aux_ev[0], 0));
    for (int k = 0; k < 3; ++k)
      NB_CUDA(cudaMemcpyAsync(dst[k], src[k], b, cudaMemcpyHostToDevice, e->stream));
    for (int k = 3; k < 7; ++k)
      NB_CUDA(cudaMemcpyAsync(dst[k], src[k], b, cudaMemcpyHostToDevice, e->aux));
    NB_CUDA(cudaEventRecord(e->aux_ev[1], e->aux));
    NB_TRY(enqueue_curve_order(e, n, own_inputs(e), e->stream, kDropInOrderLowBit));
    NB_CUDA(cudaStreamWaitEvent(e->stream, e->aux_ev[1], 0));
    // the caller's bodies gathered into Hilbert order; the split sums below
    // write the derivatives back in body order
    NB_TRY(eval_foreign_rel(e, t, n, own_inputs(e), own_derivs(e), e->stream, false));
    index = e->sort_idx + ld;
  } else {
    for (int k = 0; k < 7; ++k)
      NB_CUDA(cudaMemcpyAsync(dst[k], src[k], b, cudaMemcpyHostToDevice, e->stream));
    NB_TRY(launch_pack(e, n, own_inputs(e), e->stream, t.k->fmt, t.k->tj));
    NB_TRY(launch_pair(e, t, i_begin, i_end, e->stream));
  }
  // one field at a time: field k's download (second stream) overlaps the
  // split sums of field k + 1
  double* out[6] = {ax, ay, az, jx, jy, jz};
  const size_t rb = sizeof(double) * (i_end - i_begin);
  const int rows = i_end - i_begin;
  for (int k = 0; k < 6; ++k) {
    if (i_begin > 0) memset(out[k], 0, sizeof(double) * i_begin);
    if (i_end < n) memset(out[k] + i_end, 0, sizeof(double) * (n - i_end));
    if (!rows) continue;
    reduce_split_field_kernel<<<(rows + kBlockO1 - 1) / kBlockO1, kBlockO1, 0, e->stream>>>(
        i_begin, i_end, e->ld, partial_count(t), e->P + k * ld, e->D + k * ld, index);
    NB_CUDA(cudaGetLastError());
    NB_CUDA(cudaEventRecord(e->aux_ev[0], e->stream));
    NB_CUDA(cudaStreamWaitEvent(e->aux, e->aux_ev[0], 0));
    NB_CUDA(cudaMemcpyAsync(out[k] + i_begin, e->D + k * ld + i_begin, rb, cudaMemcpyDeviceToHost,
                            e->aux));
  }
  NB_CUDA(cudaEventRecord(e->aux_ev[1], e->aux));
  NB_CUDA(cudaStreamWaitEvent(e->stream, e->aux_ev[1], 0));
  return check_status_word(e);  // its read-back follows the outputs; one wait for all
}

extern "C" nbody_status nbody_force_calculation_release(void) {
  for (auto& kv : g_dropin.m) nbody_destroy(kv.second.e);
  g_dropin.m.clear();
  return NBODY_OK;
}
