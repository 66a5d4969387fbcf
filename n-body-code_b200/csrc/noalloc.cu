// nbody_acc_jerk_noalloc: acc + jerk on caller-owned device arrays without
// allocating any device memory.
//
// Who needs it: code that is not allowed to call cudaMalloc - a host
// application that owns the whole device memory budget through its own pool
// and forbids libraries from allocating behind its back, a real-time loop
// where cudaMalloc/cudaFree would stall (cudaFree synchronises the device),
// or a plugin called from inside someone else's stream capture or tight
// time-step loop.  Such callers pass their inputs and outputs and get the
// same result as nbody_acc_jerk_device, without creating an engine.
//
// Scratch lives in one file-scope __device__ array (g_scratch, 16 MiB): the
// j-records of the packed input, the split-j partial sums, and a status word.
// Every GPU that loads this library holds those 16 MiB until the process
// exits.  Host code cannot use the symbol g_scratch as a device address: each
// call whose stream is not capturing looks the address up again with
// cudaGetSymbolAddress, with the caller's device current (so a context that
// was reset and rebuilt, which may place the array elsewhere, is never
// written through a stale address); a call on a capturing stream uses the
// address of the last such lookup on that device, so the first call on a
// device must come before any stream capture.  All calls share the array and
// it keeps the last call's contents: each call rewrites every byte it reads
// (the j-records up to the padded size, every split slice of the partial
// sums) and clears the status word first.  Calls whose work overlaps on the
// GPU (different streams, no ordering between them) race on the array and
// corrupt each other's results; order them on one stream or serialise them.
//
// The call returns without waiting for the GPU, so it cannot report a
// bounded-wait timeout of its pair kernel as a status: the split reduction
// reads the status word instead and then writes NaN to every output, which
// the caller sees in its results.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/nbody_cuda.h"
#include "errors.h"
#include "hermite.cuh"
#include "pair.cuh"

using namespace nbody;

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;  // 16 MiB per device
constexpr int kMaxBodies = 32768;                    // largest n the scratch serves
constexpr int kPadRows = 256;
constexpr int kStatusBytes = 256;
constexpr int kMaxDevices = 64;
constexpr int kMaxSplit = 64;
constexpr int kThreads = 128;
constexpr int kTile = 128;

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct DeviceSetup {
  bool ready = false;
  unsigned char* base = nullptr;  // device address of g_scratch from the last lookup
  int sms = 0;
  int occ_fp64 = 1, occ_mixed = 1;
};
std::mutex g_mu;
DeviceSetup g_dev[kMaxDevices];

constexpr int kIptFp64 = 2, kIptMixed = 4;
const void* kernel_fp64() { return reinterpret_cast<const void*>(&pair_fp64_kernel<kThreads, kIptFp64, kTile>); }
// the packed hi/lo kernel with FP64 accumulators in registers (the engine's
// pair_variant 2 at this shape), so both entry points do identical arithmetic
const void* kernel_mixed() { return reinterpret_cast<const void*>(&pair_mixed_x2_kernel<kThreads, kIptMixed, kTile>); }

// Device set-up (once) and the scratch address (looked up on every call whose
// stream is not capturing).  Errors made here are this call's own: the entry
// point has checked that none was pending before it.
nbody_status setup(int dev, cudaStream_t cs, DeviceSetup** out) {
  std::lock_guard<std::mutex> g(g_mu);
  DeviceSetup& d = g_dev[dev];
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(cs, &cap) != cudaSuccess) {
    (void)cudaGetLastError();
    cap = cudaStreamCaptureStatusActive;  // treat an unanswerable stream as capturing
  }
  const bool capturing = cap != cudaStreamCaptureStatusNone;
  if (!d.ready) {
    if (capturing)
      return nbody_set_error(NBODY_ERR_STATE,
                             "nbody_acc_jerk_noalloc: the first call on device %d came during a "
                             "stream capture; make one call before capturing",
                             dev);
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        major != 10) {
      (void)cudaGetLastError();
      return nbody_set_error(NBODY_ERR_NO_DEVICE, "nbody_acc_jerk_noalloc: device %d is not sm_100", dev);
    }
    if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        d.sms < 1) {
      (void)cudaGetLastError();
      return nbody_set_error(NBODY_ERR_CUDA, "nbody_acc_jerk_noalloc: SM count of device %d", dev);
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_fp64, kernel_fp64(), kThreads,
                                                      2 * kTile * sizeof(JBody64)) != cudaSuccess ||
        d.occ_fp64 < 1) {
      (void)cudaGetLastError();
      d.occ_fp64 = 1;  // only sizes the j-split
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_mixed, kernel_mixed(), kThreads,
                                                      2 * kTile * sizeof(JBodyX2)) != cudaSuccess ||
        d.occ_mixed < 1) {
      (void)cudaGetLastError();
      d.occ_mixed = 1;
    }
  }
  if (!capturing) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || p == nullptr) {
      (void)cudaGetLastError();
      return nbody_set_error(NBODY_ERR_CUDA, "nbody_acc_jerk_noalloc: cudaGetSymbolAddress: %s",
                             cudaGetErrorString(e));
    }
    d.base = static_cast<unsigned char*>(p);
    d.ready = true;
  }
  *out = &d;
  return NBODY_OK;
}

// This call's launch error, if any (none was pending when the call began).
nbody_status launched(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return NBODY_OK;
  return nbody_set_error(NBODY_ERR_CUDA, "nbody_acc_jerk_noalloc: %s: %s", what, cudaGetErrorString(e));
}

}  // namespace

extern "C" nbody_status nbody_acc_jerk_noalloc(int n, double eps2, int precision, const double* x,
                                               const double* y, const double* z, const double* m,
                                               const double* vx, const double* vy,
                                               const double* vz, double* ax, double* ay,
                                               double* az, double* jx, double* jy, double* jz,
                                               void* stream) {
  if (n < 1 || n > kMaxBodies)
    return nbody_set_error(NBODY_ERR_INVALID_ARG,
                           "nbody_acc_jerk_noalloc: n = %d outside [1, %d] (the %zu MiB static "
                           "scratch limit); use nbody_acc_jerk_device for larger systems",
                           n, kMaxBodies, kScratchBytes >> 20);
  if (!(eps2 >= 1e-30 && eps2 <= 1e30))
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "nbody_acc_jerk_noalloc: eps2 = %g outside [1e-30, 1e30]", eps2);
  if (precision != NBODY_FP64 && precision != NBODY_MIXED)
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "nbody_acc_jerk_noalloc: precision = %d", precision);
  if (precision == NBODY_MIXED && eps2 < kMinEps2Mixed)
    return nbody_set_error(NBODY_ERR_INVALID_ARG,
                           "nbody_acc_jerk_noalloc: eps2 = %g below %g (mixed precision)", eps2,
                           kMinEps2Mixed);
  const void* ptrs[13] = {x, y, z, m, vx, vy, vz, ax, ay, az, jx, jy, jz};
  for (const void* p : ptrs)
    if (!p) return nbody_set_error(NBODY_ERR_INVALID_ARG, "nbody_acc_jerk_noalloc: null array");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return nbody_set_error(NBODY_ERR_NO_DEVICE, "nbody_acc_jerk_noalloc: no current device");
  // an error left pending by the caller's own earlier work stays theirs:
  // report it without clearing it, and do not run on top of it
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess)
    return nbody_set_error(NBODY_ERR_CUDA,
                           "nbody_acc_jerk_noalloc: a CUDA error was already pending in this "
                           "thread (%s); nothing was launched and the error was left in place",
                           cudaGetErrorString(pending));
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  DeviceSetup* d = nullptr;
  nbody_status st = setup(dev, cs, &d);
  if (st != NBODY_OK) return st;

  const bool fp64 = precision == NBODY_FP64;
  const int ld = (n + kPadRows - 1) / kPadRows * kPadRows;
  const size_t rec = fp64 ? sizeof(JBody64) : sizeof(JBodyX2);
  const size_t jb_bytes = (static_cast<size_t>(ld) * rec + 255) / 256 * 256;
  const size_t split_bytes = sizeof(double) * 6 * static_cast<size_t>(ld);
  const int cap = static_cast<int>((kScratchBytes - kStatusBytes - jb_bytes) / split_bytes);
  int* status = reinterpret_cast<int*>(d->base);
  unsigned char* jb = d->base + kStatusBytes;
  double* P = reinterpret_cast<double*>(jb + jb_bytes);

  // split-j from the same wave model as the engine, capped by the scratch
  const int ipt = fp64 ? kIptFp64 : kIptMixed;
  const long slots = static_cast<long>(d->sms) * (fp64 ? d->occ_fp64 : d->occ_mixed);
  const long i_blocks = (n + kThreads * ipt - 1) / (kThreads * ipt);
  const int n_tiles = ld / kTile;
  int split = 1;
  double best = 1e300;
  for (int s = 1; s <= std::min({kMaxSplit, n_tiles, cap}); ++s) {
    const long waves = (i_blocks * s + slots - 1) / slots;
    const double cost = waves * (((n_tiles + s - 1) / s) + 0.25) + 0.002 * s;
    if (cost < best - 1e-9) {
      best = cost;
      split = s;
    }
  }

  if (cudaMemsetAsync(status, 0, sizeof(int), cs) != cudaSuccess) {
    (void)cudaGetLastError();
    return nbody_set_error(NBODY_ERR_CUDA, "nbody_acc_jerk_noalloc: clearing the status word failed");
  }
  pack_kernel<<<(ld + 255) / 256, 256, 0, cs>>>(
      n, ld, SoA7{x, y, z, m, vx, vy, vz}, fp64 ? reinterpret_cast<JBody64*>(jb) : nullptr, nullptr,
      fp64 ? nullptr : reinterpret_cast<JBodyX2*>(jb));
  if ((st = launched("pack_kernel launch")) != NBODY_OK) return st;
  PairArgs a;
  a.i_begin = 0;
  a.i_end = n;
  a.n_rows_pad = ld;
  a.n_tiles = n_tiles;
  a.tiles_per_split = (n_tiles + split - 1) / split;
  a.eps2 = eps2;
  a.out = P;
  a.stride = static_cast<size_t>(ld);
  a.status = status;
  const dim3 grid(static_cast<unsigned>(i_blocks), split);
  if (fp64)
    pair_fp64_kernel<kThreads, kIptFp64, kTile><<<grid, kThreads, 2 * kTile * sizeof(JBody64), cs>>>(
        reinterpret_cast<const JBody64*>(jb), a);
  else
    pair_mixed_x2_kernel<kThreads, kIptMixed, kTile><<<grid, kThreads, 2 * kTile * sizeof(JBodyX2), cs>>>(
        reinterpret_cast<const JBodyX2*>(jb), a);
  if ((st = launched("pair kernel launch")) != NBODY_OK) return st;
  // a pair-kernel timeout (status word set) turns every output into NaN
  reduce_splits_kernel<<<(n + 255) / 256, 256, 0, cs>>>(0, n, ld, split, P,
                                                        SoA6{ax, ay, az, jx, jy, jz}, status);
  if ((st = launched("reduce_splits_kernel launch")) != NBODY_OK) return st;
  return NBODY_OK;
}
