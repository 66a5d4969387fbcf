// Pipe-throughput microkernels: the denominators of the pair kernels'
// roofline.  The device's published peaks are nominal; these measure what
// the FP64 FMA, FP32 FMA (scalar and packed f32x2) and MUFU rsqrt pipes
// deliver on this device at its current clocks.
//
// Each thread runs 8 independent dependency chains so that issue, not
// latency, bounds the rate; the chains' results feed a conditional store so
// the compiler keeps all of the work.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/nbody_cuda.h"
#include "errors.h"
#include "tma.cuh"

namespace {

// One CTA waits on an mbarrier that nothing ever arrives on: phase 0 never
// completes, so the bounded wait gives up after limit_ns and the CTA records
// the timeout in the status word - the same path every pipeline wait takes.
__global__ void selftest_wait_kernel(uint64_t limit_ns, int* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    nbody::mbar_init(&bar, 1);
    nbody::mbar_init_fence();
  }
  __syncthreads();
  const bool ok = nbody::mbar_wait_for(&bar, 0, limit_ns);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) nbody::report_status(status, nbody::kKernelTimeout);
}


constexpr int kChains = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) dfma_probe(int iters, double b, double c, double* sink) {
  double x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-3 + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], b, c);
  }
  double s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  if (s == -1.0) sink[0] = s;
}

__global__ void __launch_bounds__(kThreads) ffma_probe(int iters, float b, float c, float* sink) {
  float x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-3f + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int k = 0; k < kChains; ++k) x[k] = fmaf(x[k], b, c);
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  if (s == -1.0f) sink[0] = s;
}

// Packed single precision: one fma.rn.f32x2 performs two FMAs.
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b,
                                                    unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
  return (static_cast<unsigned long long>(__float_as_uint(hi)) << 32) | __float_as_uint(lo);
}

__global__ void __launch_bounds__(kThreads) ffma2_probe(int iters, float b, float c, float* sink) {
  unsigned long long x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = pack2(threadIdx.x * 1e-3f + k, k + 0.5f);
  const unsigned long long bb = pack2(b, b), cc = pack2(c, c);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int k = 0; k < kChains; ++k) x[k] = ffma2(x[k], bb, cc);
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += __uint_as_float(static_cast<unsigned>(x[k])) + __uint_as_float(static_cast<unsigned>(x[k] >> 32));
  if (s == -1.0f) sink[0] = s;
}

__global__ void __launch_bounds__(kThreads) rsqrt_probe(int iters, float* sink) {
  float x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) x[k] = 1.5f + threadIdx.x * 1e-3f + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int k = 0; k < kChains; ++k) {
        float y;
        asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x[k]));
        x[k] = y;
      }
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += x[k];
  if (s == -1.0f) sink[0] = s;
}

template <class Launch>
float best_ms(Launch&& launch, cudaEvent_t a, cudaEvent_t b) {
  launch();  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 3; ++r) {
    cudaEventRecord(a);
    launch();
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best) best = ms;
  }
  return best;
}

}  // namespace

extern "C" nbody_status nbody_measure_peaks(int device, nbody_peaks* out) {
  if (!out) return NBODY_ERR_INVALID_ARG;
  memset(out, 0, sizeof *out);
  if (cudaSetDevice(device) != cudaSuccess) return NBODY_ERR_NO_DEVICE;
  int sms = 0, clk = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, device);
  void* sink = nullptr;
  if (cudaMalloc(&sink, 64) != cudaSuccess) return NBODY_ERR_OOM;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const dim3 grid(sms * 8), block(kThreads);
  const double threads = static_cast<double>(grid.x) * kThreads;
  const int it64 = 20000, it32 = 40000, itmu = 5000;
  const double per_it = 8.0 * kChains;  // ops per thread per outer iteration
  float ms;
  ms = best_ms([&] { dfma_probe<<<grid, block>>>(it64, 0.999999, 1e-7, (double*)sink); }, a, b);
  out->fp64_tflops = 2.0 * per_it * it64 * threads / (ms * 1e-3) / 1e12;
  ms = best_ms([&] { ffma_probe<<<grid, block>>>(it32, 0.999999f, 1e-7f, (float*)sink); }, a, b);
  out->fp32_tflops = 2.0 * per_it * it32 * threads / (ms * 1e-3) / 1e12;
  ms = best_ms([&] { ffma2_probe<<<grid, block>>>(it32, 0.999999f, 1e-7f, (float*)sink); }, a, b);
  out->fp32x2_tflops = 4.0 * per_it * it32 * threads / (ms * 1e-3) / 1e12;
  ms = best_ms([&] { rsqrt_probe<<<grid, block>>>(itmu, (float*)sink); }, a, b);
  out->mufu_rsqrt_gops = per_it * itmu * threads / (ms * 1e-3) / 1e9;
  out->sm_clock_mhz = clk / 1000.0;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  return cudaGetLastError() == cudaSuccess ? NBODY_OK : NBODY_ERR_CUDA;
}

extern "C" nbody_status nbody_selftest_bounded_wait(int device, double limit_ms) {
  if (!(limit_ms > 0 && limit_ms <= 2000))
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "limit_ms = %g outside (0, 2000]", limit_ms);
  if (cudaSetDevice(device) != cudaSuccess) return nbody_set_error(NBODY_ERR_NO_DEVICE, "device %d", device);
  int* st = nullptr;
  if (cudaMalloc(&st, sizeof(int)) != cudaSuccess) return nbody_set_error(NBODY_ERR_OOM, "status word");
  cudaMemset(st, 0, sizeof(int));
  selftest_wait_kernel<<<1, 32>>>(static_cast<uint64_t>(limit_ms * 1e6), st);
  int h = -1;
  const cudaError_t e1 = cudaDeviceSynchronize();
  const cudaError_t e2 = cudaMemcpy(&h, st, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(st);
  if (e1 != cudaSuccess || e2 != cudaSuccess)
    return nbody_set_error(NBODY_ERR_CUDA, "self-test kernel: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
  if (h == nbody::kKernelTimeout)
    return nbody_set_error(NBODY_ERR_TIMEOUT, "in-kernel wait gave up after %.3g ms (self-test)", limit_ms);
  return NBODY_OK;
}
