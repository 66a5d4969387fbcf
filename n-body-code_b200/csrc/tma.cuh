// Shared-memory barrier and bulk-copy primitives for sm_100a (inline PTX).
//
// j-body tiles move global -> shared with the non-tensor bulk copy
// (cp.async.bulk ... mbarrier::complete_tx::bytes), issued by one thread and
// tracked by an mbarrier transaction count.  Every copy lands in the issuing
// CTA's own shared memory and reads this GPU's own global memory.  Tile
// records go the other way (shared -> global, bulk_group completion) from the
// record builder.
// Every wait is bounded by the global nanosecond timer: a wait that runs past
// its limit reports failure instead of spinning forever.
#pragma once
#include <cstdint>

namespace nbody {

// Kernel status codes written to the engine's device status word.
constexpr int kKernelOk = 0;
constexpr int kKernelTimeout = 4;

// Upper bound for one mbarrier wait: 2 s of GPU time.
constexpr uint64_t kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// Makes the initialised barriers visible to the async (bulk-copy) proxy.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// Global -> own shared memory, completion signalled on `bar` (bytes % 16 == 0,
// both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Own shared memory -> global (bytes % 16 == 0, both addresses 16-byte
// aligned), issued by one thread after the block's shared-memory writes are
// made visible to the async proxy (bulk_store_fence + __syncthreads).
// Returns once the copy has completed: its shared-memory source may then be
// reused and its global writes are done.
__device__ __forceinline__ void bulk_store_fence() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_addr(src)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for phase `parity` of `bar` to complete; false after limit_ns.
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t k = 1;; ++k) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((k & 255u) == 0 && global_ns() - t0 > limit_ns) return false;
  }
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, kWaitLimitNs);
}

__device__ __forceinline__ void report_status(int* status, int code) {
  if (status) atomicCAS(status, kKernelOk, code);
}

}  // namespace nbody
