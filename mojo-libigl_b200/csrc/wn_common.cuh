// Shared device helpers for libwn_b200: status codes, the device error word,
// and the sm_100a bulk-copy (TMA 1-D) + mbarrier primitives used to stage face
// tiles into shared memory.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace wn {

// Bits of the device error word (one int per device, cleared per call).
enum DeviceError : int {
  kErrWaitTimeout = 1,   // an mbarrier wait hit its iteration limit
  kErrBadLaunch = 2,     // a kernel found inconsistent launch parameters
};

// A bounded wait gives up after this many polls (each poll suspends the
// thread for up to the hardware time limit), i.e. well after any legitimate
// bulk copy has landed.
constexpr uint32_t kWaitPolls = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// Makes the initialised barriers visible to the async (bulk-copy) proxy.
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
// Requirements (checked by the callers' layout): src and dst 16-byte aligned,
// bytes a multiple of 16. No cluster multicast anywhere in this library.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
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

// Bounded wait on phase `parity`; false (and the error bit set) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  for (uint32_t i = 0; i < kWaitPolls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicOr(err, kErrWaitTimeout);
  return false;
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

}  // namespace wn
