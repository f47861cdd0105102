// mbarrier and bulk-copy helpers of the asynchronous pipelines (tcgen05 GEMM, the
// streamed tridiagonalisation).  Every wait is bounded: after WAIT_CYCLES of clock (about
// one second) it sets the kernel's error word and gives up, so a broken pipeline ends
// the launch with an error instead of hanging the GPU.
#pragma once
#include <cstdint>

namespace {

constexpr long long WAIT_CYCLES = 2000000000ll;   // ~1 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// waits for the phase with the given parity; false (and the error word set) after
// WAIT_CYCLES or when another thread already failed
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  const uint32_t a = smem_u32(bar);
  const long long t0 = clock64();
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255) == 255) {
      if (*(volatile int*)err != 0) return false;
      if (clock64() - t0 > WAIT_CYCLES) {
        atomicExch(err, 1);
        return false;
      }
    }
    __nanosleep(20);
  }
}

// one test of the phase with the given parity, then the bounded wait if it is not done
__device__ __forceinline__ bool mbar_wait_fast(uint64_t* bar, uint32_t parity, int* err) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done ? true : mbar_wait(bar, parity, err);
}

// bulk copy global -> this CTA's shared memory (both 16-byte aligned, bytes a multiple of
// 16), completing `bytes` transactions on `bar`
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

}  // namespace
