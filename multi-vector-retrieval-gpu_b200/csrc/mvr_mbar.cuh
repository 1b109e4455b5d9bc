// mvr_mbar.cuh -- shared-memory mbarrier helpers with bounded waits, used by
// the warp-specialised kernels of libmvr (sm_100a).
#pragma once
#include <cstdint>

namespace mvr {

constexpr uint64_t kWaitNs = 1000000000ull;  // mbarrier wait bound (1 s)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

// Bounded wait on an mbarrier phase: try_wait suspends the thread until the
// phase completes (or a hardware time slice passes); gives up after limit_ns
// of %globaltimer and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                          uint64_t limit_ns = kWaitNs) {
  const uint32_t a = smem_u32(bar);
  uint64_t t0 = 0;
  for (uint32_t i = 0;; i++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (i == 0) t0 = global_ns();
    else if (global_ns() - t0 > limit_ns) return false;
  }
}

// The same bounded wait, but a thread whose phase is not complete sleeps in
// try_wait (up to hint_ns per attempt, woken when the phase completes)
// instead of polling: for waits that are long by design, where polling warps
// would take issue slots from the warps they wait for.
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t *bar, uint32_t parity,
                                                uint64_t limit_ns = kWaitNs,
                                                uint32_t hint_ns = 20000u) {
  const uint32_t a = smem_u32(bar);
  uint64_t t0 = 0;
  for (uint32_t i = 0;; i++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(hint_ns)
        : "memory");
    if (done) return true;
    if (i == 0) t0 = global_ns();
    else if (global_ns() - t0 > limit_ns) return false;
  }
}

}  // namespace mvr
