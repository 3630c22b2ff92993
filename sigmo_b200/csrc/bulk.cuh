// Bulk asynchronous global -> shared copies (cp.async.bulk, the TMA engine)
// with completion counted on a shared-memory mbarrier, and a bounded wait.
// Used by the kernels that stage a CTA's input in shared memory before many
// threads read it (per-vertex signatures, the GMCR non-empty pass).
#pragma once

#include <cstdint>

namespace sigmo_b200 {

// try_wait polls before a wait gives up; each poll may suspend the thread
// for a hardware-chosen interval, so the bound is far above any copy's time.
constexpr uint32_t kBulkSpinLimit = 1u << 22;

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// Arrives once on `bar` and adds `bytes` to the transfer count its phase waits for.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(bytes) : "memory");
}
// Bulk global -> shared copy of `bytes` (multiple of 16; both addresses
// 16-byte aligned), its completion counted on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const unsigned b = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(d), "l"(src),
               "r"(bytes), "r"(b)
               : "memory");
}
// Waits (bounded) for phase `parity` of `bar` to complete; false if it did not.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  for (uint32_t i = 0; i < kBulkSpinLimit; ++i) {
    uint32_t done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// The same wait, letting the hardware suspend the thread for up to
// `hint_ns` nanoseconds per poll (it resumes as soon as the phase completes),
// so waiting warps take fewer issue slots; at most `polls` polls.
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t hint_ns, uint32_t polls) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  for (uint32_t i = 0; i < polls; ++i) {
    uint32_t done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(hint_ns)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace sigmo_b200
