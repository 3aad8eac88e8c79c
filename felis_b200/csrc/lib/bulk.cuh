// Bulk copies global -> shared memory by the TMA engine (the untiled
// cp.async.bulk form, this GPU's own memory, no multicast), counted on an
// mbarrier whose wait is bounded.
#pragma once

namespace felis {

// One instruction moves a whole row: both addresses 16-byte aligned, the size
// a multiple of 16 bytes.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst_smem)),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// Wait for phase 0 of the barrier, at most `tries` polls; false when it ran out.
__device__ __forceinline__ bool bar_wait0(unsigned bar, int tries) {
  for (int it = 0; it < tries; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar)
        : "memory");
    if (done) return true;
  }
  return false;
}
constexpr int kBulkWaitTries = 1 << 20;

}  // namespace felis
