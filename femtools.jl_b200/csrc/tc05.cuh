// tc05.cuh — the sm_100a tensor-core primitives (tcgen05) used by the warm-start
// network's convolutions: shared-memory matrix descriptors, the instruction descriptor
// of a BF16 × BF16 → FP32 MMA, tensor-memory (TMEM) allocation, the single-thread MMA
// issue with its mbarrier commit, and the warp-wide TMEM → register load.
//
// Operand layout (no swizzle, K-major): a "core matrix" is 8 rows × 16 bytes stored as
// 128 contiguous bytes (row r at byte 16·r). One MMA reads, for each group of 8 rows,
// the two core matrices that hold its K = 16 BF16 values: the second one LBO bytes
// after the first; consecutive groups of 8 rows lie SBO bytes apart. Addresses, LBO
// and SBO are multiples of 16 bytes.
//
// Every wait on an mbarrier is bounded (mbar_poll gives up after 2^22 test_wait polls) and
// reports whether it gave up; the caller then records the failure in an error word and
// still frees its TMEM.
#pragma once
#include <stdint.h>
#include "common.cuh"

namespace femb {
namespace tc05 {

FEMB_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (sm_100 format): start address, leading and stride
// byte offsets in 16-byte units (14 bits each), version 1 at bits 46–47, no swizzle.
FEMB_D uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B and an FP32 accumulator: D format
// at bits 4–5, A/B formats at 7–9 / 10–12, N/8 at 17–22, M/16 at 24–28; both operands
// K-major (bits 15 and 16 select MN-major for A and B).
template <int M, int N>
FEMB_HD constexpr uint32_t idesc_bf16_f32() {
    static_assert(M == 128 && N % 16 == 0 && N >= 16 && N <= 256, "cta_group::1, M = 128 shapes only");
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// TMEM allocation of `ncols` columns (a power of two ≥ 32) by one whole warp; the base
// address is written to shared memory at `slot`.
FEMB_D void tmem_alloc(uint32_t slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
FEMB_D void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
FEMB_D void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
FEMB_D void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// makes this thread's generic-proxy shared-memory writes visible to the tensor core
FEMB_D void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (TMEM) = A·B (accumulate = false) or D + A·B; issued by one thread.
FEMB_D void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}
// arrives once on the mbarrier when every MMA this thread issued before has completed
FEMB_D void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

FEMB_D void mbar_init(uint32_t m) { asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m) : "memory"); }
FEMB_D void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Polling form for a completion that is only a few hundred cycles away (the MMAs just
// issued): mbarrier.test_wait never suspends the thread, so the caller resumes as soon as
// the phase completes; false after 2^22 polls.
FEMB_D bool mbar_poll(uint32_t m, uint32_t parity) {
    uint32_t done = 0;
    for (int it = 0; it < (1 << 22) && !done; ++it)
        asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(done)
                     : "r"(m), "r"(parity)
                     : "memory");
    return done != 0;
}

// Columns [col, col + 16) of the TMEM lane that belongs to this thread (warp w of the
// CTA reads lanes 32·(w mod 4) + lane); `taddr` carries the warp's lane base in bits 16+.
FEMB_D void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    // the load and its wait in one statement: the outputs are defined only after the wait
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc05
}  // namespace femb
