// 5th-generation tensor-core (tcgen05) building blocks for sm_100a, in inline PTX: shared-memory matrix
// descriptors for the no-swizzle K-major layout, the instruction descriptor of kind::f16 (BF16 in, FP32
// accumulate), tensor-memory allocation, MMA issue and commit, a bounded mbarrier wait and TMEM loads.
//
// Operand layout in shared memory (K-major, no swizzle): a tile of R rows x KT bf16 values is stored as
// 8x8 "core matrices" of 128 contiguous bytes (8 rows x 16 bytes).  Element (r, k) lives at byte
//     ((r / 8) * (KT / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// so the core matrices of one 8-row group follow each other along K (leading byte offset 128) and
// consecutive 8-row groups are KT*16 bytes apart (stride byte offset).  One MMA consumes K = 16, i.e. two
// core matrices per row group; the descriptor of step s starts 256*s bytes into the tile.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dmolp {
namespace umma {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of element (r, k) in a K-major no-swizzle tile with KT columns.
__host__ __device__ __forceinline__ uint32_t tile_offset(int r, int k, int KT) {
    return (uint32_t)((((r >> 3) * (KT >> 3) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// Shared-memory matrix descriptor (sm_100 format): start address, leading / stride byte offsets (all in
// 16-byte units, 14 bits each), version 1 at bits 46-47, base offset 0, no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bits 4-5 = 1), A and B BF16 (bits 7-9,
// 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---- tensor memory ----
// Allocate ncols (a power of two >= 32) columns for this CTA; the base address is written to *slot
// (shared memory).  Called by one whole warp.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// ---- MMA: D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread ----
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate));
}

// Arrive on the mbarrier once every MMA this thread issued so far has completed.
__device__ __forceinline__ void mma_commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        smem_addr(mbar)));
}

// ---- mbarrier ----
__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count));
}
// Wait for the phase with parity `phase` to complete; gives up after `limit` polls and returns false.  Each
// poll is the non-blocking test_wait, so a limit is a fixed number of checks.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t phase, uint32_t limit) {
    const uint32_t a = smem_addr(mbar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(phase));
        if (done) return true;
    }
    return false;
}

// Generic-proxy shared-memory writes become visible to the tensor cores (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// ---- TMEM -> registers: 32 lanes x 16 consecutive 32-bit columns; the warp reads its lane quarter ----
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace dmolp
