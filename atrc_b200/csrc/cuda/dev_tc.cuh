// Fifth-generation tensor core (tcgen05) primitives for sm_100a, written as
// inline PTX: tensor-memory (TMEM) allocation, shared-memory matrix
// descriptors, the kind::f16 MMA (BF16 inputs, FP32 accumulators in TMEM),
// completion through an mbarrier, and TMEM -> register loads.
//
// Operand layout.  Every MMA operand lives in shared memory in the canonical
// K-major layout without swizzle: the matrix is cut into core matrices of
// 8 rows x 16 bytes (8 BF16 values along K), each stored as 128 contiguous
// bytes (row r at byte 16 r).  Core matrix (row group g, K chunk j) of an
// operand with K columns sits at byte (g * K / 8 + j) * 128: the descriptor's
// leading byte offset (between K chunks) is 128 and its stride byte offset
// (between 8-row groups) is K * 16.  One MMA consumes K = 16, two K chunks.
// Row groups are outermost, so an operand read with more rows than it holds
// (M = 128 over a 64-row matrix) reads past its end, never inside it.
//
// Every wait on an mbarrier is bounded; a wait that gives up sets *err and
// returns, and the kernels then skip their remaining MMAs but still free
// their TMEM.
#pragma once

#include <cstdint>

namespace atrc {
namespace dev {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (row, k) of an operand with K columns.
__device__ __forceinline__ uint32_t kmajor_offset(int K, int row, int k) {
    return uint32_t(((row >> 3) * (K >> 3) + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (tcgen05 format, no swizzle).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFF);
    d |= uint64_t((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= uint64_t((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= uint64_t(1) << 46;  // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Descriptor of the K-step `ks` (16 values of K) of an operand with K columns.
__device__ __forceinline__ uint64_t operand_desc(uint32_t base_saddr, int K, int ks) {
    return make_desc(base_saddr + uint32_t(ks) * 256, 128, uint32_t(K) * 16);
}

// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

// ---- TMEM allocation (one full warp executes these)
__device__ __forceinline__ void tmem_alloc(uint32_t* smem_dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_addr(smem_dst)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- MMA issue (one thread)
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1u : 0u) : "memory");
}

// D[128 x N] (+)= A[128 x K] B[N x K]^T, both operands K-major with K
// columns in shared memory.
__device__ __forceinline__ void mma_tile(uint32_t tmem_d, uint32_t a_saddr, uint32_t b_saddr, int k, int n,
                                         bool accumulate) {
    const uint32_t id = idesc_bf16(128, n);
    for (int ks = 0; ks < k / 16; ++ks)
        mma_bf16(tmem_d, operand_desc(a_saddr, k, ks), operand_desc(b_saddr, k, ks), id, accumulate || ks > 0);
}

// ---- completion
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// All MMAs issued so far by this thread arrive on `bar` when complete.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_addr(bar)) : "memory");
}
// Wait for phase `parity` of `bar` to complete; gives up after `limit`
// polls (each try_wait may suspend the thread for a while) and sets *err.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, uint32_t limit = 1u << 20) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    atomicExch(err, 1);
    return false;
}

// ---- bulk copies (TMA engine, untiled, no multicast)
// Arm `bar` for one arrival that also expects `bytes` of transactions.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// Copy `bytes` (a multiple of 16; both addresses 16-byte aligned) from
// global to this CTA's shared memory; completion is counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// ---- TMEM -> registers: this warp's 32 lanes, 16 consecutive columns
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr) : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// TMEM address of (lane, column) relative to an allocation base.
__device__ __forceinline__ uint32_t tmem_at(uint32_t base, int lane, int col) {
    return base + (uint32_t(lane) << 16) + uint32_t(col);
}

}  // namespace tc
}  // namespace dev
}  // namespace atrc
