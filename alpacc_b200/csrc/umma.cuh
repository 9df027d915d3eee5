// Fifth-generation tensor core primitives for sm_100a (tcgen05): shared-memory
// matrix descriptors for K-major operands in the 128-byte swizzle layout, the
// instruction descriptor of a BF16 x BF16 -> FP32 MMA, the MMA itself issued
// by one thread, its completion through an mbarrier (waits bounded), and
// tensor-memory allocation and loads.  Written after the PTX ISA's tcgen05
// chapter; the descriptor bit positions match CUTLASS's cute::UMMA
// SmemDescriptor and InstrDescriptor.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace alp {

// ---- operand layout ----------------------------------------------------------------
// A K-major operand tile is R rows of 64 BF16 values (128 bytes each), the tile
// 1024-byte aligned.  The 16-byte chunk c of row r sits at chunk c ^ (r & 7) of
// its row (the 128-byte swizzle); 8-row groups are 1024 bytes apart.
__device__ __forceinline__ uint32_t sw128_offset(uint32_t row, uint32_t chunk) {
    return row * 128u + ((chunk ^ (row & 7u)) << 4);
}

// Shared-memory descriptor of such a tile: start address >> 4 in bits [0,14),
// leading byte offset (16 bytes, unused by the swizzled K-major form) in
// [16,30), stride byte offset 1024 >> 4 in [32,46), version 1 in [46,48),
// layout SWIZZLE_128B (2) in [61,64).  Advancing K by 16 BF16 values within the
// 64-wide row adds 32 bytes to the start address.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3fffu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

// Instruction descriptor, kind::f16: D FP32 (bits [4,6) = 1), A and B BF16
// ([7,10) = 1, [10,13) = 1), both K-major (bits 15, 16 = 0), N >> 3 in [17,23),
// M >> 4 in [24,29).
__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[desc_a] * B[desc_b]^T for one K = 16 step; accumulate = 0 overwrites.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t desc_a, uint64_t desc_b, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(desc_a), "l"(desc_b), "r"(idesc), "r"(accumulate));
}

// The same with A from tensor memory: lane m holds row m, 32-bit column c
// holds K elements 2c and 2c + 1 (low half first).
__device__ __forceinline__ void umma_bf16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t desc_b, uint32_t idesc,
                                             uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "r"(tmem_a), "l"(desc_b), "r"(idesc), "r"(accumulate));
}

// The mbarrier arrives once every MMA this thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(mbar);
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(a) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(mbar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}

// Wait for the phase with parity `parity` to complete; false (and *err set)
// when it does not within ALP_SPIN_LIMIT polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, unsigned int* err) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(mbar);
    for (uint32_t it = 0; it < ALP_SPIN_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(64);
    }
    atomicOr(err, ALP_DEV_ERR_TIMEOUT);
    return false;
}

// Non-blocking test of the phase with parity `parity`.
__device__ __forceinline__ bool mbar_test(uint64_t* mbar, uint32_t parity) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(mbar);
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    return done != 0;
}

// mbarrier initialisation becomes visible to the async proxy (bulk copies, tensor core).
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Arrive once on the mbarrier and add `bytes` to the transaction count its
// current phase waits for (the bulk copies below complete them).
__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(mbar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}

// Bulk (non-tensor) asynchronous copy global -> shared through the TMA unit:
// both addresses 16-byte aligned, `bytes` a multiple of 16; completion is
// counted on the mbarrier in bytes.  No multicast.
__device__ __forceinline__ void bulk_g2s(uint32_t dst_smem, const void* src, uint32_t bytes, uint64_t* mbar) {
    const uint32_t m = (uint32_t)__cvta_generic_to_shared(mbar);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst_smem),
                 "l"(src), "r"(bytes), "r"(m)
                 : "memory");
}

// Shared-memory writes of the generic proxy become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Tensor memory: one warp allocates `ncols` columns (a power of two >= 32) and
// writes the base address to *dst (shared memory); the same warp frees them.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(a), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols));
}

// 32 consecutive FP32 columns of this thread's lane (row): lane 32 * (warp % 4)
// + laneid of the accumulator, columns [col, col + 32).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 8 consecutive 32-bit columns of this thread's lane, from registers
// (lane 32 * (warp % 4) + laneid, columns [col, col + 8)); tmem_wait_st waits
// for this thread's stores.
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

}  // namespace alp
