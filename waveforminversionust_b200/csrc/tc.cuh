// tcgen05 (5th-generation tensor core) building blocks for sm_100a.
//
// One CTA computes a 128 x TN fp32 tile D = A * B^T in tensor memory:
//   A: 128 rows x K, B: TN rows x K, both K-major in the no-swizzle
//      core-matrix layout (8 rows x 16 bytes per core matrix), stored in
//      global memory already cut into K-chunks of 128 bytes per row, so one
//      chunk of a tile is one contiguous block that a single cp.async.bulk
//      moves into shared memory.
//   Inside a chunk: core matrix (row group g, k group q) sits at
//      g * 1024 + q * 128 bytes; rows of a core matrix are 16 bytes apart.
//      -> leading byte offset (K direction) 128 B, stride byte offset
//         (row-group direction) 1024 B.
//   One MMA consumes 32 bytes of K (bf16: K = 16, tf32: K = 8), i.e. two
//   core matrices, so the descriptor start advances 256 B per MMA.
// A single thread issues the bulk copies (mbarrier complete_tx), the MMAs
// (accumulating in TMEM) and the tcgen05.commit arrivals; every wait is
// bounded by a %globaltimer budget and reports failure.
#pragma once

#include <stdint.h>

#include "common.cuh"

namespace wust {
namespace tc {

constexpr int kChunkBytes = 128;                 // K bytes per row per chunk
constexpr int kRowGroupBytes = 8 * kChunkBytes;  // 1024: one 8-row group of a chunk
constexpr int kTileRows = 128;                   // MMA M
constexpr int kAChunk = kTileRows * kChunkBytes; // 16 KB

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (row, ke) inside one K chunk (128 bytes per row) of a
// tile in the layout above.
__host__ __device__ __forceinline__ size_t chunk_off(int row, int ke) {
    return (size_t)(row >> 3) * kRowGroupBytes + (size_t)(ke >> 2) * 128 + (size_t)(row & 7) * 16 + (ke & 3) * 4;
}

// The same layout for 16-bit operands: 64 K values per 128-byte chunk row,
// 8 per 16-byte core-matrix row.
__host__ __device__ __forceinline__ size_t chunk_off16(int row, int ke) {
    return (size_t)(row >> 3) * kRowGroupBytes + (size_t)(ke >> 3) * 128 + (size_t)(row & 7) * 16 + (ke & 7) * 2;
}

// fp32 -> bf16 bits, round to nearest even; Inf and NaN keep their class.
__device__ __forceinline__ uint16_t to_bf16_bits(float x) {
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)((u >> 16) | ((u & 0xffffu) ? 0x40u : 0u));
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

// Round to TF32 (10-bit mantissa, nearest, ties away).  The tensor core
// would otherwise drop the low mantissa bits of fp32 operands (truncation),
// a bias that accumulates over long products.  Integer form (two ALU ops):
// add half of the 13 dropped bits to the magnitude, clear them.  Inf and NaN
// pass unchanged.
__device__ __forceinline__ float to_tf32(float x) {
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    return __uint_as_float(u);
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// Bounded parity wait: false when the budget ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase, unsigned long long timeout_ns) {
    const uint32_t a = smem_u32(bar);
    unsigned long long t0 = 0;
    for (uint32_t spin = 0;; ++spin) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
        if ((spin & 63u) == 0) {
            const unsigned long long t = global_timer_ns();
            if (!t0) t0 = t;
            else if (t - t0 > timeout_ns) return false;
        }
    }
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// L2 eviction priorities for bulk copies: a stream read once (evict first)
// and lines that several CTAs read shortly after (evict last).
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar, uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
}
__device__ __forceinline__ uint64_t smem_desc(const void *p) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_u32(p) >> 4) & 0x3FFF);                 // start address
    d |= (uint64_t)((kChunkBytes >> 4) & 0x3FFF) << 16;           // leading byte offset (K direction)
    d |= (uint64_t)((kRowGroupBytes >> 4) & 0x3FFF) << 32;        // stride byte offset (row groups)
    d |= (uint64_t)1 << 46;                                       // descriptor version for sm_100
    return d;                                                     // base offset 0, no swizzle
}
// Instruction descriptor: D fp32, A/B tf32 (kind::tf32) or bf16 (kind::f16), both K-major.
template <bool TF32>
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
    return (1u << 4) | ((TF32 ? 2u : 1u) << 7) | ((TF32 ? 2u : 1u) << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

template <bool TF32>
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    if (TF32)
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p; }" ::"r"(
                         tmem_d),
                     "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
                     : "memory");
    else
        asm volatile("{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }" ::"r"(
                         tmem_d),
                     "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
                     : "memory");
}
__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Warp-wide TMEM allocation (ncols: power of two >= 32); address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// 8 consecutive fp32 columns of this thread's TMEM lane (warp w reads lanes 32(w%4)..).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = __uint_as_float(r[q]);
}

// 32 consecutive fp32 columns of this thread's TMEM lane, one wait.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

}  // namespace tc
}  // namespace wust
