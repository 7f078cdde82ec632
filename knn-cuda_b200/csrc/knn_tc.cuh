// knn_tc.cuh -- tcgen05 / TMEM helpers (sm_100a): TMEM allocation, UMMA
// shared-memory and instruction descriptors, MMA issue / commit, TMEM loads.
#pragma once

#include "knn_common.cuh"

namespace knnb200 {

KNN_DI void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
KNN_DI void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor for a K-major operand stored with the
// 128-byte swizzle (the layout a TMA SWIZZLE_128B box of 64 bf16 x rows
// produces): rows of 128 B, 8-row swizzle atoms 1024 B apart.
//   start address >> 4 in [0,14), LBO = 1 (16 B, unused for swizzled K-major)
//   in [16,30), SBO = 1024 B >> 4 in [32,46), version 1 in [46,48),
//   layout type SWIZZLE_128B (2) in [61,64).  The buffer is 1024-B aligned.
KNN_DI uint64_t umma_desc_sw128(const void *smem_ptr) {
    const uint64_t addr = smem_u32(smem_ptr);
    uint64_t d = (addr >> 4) & 0x3FFFull;
    d |= 1ull << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= 1ull << 46;
    d |= 2ull << 61;
    return d;
}

// Same for the 32-byte swizzle (a TMA SWIZZLE_32B box of 16 bf16 x rows):
// rows of 32 B (one K=16 step), 8-row atoms 256 B apart, layout type
// SWIZZLE_32B (6).  The buffer is 256-B aligned.
KNN_DI uint64_t umma_desc_sw32(const void *smem_ptr) {
    const uint64_t addr = smem_u32(smem_ptr);
    uint64_t d = (addr >> 4) & 0x3FFFull;
    d |= 1ull << 16;
    d |= (uint64_t)(256 >> 4) << 32;
    d |= 1ull << 46;
    d |= 6ull << 61;
    return d;
}

// Make this thread's generic-proxy shared-memory writes visible to the
// async proxy (tensor-core operand reads) after the next barrier.
KNN_DI void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Instruction descriptor, kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 in
// [17,23), M >> 4 in [24,29).
constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}
// Instruction descriptor, kind::f8f6f4: D = F32, A = B = E4M3 (format 0 in
// bits 7-9 and 10-12), both K-major, N >> 3 in [17,23), M >> 4 in [24,29).
constexpr uint32_t umma_idesc_e4m3(int M, int N) {
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---------------------------------------------------------------------------
// CTA pairs (cluster of 2, cta_group::2): one MMA spans both CTAs' tensor
// cores.  A (M = 256) is split by rows between the two CTAs' shared memory,
// B (N) by rows (reference points) likewise, at the same shared-memory
// offsets; CTA r's TMEM receives accumulator rows r * 128 .. + 127, all N
// columns.  The even CTA of the pair (rank 0) issues the MMAs.
// ---------------------------------------------------------------------------
KNN_DI uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// Address of the same shared-memory offset in CTA `rank` of the cluster.
KNN_DI uint32_t mapa_shared(uint32_t local_addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local_addr), "r"(rank));
    return r;
}
// All threads of both CTAs; orders shared-memory (and barrier-init) writes
// before the barrier against reads after it, cluster-wide.
KNN_DI void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                     : "memory");
}
// Arrive on an mbarrier of another CTA of the cluster (shared::cluster
// address).  Used after tcgen05.wait::ld + tcgen05.fence::before_thread_sync:
// the TMEM data already sits in registers when the arrive executes.
KNN_DI void mbar_arrive_cluster(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
// TMA 2-D load into this CTA's shared memory whose completion is counted on
// an mbarrier of either CTA of the pair (shared::cluster address).
KNN_DI void tma_load_2d_pair(void *smem_dst, const CUtensorMap *map, uint32_t bar_cluster_addr,
                             int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar_cluster_addr), "r"(x), "r"(y)
        : "memory");
}
// Both CTAs of the pair execute these (same warp), with the same holder
// offset.
KNN_DI void tmem_alloc_pair(uint32_t *smem_holder, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(smem_holder)),
                 "r"(ncols)
                 : "memory");
}
KNN_DI void tmem_relinquish_pair() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
KNN_DI void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
KNN_DI void umma_bf16_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                           uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// The same MMA on FP8 operands (kind::f8f6f4; K = 32 per instruction, so a
// K step is again 32 bytes of each operand row).
KNN_DI void umma_f8_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive on the mbarrier at this shared-memory offset in every CTA of
// cta_mask once the pair MMAs issued so far have completed.
KNN_DI void umma_commit_pair_mc(uint64_t *bar, uint16_t cta_mask) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
        " [%0], %1;" ::"r"(smem_u32(bar)),
        "h"(cta_mask)
        : "memory");
}
KNN_DI void umma_commit_pair(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns: thread i of the warp receives
// lane (taddr.lane + i), columns taddr.col .. +31.
KNN_DI void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
          "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
          "=r"(v[31])
        : "r"(taddr));
}
// Wait for this thread's outstanding TMEM loads.  The loaded registers are
// passed through the asm so no use of them can be scheduled before the wait.
KNN_DI void tmem_ld_wait(uint32_t (&v)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]),
                   "+r"(v[6]), "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]),
                   "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15]), "+r"(v[16]), "+r"(v[17]),
                   "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]), "+r"(v[22]), "+r"(v[23]),
                   "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]), "+r"(v[29]),
                   "+r"(v[30]), "+r"(v[31])
                 :
                 : "memory");
}

// Three-input minimum (sm_100): min of a, b, c; a NaN operand is ignored
// like fminf.
KNN_DI float min3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Smallest of 32 accumulator values (FP32 bit patterns): a depth-4 tree
// of 17 min instructions.
KNN_DI float min32(const uint32_t (&v)[32]) {
    float m[11];
#pragma unroll
    for (int i = 0; i < 10; ++i)
        m[i] = min3f(__uint_as_float(v[3 * i]), __uint_as_float(v[3 * i + 1]),
                     __uint_as_float(v[3 * i + 2]));
    m[10] = fminf(__uint_as_float(v[30]), __uint_as_float(v[31]));
    const float n0 = min3f(m[0], m[1], m[2]), n1 = min3f(m[3], m[4], m[5]);
    const float n2 = min3f(m[6], m[7], m[8]), n3 = fminf(m[9], m[10]);
    return fminf(min3f(n0, n1, n2), n3);
}

}  // namespace knnb200
