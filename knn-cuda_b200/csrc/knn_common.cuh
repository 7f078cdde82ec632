// knn_common.cuh -- device helpers shared by the k-NN kernels (sm_100a only).
//
// * mbarrier init / arrive / bounded wait (every wait gives up after a time
//   limit and reports it instead of spinning forever),
// * 2-D TMA tile loads (cp.async.bulk.tensor, no multicast),
// * packed FP32 pair arithmetic (sub/fma .f32x2, sm_100+),
// * the 64-bit (distance, index) selection key.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define KNN_DI __device__ __forceinline__

namespace knnb200 {

// ---------------------------------------------------------------------------
// Error codes written by kernels into a device status word.
// ---------------------------------------------------------------------------
enum DeviceStatus : int {
    kDevOk = 0,
    kDevTimeoutFull = 1,   // consumer gave up waiting for a TMA stage
    kDevTimeoutEmpty = 2,  // producer gave up waiting for consumers to free a stage
    kDevTimeoutDrain = 3,  // producer gave up waiting for its own copies at exit
};

// Wait limit for any spin on an mbarrier: 2 s of %globaltimer.  A pipeline
// stage normally completes in microseconds.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

KNN_DI uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

KNN_DI unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

KNN_DI void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Make mbarrier initialisation visible to the async (TMA) proxy.
KNN_DI void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

KNN_DI void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

KNN_DI void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

KNN_DI bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete.  Returns false if it
// did not complete within kWaitLimitNs (the caller records an error and
// leaves its loop; nothing spins forever).
KNN_DI bool mbar_wait(uint64_t *bar, uint32_t parity,
                      unsigned long long limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        for (int i = 0; i < 64; ++i)
            if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// 2-D tiled TMA load of box {x .. x+box0, y .. y+box1} into shared memory,
// completing on `bar` (complete_tx).  x * elemsize must be a multiple of 16 B.
KNN_DI void tma_load_2d(void *smem_dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

KNN_DI void prefetch_tensormap(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ---------------------------------------------------------------------------
// Packed FP32 pairs (two lanes of work per instruction; IEEE round-to-nearest,
// so results equal the scalar sub / fma on each half).
// ---------------------------------------------------------------------------
typedef unsigned long long f32x2_t;

KNN_DI f32x2_t f2_pack(float lo, float hi) {
    f32x2_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
KNN_DI float f2_lo(f32x2_t v) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
    return lo;
}
KNN_DI float f2_hi(f32x2_t v) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
    return hi;
}
KNN_DI f32x2_t f2_sub(f32x2_t a, f32x2_t b) {
    f32x2_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
KNN_DI f32x2_t f2_fma(f32x2_t a, f32x2_t b, f32x2_t c) {
    f32x2_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// ---------------------------------------------------------------------------
// Selection key: (squared distance bits << 32) | reference index.  For
// non-negative floats the bit pattern is monotonic, so ascending keys give
// ascending distance with ties broken by ascending index -- the order the
// reference's insertion sort produces (code/knncuda.cu:172, :178).
// ---------------------------------------------------------------------------
constexpr unsigned long long kKeyInf = ~0ull;

KNN_DI unsigned long long make_key(float d2, uint32_t idx) {
    return (static_cast<unsigned long long>(__float_as_uint(d2)) << 32) | idx;
}
KNN_DI float key_dist2(unsigned long long key) {
    return __uint_as_float(static_cast<uint32_t>(key >> 32));
}
KNN_DI int key_index(unsigned long long key) { return static_cast<int>(key & 0xffffffffu); }

}  // namespace knnb200
