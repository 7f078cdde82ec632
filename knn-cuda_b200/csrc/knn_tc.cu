// knn_tc.cu -- the expansion method (knn_cublas) on tcgen05 tensor cores,
// returning EXACT results.
//
// The reference computes D = ||r||^2 - 2 Q^T R + ||q||^2 with cublasSgemm
// plus norm kernels, sorts the full matrix and adds ||q||^2 to the survivors
// (code/knncuda.cu:709-794).  Here the contraction runs in BF16 on the 5th-gen
// tensor cores with FP32 accumulation in TMEM, and the selection lives in the
// GEMM epilogue; nothing of size ref_nb x query_nb is stored.
//
// The norm term is part of the contraction: the query operand is
// bf16(-2 q) (exact scaling of bf16(q)), and one extra K=16 step multiplies
// a tile of ones by the reference's squared norm split into three BF16 parts
// (h + m + l = ||r||^2 to 2^-27 relative), so the accumulator holds
// a = ||r||^2 - 2 r.q directly and the epilogue reads nothing but TMEM.
//
//   prep      reference / query sets -> BF16 point-major (K-major) copies,
//             FP32 point-major copy of the reference set (for re-ranking),
//             the reference norm parts, FP32 query norms and the largest
//             reference norm.
//   pass 1    tensor scan of a 1/G sample of the reference tiles (runs of
//             consecutive tiles, one run every G runs' worth); each
//             epilogue thread keeps the KS smallest a of its query row in
//             registers -> threshold T_q (KS-th smallest over the sample;
//             over the full set about KS*G points lie below it).
//   pass 2    tensor scan of all reference tiles; the epilogue emits every
//             reference with a < T_q into the query's candidate list.
//   rerank    exact FP32 direct-form distances of the candidates, in the same
//             arithmetic and order as the fused exact kernel, sorted by
//             (distance, index).  The result is CERTIFIED when the k-th exact
//             distance D_k satisfies D_k (1+g) + E_q < T_q + ||q||^2, where
//             E_q bounds |(BF16 expansion) - (exact squared distance)| for
//             every reference: then every point that could belong to the
//             exact top-k was emitted, and the output is bit-identical to
//             the exact kernel's.  Uncertified queries (sample too small, list
//             overflow) are scanned again or recomputed by the exact kernel.
//             When the set streams in from the host in pieces, the re-rank
//             runs piece by piece into running top-k lists and only the
//             certification waits for the last piece.
//
// Error bound (u = 2^-8, BF16 unit roundoff; K = d_pad + 16 accumulated
// terms): |bf16(r).bf16(q) - r.q| <= (2u + u^2) sum|r_i q_i|, and the FP32
// accumulation of the K products adds at most K 2^-23 of the sum of their
// magnitudes (2 ||r|| ||q|| (1 + u)^2 + ||r||^2 (1 + 2^-8)); the norm itself
// carries the FP32 rounding of its d-term FMA chain and the 2^-27 of the
// split.  With g = K 2^-22 (twice the accumulation term) and eps = 2^-7 +
// 2^-16 + g, E_q = 2 eps ||q|| max||r|| + g (max||r||^2 + ||q||^2) + 2^-20
// (|T_q| + ||q||^2) covers all of them and the roundings of ||q||^2 and T_q.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdio>

#include "knn_exact_core.cuh"
#include "knn_kernels.h"
#include "knn_tc.cuh"

namespace knnb200 {

constexpr int TC_BM = 128;            // rows (queries) per CTA of a pair, points per CTA half-tile
constexpr int TC_QT = 2 * TC_BM;      // queries per CTA pair
constexpr int TC_BK = 64;             // K block: 64 bf16 = 128 B (one swizzle row)
constexpr int TC_KBMAX = 4;           // d_pad <= 256
constexpr int TC_TILE_BYTES = TC_BM * TC_BK * 2;   // 16 KB (A or B K-block tile of one CTA)
constexpr int TC_NK = 16;             // norm step: K = 16 (h, m, l, 13 zeros)
constexpr int TC_NORM_BYTES = TC_BM * TC_NK * 2;   // 4 KB norm tile (32-byte swizzle)
constexpr int TC_KS = 16;             // pass-1 per-row list length
constexpr uint32_t TC_TMEM_COLS = 512;   // 2 accumulator buffers x 256 columns
constexpr int kCenterStride = 64;     // the translation is the mean of every 64th tile

// Candidate entries: (order-preserving bits of a) << 32 | reference index,
// so that unsigned order is (a, index) order for every non-NaN a.
KNN_DI uint32_t ord_bits(uint32_t f) { return (f & 0x80000000u) ? ~f : (f | 0x80000000u); }
KNN_DI float ord_float(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// Bit e set iff v[e] < lim: independent compares, then a 3-input OR tree
// (depth 4) instead of a 32-long dependent chain.
KNN_DI uint32_t below_mask(const uint32_t (&v)[32], float lim) {
    uint32_t b[32];
#pragma unroll
    for (int e = 0; e < 32; ++e) b[e] = __uint_as_float(v[e]) < lim ? (1u << e) : 0u;
    uint32_t t[11];
#pragma unroll
    for (int i = 0; i < 10; ++i) t[i] = b[3 * i] | b[3 * i + 1] | b[3 * i + 2];
    t[10] = b[30] | b[31];
    const uint32_t u0 = t[0] | t[1] | t[2], u1 = t[3] | t[4] | t[5];
    const uint32_t u2 = t[6] | t[7] | t[8], u3 = t[9] | t[10];
    return u0 | u1 | u2 | u3;
}

// v[e] for a run-time e: a binary select tree on e's bits (depth 5)
// instead of a 31-long dependent chain; v stays in registers.
KNN_DI uint32_t select32(const uint32_t (&v)[32], int e) {
    uint32_t s16[16], s8[8], s4[4];
#pragma unroll
    for (int i = 0; i < 16; ++i) s16[i] = (e & 1) ? v[2 * i + 1] : v[2 * i];
#pragma unroll
    for (int i = 0; i < 8; ++i) s8[i] = (e & 2) ? s16[2 * i + 1] : s16[2 * i];
#pragma unroll
    for (int i = 0; i < 4; ++i) s4[i] = (e & 4) ? s8[2 * i + 1] : s8[2 * i];
    const uint32_t s2a = (e & 8) ? s4[1] : s4[0], s2b = (e & 8) ? s4[3] : s4[2];
    return (e & 16) ? s2b : s2a;
}

// Candidates found by one epilogue thread, appended to its query's list
// later with one atomicAdd that reserves all their slots: the append's
// round trip then overlaps the wait for the next accumulator instead of
// lengthening the test of the current one (the next tile's TMEM load waits
// for that test).
struct PendingCands {
    static constexpr int kMax = 4;
    unsigned long long e[kMax];
    int n = 0;
    KNN_DI void flush(int *count, unsigned long long *cand, int cmax, int qrow) {
        if (n == 0) return;
        const int pos = atomicAdd(&count[qrow], n);
#pragma unroll
        for (int p = 0; p < kMax; ++p)
            if (p < n && pos + p < cmax) cand[(size_t)qrow * cmax + pos + p] = e[p];
        n = 0;
    }
    KNN_DI void push(unsigned long long key, int *count, unsigned long long *cand, int cmax,
                     int qrow) {
        if (n == kMax) flush(count, cand, cmax, qrow);
#pragma unroll
        for (int p = 0; p < kMax; ++p)
            if (p == n) e[p] = key;
        ++n;
    }
};

// ---------------------------------------------------------------------------
// The tensor scan on CTA pairs (cta_group::2): pass 1 (MODE 0, the tiles
// of a sample pattern), pass 2 and the second-chance scan (MODE 1).  A
// cluster of two CTAs owns 256 queries (128 per CTA, resident) and walks its
// reference range in tiles of 256 points, each CTA loading its 128-point
// half of every K block.  The even CTA issues M = 256, N = 256 MMAs whose
// operands come from both CTAs' shared memory, so each SM's tensor core
// reads 8 KB of operands per 1 MFLOP instead of the 16 KB of two 128 x 128
// MMAs sharing one B tile: the scan is tensor-bound rather than
// shared-memory-bound.  Each CTA's epilogue reads its own 128 accumulator
// rows x 256 columns from TMEM.
//
// Synchronisation: the full barriers live in the even CTA and count the TMA
// bytes of both CTAs (the even CTA's producer expects both shares); the
// MMA commits arrive on the empty / accumulator-full barriers of both CTAs;
// both CTAs' epilogue warps arrive on the even CTA's accumulator-empty
// barriers.  Every wait is bounded; both CTAs reach the closing cluster
// barrier on every path.
// ---------------------------------------------------------------------------
constexpr int TP_BN = 256;            // reference points per pair tile
constexpr int TP_EPI_WARPS = 8;       // two per TMEM lane quadrant, 128 columns each
constexpr int TP_COLS = TP_BN / (TP_EPI_WARPS / 4);   // columns per epilogue warp
constexpr int TP_CHUNKS = TP_COLS / 32;
constexpr int TP_THREADS = 32 * (2 + TP_EPI_WARPS);   // warp 0 TMA, warp 1 MMA, epilogue
constexpr int TP_LISTS = TP_EPI_WARPS / 4;             // pass-1 lists per query and split
constexpr int TP_STAGES = 8;
constexpr int TP_NSLOTS = 4;
constexpr uint32_t TP_IDESC = umma_idesc_bf16(2 * TC_BM, TP_BN);

constexpr size_t TP_OFF_A = 0;
constexpr size_t TP_OFF_ONES = (size_t)TC_KBMAX * TC_TILE_BYTES;                // 64 KB
constexpr size_t TP_OFF_B = TP_OFF_ONES + (size_t)TC_BM * TC_NK * 2;            // +4 KB
constexpr size_t TP_OFF_N = TP_OFF_B + (size_t)TP_STAGES * TC_TILE_BYTES;        // +128 KB
constexpr size_t TP_OFF_BAR = TP_OFF_N + (size_t)TP_NSLOTS * TC_NORM_BYTES;      // +16 KB
constexpr int TP_NBARS = 1 + 2 * TP_STAGES + 2 * TP_NSLOTS + 2 + 2 + 1;
constexpr size_t TP_SMEM = 1024 + TP_OFF_BAR + TP_NBARS * 8 + 16;
static_assert(TP_SMEM <= 232448, "pair scan kernel shared memory");

struct TpArgs {
    int N, Q, kb_count;
    int tile_base, n_splits;
    TileRuns tiles;         // scan tiles tile_base + tiles.tile(u), u < tiles.units
    const float *thr;       // emit pass: [Q] thresholds (a units)
    float *p1;              // sample pass: [TP_LISTS n_splits][Q][TC_KS] (per column range)
    unsigned long long *cand;   // [Q][cmax] (a, index) entries
    int *count;             // [Q]
    int cmax;
    int *status;
};

template <int MODE>   // 0: threshold sample pass, 1: emit pass
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TP_THREADS, 1)
    knn_tc_pair_scan_kernel(const __grid_constant__ CUtensorMap tmA,
                            const __grid_constant__ CUtensorMap tmB,
                            const __grid_constant__ CUtensorMap tmN, TpArgs a) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char *sA = base + TP_OFF_A;
    unsigned char *sOnes = base + TP_OFF_ONES;
    unsigned char *sB = base + TP_OFF_B;
    unsigned char *sN = base + TP_OFF_N;
    uint64_t *bars = reinterpret_cast<uint64_t *>(base + TP_OFF_BAR);
    uint64_t *a_full = bars;
    uint64_t *b_full = bars + 1;
    uint64_t *b_empty = b_full + TP_STAGES;
    uint64_t *n_full = b_empty + TP_STAGES;
    uint64_t *n_empty = n_full + TP_NSLOTS;
    uint64_t *acc_full = n_empty + TP_NSLOTS;
    uint64_t *acc_empty = acc_full + 2;
    uint64_t *drain = acc_empty + 2;
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(bars + TP_NBARS);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_holder + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const bool lead = rank == 0;
    const int qpair = blockIdx.x >> 1, split = blockIdx.y;
    const int KB = a.kb_count;
    // this split's units [u0, u0 + n_my)
    const int u0 = (int)((long long)a.tiles.units * split / a.n_splits);
    const int n_my = (int)((long long)a.tiles.units * (split + 1) / a.n_splits) - u0;

    for (int i = threadIdx.x; i < TC_BM * TC_NK / 2; i += TP_THREADS)
        reinterpret_cast<uint32_t *>(sOnes)[i] = 0x3F803F80u;
    fence_proxy_async_smem();
    if (warp == 0 && lane == 0) {
        mbar_init(a_full, 1);
        for (int s = 0; s < TP_STAGES; ++s) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 1);
        }
        for (int s = 0; s < TP_NSLOTS; ++s) {
            mbar_init(&n_full[s], 1);
            mbar_init(&n_empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 2 * TP_EPI_WARPS);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        fence_mbar_init();
        prefetch_tensormap(&tmA);
        prefetch_tensormap(&tmB);
        prefetch_tensormap(&tmN);
    }
    if (warp == 1) {
        tmem_alloc_pair(tmem_holder, TC_TMEM_COLS);
        tmem_relinquish_pair();
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();   // both CTAs' barriers are initialised before any use
    tc_fence_after();
    const uint32_t tmem = *tmem_holder;

    if (warp == 0) {
        // ---------------- TMA producer (both CTAs) ----------------
        if (lane == 0) {
            int issued = 0, n_issued = 0;
            bool a_issued = false, ok = true;
            const int half_row = (int)rank * TC_BM;
            if (n_my > 0) {
                if (lead) mbar_arrive_expect_tx(a_full, (uint32_t)(2 * KB * TC_TILE_BYTES));
                const uint32_t bar = mapa_shared(smem_u32(a_full), 0);
                for (int kb = 0; kb < KB; ++kb)
                    tma_load_2d_pair(sA + (size_t)kb * TC_TILE_BYTES, &tmA, bar, kb * TC_BK,
                                     qpair * TC_QT + half_row);
                a_issued = true;
            }
            for (int j = 0; j < n_my && ok; ++j) {
                const int row0 = (a.tile_base + a.tiles.tile(u0 + j)) * TP_BN + half_row;
                const int ns = j % TP_NSLOTS;
                if (j >= TP_NSLOTS && !mbar_wait(&n_empty[ns], ((j / TP_NSLOTS) - 1) & 1)) {
                    ok = false;
                    break;
                }
                if (*abort_flag) break;
                if (lead) mbar_arrive_expect_tx(&n_full[ns], 2 * TC_NORM_BYTES);
                tma_load_2d_pair(sN + (size_t)ns * TC_NORM_BYTES, &tmN,
                                 mapa_shared(smem_u32(&n_full[ns]), 0), 0, row0);
                n_issued = j + 1;
                const int row_ahead = j + 2 < n_my
                                          ? (a.tile_base + a.tiles.tile(u0 + j + 2)) * TP_BN + half_row
                                          : a.N;
                for (int kb = 0; kb < KB; ++kb) {
                    const int it = j * KB + kb, s = it % TP_STAGES;
                    if (it >= TP_STAGES && !mbar_wait(&b_empty[s], ((it / TP_STAGES) - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    if (*abort_flag) break;
                    if (lead) mbar_arrive_expect_tx(&b_full[s], 2 * TC_TILE_BYTES);
                    tma_load_2d_pair(sB + (size_t)s * TC_TILE_BYTES, &tmB,
                                     mapa_shared(smem_u32(&b_full[s]), 0), kb * TC_BK, row0);
                    if (row_ahead < a.N) tma_prefetch_l2_2d(&tmB, kb * TC_BK, row_ahead);
                    issued = it + 1;
                }
                if (*abort_flag) break;
            }
            if (!ok) {
                atomicMax(a.status, (int)kDevTimeoutEmpty);
                *abort_flag = 1;
            }
            // The even CTA's full barriers count both CTAs' bytes: once its
            // last phases completed, no TMA write into either CTA is in
            // flight (the closing cluster barrier orders the odd CTA's exit
            // after this).
            if (lead) {
                for (int it = max(0, issued - TP_STAGES); it < issued; ++it)
                    if (!mbar_wait(&b_full[it % TP_STAGES], (it / TP_STAGES) & 1))
                        atomicMax(a.status, (int)kDevTimeoutDrain);
                for (int j = max(0, n_issued - TP_NSLOTS); j < n_issued; ++j)
                    if (!mbar_wait(&n_full[j % TP_NSLOTS], (j / TP_NSLOTS) & 1))
                        atomicMax(a.status, (int)kDevTimeoutDrain);
                if (a_issued && !mbar_wait(a_full, 0)) atomicMax(a.status, (int)kDevTimeoutDrain);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issuer (even CTA) ----------------
        if (lead && lane == 0) {
            bool ok = n_my == 0 || mbar_wait(a_full, 0);
            bool issued_mma = false;
            tc_fence_after();
            const uint64_t odesc = umma_desc_sw32(sOnes);
            for (int j = 0; j < n_my && ok; ++j) {
                const int b = j & 1;
                if (j >= 2 && !mbar_wait(&acc_empty[b], ((j >> 1) - 1) & 1)) {
                    ok = false;
                    break;
                }
                const int ns = j % TP_NSLOTS;
                if (!mbar_wait(&n_full[ns], (j / TP_NSLOTS) & 1) || *abort_flag) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                umma_bf16_pair(tmem + (uint32_t)(b * TP_BN), odesc,
                               umma_desc_sw32(sN + (size_t)ns * TC_NORM_BYTES), TP_IDESC, 0u);
                umma_commit_pair_mc(&n_empty[ns], 0x3);
                issued_mma = true;
                for (int kb = 0; kb < KB; ++kb) {
                    const int it = j * KB + kb, s = it % TP_STAGES;
                    if (!mbar_wait(&b_full[s], (it / TP_STAGES) & 1) || *abort_flag) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t adesc = umma_desc_sw128(sA + (size_t)kb * TC_TILE_BYTES);
                    const uint64_t bdesc = umma_desc_sw128(sB + (size_t)s * TC_TILE_BYTES);
#pragma unroll
                    for (int k = 0; k < TC_BK / 16; ++k)
                        umma_bf16_pair(tmem + (uint32_t)(b * TP_BN), adesc + (uint64_t)(2 * k),
                                       bdesc + (uint64_t)(2 * k), TP_IDESC, 1u);
                    umma_commit_pair_mc(&b_empty[s], 0x3);
                }
                if (!ok) break;
                umma_commit_pair_mc(&acc_full[b], 0x3);
            }
            if (!ok) {
                atomicMax(a.status, (int)kDevTimeoutFull);
                *abort_flag = 1;
            }
            if (issued_mma) {
                umma_commit_pair(drain);
                if (!mbar_wait(drain, 0)) atomicMax(a.status, (int)kDevTimeoutDrain);
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue (TP_EPI_WARPS warps per CTA) ----------------
        // Warp w: TMEM lane quadrant w % 4 (32 query rows), column range
        // (w - 2) / 4 (TP_COLS of the tile's 256 reference points).
        const int qd = warp & 3;
        const int hc = (warp - 2) >> 2;
        const int qrow = qpair * TC_QT + (int)rank * TC_BM + qd * 32 + lane;
        float thr = -INFINITY;
        if (MODE == 1 && qrow < a.Q) thr = a.thr[qrow];
        float L[TC_KS];
#pragma unroll
        for (int i = 0; i < TC_KS; ++i) L[i] = INFINITY;
        PendingCands pend;
        for (int j = 0; j < n_my; ++j) {
            const int b = j & 1;
            if (MODE == 1) pend.flush(a.count, a.cand, a.cmax, qrow);
            const bool got = mbar_wait(&acc_full[b], (j >> 1) & 1);
            if (__any_sync(0xffffffffu, !got || *abort_flag != 0)) {
                if (lane == 0) {
                    if (!got) atomicMax(a.status, (int)kDevTimeoutFull);
                    *abort_flag = 1;
                }
                break;
            }
            tc_fence_after();
            // the warp's 128 columns in one go; the buffer goes back to the
            // MMA as soon as the values sit in registers
            uint32_t v[TP_CHUNKS][32];
            {
                const uint32_t tb =
                    tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(b * TP_BN + hc * TP_COLS);
#pragma unroll
                for (int c = 0; c < TP_CHUNKS; ++c) tmem_ld32(tb + 32 * c, v[c]);
#pragma unroll
                for (int c = 0; c < TP_CHUNKS; ++c) tmem_ld_wait(v[c]);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                if (lead)
                    mbar_arrive(&acc_empty[b]);
                else
                    mbar_arrive_cluster(mapa_shared(smem_u32(&acc_empty[b]), 0));
            }
            // first reference of this warp
            const int col0 = (a.tile_base + a.tiles.tile(u0 + j)) * TP_BN + hc * TP_COLS;
            const int valid = a.N - col0;
#pragma unroll
            for (int c = 0; c < TP_CHUNKS; ++c) {
                const int cvalid = valid - c * 32;
                if (cvalid < 32) {
#pragma unroll
                    for (int e = 0; e < 32; ++e)
                        if (e >= cvalid) v[c][e] = 0x7f800000u;   // +inf
                }
                const float lim = MODE == 1 ? thr : L[TC_KS - 1];
                if (!(min32(v[c]) < lim)) continue;
                uint32_t m = below_mask(v[c], lim);
                const int cbase = col0 + c * 32;
                while (m) {
                    const int e = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t xb = select32(v[c], e);
                    if (MODE == 1) {
                        pend.push(((unsigned long long)ord_bits(xb) << 32) | (uint32_t)(cbase + e),
                                  a.count, a.cand, a.cmax, qrow);
                    } else {
                        const float x = __uint_as_float(xb);
                        if (x < L[TC_KS - 1]) {
#pragma unroll
                            for (int i = TC_KS - 1; i > 0; --i)
                                L[i] = x < L[i - 1] ? L[i - 1] : (x < L[i] ? x : L[i]);
                            L[0] = fminf(L[0], x);
                        }
                    }
                }
            }
        }
        if (MODE == 1) pend.flush(a.count, a.cand, a.cmax, qrow);
        if (MODE == 0 && !*abort_flag && qrow < a.Q) {
            float *dst = a.p1 + ((size_t)(TP_LISTS * split + hc) * a.Q + qrow) * TC_KS;
#pragma unroll
            for (int i = 0; i < TC_KS; ++i) dst[i] = L[i];
        }
    }

    tc_fence_before();
    __syncthreads();
    cluster_sync();   // no MMA / TMA of the pair touches either CTA after this
    tc_fence_after();
    if (warp == 1) tmem_dealloc_pair(tmem, TC_TMEM_COLS);
}

// ---------------------------------------------------------------------------
// error bound of the BF16 expansion (see the file comment)
// ---------------------------------------------------------------------------
KNN_DI float tc_error_bound(float qq, float r2, float T, int d_pad) {
    const float g = (float)(d_pad + TC_NK) * 2.384185791015625e-07f;   // K * 2^-22
    const float eps = 0.0078125f + 1.52587890625e-05f + g;              // 2^-7 + 2^-16 + g
    return 2.f * eps * sqrtf(qq * r2) + g * (r2 + qq) + 9.5367431640625e-07f * (fabsf(T) + qq);
}

// ---------------------------------------------------------------------------
// prep kernels
// ---------------------------------------------------------------------------

// The norm-step row of point p: h, m, l = successive BF16 roundings of the
// remainder of the squared norm s (each subtraction is exact by Sterbenz'
// lemma, and h + m + l equals s to 2^-27 relative), then 13 zeros.
KNN_DI void write_norm_row(__nv_bfloat16 *parts, int p, float s) {
    __nv_bfloat16 hml[3];
    if (isfinite(s)) {
        float rem = s;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            hml[i] = __float2bfloat16_rn(rem);
            rem = rem - __bfloat162float(hml[i]);
        }
    } else {
        hml[0] = __float2bfloat16_rn(INFINITY);
        hml[1] = hml[2] = __float2bfloat16_rn(0.f);
    }
    uint4 row[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
    __nv_bfloat16 *e = reinterpret_cast<__nv_bfloat16 *>(row);
    e[0] = hml[0];
    e[1] = hml[1];
    e[2] = hml[2];
    uint4 *dst = reinterpret_cast<uint4 *>(parts + (size_t)p * TC_NK);
    dst[0] = row[0];
    dst[1] = row[1];
}

// Squared norm of each point of a dim x n set, translated by -center
// (sequential FP32 fma over d), and optionally the largest squared norm
// (non-negative float bits compare as unsigned).
__global__ void tc_norms_kernel(const float *__restrict__ x, int n, long long ld, int d,
                                const float *__restrict__ center, float *__restrict__ nrm,
                                unsigned *__restrict__ max_bits) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    float s = 0.f;
    if (p < n) {
        for (int dd = 0; dd < d; ++dd) {
            const float v = x[(size_t)dd * ld + p] - center[dd];
            s = fmaf(v, v, s);
        }
        nrm[p] = s;
    }
    unsigned m = __float_as_uint(s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && max_bits) atomicMax(max_bits, m);
}

// dim x n (row pitch ld) FP32 -> n x d_pad BF16 of scale * (x - center)
// (scale a power of two, so bf16(scale y) = scale bf16(y)), zero-padded in
// [d, d_pad).  32 x 32 tiles through shared memory.
__global__ void tc_pack_kernel(const float *__restrict__ x, int n, long long ld, int d,
                               int d_pad, const float *__restrict__ center, float scale,
                               __nv_bfloat16 *__restrict__ xb) {
    __shared__ float tile[32][33];
    const int p0 = blockIdx.x * 32, d0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int dd = d0 + ty + 8 * i, p = p0 + tx;
        tile[ty + 8 * i][tx] = (dd < d && p < n) ? x[(size_t)dd * ld + p] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int p = p0 + ty + 8 * i, dd = d0 + tx;
        if (p < n && dd < d_pad) {
            const float v = dd < d ? tile[tx][ty + 8 * i] - center[dd] : 0.f;
            xb[(size_t)p * d_pad + dd] = __float2bfloat16_rn(v * scale);
        }
    }
}

// The translation c applied to both sets before the BF16 expansion (squared
// distances do not change, but the expansion's error bound scales with the
// norms): the mean of the 256-point tiles of units 0, step, 2 step, ... of
// a tile pattern (n_used of them), one block per dimension, a fixed-order
// reduction.  c = 0 in [d, d_pad).
__global__ void __launch_bounds__(256)
    tc_center_kernel(const float *__restrict__ x, int n, long long ld, int d, TileRuns tiles,
                     int step, int n_used, float *__restrict__ center) {
    __shared__ float part[256];
    __shared__ int cnt[256];
    const int dd = blockIdx.x;
    // thread t sums point t of every sample tile, in four independent chains
    float s4[4] = {0.f, 0.f, 0.f, 0.f};
    int c = 0;
    if (dd < d) {
        const float *row = x + (size_t)dd * ld;
#pragma unroll 4
        for (int t = 0; t < n_used; ++t) {
            const long long p = (long long)tiles.tile(t * step) * TP_BN + threadIdx.x;
            if (p < n) {
                s4[t & 3] += row[p];
                ++c;
            }
        }
    }
    part[threadIdx.x] = (s4[0] + s4[1]) + (s4[2] + s4[3]);
    cnt[threadIdx.x] = c;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            part[threadIdx.x] += part[threadIdx.x + h];
            cnt[threadIdx.x] += cnt[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) center[dd] = cnt[0] > 0 ? part[0] / (float)cnt[0] : 0.f;
}

// Reference-set prep in one pass over the input: point-major BF16 and FP32
// copies (zero-padded to d_pad; the BF16 one of x - center, the FP32 one of
// x itself) plus the norm-step row and the largest squared norm of
// x - center, for the 256-point tiles tile0 + tiles.tile(u) (eight blocks
// per tile).  A block owns 32 points and walks the dimensions in
// 32 x 32 tiles through shared memory (coalesced on both sides); one thread
// per point accumulates the squared norm in increasing d with FP32 fma, the
// order tc_norms_kernel uses.
__global__ void tc_prep_ref_kernel(const float *__restrict__ x, int n, long long ld, int d,
                                   int d_pad, int tile0, TileRuns tiles,
                                   const float *__restrict__ center,
                                   __nv_bfloat16 *__restrict__ xb, float *__restrict__ xt,
                                   __nv_bfloat16 *__restrict__ parts,
                                   unsigned *__restrict__ max_bits) {
    __shared__ float tile[32][33];
    __shared__ float cs[32];   // the chunk's translation
    const int p0 = (tile0 + tiles.tile((int)(blockIdx.x >> 3))) * TP_BN + (blockIdx.x & 7) * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    float s = 0.f;
    // the next chunk's values are loaded into registers while this chunk
    // is processed
    float nx[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int dd = ty + 8 * i, p = p0 + tx;
        nx[i] = (dd < d && p < n) ? x[(size_t)dd * ld + p] : 0.f;
    }
    for (int d0 = 0; d0 < d_pad; d0 += 32) {
#pragma unroll
        for (int i = 0; i < 4; ++i) tile[ty + 8 * i][tx] = nx[i];
        if (ty == 1) cs[tx] = d0 + tx < d ? center[d0 + tx] : 0.f;
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int dd = d0 + 32 + ty + 8 * i, p = p0 + tx;
            nx[i] = (dd < d && p < n) ? x[(size_t)dd * ld + p] : 0.f;
        }
        if (ty == 0) {
            const int dm = min(32, d - d0);
            for (int dd = 0; dd < dm; ++dd) {
                const float v = tile[dd][tx] - cs[dd];
                s = fmaf(v, v, s);
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int p = p0 + ty + 8 * i, dd = d0 + tx;
            if (p < n) {
                const float v = tile[tx][ty + 8 * i];
                xb[(size_t)p * d_pad + dd] = __float2bfloat16_rn(dd < d ? v - cs[tx] : 0.f);
                xt[(size_t)p * d_pad + dd] = v;
            }
        }
        __syncthreads();
    }
    if (ty == 0) {
        const int p = p0 + tx;
        if (p < n) write_norm_row(parts, p, s);
        unsigned m = p < n ? __float_as_uint(s) : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (tx == 0) atomicMax(max_bits, m);
    }
}

// Emission threshold: the KS-th smallest of the per-split pass-1 lists plus
// the error bound E_q (so that the k-th exact distance only has to lie below
// the sample's KS-th approximate one to certify); resets candidate counts.
__global__ void tc_threshold_kernel(const float *__restrict__ p1, int S, int Q,
                                    const float *__restrict__ qn,
                                    const unsigned *__restrict__ rmax_bits, int d_pad,
                                    float *__restrict__ thr, int *__restrict__ count) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    float L[TC_KS];
#pragma unroll
    for (int i = 0; i < TC_KS; ++i) L[i] = INFINITY;
    for (int s = 0; s < S; ++s) {
        const float *src = p1 + ((size_t)s * Q + q) * TC_KS;
        for (int i = 0; i < TC_KS; ++i) {
            const float v = src[i];
            if (!(v < L[TC_KS - 1])) break;   // lists are ascending
#pragma unroll
            for (int t = TC_KS - 1; t > 0; --t)
                L[t] = v < L[t - 1] ? L[t - 1] : (v < L[t] ? v : L[t]);
            L[0] = fminf(L[0], v);
        }
    }
    const float T = L[TC_KS - 1];
    thr[q] = T + tc_error_bound(qn[q], __uint_as_float(*rmax_bits), T, d_pad);
    count[q] = 0;
}

// Ascending bitonic sort of keys[0..P) (P a power of two) by one warp.
KNN_DI void warp_bitonic_sort(unsigned long long *keys, int P, int lane) {
    for (int size = 2; size <= P; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < P / 2; t += 32) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const unsigned long long x = keys[lo], y = keys[hi];
                if ((x > y) == up) {
                    keys[lo] = y;
                    keys[hi] = x;
                }
            }
            __syncwarp();
        }
    }
}

// Exact FP32 re-rank of each query's candidates + certification.
// One warp per query (TC_RR_WARPS queries per block, no block-wide syncs).
//
// Pruning: the candidates are first sorted by their BF16-expansion value a.
// With a_k the k-th smallest, every candidate i of the first k has exact
// FP32 distance <= (a_k + ||q||^2 + E)(1 + gamma), and a candidate r has
// exact FP32 distance >= (a_r + ||q||^2 - E)(1 - gamma) (E as for the
// threshold, gamma the relative rounding of the FP32 distance chain).  A
// candidate whose lower bound exceeds that upper bound has k strictly
// closer candidates and cannot be in the top-k, so only the prefix with
// a_r <= a_k + 2 E + 2 g (|a_k| + ||q||^2 + E) (g = K 2^-22 >= 4 gamma, which
// also absorbs the roundings of this bound) is re-ranked; the k-th exact
// distance of that prefix is the k-th of all candidates.
//
// The prefix is handled 32 candidates at a time, one per lane: the warp
// copies the 32 candidate rows of the FP32 point-major copy, TC_RR_DCH
// dimensions at a time, into a padded shared tile with asynchronous 16-byte
// copies (cp.async, several rows per instruction, coalesced), through a ring
// of TC_RR_NBUF buffers so the next chunks are in flight while each lane
// runs its candidate's FMA chain in increasing d -- the fused exact kernel's
// arithmetic and order, so distances are identical.  The (distance, index)
// keys are bitonic-sorted by the warp.  One warp per block: the gather is
// latency-bound, and single-warp blocks let the SM hold as many warps as
// its shared memory allows (about 14 at d = 256).
//
// An uncertified query is appended to fail_list and retry[q] receives a
// threshold for a second scan: when it had at least k candidates, their k-th
// exact distance D_k bounds the true k-th from above, so every point of the
// true top-k has a < D_k (1+g) + E - ||q||^2 and a second scan emitting below
// D_k (1+g) + 2.5 E - ||q||^2 passes the check; with fewer than k candidates
// the threshold is widened by 8 E; an overflowing list keeps its threshold
// for a second scan with a longer list (final_pass = 0) or gets NaN (exact
// kernel).
constexpr int TC_RR_WARPS = 1;
constexpr int TC_RR_DCH = 32;                 // dimensions per staged chunk
constexpr int TC_RR_NBUF = 2;                 // staging buffers per warp (ring)
// padded row (floats): 16-byte aligned, and 16-byte reads of one row per lane
// fall in distinct bank groups for every 8 consecutive lanes
constexpr int TC_RR_STRIDE = TC_RR_DCH + 4;
constexpr int TC_RR_BUF = 32 * TC_RR_STRIDE;  // floats per staging buffer

__host__ __device__ inline size_t tc_rr_warp_bytes(int d_pad, int cpow) {
    return (size_t)d_pad * 4 + TC_RR_NBUF * TC_RR_BUF * 4 + (size_t)cpow * 8;
}

KNN_DI void cp_async16(void *smem_dst, const void *gmem_src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)),
                 "l"(gmem_src)
                 : "memory");
}
KNN_DI void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
KNN_DI void cp_async_wait_n() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// A candidate list that cannot be re-ranked -- more entries than it holds
// (overflow) or fewer than k: the query joins fail_list with the threshold
// of a second scan.  Too few candidates mean the threshold was low, so it is
// widened by 8 E; an overflowing list is scanned again with the same
// threshold and a longer list, and overflowing that too (final_pass) it
// goes to the exact kernel (NaN).  Warp-uniform; true if rejected.
KNN_DI bool rr_reject_list(int c, int cmax, int k, int q, float qq, float r2, float T, int d_pad,
                           int final_pass, int *fail_list, int *n_fail, float *retry, int lane) {
    if (c <= cmax && c >= k) return false;
    if (lane == 0) {
        fail_list[atomicAdd(n_fail, 1)] = q;
        retry[q] = c < k ? T + 8.f * tc_error_bound(qq, r2, T, d_pad)
                         : (final_pass ? __int_as_float(0x7fc00000) : T);
    }
    return true;
}

// Exact FP32 distances of the candidates keys[0..n) (point index in the low
// 32 bits), in place: keys[t] = (distance, index).  One warp, 32 candidates
// at a time, one per lane: the rows of the FP32 point-major copy are staged
// TC_RR_DCH dimensions at a time through the TC_RR_NBUF buffers `rows`
// (steps s = (group, chunk); the copies of steps s + 1 .. s + NBUF - 1
// overlap step s), and each lane runs its candidate's FMA chain against the
// query qv (d_pad floats) in increasing d.
//
// Bound check (STAT, a test-only instantiation): before a key is replaced,
// its entry still holds the BF16-expansion value a of that candidate; the
// lane records |a + ||q||^2 - D| / E_q (D the exact FP32 distance, qq =
// ||q||^2, E_q = e_q) as float bits in stat[0] (atomic max) and counts the
// candidates checked in the 64-bit counter at stat + 2.
struct BoundStat {
    float qq, e_q;
    unsigned *stat;
};

template <bool STAT = false>
KNN_DI void rr_exact_distances(unsigned long long *keys, int n, const float *__restrict__ refT,
                               int d_pad, const float *qv, float *rows, int lane,
                               BoundStat bs = BoundStat{0.f, 0.f, nullptr}) {
    const int nch = d_pad / TC_RR_DCH;
    const int total = ((n + 31) / 32) * nch;
    constexpr int CPL = TC_RR_DCH / 4;   // 16-byte copies per row and chunk
    constexpr int RPI = 32 / CPL;        // rows per copy instruction
    auto issue = [&](int buf, int rr, int ch) {
        float *dstb = rows + buf * TC_RR_BUF;
#pragma unroll
        for (int i = 0; i < 32 / RPI; ++i) {
            const int row = RPI * i + lane / CPL;
            const int r = __shfl_sync(0xffffffffu, rr, row);
            if (r >= 0)
                cp_async16(dstb + row * TC_RR_STRIDE + (lane % CPL) * 4,
                           refT + (size_t)r * d_pad + ch + (lane % CPL) * 4);
        }
    };
    auto row_of = [&](int grp) {
        const int t = grp * 32 + lane;
        return t < n ? (int)(uint32_t)keys[t] : -1;
    };
#pragma unroll
    for (int s = 0; s < TC_RR_NBUF - 1; ++s) {
        if (s < total) issue(s, row_of(s / nch), (s % nch) * TC_RR_DCH);
        cp_async_commit();
    }
    float acc = 0.f;
    int r_cur = -1;
    for (int s = 0; s < total; ++s) {
        const int g = s / nch, ch = s - g * nch;
        if (ch == 0) r_cur = row_of(g);
        const int s1 = s + TC_RR_NBUF - 1;
        if (s1 < total) issue(s1 % TC_RR_NBUF, row_of(s1 / nch), (s1 % nch) * TC_RR_DCH);
        cp_async_commit();
        cp_async_wait_n<TC_RR_NBUF - 1>();   // step s's copies have landed
        __syncwarp();
        const float4 *myrow = reinterpret_cast<const float4 *>(
            rows + (s % TC_RR_NBUF) * TC_RR_BUF + lane * TC_RR_STRIDE);
        const float4 *qc = reinterpret_cast<const float4 *>(qv + ch * TC_RR_DCH);
#pragma unroll
        for (int j = 0; j < TC_RR_DCH / 4; ++j) {
            const float4 rv = myrow[j], qq4 = qc[j];
            float t0 = __fsub_rn(rv.x, qq4.x);
            acc = __fmaf_rn(t0, t0, acc);
            t0 = __fsub_rn(rv.y, qq4.y);
            acc = __fmaf_rn(t0, t0, acc);
            t0 = __fsub_rn(rv.z, qq4.z);
            acc = __fmaf_rn(t0, t0, acc);
            t0 = __fsub_rn(rv.w, qq4.w);
            acc = __fmaf_rn(t0, t0, acc);
        }
        __syncwarp();   // this buffer is refilled NBUF - 1 steps later
        if (ch == nch - 1) {
            const int t = g * 32 + lane;
            if (STAT && t < n) {
                const float a = ord_float((uint32_t)(keys[t] >> 32));
                const float ratio = fabsf(a + bs.qq - acc) / bs.e_q;
                atomicMax(bs.stat, __float_as_uint(ratio));
                atomicAdd(reinterpret_cast<unsigned long long *>(bs.stat + 2), 1ull);
            }
            if (t < n) keys[t] = make_key(acc, (uint32_t)r_cur);
            acc = 0.f;
        }
    }
}

// Certification from a query's k smallest exact keys (sorted; keys[k - 1]
// the k-th): certified, the query's sqrt distances and indices are written;
// otherwise it joins fail_list with the threshold of a second scan that
// certifies (see tc_rerank_kernel).  Warp-uniform.
KNN_DI void rr_certify(const unsigned long long *keys, int q, float qq, float r2, float T,
                       int d_pad, int k, float *__restrict__ out_dist, int *__restrict__ out_idx,
                       long long ld_out, int *fail_list, int *n_fail, float *retry, int lane) {
    int failed = 0;
    if (lane == 0) {
        const float dk = key_dist2(keys[k - 1]);
        const float E = tc_error_bound(qq, r2, T, d_pad);
        const float dkg = dk * (1.f + (float)d_pad * 2.384185791015625e-07f);
        failed = !(dkg + E < T + qq);
        if (failed) {
            fail_list[atomicAdd(n_fail, 1)] = q;
            const float T2 = dkg - qq;
            retry[q] = T2 + 2.5f * tc_error_bound(qq, r2, T2, d_pad);
        }
    }
    if (__shfl_sync(0xffffffffu, failed, 0)) return;
    for (int j = lane; j < k; j += 32) {
        const unsigned long long key = keys[j];
        out_dist[(size_t)j * ld_out + q] = sqrtf(key_dist2(key));
        out_idx[(size_t)j * ld_out + q] = key_index(key);
    }
}

template <bool STAT>
__global__ void __launch_bounds__(TC_RR_WARPS * 32)
    tc_rerank_kernel(const float *__restrict__ refT, int d, int d_pad,
                     const float *__restrict__ qry, long long ldq, const float *__restrict__ qn,
                     const unsigned *__restrict__ rmax_bits, const float *__restrict__ thr,
                     const unsigned long long *__restrict__ cand, const int *__restrict__ count,
                     int cmax, int cpow, int Q, int k, float *__restrict__ out_dist,
                     int *__restrict__ out_idx, long long ld_out, int *__restrict__ fail_list,
                     int *__restrict__ n_fail, float *__restrict__ retry,
                     unsigned long long *__restrict__ cand_total, int final_pass,
                     unsigned *__restrict__ bound_stat) {
    extern __shared__ unsigned char rsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * (blockDim.x >> 5) + warp;
    if (q >= Q) return;
    unsigned char *mine = rsm + (size_t)warp * tc_rr_warp_bytes(d_pad, cpow);
    float *qv = reinterpret_cast<float *>(mine);
    float *rows = qv + d_pad;   // two staging buffers
    unsigned long long *keys = reinterpret_cast<unsigned long long *>(rows + TC_RR_NBUF * TC_RR_BUF);

    const int c = count[q];
    if (lane == 0) atomicAdd(cand_total, (unsigned long long)c);
    const float qq = qn[q];
    const float r2 = __uint_as_float(*rmax_bits);
    const float T = thr[q];
    if (rr_reject_list(c, cmax, k, q, qq, r2, T, d_pad, final_pass, fail_list, n_fail, retry,
                       lane))
        return;
    // candidates sorted by (a, index)
    const unsigned long long *cq = cand + (size_t)q * cmax;
    int P = 32;
    while (P < c) P <<= 1;
    for (int t = lane; t < P; t += 32) keys[t] = t < c ? cq[t] : ~0ull;
    for (int dd = lane; dd < d_pad; dd += 32) qv[dd] = dd < d ? qry[(size_t)dd * ldq + q] : 0.f;
    __syncwarp();
    warp_bitonic_sort(keys, P, lane);
    // the prefix that can still reach the top-k
    int n_s;
    {
        const float ak = ord_float((uint32_t)(keys[k - 1] >> 32));
        const float E = tc_error_bound(qq, r2, ak, d_pad);
        const float g = (float)(d_pad + TC_NK) * 2.384185791015625e-07f;
        const float lim = ak + 2.f * E + 2.f * g * (fabsf(ak) + qq + E);
        const uint32_t lim_o = ord_bits(__float_as_uint(lim));
        int cnt = 0;
        for (int t0 = 0; t0 < c; t0 += 32) {
            const int t = t0 + lane;
            const bool in = t < c && (uint32_t)(keys[t] >> 32) <= lim_o;
            cnt += __popc(__ballot_sync(0xffffffffu, in));
        }
        n_s = max(cnt, k);   // keys are sorted, so the kept ones are a prefix
    }
    rr_exact_distances<STAT>(keys, n_s, refT, d_pad, qv, rows, lane,
                             BoundStat{qq, tc_error_bound(qq, r2, T, d_pad), bound_stat});
    int P2 = 32;
    while (P2 < n_s) P2 <<= 1;
    for (int t = n_s + lane; t < P2; t += 32) keys[t] = kKeyInf;
    __syncwarp();
    warp_bitonic_sort(keys, P2, lane);
    rr_certify(keys, q, qq, r2, T, d_pad, k, out_dist, out_idx, ld_out, fail_list, n_fail, retry,
               lane);
}

// Incremental re-rank for a reference set that arrives in pieces (the
// streamed host entry).  After each piece's scan, the candidates a query
// gained since the last call (list entries done[q] .. min(count, cmax)) get
// their exact FP32 distances and are merged into its running k smallest
// keys run[q][0..k) (a sort of the new keys, then every key placed at its
// index plus its rank in the other array).  Nothing is pruned -- the k-th a
// is not known yet -- so about twice the rows of tc_rerank_kernel are
// gathered, while the rest of the set is still being copied in.  After the
// last piece run[q] holds the k smallest exact keys of all candidates: the
// certification and the output are those of tc_rerank_kernel.  One warp
// (block) per query.
template <int KCAP>
__global__ void __launch_bounds__(32)
    tc_rerank_piece_kernel(const float *__restrict__ refT, int d, int d_pad,
                           const float *__restrict__ qry, long long ldq,
                           const unsigned long long *__restrict__ cand,
                           const int *__restrict__ count, int cmax, int k,
                           unsigned long long *__restrict__ run, int *__restrict__ done) {
    extern __shared__ unsigned char rsm[];
    const int q = blockIdx.x, lane = threadIdx.x;
    const int c = min(count[q], cmax);
    const int s0 = done[q];
    if (s0 >= c) return;
    float *qv = reinterpret_cast<float *>(rsm);
    float *rows = qv + d_pad;
    unsigned long long *L = reinterpret_cast<unsigned long long *>(rows + TC_RR_NBUF * TC_RR_BUF);
    unsigned long long *C = L + KCAP;   // warp_merge's candidate slots (EX_CB)
    for (int dd = lane; dd < d_pad; dd += 32) qv[dd] = dd < d ? qry[(size_t)dd * ldq + q] : 0.f;
    for (int t = lane; t < KCAP; t += 32) L[t] = t < k ? run[(size_t)q * k + t] : kKeyInf;
    __syncwarp();
    const unsigned long long *cq = cand + (size_t)q * cmax;
    for (int b0 = s0; b0 < c; b0 += EX_CB) {
        const int n = min(EX_CB, c - b0);
        for (int t = lane; t < n; t += 32) C[t] = cq[b0 + t];
        __syncwarp();
        rr_exact_distances(C, n, refT, d_pad, qv, rows, lane);
        __syncwarp();
        warp_merge<KCAP>(L, n, k, lane);
    }
    for (int t = lane; t < k; t += 32) run[(size_t)q * k + t] = L[t];
    if (lane == 0) done[q] = c;
}

// Certification after the last piece: tc_rerank_kernel's first-pass checks
// on the running k smallest keys of tc_rerank_piece_kernel.  One warp per
// query.
__global__ void tc_certify_pieces_kernel(const int *__restrict__ count, int cmax,
                                         const float *__restrict__ qn,
                                         const unsigned *__restrict__ rmax_bits,
                                         const float *__restrict__ thr,
                                         const unsigned long long *__restrict__ run, int Q, int k,
                                         int d_pad, float *__restrict__ out_dist,
                                         int *__restrict__ out_idx, long long ld_out,
                                         int *__restrict__ fail_list, int *__restrict__ n_fail,
                                         float *__restrict__ retry,
                                         unsigned long long *__restrict__ cand_total) {
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (q >= Q) return;
    const int c = count[q];
    if (lane == 0) atomicAdd(cand_total, (unsigned long long)c);
    const float qq = qn[q];
    const float r2 = __uint_as_float(*rmax_bits);
    const float T = thr[q];
    if (rr_reject_list(c, cmax, k, q, qq, r2, T, d_pad, 0, fail_list, n_fail, retry, lane)) return;
    rr_certify(run + (size_t)q * k, q, qq, r2, T, d_pad, k, out_dist, out_idx, ld_out, fail_list,
               n_fail, retry, lane);
}

// Fallback plumbing: gather the uncertified queries into a dense d x m set
// and scatter the exact results back.
__global__ void gather_queries_kernel(const float *__restrict__ qry, long long ldq, int d,
                                      const int *__restrict__ list, int m, float *__restrict__ dst,
                                      long long ldd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int dd = blockIdx.y;
    if (i < m) dst[(size_t)dd * ldd + i] = qry[(size_t)dd * ldq + list[i]];
}

__global__ void scatter_results_kernel(const float *__restrict__ sd, const int *__restrict__ si,
                                       long long lds, const int *__restrict__ list, int m,
                                       float *__restrict__ out_dist, int *__restrict__ out_idx,
                                       long long ld_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i < m) {
        out_dist[(size_t)j * ld_out + list[i]] = sd[(size_t)j * lds + i];
        out_idx[(size_t)j * ld_out + list[i]] = si[(size_t)j * lds + i];
    }
}

// Second-chance scan of the uncertified queries: compact thresholds.
__global__ void tc_retry_prep_kernel(const int *__restrict__ list, int m,
                                     const float *__restrict__ retry, float *__restrict__ thr,
                                     int *__restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        thr[i] = retry[list[i]];
        count[i] = 0;
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

bool encode_bf16_kmajor(CUtensorMap *m, const void *base, int rows, int d_pad) {
    return encode_2d(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, (uint64_t)d_pad,
                     (uint64_t)rows, (uint64_t)d_pad, TC_BK, TC_BM, CU_TENSOR_MAP_SWIZZLE_128B);
}

// Norm-step rows [rows][16] BF16, 128-row boxes with the 32-byte swizzle.
bool encode_norm_rows(CUtensorMap *m, const void *base, int rows) {
    return encode_2d(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, (uint64_t)TC_NK, (uint64_t)rows,
                     (uint64_t)TC_NK, TC_NK, TC_BM, CU_TENSOR_MAP_SWIZZLE_32B);
}

// Candidate lists: first scan cmax = 4 * KS * stride (<= 1280 for k <=
// 128); the second scan of the queries whose list overflowed reuses the
// whole list buffer, up to kTcCmaxRetry entries per query.  The re-rank
// kernel's shared memory (keys padded to a power of two) is capped at
// kRerankSmem per block: fewer warps per block for long lists.
constexpr int kTcCmaxRetry = 8192;
constexpr size_t kRerankSmem = 200 * 1024;

struct TcPlan {
    int d_pad, kb, qtiles, cmax;
    int n_tiles2, splits1;   // 256-point tiles; pass-1 splits over CTA pairs
    TileRuns sample;         // pass-1 tiles
};

// Splits that fill whole waves of one CTA per SM for `tiles` tiles per
// query tile, with at least min_tiles per CTA; modelled per-CTA cost =
// tiles per split + a fixed set-up cost of `fixed` tiles.
static int choose_splits(int qtiles, int tiles, int min_tiles, double fixed, int num_sms) {
    int best = 1;
    double best_t = 1e300;
    const int max_s = std::max(1, std::min(256, tiles / std::max(1, min_tiles)));
    for (int S = 1; S <= max_s; ++S) {
        const long long ctas = (long long)qtiles * S;
        const double t = (double)((ctas + num_sms - 1) / num_sms) * ((double)tiles / S + fixed);
        if (t < best_t * 0.999) {
            best_t = t;
            best = S;
        }
    }
    return best;
}

TcPlan plan_tc(int N, int Q, int d, int k, int num_sms) {
    TcPlan p;
    p.d_pad = (d + 63) / 64 * 64;
    p.kb = p.d_pad / 64;
    p.qtiles = (Q + TC_QT - 1) / TC_QT;
    // pass 1 samples one tile in `stride`: the sample must hold about 2.5k
    // points below T_q, KS * stride >= 2.5k
    const int stride = std::max(16, (5 * k + 2 * TC_KS - 1) / (2 * TC_KS));
    p.cmax = 4 * TC_KS * stride;
    p.n_tiles2 = (N + TP_BN - 1) / TP_BN;
    // in runs of up to 16 consecutive tiles (one every stride tiles when
    // the set is small), at least 32 runs across the set
    const int run = std::max(1, std::min(16, p.n_tiles2 / (32 * stride)));
    p.sample.run = run;
    p.sample.period = run * stride;
    p.sample.units = p.sample.count_below(p.n_tiles2);
    // coarser pass-1 splits amortise each pair's set-up (query tile load,
    // TMEM allocation, pipeline fill)
    p.splits1 = choose_splits(p.qtiles, p.sample.units, 16, 8.0, std::max(1, num_sms / 2));
    return p;
}

struct Carve {
    unsigned char *p;
    size_t used, cap;
    template <typename T>
    T *take(size_t count) {
        used = (used + 255) & ~size_t(255);
        T *r = reinterpret_cast<T *>(p + used);
        used += count * sizeof(T);
        return r;
    }
};

}  // namespace

bool tc_supported(int N, int Q, int d, int k) {
    return d >= 16 && d <= TC_KBMAX * TC_BK && k >= 1 && k <= 128 && N >= 32768 && Q >= 1;
}

size_t tc_ref_bytes(int N, int d) {
    const int d_pad = (d + 63) / 64 * 64;
    return (size_t)N * d_pad * 2 + (size_t)N * d_pad * 4 + (size_t)N * TC_NK * 2 +
           (size_t)d_pad * 4 + 5 * 256;
}

static size_t fallback_bytes(int N, int Q, int d, int k, int num_sms) {
    const long long ldf = (Q + 3) / 4 * 4;
    return (size_t)d * ldf * 4 + (size_t)k * ldf * 8 + exact_scratch_bytes(N, Q, d, k, num_sms) +
           4 * 256;
}

size_t tc_scratch_bytes(int N, int Q, int d, int k, int num_sms) {
    const TcPlan p = plan_tc(N, Q, d, k, num_sms);
    size_t b = (size_t)p.qtiles * TC_QT * p.d_pad * 2 + (size_t)Q * 4 * 6 + 16;
    b += (size_t)TP_LISTS * p.splits1 * Q * TC_KS * 4;
    b += (size_t)Q * p.cmax * 8;
    b += fallback_bytes(N, Q, d, k, num_sms);   // worst case: every query uncertified
    return b + 16 * 256;
}

int tc_prepare_ref(const TcRefView &v, const float *ref, int N, long long ldr, int d,
                   cudaStream_t st) {
    if (cudaMemsetAsync(v.rmax_bits, 0, sizeof(unsigned), st) != cudaSuccess) return kErrCuda;
    const int n_tiles = (N + TP_BN - 1) / TP_BN;
    const int rc = tc_center_from_tiles(v, ref, N, ldr, d, contiguous_tiles(n_tiles),
                                        kCenterStride, st);
    return rc != kOk ? rc
                     : tc_prepare_ref_tiles(v, ref, N, ldr, d, 0, contiguous_tiles(n_tiles), st);
}

int tc_center_from_tiles(const TcRefView &v, const float *ref, int N, long long ldr, int d,
                         const TileRuns &tiles, int step, cudaStream_t st) {
    if (step < 1 || tiles.run < 1 || tiles.period < tiles.run) return kErrInvalid;
    const int d_pad = (d + 63) / 64 * 64;
    const int n_used = (tiles.units + step - 1) / step;
    tc_center_kernel<<<d_pad, 256, 0, st>>>(ref, N, ldr, d, tiles, step, n_used, v.center);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrLaunch;
}

int tc_prepare_ref_tiles(const TcRefView &v, const float *ref, int N, long long ldr, int d,
                         int tile0, const TileRuns &tiles, cudaStream_t st) {
    if (tiles.units <= 0) return kOk;
    if (tiles.run < 1 || tiles.period < tiles.run) return kErrInvalid;
    const int d_pad = (d + 63) / 64 * 64;
    tc_prep_ref_kernel<<<tiles.units * 8, dim3(32, 8), 0, st>>>(ref, N, ldr, d, d_pad, tile0,
                                                                tiles, v.center, v.refB, v.refT,
                                                                v.refN, v.rmax_bits);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrLaunch;
}

int tc_tile_points() { return TP_BN; }

TcRefView tc_carve_ref(void *mem, int N, int d) {
    const int d_pad = (d + 63) / 64 * 64;
    Carve cv{static_cast<unsigned char *>(mem), 0, 0};
    TcRefView v;
    v.refB = cv.take<__nv_bfloat16>((size_t)N * d_pad);
    v.refT = cv.take<float>((size_t)N * d_pad);
    v.refN = cv.take<__nv_bfloat16>((size_t)N * TC_NK);
    v.rmax_bits = cv.take<unsigned>(1);
    v.center = cv.take<float>(d_pad);
    return v;
}

namespace {

// Emission scan of the reference tiles [tb, te) (256-point tiles) for the Q
// queries whose BF16 copy is qB, lists of stride cmax.
int emit_scan(const TcRun &r, cudaStream_t st, const __nv_bfloat16 *qB, int Q, const float *thr,
              int cmax, int tb, int te) {
    const TcProblem &P = r.P;
    CUtensorMap tmA, tmB, tmN;
    if (!encode_bf16_kmajor(&tmA, qB, Q, r.d_pad)) return kErrTensorMap;
    if (!encode_bf16_kmajor(&tmB, r.R.refB, P.N, r.d_pad)) return kErrTensorMap;
    if (!encode_norm_rows(&tmN, r.R.refN, P.N)) return kErrTensorMap;
    const int qtiles = (Q + TC_QT - 1) / TC_QT;
    TpArgs a;
    a.N = P.N;
    a.Q = Q;
    a.kb_count = r.kb;
    a.tile_base = tb;
    a.tiles = contiguous_tiles(te - tb);
    a.n_splits = choose_splits(qtiles, te - tb, 8, 2.0, std::max(1, P.num_sms / 2));
    a.thr = thr;
    a.p1 = nullptr;
    a.cand = r.cand;
    a.count = r.count;
    a.cmax = cmax;
    a.status = P.status;
    knn_tc_pair_scan_kernel<1><<<dim3(2 * qtiles, a.n_splits), TP_THREADS, TP_SMEM, st>>>(
        tmA, tmB, tmN, a);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrLaunch;
}

// Exact re-rank + certification of Q queries (see tc_rerank_kernel) whose
// candidate lists have stride cmax.
int rerank(const TcRun &r, cudaStream_t st, int Q, int cmax, const float *qry, long long ldq,
           const float *qn, const float *thr, float *out_dist, int *out_idx, long long ld_out,
           int *fail, bool final_pass) {
    const TcProblem &P = r.P;
    if (cudaMemsetAsync(r.nfail, 0, sizeof(int), st) != cudaSuccess) return kErrCuda;
    int cpow = 1;
    while (cpow < cmax) cpow <<= 1;
    int warps = TC_RR_WARPS;
    while (warps > 1 && (size_t)warps * tc_rr_warp_bytes(r.d_pad, cpow) > kRerankSmem) warps >>= 1;
    const size_t rsmem = (size_t)warps * tc_rr_warp_bytes(r.d_pad, cpow);
    // one fixed limit for every launch, so that calls from several host
    // threads never lower it under each other
    // the bound statistic runs in its own instantiation, only when asked for
    auto kern = P.bound_stat ? tc_rerank_kernel<true> : tc_rerank_kernel<false>;
    if (rsmem > kRerankSmem ||
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kRerankSmem) != cudaSuccess)
        return kErrLaunch;
    kern<<<(Q + warps - 1) / warps, warps * 32, rsmem, st>>>(
        r.R.refT, P.d, r.d_pad, qry, ldq, qn, r.R.rmax_bits, thr, r.cand, r.count, cmax, cpow,
        Q, P.k, out_dist, out_idx, ld_out, fail, r.nfail, r.retry, r.cand_total,
        final_pass ? 1 : 0, P.bound_stat);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrLaunch;
}

int read_count(const int *dev, int *host_pinned, cudaStream_t st, int &out) {
    if (cudaMemcpyAsync(host_pinned, dev, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return kErrCuda;
    out = *host_pinned;
    return kOk;
}

}  // namespace

TileRuns tc_sample_runs(int N, int Q, int d, int k, int num_sms) {
    return plan_tc(N, Q, d, k, num_sms).sample;
}

int tc_run_begin(const TcProblem &P, const TcRefView &R, cudaStream_t st, TcRun &r) {
    if (!tc_supported(P.N, P.Q, P.d, P.k)) return kErrUnsupported;
    const TcPlan p = plan_tc(P.N, P.Q, P.d, P.k, P.num_sms);
    r.P = P;
    r.R = R;
    r.d_pad = p.d_pad;
    r.kb = p.kb;
    r.qtiles = p.qtiles;
    r.n_tiles2 = p.n_tiles2;
    r.splits1 = p.splits1;
    r.sample = p.sample;
    r.cmax = p.cmax;
    Carve cv{static_cast<unsigned char *>(P.scratch), 0, P.scratch_bytes};
    r.qB = cv.take<__nv_bfloat16>((size_t)p.qtiles * TC_QT * p.d_pad);
    r.qn = cv.take<float>(P.Q);
    r.thr = cv.take<float>(P.Q);
    r.retry = cv.take<float>(P.Q);
    r.count = cv.take<int>(P.Q);
    r.fail = cv.take<int>(P.Q);
    r.fail2 = cv.take<int>(P.Q);
    r.nfail = cv.take<int>(4);
    r.cand_total = cv.take<unsigned long long>(1);
    r.p1 = cv.take<float>((size_t)TP_LISTS * p.splits1 * P.Q * TC_KS);
    r.cand = cv.take<unsigned long long>((size_t)P.Q * p.cmax);
    r.ldf = (P.Q + 3) / 4 * 4;   // second-chance buffers, sized for all queries
    r.qsub = cv.take<float>((size_t)P.d * r.ldf);
    r.sd = cv.take<float>((size_t)P.k * r.ldf);
    r.si = cv.take<int>((size_t)P.k * r.ldf);
    r.xs = cv.take<unsigned char>(0);
    if (cv.used > P.scratch_bytes) return kErrScratch;
    r.xcap = P.scratch_bytes - cv.used;
    r.pieces = false;
    r.run_keys = nullptr;
    r.done = nullptr;

    // queries: norms + BF16 K-major copy of -2 q
    tc_norms_kernel<<<(P.Q + 255) / 256, 256, 0, st>>>(P.qry, P.Q, P.ldq, P.d, R.center, r.qn,
                                                       nullptr);
    tc_pack_kernel<<<dim3((P.Q + 31) / 32, p.d_pad / 32), dim3(32, 8), 0, st>>>(
        P.qry, P.Q, P.ldq, P.d, p.d_pad, R.center, -2.0f, r.qB);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    if (P.timer) P.timer->mark(st, kPhaseTcPrepQuery);
    if (cudaFuncSetAttribute(knn_tc_pair_scan_kernel<0>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TP_SMEM) != cudaSuccess ||
        cudaFuncSetAttribute(knn_tc_pair_scan_kernel<1>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TP_SMEM) != cudaSuccess)
        return kErrLaunch;
    if (cudaMemsetAsync(r.cand_total, 0, sizeof(unsigned long long), st) != cudaSuccess)
        return kErrCuda;
    return kOk;
}

int tc_run_pass1(TcRun &r, cudaStream_t st) {
    const TcProblem &P = r.P;
    CUtensorMap tmA, tmB, tmN;
    if (!encode_bf16_kmajor(&tmA, r.qB, P.Q, r.d_pad)) return kErrTensorMap;
    if (!encode_bf16_kmajor(&tmB, r.R.refB, P.N, r.d_pad)) return kErrTensorMap;
    if (!encode_norm_rows(&tmN, r.R.refN, P.N)) return kErrTensorMap;
    TpArgs a;
    a.N = P.N;
    a.Q = P.Q;
    a.kb_count = r.kb;
    a.tile_base = 0;
    a.tiles = r.sample;
    a.n_splits = r.splits1;
    a.thr = nullptr;
    a.p1 = r.p1;
    a.cand = r.cand;
    a.count = r.count;
    a.cmax = r.cmax;
    a.status = P.status;
    knn_tc_pair_scan_kernel<0><<<dim3(2 * r.qtiles, r.splits1), TP_THREADS, TP_SMEM, st>>>(
        tmA, tmB, tmN, a);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    if (P.timer) P.timer->mark(st, kPhaseTcPass1);
    // TP_LISTS lists (column ranges) per pair and split; resets the counts
    tc_threshold_kernel<<<(P.Q + 255) / 256, 256, 0, st>>>(r.p1, TP_LISTS * r.splits1, P.Q, r.qn,
                                                           r.R.rmax_bits, r.d_pad, r.thr,
                                                           r.count);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    if (P.timer) P.timer->mark(st, kPhaseTcThreshold);
    return kOk;
}

int tc_run_pass2(TcRun &r, int tile_begin, int tile_end, cudaStream_t st) {
    tile_end = std::min(tile_end, r.n_tiles2);
    if (tile_begin >= tile_end) return kOk;
    const int rc = emit_scan(r, st, r.qB, r.P.Q, r.thr, r.cmax, tile_begin, tile_end);
    if (rc == kOk && r.P.timer) r.P.timer->mark(st, kPhaseTcPass2);
    return rc;
}

int tc_run_rerank_piece(TcRun &r, cudaStream_t st) {
    const TcProblem &P = r.P;
    if (!r.pieces) {
        // the running lists take the exact-fallback scratch, which nothing
        // uses before the certification; without room the full re-rank
        // runs in tc_run_finish instead
        Carve cv{r.xs, 0, r.xcap};
        unsigned long long *keys = cv.take<unsigned long long>((size_t)P.Q * P.k);
        int *done = cv.take<int>(P.Q);
        if (cv.used > r.xcap) return kOk;
        if (cudaMemsetAsync(keys, 0xff, (size_t)P.Q * P.k * 8, st) != cudaSuccess ||
            cudaMemsetAsync(done, 0, (size_t)P.Q * 4, st) != cudaSuccess)
            return kErrCuda;
        r.run_keys = keys;
        r.done = done;
        r.pieces = true;
    }
    const int kcap = P.k <= 32 ? 32 : (P.k <= 64 ? 64 : 128);
    const size_t smem = (size_t)r.d_pad * 4 + (size_t)TC_RR_NBUF * TC_RR_BUF * 4 +
                        (size_t)(kcap + EX_CB) * 8;   // < 48 KB for d_pad <= 256
    auto go = [&](auto kern) {
        kern<<<P.Q, 32, smem, st>>>(r.R.refT, P.d, r.d_pad, P.qry, P.ldq, r.cand, r.count, r.cmax,
                                    P.k, r.run_keys, r.done);
    };
    if (kcap == 32)
        go(tc_rerank_piece_kernel<32>);
    else if (kcap == 64)
        go(tc_rerank_piece_kernel<64>);
    else
        go(tc_rerank_piece_kernel<128>);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrLaunch;
}

int tc_run_finish(TcRun &r, cudaStream_t st, int *host_stats) {
    const TcProblem &P = r.P;
    PhaseTimer *tm = P.timer;
    int *host_tmp = host_stats + 2;
    host_stats[0] = host_stats[1] = 0;
    host_stats[4] = host_stats[5] = 0;
    int rc = kOk;
    if (r.pieces) {
        // every candidate was re-ranked piece by piece: certify
        if (cudaMemsetAsync(r.nfail, 0, sizeof(int), st) != cudaSuccess) return kErrCuda;
        constexpr int W = 4;
        tc_certify_pieces_kernel<<<(P.Q + W - 1) / W, W * 32, 0, st>>>(
            r.count, r.cmax, r.qn, r.R.rmax_bits, r.thr, r.run_keys, P.Q, P.k, r.d_pad,
            P.out_dist, P.out_idx, P.ld_out, r.fail, r.nfail, r.retry, r.cand_total);
        if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    } else {
        rc = rerank(r, st, P.Q, r.cmax, P.qry, P.ldq, r.qn, r.thr, P.out_dist, P.out_idx,
                    P.ld_out, r.fail, false);
    }
    if (rc != kOk) return rc;
    if (tm) tm->mark(st, kPhaseTcRerank);
    int nf = 0;
    if (cudaMemcpyAsync(host_stats + 4, r.cand_total, sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return kErrCuda;
    if ((rc = read_count(r.nfail, host_tmp, st, nf)) != kOk) return rc;
    host_stats[0] = nf;
    if (nf == 0) return kOk;

    // second chance: the uncertified queries, compacted, scanned again with
    // thresholds that certify (list overflows excepted)
    gather_queries_kernel<<<dim3((nf + 127) / 128, P.d), 128, 0, st>>>(P.qry, P.ldq, P.d, r.fail,
                                                                       nf, r.qsub, r.ldf);
    tc_norms_kernel<<<(nf + 255) / 256, 256, 0, st>>>(r.qsub, nf, r.ldf, P.d, r.R.center, r.qn,
                                                      nullptr);
    tc_pack_kernel<<<dim3((nf + 31) / 32, r.d_pad / 32), dim3(32, 8), 0, st>>>(
        r.qsub, nf, r.ldf, P.d, r.d_pad, r.R.center, -2.0f, r.qB);
    tc_retry_prep_kernel<<<(nf + 255) / 256, 256, 0, st>>>(r.fail, nf, r.retry, r.thr, r.count);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    // the compacted queries share the whole list buffer (Q * cmax entries)
    const int cmax2 = (int)std::min<long long>(
        kTcCmaxRetry, std::max<long long>(r.cmax, (long long)P.Q * r.cmax / nf));
    if ((rc = emit_scan(r, st, r.qB, nf, r.thr, cmax2, 0, r.n_tiles2)) != kOk) return rc;
    if (tm) tm->mark(st, kPhaseTcRetryScan);
    rc = rerank(r, st, nf, cmax2, r.qsub, r.ldf, r.qn, r.thr, r.sd, r.si, r.ldf, r.fail2, true);
    if (rc != kOk) return rc;
    if (tm) tm->mark(st, kPhaseTcRetryRerank);
    int nf2 = 0;
    if ((rc = read_count(r.nfail, host_tmp, st, nf2)) != kOk) return rc;
    host_stats[1] = nf2;
    if (nf2 > 0) {
        // still uncertified (list overflow): the exact kernel recomputes the
        // compacted batch
        const long long per_split = (long long)nf * P.k * 8;
        const int splits = (int)std::max<long long>(
            1, std::min<long long>(exact_plan_splits(P.N, nf, P.d, P.k, P.num_sms),
                                   (long long)(r.xcap / per_split)));
        ExactProblem x;
        x.ref = P.ref;
        x.N = P.N;
        x.ldr = P.ldr;
        x.qry = r.qsub;
        x.Q = nf;
        x.ldq = r.ldf;
        x.d = P.d;
        x.k = P.k;
        x.out_dist = r.sd;
        x.out_idx = r.si;
        x.ld_out = r.ldf;
        x.scratch = r.xs;
        x.scratch_bytes = r.xcap;
        x.status = P.status;
        x.num_sms = P.num_sms;
        x.force_splits = splits;
        x.timer = nullptr;
        if ((rc = launch_exact(x, st)) != kOk) return rc;
    }
    scatter_results_kernel<<<dim3((nf + 127) / 128, P.k), 128, 0, st>>>(
        r.sd, r.si, r.ldf, r.fail, nf, P.out_dist, P.out_idx, P.ld_out);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    if (tm) tm->mark(st, kPhaseTcFallback);
    return kOk;
}

int launch_tc(const TcProblem &P, const TcRefView &R, cudaStream_t st, int *host_stats) {
    TcRun r;
    int rc = tc_run_begin(P, R, st, r);
    if (rc == kOk) rc = tc_run_pass1(r, st);
    if (rc == kOk) rc = tc_run_pass2(r, 0, r.n_tiles2, st);
    if (rc == kOk) rc = tc_run_finish(r, st, host_stats);
    return rc;
}

}  // namespace knnb200
