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
#include <cuda_fp8.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "knn_exact_core.cuh"
#include "knn_kernels.h"
#include "knn_tc.cuh"

namespace knnb200 {

constexpr int TC_BM = 128;            // rows (queries) per CTA of a pair, points per CTA half-tile
constexpr int TC_QT = 2 * TC_BM;      // queries per CTA pair
constexpr int TC_BK = 64;             // K block: 64 bf16 = 128 B (one swizzle row)
constexpr int TC_NK = 16;             // norm step: K = 16 (h, m, l, 13 zeros)
constexpr int TC_KS = 16;             // pass-1 per-row list length
constexpr int TC_SAMPLE_EVERY = 16;   // point sample: every 16th point (pass 1 takes every m-th of those)
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
// later with one atomicAdd that reserves all their slots.  The atomic is
// issued before the wait for the next accumulator and the entries are
// written once that accumulator has been read and released, so the
// round trip overlaps the wait instead of delaying the release.
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
    // the slots for the buffered entries: issue the atomic now, use `pos`
    // later (the round trip overlaps whatever runs in between)
    KNN_DI int reserve(int *count, int qrow) const { return n ? atomicAdd(&count[qrow], n) : 0; }
    KNN_DI void commit(int pos, unsigned long long *cand, int cmax, int qrow) {
        if (n == 0) return;
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
constexpr int TP_NSLOTS = 2;          // norm-step ring slots

// Operand kinds of the scan.  Every kind keeps the same epilogue: the
// accumulator holds a (scaled for FP8) and the threshold test is the same.
enum TcKind : int {
    kTcBf16 = 0,     // BF16 operands (kind::f16): one MMA per 16-element K step
    kTcBf16x3 = 1,   // split BF16: hi + lo parts of both sets, hi.hi + lo.hi + hi.lo
    kTcFp8 = 2,      // FP8 e4m3 operands (kind::f8f6f4), power-of-two scales
};

// Shared memory: a region of TP_REGION_TILES operand tiles (128 rows x
// 128 bytes, 16 KB each) holds the resident query tiles (A) followed by the
// reference ring (B), or -- when A does not fit, d_pad > 512 in BF16 -- a
// ring whose stages carry an A tile and a B tile each; then the ones tile,
// the norm-step ring and the barriers.
constexpr int TP_TILE_BYTES = TC_BM * 128;            // 16 KB
constexpr int TP_REGION_TILES = 13;
constexpr int TP_MAX_RESIDENT_A = 8;                   // leaves >= 5 ring stages
constexpr int TP_MAX_STAGES = TP_REGION_TILES - 1;
constexpr int TP_NORM_BYTES = TC_BM * 32;              // 4 KB: 32-byte norm-step rows
constexpr size_t TP_OFF_REGION = 0;
constexpr size_t TP_OFF_ONES = (size_t)TP_REGION_TILES * TP_TILE_BYTES;   // 208 KB
constexpr size_t TP_OFF_N = TP_OFF_ONES + TP_NORM_BYTES;                   // +4 KB
constexpr size_t TP_OFF_BAR = TP_OFF_N + (size_t)TP_NSLOTS * TP_NORM_BYTES;  // +8 KB
constexpr int TP_NBARS = 1 + 2 * TP_MAX_STAGES + 2 * TP_NSLOTS + 2 + 2 + 1;
constexpr size_t TP_SMEM = 1024 + TP_OFF_BAR + TP_NBARS * 8 + 16;
static_assert(TP_SMEM <= 232448, "pair scan kernel shared memory");
static_assert(TP_OFF_N % 1024 == 0 && TP_OFF_ONES % 1024 == 0, "tile alignment");

struct TpArgs {
    int N, Q;
    int kb;                 // K blocks per operand row (128 bytes each)
    int ka;                 // resident A tiles (0: A streamed with B)
    int stages;             // ring stages
    int items;              // ring items per reference tile
    int tile_base, n_splits;
    TileRuns tiles;         // scan tiles tile_base + tiles.tile(u), u < tiles.units
    const float *thr;       // emit pass: [Q] thresholds (a units)
    float thr_scale;        // accumulator units per a unit (FP8: s_q s_r; else 1)
    uint32_t ones_word;     // four bytes of the ones tile (1.0 BF16 x2, or the FP8 c1 x4)
    float *p1;              // sample pass: [TP_LISTS n_splits][Q][TC_KS] (accumulator units)
    unsigned long long *cand;   // [Q][cmax] (accumulator bits, index) entries
    int *count;             // [Q]
    int cmax;
    int *status;
};

// Norm step and one ring item's MMAs for each kind, issued by the even
// CTA's MMA thread.  K steps advance the descriptors by 32 bytes (2 in
// 16-byte units) for every kind: 16 BF16 or 32 FP8 elements.
template <int KIND>
KNN_DI void tp_mma_norm(uint32_t acc, uint64_t odesc, uint64_t ndesc) {
    if (KIND == kTcFp8)
        umma_f8_pair(acc, odesc, ndesc, umma_idesc_e4m3(2 * TC_BM, TP_BN), 0u);
    else
        umma_bf16_pair(acc, odesc, ndesc, umma_idesc_bf16(2 * TC_BM, TP_BN), 0u);
}
template <int KIND>
KNN_DI void tp_mma_block(uint32_t acc, uint64_t adesc, uint64_t bdesc) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (KIND == kTcFp8)
            umma_f8_pair(acc, adesc + (uint64_t)(2 * k), bdesc + (uint64_t)(2 * k),
                         umma_idesc_e4m3(2 * TC_BM, TP_BN), 1u);
        else
            umma_bf16_pair(acc, adesc + (uint64_t)(2 * k), bdesc + (uint64_t)(2 * k),
                           umma_idesc_bf16(2 * TC_BM, TP_BN), 1u);
    }
}

template <int MODE, int KIND>   // MODE 0: threshold sample pass, 1: emit pass
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TP_THREADS, 1)
    knn_tc_pair_scan_kernel(const __grid_constant__ CUtensorMap tmA,
                            const __grid_constant__ CUtensorMap tmA2,
                            const __grid_constant__ CUtensorMap tmB,
                            const __grid_constant__ CUtensorMap tmB2,
                            const __grid_constant__ CUtensorMap tmN, TpArgs a) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char *sR = base + TP_OFF_REGION;
    unsigned char *sOnes = base + TP_OFF_ONES;
    unsigned char *sN = base + TP_OFF_N;
    uint64_t *bars = reinterpret_cast<uint64_t *>(base + TP_OFF_BAR);
    uint64_t *a_full = bars;
    uint64_t *b_full = bars + 1;
    uint64_t *b_empty = b_full + TP_MAX_STAGES;
    uint64_t *n_full = b_empty + TP_MAX_STAGES;
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
    const int KB = a.kb, KA = a.ka, NST = a.stages, ITEMS = a.items;
    const bool streamed = KA == 0;
    const int stage_tiles = streamed ? 2 : 1;
    const uint32_t stage_bytes = (uint32_t)(stage_tiles * TP_TILE_BYTES);
    // K-block width in elements of the operand type (128 bytes)
    const int kx = KIND == kTcFp8 ? 128 : 64;
    // this split's units [u0, u0 + n_my)
    const int u0 = (int)((long long)a.tiles.units * split / a.n_splits);
    const int n_my = (int)((long long)a.tiles.units * (split + 1) / a.n_splits) - u0;

    for (int i = threadIdx.x; i < TP_NORM_BYTES / 4; i += TP_THREADS)
        reinterpret_cast<uint32_t *>(sOnes)[i] = a.ones_word;
    fence_proxy_async_smem();
    if (warp == 0 && lane == 0) {
        mbar_init(a_full, 1);
        for (int s = 0; s < NST; ++s) {
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
        if (KIND == kTcBf16x3) {
            prefetch_tensormap(&tmA2);
            prefetch_tensormap(&tmB2);
        }
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
    // ring stage s: tiles [KA + s * stage_tiles, + stage_tiles) of the region
    auto stage_ptr = [&](int s) { return sR + (size_t)(KA + s * stage_tiles) * TP_TILE_BYTES; };

    if (warp == 0) {
        // ---------------- TMA producer (both CTAs) ----------------
        if (lane == 0) {
            int issued = 0, n_issued = 0;
            int ps = 0;          // ring stage of the next item
            uint32_t pph = 0;    // its phase parity
            bool a_issued = false, ok = true;
            const int half_row = (int)rank * TC_BM;
            const int qrow0 = qpair * TC_QT + half_row;
            if (n_my > 0 && KA > 0) {
                if (lead) mbar_arrive_expect_tx(a_full, (uint32_t)(2 * KA * TP_TILE_BYTES));
                const uint32_t bar = mapa_shared(smem_u32(a_full), 0);
                for (int t = 0; t < KA; ++t) {
                    // split BF16: hi tiles 0 .. KB-1, lo tiles KB .. 2 KB-1
                    const CUtensorMap *m = (KIND == kTcBf16x3 && t >= KB) ? &tmA2 : &tmA;
                    tma_load_2d_pair(sR + (size_t)t * TP_TILE_BYTES, m, bar, (t % KB) * kx, qrow0);
                }
                a_issued = true;
            }
            TileRuns::Iter tile = a.tiles.from(u0);
            // the even CTA's full barriers (shared::cluster addresses) and
            // the ring's first stage; stage s is 8 B and s stage_bytes on
            const uint32_t bfull0 = mapa_shared(smem_u32(&b_full[0]), 0);
            unsigned char *const stage0 = stage_ptr(0);
            for (int j = 0; j < n_my && ok; ++j, tile.next()) {
                const int row0 = (a.tile_base + *tile) * TP_BN + half_row;
                const int ns = j % TP_NSLOTS;
                if (j >= TP_NSLOTS && !mbar_wait(&n_empty[ns], ((j / TP_NSLOTS) - 1) & 1)) {
                    ok = false;
                    break;
                }
                if (*abort_flag) break;
                if (lead) mbar_arrive_expect_tx(&n_full[ns], 2 * TP_NORM_BYTES);
                tma_load_2d_pair(sN + (size_t)ns * TP_NORM_BYTES, &tmN,
                                 mapa_shared(smem_u32(&n_full[ns]), 0), 0, row0);
                n_issued = j + 1;
                for (int i = 0; i < ITEMS; ++i) {
                    const int it = j * ITEMS + i, s = ps;
                    const uint32_t ph = pph;
                    if (++ps == NST) { ps = 0; pph ^= 1u; }
                    if (it >= NST && !mbar_wait(&b_empty[s], ph ^ 1u)) {
                        ok = false;
                        break;
                    }
                    if (lead) mbar_arrive_expect_tx(&b_full[s], 2 * stage_bytes);
                    const uint32_t bar = bfull0 + 8u * (uint32_t)s;
                    unsigned char *dst = stage0 + (size_t)s * stage_bytes;
                    // split BF16: items alternate hi, lo of K block i / 2
                    const int kb = KIND == kTcBf16x3 ? (i >> 1) : i;
                    const CUtensorMap *mb = (KIND == kTcBf16x3 && (i & 1)) ? &tmB2 : &tmB;
                    if (streamed) {
                        tma_load_2d_pair(dst, &tmA, bar, kb * kx, qrow0);
                        dst += TP_TILE_BYTES;
                    }
                    tma_load_2d_pair(dst, mb, bar, kb * kx, row0);
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
                for (int it = max(0, issued - NST); it < issued; ++it)
                    if (!mbar_wait(&b_full[it % NST], (it / NST) & 1))
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
            bool ok = n_my == 0 || KA == 0 || mbar_wait(a_full, 0);
            bool issued_mma = false;
            int ms = 0;          // ring stage of the next item
            uint32_t mph = 0;    // its phase parity
            tc_fence_after();
            const uint64_t odesc = umma_desc_sw32(sOnes);
            // descriptors advance by the operand offset in 16-byte units
            const uint64_t a_desc0 = umma_desc_sw128(sR);
            const uint64_t s_desc0 = umma_desc_sw128(stage_ptr(0));
            constexpr uint64_t kTileDesc = TP_TILE_BYTES >> 4;
            for (int j = 0; j < n_my && ok; ++j) {
                const int b = j & 1;
                const uint32_t acc = tmem + (uint32_t)(b * TP_BN);
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
                tp_mma_norm<KIND>(acc, odesc, umma_desc_sw32(sN + (size_t)ns * TP_NORM_BYTES));
                umma_commit_pair_mc(&n_empty[ns], 0x3);
                issued_mma = true;
                for (int i = 0; i < ITEMS; ++i) {
                    const int s = ms;
                    const uint32_t ph = mph;
                    if (++ms == NST) { ms = 0; mph ^= 1u; }
                    // (an abort elsewhere ends this wait by its time limit)
                    if (!mbar_wait(&b_full[s], ph)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t sdesc = s_desc0 + (uint64_t)(s * stage_tiles) * kTileDesc;
                    const uint64_t bdesc = sdesc + (streamed ? kTileDesc : 0);
                    if (streamed) {
                        tp_mma_block<KIND>(acc, sdesc, bdesc);
                    } else if (KIND == kTcBf16x3) {
                        const int kb = i >> 1;
                        const uint64_t ahi = a_desc0 + (uint64_t)kb * kTileDesc;
                        if ((i & 1) == 0) {
                            // B hi: A hi . B hi + A lo . B hi
                            tp_mma_block<KIND>(acc, ahi, bdesc);
                            tp_mma_block<KIND>(acc, a_desc0 + (uint64_t)(KB + kb) * kTileDesc,
                                               bdesc);
                        } else {
                            tp_mma_block<KIND>(acc, ahi, bdesc);   // A hi . B lo
                        }
                    } else {
                        tp_mma_block<KIND>(acc, a_desc0 + (uint64_t)i * kTileDesc, bdesc);
                    }
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
        if (MODE == 1 && qrow < a.Q) thr = a.thr[qrow] * a.thr_scale;
        float L[TC_KS];
#pragma unroll
        for (int i = 0; i < TC_KS; ++i) L[i] = INFINITY;
        PendingCands pend;
        TileRuns::Iter tile = a.tiles.from(u0);
        for (int j = 0; j < n_my; ++j, tile.next()) {
            const int b = j & 1;
            const int pos = MODE == 1 ? pend.reserve(a.count, qrow) : 0;
            const bool got = mbar_wait(&acc_full[b], (j >> 1) & 1);
            if (__any_sync(0xffffffffu, !got || *abort_flag != 0)) {
                if (MODE == 1) pend.commit(pos, a.cand, a.cmax, qrow);
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
            if (MODE == 1) pend.commit(pos, a.cand, a.cmax, qrow);
            // first reference of this warp
            const int col0 = (a.tile_base + *tile) * TP_BN + hc * TP_COLS;
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
                            // sorted insertion: L[i] becomes the median of
                            // L[i - 1], x, L[i] (no NaN reaches here)
#pragma unroll
                            for (int i = TC_KS - 1; i > 0; --i)
                                L[i] = fmaxf(L[i - 1], fminf(x, L[i]));
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
// error bound of the expansion (see the file comment), per scan kind
// ---------------------------------------------------------------------------
// E_q = 2 eps ||q|| R + g (R^2 + ||q||^2) + abs_q ||q|| + abs_r R + abs_c
//       + 2^-20 (|T| + ||q||^2),   R^2 = max ||r||^2:
//   BF16        eps = 2^-7 + 2^-16 + g, g = (d_pad + 16) 2^-22
//   split BF16  eps = 3 2^-16 + 2^-20 + g, g = (3 d_pad + 16) 2^-22: the
//               dropped lo.lo product and the second roundings are 3u^2 +
//               O(u^3) of sum |q_i r_i| (u = 2^-8)
//   FP8 e4m3    eps = 2^-3 + 2^-8 + g, g = (d_pad8 + 32) 2^-22 (u = 2^-4),
//               plus the absolute error of values below the normal range
//               (half the subnormal spacing, 2^-10, in scaled units):
//               abs_q = 2 (1 + u) 2^-10 sqrt(d) / s_r,
//               abs_r = (1 + u) 2^-10 sqrt(d) / s_q,
//               abs_c = d 2^-20 / (s_q s_r) + the norm split's residual.
struct TcBound {
    float eps, g, abs_q, abs_r, abs_c;
};

KNN_DI float tc_error_bound(float qq, float r2, float T, const TcBound &b) {
    float e = 2.f * b.eps * sqrtf(qq * r2) + b.g * (r2 + qq) +
              9.5367431640625e-07f * (fabsf(T) + qq);
    if (b.abs_q != 0.f || b.abs_r != 0.f) e += b.abs_q * sqrtf(qq) + b.abs_r * sqrtf(r2);
    return e + b.abs_c;
}

// Relative rounding of the FP32 direct-form distance chain used by the
// re-rank's pruning: g = (d_pad + 16) 2^-22 (>= 4 gamma_d).
KNN_DI float tc_fp32_gamma(int d_pad) { return (float)(d_pad + TC_NK) * 2.384185791015625e-07f; }

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
// With absmax_bits, also the largest |x - c| of any coordinate (FP8 scale).
__global__ void tc_norms_kernel(const float *__restrict__ x, int n, long long ld, int d,
                                const float *__restrict__ center, float *__restrict__ nrm,
                                unsigned *__restrict__ max_bits,
                                unsigned *__restrict__ absmax_bits = nullptr) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    float s = 0.f, am = 0.f;
    if (p < n) {
        for (int dd = 0; dd < d; ++dd) {
            const float v = x[(size_t)dd * ld + p] - center[dd];
            s = fmaf(v, v, s);
            am = fmaxf(am, fabsf(v));
        }
        nrm[p] = s;
    }
    unsigned m = __float_as_uint(s), ma = __float_as_uint(am);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        ma = max(ma, __shfl_xor_sync(0xffffffffu, ma, o));
    }
    if ((threadIdx.x & 31) == 0 && max_bits) atomicMax(max_bits, m);
    if ((threadIdx.x & 31) == 0 && absmax_bits) atomicMax(absmax_bits, ma);
}

// dim x n (row pitch ld) FP32 -> n x d_pad BF16 of scale * (x - center)
// (scale a power of two, so bf16(scale y) = scale bf16(y)), zero-padded in
// [d, d_pad); with xlo also the lo part bf16(scale y - hi) of split BF16.
// 32 x 32 tiles through shared memory.
__global__ void tc_pack_kernel(const float *__restrict__ x, int n, long long ld, int d,
                               int d_pad, const float *__restrict__ center, float scale,
                               __nv_bfloat16 *__restrict__ xb,
                               __nv_bfloat16 *__restrict__ xlo = nullptr) {
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
            const __nv_bfloat16 hi = __float2bfloat16_rn(v * scale);
            xb[(size_t)p * d_pad + dd] = hi;
            if (xlo)
                xlo[(size_t)p * d_pad + dd] = __float2bfloat16_rn(v * scale - __bfloat162float(hi));
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
// x - center, for the 256-point tiles tile0 + tiles.tile(u) (two blocks of
// four warps per tile).  A warp owns 32 points (one per lane) and walks the
// dimensions in chunks of 32: each lane loads its point's 32 values of the
// chunk (coalesced rows, the next chunk's loads in flight meanwhile),
// accumulates its squared norm in increasing d with FP32 fma (the order
// tc_norms_kernel uses), and the chunk is transposed through a padded
// shared tile so that every store writes four points' 128-byte rows.
constexpr int TC_PREP_WARPS = 4;
constexpr int TC_PREP_LD = 36;   // floats per point row of the transpose tile
__global__ void __launch_bounds__(32 * TC_PREP_WARPS)
    tc_prep_ref_kernel(const float *__restrict__ x, int n, long long ld, int d, int d_pad,
                       int tile0, TileRuns tiles, const float *__restrict__ center,
                       __nv_bfloat16 *__restrict__ xb, float *__restrict__ xt,
                       __nv_bfloat16 *__restrict__ parts, unsigned *__restrict__ max_bits,
                       unsigned *__restrict__ absmax_bits) {
    __shared__ __align__(16) float tile_all[TC_PREP_WARPS][32 * TC_PREP_LD];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *tt = tile_all[warp];
    const int p0 = (tile0 + tiles.tile((int)(blockIdx.x >> 1))) * TP_BN +
                   (int)(blockIdx.x & 1) * (TP_BN / 2) + warp * 32;
    const int p = p0 + lane;       // this lane's point (loads, norm)
    const bool pin = p < n;
    float s = 0.f;                 // squared norm of x_p - c
    float am = 0.f;                // largest |x - c| this lane wrote
    float cur[32], nxt[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) cur[j] = (j < d && pin) ? x[(size_t)j * ld + p] : 0.f;
    // write-out roles: 8 rounds of 4 points, lane -> point 4 r + lane / 8,
    // dimensions 4 (lane % 8) .. + 3
    const int wp = lane >> 3, wm = lane & 7;
    for (int d0 = 0; d0 < d_pad; d0 += 32) {
        if (d0 + 32 < d_pad) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int dd = d0 + 32 + j;
                nxt[j] = (dd < d && pin) ? x[(size_t)dd * ld + p] : 0.f;
            }
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            if (d0 + j < d) {
                const float v = cur[j] - __ldg(center + d0 + j);
                s = fmaf(v, v, s);
            }
        }
#pragma unroll
        for (int m = 0; m < 8; ++m)
            *reinterpret_cast<float4 *>(tt + lane * TC_PREP_LD + 4 * m) =
                make_float4(cur[4 * m], cur[4 * m + 1], cur[4 * m + 2], cur[4 * m + 3]);
        __syncwarp();
        const int dd = d0 + 4 * wm;
        float c4[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) c4[e] = dd + e < d ? __ldg(center + dd + e) : 0.f;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int pp = 4 * r + wp, q = p0 + pp;
            const float4 v = *reinterpret_cast<const float4 *>(tt + pp * TC_PREP_LD + 4 * wm);
            if (q < n) {
                const float ve[4] = {v.x, v.y, v.z, v.w};
                __nv_bfloat16 yb[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float y = dd + e < d ? ve[e] - c4[e] : 0.f;
                    yb[e] = __float2bfloat16_rn(y);
                    am = fmaxf(am, fabsf(y));
                }
                *reinterpret_cast<float4 *>(xt + (size_t)q * d_pad + dd) = v;
                *reinterpret_cast<uint2 *>(xb + (size_t)q * d_pad + dd) =
                    *reinterpret_cast<const uint2 *>(yb);
            }
        }
        __syncwarp();
        if (d0 + 32 < d_pad) {
#pragma unroll
            for (int j = 0; j < 32; ++j) cur[j] = nxt[j];
        }
    }
    {
        unsigned ma = __float_as_uint(am);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ma = max(ma, __shfl_xor_sync(0xffffffffu, ma, o));
        if (lane == 0) atomicMax(absmax_bits, ma);
    }
    if (pin) write_norm_row(parts, p, s);
    unsigned m = pin ? __float_as_uint(s) : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) atomicMax(max_bits, m);
}

// The threshold sample of a prepared set: the BF16 row and the norm-step row
// of every TC_SAMPLE_EVERY-th point, copied into compact arrays (16-byte
// words; one warp per row).
__global__ void tc_sample_rows_kernel(const __nv_bfloat16 *__restrict__ xb,
                                      const __nv_bfloat16 *__restrict__ parts, int ns,
                                      int d_pad, __nv_bfloat16 *__restrict__ sb,
                                      __nv_bfloat16 *__restrict__ sparts) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= ns) return;
    const size_t p = (size_t)row * TC_SAMPLE_EVERY;
    const uint4 *src = reinterpret_cast<const uint4 *>(xb + p * d_pad);
    uint4 *dst = reinterpret_cast<uint4 *>(sb + (size_t)row * d_pad);
    for (int w = lane; w < d_pad / 8; w += 32) dst[w] = src[w];
    if (lane < TC_NK / 8)
        reinterpret_cast<uint4 *>(sparts + (size_t)row * TC_NK)[lane] =
            reinterpret_cast<const uint4 *>(parts + p * TC_NK)[lane];
}

// Lo parts of split BF16 for the whole prepared set: from the FP32
// point-major copy r and the translation c, lo = bf16(y - bf16(y)) with
// y = r - c computed as tc_prep_ref_kernel computes it (so hi + lo splits
// the same y the BF16 copy rounded).  Four consecutive elements per thread.
__global__ void tc_ref_lo_kernel(const float *__restrict__ xt, long long n_elems, int d,
                                 int d_pad, const float *__restrict__ center,
                                 __nv_bfloat16 *__restrict__ xlo) {
    const long long e0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (e0 >= n_elems) return;
    const float4 v = *reinterpret_cast<const float4 *>(xt + e0);
    const float vv[4] = {v.x, v.y, v.z, v.w};
    __nv_bfloat16 out[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int dd = (int)((e0 + i) % d_pad);
        const float y = dd < d ? vv[i] - center[dd] : 0.f;
        const __nv_bfloat16 hi = __float2bfloat16_rn(y);
        out[i] = __float2bfloat16_rn(y - __bfloat162float(hi));
    }
    *reinterpret_cast<uint2 *>(xlo + e0) = *reinterpret_cast<const uint2 *>(out);
}

// FP8 (e4m3) copy of the prepared set: byte (p, dd) = e4m3(s_r (r - c)), one
// warp per point (coalesced reads of the FP32 point-major copy), rows of
// d_pad8 bytes (d rounded up to 128, one K block; the FP32 rows are d_pad
// <= d_pad8 floats), and the norm-step row: ||r - c||^2 (FP32) as
// v = s_r ||r - c||^2 / kappa split greedily into up to 8 e4m3 parts (each
// at most 448, the format's largest value; the remainder carried in
// double), then zeros.  The A side's ones tile holds c1 = s_q kappa, so the
// parts contribute s_q s_r ||r - c||^2 to the accumulator.  resid_bits: the
// largest residual |v - sum parts| in unscaled units (kappa / s_r per unit
// of v), a term of the error bound.
__global__ void tc_pack_ref_f8_kernel(const float *__restrict__ xt, int n, int d, int d_pad,
                                      int d_pad8, const float *__restrict__ center, float s_r,
                                      float kappa, unsigned char *__restrict__ x8,
                                      unsigned char *__restrict__ parts8,
                                      unsigned *__restrict__ resid_bits) {
    const int warps = blockDim.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * warps + (threadIdx.x >> 5);
    if (p >= n) return;
    const float *row = xt + (size_t)p * d_pad;
    float s = 0.f;
    for (int d0 = lane * 4; d0 < d_pad8; d0 += 128) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (d0 < d_pad) v = *reinterpret_cast<const float4 *>(row + d0);
        const float vv[4] = {v.x, v.y, v.z, v.w};
        uint32_t packed = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float y = d0 + i < d ? vv[i] - center[d0 + i] : 0.f;
            s = fmaf(y, y, s);
            const __nv_fp8_e4m3 f(y * s_r);
            packed |= (uint32_t)f.__x << (8 * i);
        }
        *reinterpret_cast<uint32_t *>(x8 + (size_t)p * d_pad8 + d0) = packed;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        double rem = (double)s * (double)s_r / (double)kappa;
        unsigned char row8[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) row8[j] = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const __nv_fp8_e4m3 f((float)fmin(rem, 448.0));
            row8[j] = f.__x;
            rem -= (double)(float)f;
        }
        uint4 *dst = reinterpret_cast<uint4 *>(parts8 + (size_t)p * 32);
        dst[0] = *reinterpret_cast<const uint4 *>(row8);
        dst[1] = *reinterpret_cast<const uint4 *>(row8 + 16);
        const float resid = (float)(fabs(rem) * (double)kappa / (double)s_r);
        atomicMax(resid_bits, __float_as_uint(resid * 1.0000001f));
    }
}

// dim x n FP32 queries -> n x d_pad8 e4m3 of scale (x - c) (scale = -2 s_q),
// zero-padded; 32 x 32 tiles through shared memory as in tc_pack_kernel.
__global__ void tc_pack_f8_kernel(const float *__restrict__ x, int n, long long ld, int d,
                                  int d_pad8, const float *__restrict__ center, float scale,
                                  unsigned char *__restrict__ x8) {
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
        if (p < n && dd < d_pad8) {
            const float v = dd < d ? tile[tx][ty + 8 * i] - center[dd] : 0.f;
            x8[(size_t)p * d_pad8 + dd] = __nv_fp8_e4m3(v * scale).__x;
        }
    }
}

// Emission threshold: the KS-th smallest of the per-split pass-1 lists plus
// the error bound E_q (so that the k-th exact distance only has to lie below
// the sample's KS-th approximate one to certify); resets candidate counts.
// thr_raw keeps the sample's KS-th value itself (a scan of another kind
// re-derives its threshold from it).  Overflow prediction: a query whose
// bound under a probe kind exceeds the spread of its KS sample values
// (T - L_0) is expected to overflow its candidate list in that kind: about
// KS x stride points lie below T, and the density of points grows steeply
// above the sample's smallest values, so a band [T, T + E] wider than
// [L_0, T] holds many times that; n_wide[0] counts them for probe0 (BF16:
// switch to split BF16), n_wide[1] for probe1 (FP8: whether an FP8 pass 2
// pays).
__global__ void tc_threshold_kernel(const float *__restrict__ p1, int S, int Q,
                                    const float *__restrict__ qn,
                                    const unsigned *__restrict__ rmax_bits, TcBound bound,
                                    TcBound probe0, TcBound probe1, float *__restrict__ thr,
                                    float *__restrict__ thr_raw, int *__restrict__ count,
                                    int *__restrict__ n_wide) {
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
    const float r2 = __uint_as_float(*rmax_bits);
    thr[q] = T + tc_error_bound(qn[q], r2, T, bound);
    thr_raw[q] = T;
    count[q] = 0;
    if (n_wide) {
        const float spread = T - L[0];
        if (tc_error_bound(qn[q], r2, T, probe0) > spread) atomicAdd(n_wide, 1);
        if (tc_error_bound(qn[q], r2, T, probe1) > spread) atomicAdd(n_wide + 1, 1);
    }
}

// Thresholds of a scan of another kind from the raw sample thresholds:
// thr = T + E_q(T) under that kind's bound, plus E_q(T) under `extra` (the
// sample's own kind when it differs from the scan's: the sample value
// itself is then off by up to that bound).
__global__ void tc_rethreshold_kernel(const float *__restrict__ thr_raw, int Q,
                                      const float *__restrict__ qn,
                                      const unsigned *__restrict__ rmax_bits, TcBound bound,
                                      TcBound extra, int use_extra, float *__restrict__ thr) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    const float T = thr_raw[q], r2 = __uint_as_float(*rmax_bits);
    float t = T + tc_error_bound(qn[q], r2, T, bound);
    if (use_extra) t += tc_error_bound(qn[q], r2, T, extra);
    thr[q] = t;
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

// Exact FP32 re-rank of each query's candidates + certification, in three
// kernels of one warp per query: select (tc_rerank_select_kernel: the k-th
// smallest a by radix selection, the pruning below, the kept candidates
// compacted in place), gather (tc_rerank_gather_kernel: their exact
// distances) and certify (tc_rerank_certify_kernel: sort, check, output).
// The gather, which moves the bytes, then runs with nothing but its staging
// ring and the query in shared memory, so the SM holds about twice the warps
// (copies in flight) of one kernel that also keeps the sort keys there.
//
// Pruning: with a_k the k-th smallest BF16-expansion value a among the
// candidates, every candidate i of the first k has exact
// FP32 distance <= (a_k + ||q||^2 + E)(1 + gamma), and a candidate r has
// exact FP32 distance >= (a_r + ||q||^2 - E)(1 - gamma) (E as for the
// threshold, gamma the relative rounding of the FP32 distance chain).  A
// candidate whose lower bound exceeds that upper bound has k strictly
// closer candidates and cannot be in the top-k, so only the prefix with
// a_r <= a_k + 2 E + 2 g (|a_k| + ||q||^2 + E) (g = K 2^-22 >= 4 gamma, which
// also absorbs the roundings of this bound) is re-ranked; the k-th exact
// distance of the kept candidates is the k-th of all candidates.
//
// The kept candidates are handled 32 at a time, one per lane: the warp
// copies the 32 candidate rows of the FP32 point-major copy, TC_RR_DCH
// dimensions at a time, into a padded shared tile with asynchronous 16-byte
// copies (cp.async, several rows per instruction, coalesced), through a ring
// of TC_RR_NBUF buffers so the next chunks are in flight while each lane
// runs its candidate's FMA chain in increasing d -- the fused exact kernel's
// arithmetic and order, so distances are identical.  The (distance, index)
// keys are bitonic-sorted by the warp.  One warp per block: the gather is
// latency-bound, and single-warp blocks let the SM hold as many warps as
// its shared memory allows.
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

__host__ __device__ inline size_t tc_rr_gather_bytes(int d_pad) {
    return (size_t)d_pad * 4 + TC_RR_NBUF * TC_RR_BUF * 4;
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
// Bounds a re-rank works with: those of the scan that emitted the
// candidates, whose accumulator values are a / a_scale.
struct RrBounds {
    TcBound cur;
    float a_scale;
};

// A query that fails leaves the threshold of its second scan as a base
// value and a factor: thr = base + f E_q(base) under the bound of the kind
// the second scan uses (chosen once the failures are counted; f = 0: base
// is the threshold, NaN: exact kernel), and optionally a "sure" base s:
// then thr = min(that, s + 2.5 E_q(s)).  Overflowing lists count in
// n_fail[1].
//
// Returns 0 for a list to re-rank and certify, 1 for a list rejected here,
// 2 for an overflowing list of the first scan: its cmax entries are
// re-ranked all the same, and their k-th exact distance D -- not below the
// true k-th, since they are genuine points -- gives the sure base
// D (1 + g) - ||q||^2 (rr_certify), which keeps every point of the exact
// top-k below the second scan's threshold and certifies it there.
KNN_DI int rr_reject_list(int c, int cmax, int k, int q, float qq, float r2, float T,
                          float T_raw, const RrBounds &rb, int final_pass, int *fail_list,
                          int *n_fail, float *retry, float *retry_f, float *retry_s,
                          int lane) {
    if (c <= cmax && c >= k) return 0;
    if (lane == 0) {
        fail_list[atomicAdd(n_fail, 1)] = q;
        retry_s[q] = INFINITY;
        if (c < k) {
            retry[q] = T + 8.f * tc_error_bound(qq, r2, T, rb.cur);
            retry_f[q] = 0.f;
        } else {
            atomicAdd(n_fail + 1, 1);
            retry[q] = final_pass ? __int_as_float(0x7fc00000) : T_raw;
            retry_f[q] = final_pass ? 0.f : 1.f;
        }
    }
    return (c > cmax && !final_pass) ? 2 : 1;
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
    float qq, e_q, a_scale;
    unsigned *stat;
};

template <bool STAT = false>
KNN_DI void rr_exact_distances(unsigned long long *keys, int n, const float *__restrict__ refT,
                               int d_pad, const float *qv, float *rows, int lane,
                               BoundStat bs = BoundStat{0.f, 0.f, 1.f, nullptr}) {
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
                const float a = ord_float((uint32_t)(keys[t] >> 32)) * bs.a_scale;
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
// otherwise it joins fail_list with the base threshold of a second scan
// that certifies (see tc_rerank_select_kernel).  Warp-uniform.
KNN_DI void rr_certify(const unsigned long long *keys, int q, float qq, float r2, float T,
                       int d_pad, int k, const RrBounds &rb, float *__restrict__ out_dist,
                       int *__restrict__ out_idx, long long ld_out, int *fail_list, int *n_fail,
                       float *retry, float *retry_f, float *retry_s, bool overflow, int lane) {
    int failed = 0;
    if (lane == 0) {
        const float dk = key_dist2(keys[k - 1]);
        const float E = tc_error_bound(qq, r2, T, rb.cur);
        const float dkg = dk * (1.f + (float)d_pad * 2.384185791015625e-07f);
        if (overflow) {
            // an overflowing list (already counted as a failure): the sure
            // base from its entries' k-th exact distance
            retry_s[q] = dkg - qq;
            failed = 1;
        } else {
            failed = !(dkg + E < T + qq);
            if (failed) {
                fail_list[atomicAdd(n_fail, 1)] = q;
                retry[q] = dkg - qq;
                retry_f[q] = 2.5f;
                retry_s[q] = INFINITY;
            }
        }
    }
    if (__shfl_sync(0xffffffffu, failed, 0)) return;
    for (int j = lane; j < k; j += 32) {
        const unsigned long long key = keys[j];
        out_dist[(size_t)j * ld_out + q] = sqrtf(key_dist2(key));
        out_idx[(size_t)j * ld_out + q] = key_index(key);
    }
}

// Select: reject lists that cannot be re-ranked, find the k-th smallest
// entry key (the order-preserving bits of a) by an 8-bit radix selection
// over the list, and compact the entries with a <= the pruning limit to the
// front of the list (in place: an entry moves only to a position already
// read).  nsel[q] = their number, or -1 for a rejected list.
__global__ void __launch_bounds__(32)
    tc_rerank_select_kernel(unsigned long long *__restrict__ cand, const int *__restrict__ count,
                            int cmax, int Q, int k, const float *__restrict__ qn,
                            const unsigned *__restrict__ rmax_bits,
                            const float *__restrict__ thr, const float *__restrict__ thr_raw,
                            RrBounds rb, int d_pad, int final_pass, int *__restrict__ fail_list,
                            int *__restrict__ n_fail, float *__restrict__ retry,
                            float *__restrict__ retry_f, float *__restrict__ retry_s,
                            unsigned long long *__restrict__ cand_total, int *__restrict__ nsel) {
    __shared__ unsigned hist[256];
    const int q = blockIdx.x, lane = threadIdx.x;
    if (q >= Q) return;
    int c = count[q];
    if (lane == 0) atomicAdd(cand_total, (unsigned long long)c);
    const float qq = qn[q];
    const float r2 = __uint_as_float(*rmax_bits);
    const float T = thr[q];
    const int rj = rr_reject_list(c, cmax, k, q, qq, r2, T, thr_raw ? thr_raw[q] : T, rb,
                                  final_pass, fail_list, n_fail, retry, retry_f, retry_s, lane);
    if (rj == 1) {
        if (lane == 0) nsel[q] = -1;
        return;
    }
    if (rj == 2) c = cmax;   // the entries that were kept
    unsigned long long *cq = cand + (size_t)q * cmax;
    // k-th smallest key, 8 bits per round from the top
    uint32_t prefix = 0, hmask = 0;
    unsigned rank = (unsigned)k;   // 1-based rank among the keys matching prefix
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = lane; i < 256; i += 32) hist[i] = 0u;
        __syncwarp();
        for (int t = lane; t < c; t += 32) {
            const uint32_t key = (uint32_t)(cq[t] >> 32);
            if ((key & hmask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncwarp();
        unsigned h[8], sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            h[j] = hist[8 * lane + j];
            sum += h[j];
        }
        unsigned incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const unsigned excl = incl - sum;
        const unsigned owner = __ballot_sync(0xffffffffu, excl < rank && rank <= incl);
        const int src = __ffs(owner) - 1;
        int bin = 0;
        unsigned below = 0;
        if (lane == src) {
            unsigned run = excl;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (bin == 0 && run + h[j] >= rank) {
                    bin = 8 * lane + j + 1;   // +1: found
                    below = run;
                }
                run += h[j];
            }
        }
        bin = __shfl_sync(0xffffffffu, bin, src) - 1;
        below = __shfl_sync(0xffffffffu, below, src);
        prefix |= (uint32_t)bin << shift;
        hmask |= 255u << shift;
        rank -= below;
        __syncwarp();
    }
    const float ak = ord_float(prefix) * rb.a_scale;
    const float E = tc_error_bound(qq, r2, ak, rb.cur);
    const float g = tc_fp32_gamma(d_pad);
    const float lim = (ak + 2.f * E + 2.f * g * (fabsf(ak) + qq + E)) / rb.a_scale;
    const uint32_t lim_o = ord_bits(__float_as_uint(lim));
    int kept = 0;
    for (int t0 = 0; t0 < c; t0 += 32) {
        const int t = t0 + lane;
        kept += __popc(__ballot_sync(0xffffffffu, t < c && (uint32_t)(cq[t] >> 32) <= lim_o));
    }
    if (kept >= k) {
        int pos0 = 0;
        for (int t0 = 0; t0 < c; t0 += 32) {
            const int t = t0 + lane;
            const unsigned long long e = t < c ? cq[t] : kKeyInf;
            const bool in = t < c && (uint32_t)(e >> 32) <= lim_o;
            const unsigned b = __ballot_sync(0xffffffffu, in);
            if (in) cq[pos0 + __popc(b & ((1u << lane) - 1u))] = e;
            pos0 += __popc(b);
        }
    } else {
        kept = c;   // not reached for finite values (lim >= a_k); keep the whole list
    }
    if (lane == 0) nsel[q] = kept;
}

// Gather: exact FP32 distances of the nsel[q] selected candidates, keys
// replaced in place by (distance, index).  Shared memory: the query and the
// staging ring (rr_exact_distances).
template <bool STAT>
__global__ void __launch_bounds__(32)
    tc_rerank_gather_kernel(const float *__restrict__ refT, int d, int d_pad,
                            const float *__restrict__ qry, long long ldq,
                            const float *__restrict__ qn, const unsigned *__restrict__ rmax_bits,
                            const float *__restrict__ thr, RrBounds rb,
                            unsigned long long *__restrict__ cand, const int *__restrict__ nsel,
                            int cmax, int Q, unsigned *__restrict__ bound_stat) {
    extern __shared__ __align__(16) unsigned char rsm[];
    const int q = blockIdx.x, lane = threadIdx.x;
    if (q >= Q) return;
    const int n = nsel[q];
    if (n <= 0) return;
    float *qv = reinterpret_cast<float *>(rsm);
    float *rows = qv + d_pad;
    for (int dd = lane; dd < d_pad; dd += 32) qv[dd] = dd < d ? qry[(size_t)dd * ldq + q] : 0.f;
    __syncwarp();
    const float qq = qn[q];
    const float E = STAT ? tc_error_bound(qq, __uint_as_float(*rmax_bits), thr[q], rb.cur) : 0.f;
    rr_exact_distances<STAT>(cand + (size_t)q * cmax, n, refT, d_pad, qv, rows, lane,
                             BoundStat{qq, E, rb.a_scale, bound_stat});
}

// Certify: sort the exact keys of the selected candidates (their k-th is
// the k-th of all candidates) and certify (rr_certify).
__global__ void __launch_bounds__(32)
    tc_rerank_certify_kernel(const unsigned long long *__restrict__ cand,
                             const int *__restrict__ nsel, const int *__restrict__ count,
                             int cmax, int Q, int k, int d_pad,
                             const float *__restrict__ qn, const unsigned *__restrict__ rmax_bits,
                             const float *__restrict__ thr, RrBounds rb,
                             float *__restrict__ out_dist, int *__restrict__ out_idx,
                             long long ld_out, int *__restrict__ fail_list,
                             int *__restrict__ n_fail, float *__restrict__ retry,
                             float *__restrict__ retry_f, float *__restrict__ retry_s) {
    extern __shared__ unsigned long long keys[];
    const int q = blockIdx.x, lane = threadIdx.x;
    if (q >= Q) return;
    const int n = nsel[q];
    if (n < 0) return;
    const unsigned long long *cq = cand + (size_t)q * cmax;
    int P = 32;
    while (P < n) P <<= 1;
    for (int t = lane; t < P; t += 32) keys[t] = t < n ? cq[t] : kKeyInf;
    __syncwarp();
    warp_bitonic_sort(keys, P, lane);
    rr_certify(keys, q, qn[q], __uint_as_float(*rmax_bits), thr[q], d_pad, k, rb, out_dist,
               out_idx, ld_out, fail_list, n_fail, retry, retry_f, retry_s, count[q] > cmax,
               lane);
}

// Incremental re-rank for a reference set that arrives in pieces (the
// streamed host entry).  After each piece's scan, the candidates a query
// gained since the last call (list entries done[q] .. min(count, cmax)) get
// their exact FP32 distances and are merged into its running k smallest
// keys run[q][0..k) (a sort of the new keys, then every key placed at its
// index plus its rank in the other array).  Nothing is pruned -- the k-th a
// is not known yet -- so about twice the rows of the select and gather
// kernels are gathered, while the rest of the set is still being copied in.
// After the last piece run[q] holds the k smallest exact keys of all
// candidates: the certification and the output are those of
// tc_rerank_certify_kernel.  One warp (block) per query.
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

// Certification after the last piece: the first-pass checks of
// tc_rerank_select_kernel and tc_rerank_certify_kernel on the running k
// smallest keys of tc_rerank_piece_kernel.  One warp per query.
__global__ void tc_certify_pieces_kernel(const int *__restrict__ count, int cmax,
                                         const float *__restrict__ qn,
                                         const unsigned *__restrict__ rmax_bits,
                                         const float *__restrict__ thr,
                                         const float *__restrict__ thr_raw, RrBounds rb,
                                         const unsigned long long *__restrict__ run, int Q, int k,
                                         int d_pad, float *__restrict__ out_dist,
                                         int *__restrict__ out_idx, long long ld_out,
                                         int *__restrict__ fail_list, int *__restrict__ n_fail,
                                         float *__restrict__ retry, float *__restrict__ retry_f,
                                         float *__restrict__ retry_s,
                                         unsigned long long *__restrict__ cand_total) {
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (q >= Q) return;
    const int c = count[q];
    if (lane == 0) atomicAdd(cand_total, (unsigned long long)c);
    const float qq = qn[q];
    const float r2 = __uint_as_float(*rmax_bits);
    const float T = thr[q];
    const int rj = rr_reject_list(c, cmax, k, q, qq, r2, T, thr_raw[q], rb, 0, fail_list,
                                  n_fail, retry, retry_f, retry_s, lane);
    if (rj == 1) return;
    // run holds the k smallest exact keys of the list's entries (all of
    // them, or the cmax kept of an overflowing list)
    rr_certify(run + (size_t)q * k, q, qq, r2, T, d_pad, k, rb, out_dist, out_idx, ld_out,
               fail_list, n_fail, retry, retry_f, retry_s, rj == 2, lane);
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

// Second-chance scan of the uncertified queries: compacted thresholds
// under the bound of the second scan's kind (qn already holds the
// compacted queries' norms).
__global__ void tc_retry_prep_kernel(const int *__restrict__ list, int m,
                                     const float *__restrict__ retry,
                                     const float *__restrict__ retry_f,
                                     const float *__restrict__ retry_s,
                                     const float *__restrict__ qn,
                                     const unsigned *__restrict__ rmax_bits, TcBound bound,
                                     float *__restrict__ thr, int *__restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        const float r2 = __uint_as_float(*rmax_bits);
        const float base = retry[list[i]], f = retry_f[list[i]], sure = retry_s[list[i]];
        float t = f == 0.f ? base : base + f * tc_error_bound(qn[i], r2, base, bound);
        if (isfinite(sure)) t = fminf(t, sure + 2.5f * tc_error_bound(qn[i], r2, sure, bound));
        thr[i] = t;
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

// FP8 operand rows [rows][d_pad8] bytes: 128-byte x 128-row boxes.
bool encode_u8_kmajor(CUtensorMap *m, const void *base, int rows, int d_pad8) {
    return encode_2d(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, base, (uint64_t)d_pad8, (uint64_t)rows,
                     (uint64_t)d_pad8, 128, TC_BM, CU_TENSOR_MAP_SWIZZLE_128B);
}

// Norm-step rows, 32 bytes each (16 BF16 or 32 FP8), 128-row boxes with the
// 32-byte swizzle.
bool encode_norm_rows(CUtensorMap *m, const void *base, int rows, bool fp8) {
    return fp8 ? encode_2d(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, base, 32, (uint64_t)rows, 32, 32,
                           TC_BM, CU_TENSOR_MAP_SWIZZLE_32B)
               : encode_2d(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, (uint64_t)TC_NK,
                           (uint64_t)rows, (uint64_t)TC_NK, TC_NK, TC_BM,
                           CU_TENSOR_MAP_SWIZZLE_32B);
}

// Candidate lists: first scan cmax = 4 * KS * stride (<= 2560 for k <=
// 256); the second scan of the queries whose list overflowed reuses the
// whole list buffer, up to kTcCmaxRetry entries per query.  The re-rank
// kernel's shared memory (keys padded to a power of two) is capped at
// kRerankSmem per block: fewer warps per block for long lists.
constexpr int kTcCmaxRetry = 8192;
constexpr size_t kSplitBytes = 26u << 20;   // reference bytes per pass-2 split (L2 126 MB)
constexpr size_t kRerankSmem = 200 * 1024;
constexpr int kTcMaxDim = 4096;
constexpr int kTcMaxK = 256;

struct TcPlan {
    int d_pad, d_pad8, qtiles, cmax;
    int n_tiles2, splits1;   // 256-point tiles; pass-1 splits over CTA pairs
    TileRuns sample;         // pass-1 tiles
    int p1_rows, p1_every;   // point sample: pass 1 scans rows 0, m, 2m, ... of
                             // the every-16th-point copy (p1_every = m; 0: tile runs)
};

// Operand feed of one scan kind: K blocks of 128 bytes per operand row,
// resident A tiles (0: A streams beside B), ring stages and items per
// reference tile.
struct TcOp {
    int kind, kb, ka, stages, items;
};

TcOp tc_op(int kind, int d_pad, int d_pad8) {
    TcOp o;
    o.kind = kind;
    if (kind == kTcFp8) {
        o.kb = d_pad8 / 128;
        o.ka = o.kb;
        o.items = o.kb;
    } else if (kind == kTcBf16x3) {
        o.kb = d_pad / 64;
        o.ka = 2 * o.kb;
        o.items = 2 * o.kb;
    } else {
        o.kb = d_pad / 64;
        o.ka = o.kb <= TP_MAX_RESIDENT_A ? o.kb : 0;
        o.items = o.kb;
    }
    o.stages = o.ka > 0 ? TP_REGION_TILES - o.ka : TP_REGION_TILES / 2;
    return o;
}

bool kind_fits(int kind, int d_pad, int d_pad8) {
    if (kind == kTcBf16x3) return 2 * (d_pad / 64) <= TP_MAX_RESIDENT_A;
    if (kind == kTcFp8) return d_pad8 / 128 <= TP_MAX_RESIDENT_A;
    return true;
}

// Splits that fill whole waves of one CTA per SM for `tiles` tiles per
// query tile, with at least min_tiles per CTA; modelled per-CTA cost =
// tiles per split + a fixed set-up cost of `fixed` tiles.  With max_tiles >
// 0 only splits of at most max_tiles tiles are considered (when there are
// such splits): the CTAs that share a split do not all run in the same
// wave, and the later ones find its tiles in L2 only if a wave's splits
// fit there.
static int choose_splits(int qtiles, int tiles, int min_tiles, double fixed, int num_sms,
                         int max_tiles = 0) {
    int best = 1;
    double best_t = 1e300;
    const int max_s = std::max(1, std::min(256, tiles / std::max(1, min_tiles)));
    const int min_s = max_tiles > 0 ? std::min(max_s, (tiles + max_tiles - 1) / max_tiles) : 1;
    for (int S = min_s; S <= max_s; ++S) {
        const long long ctas = (long long)qtiles * S;
        const double t = (double)((ctas + num_sms - 1) / num_sms) * ((double)tiles / S + fixed);
        if (t < best_t * 0.999) {
            best_t = t;
            best = S;
        }
    }
    return best;
}

TcPlan plan_tc(int N, int Q, int d, int k, int num_sms, bool point_sample = false) {
    TcPlan p;
    p.d_pad = (d + 63) / 64 * 64;
    p.d_pad8 = (d + 127) / 128 * 128;
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
    p.p1_rows = p.p1_every = 0;
    if (point_sample) {
        // every (16 m)-th point, 16 m >= stride: rows 0, m, 2m, ... of the
        // every-16th-point copy, scanned as contiguous 256-row tiles
        const int m = (stride + TC_SAMPLE_EVERY - 1) / TC_SAMPLE_EVERY;
        const int ns = (N + TC_SAMPLE_EVERY - 1) / TC_SAMPLE_EVERY;
        p.p1_every = m;
        p.p1_rows = (ns + m - 1) / m;
        p.sample = contiguous_tiles((p.p1_rows + TP_BN - 1) / TP_BN);
    }
    // coarser pass-1 splits amortise each pair's set-up (query tile load,
    // TMEM allocation, pipeline fill)
    p.splits1 = choose_splits(p.qtiles, p.sample.units, 16, 8.0, std::max(1, num_sms / 2));
    return p;
}

// Error-bound constants of each kind (see tc_error_bound).
TcBound bound_of(int kind, int d, int d_pad, int d_pad8, float s_q, float s_r, float resid8) {
    TcBound b{0.f, 0.f, 0.f, 0.f, 0.f};
    const double two22 = 2.384185791015625e-07;   // 2^-22
    if (kind == kTcBf16x3) {
        b.g = (float)((3.0 * d_pad + TC_NK) * two22);
        b.eps = (float)(3.0 * 1.52587890625e-05 + 9.5367431640625e-07) + b.g;
    } else if (kind == kTcFp8) {
        const double u = 0.0625, eta = 9.765625e-04;   // 2^-4, 2^-10
        b.g = (float)((d_pad8 + 32.0) * two22);
        b.eps = (float)(2.0 * u + u * u) + b.g;
        const double sd = std::sqrt((double)d);
        b.abs_q = (float)(2.0 * (1.0 + u) * eta * sd / s_r * 1.0000001);
        b.abs_r = (float)((1.0 + u) * eta * sd / s_q * 1.0000001);
        b.abs_c = (float)(((double)d * eta * eta / ((double)s_q * s_r) + resid8) * 1.0000001);
    } else {
        b.g = (float)((d_pad + TC_NK) * two22);
        b.eps = 0.0078125f + 1.52587890625e-05f + b.g;
    }
    return b;
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

int read_count(const int *dev, int *host_pinned, cudaStream_t st, int &out, int n = 1) {
    if (cudaMemcpyAsync(host_pinned, dev, n * sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return kErrCuda;
    out = *host_pinned;
    return kOk;
}

float pow2_floor(double x) { return (float)std::ldexp(1.0, (int)std::floor(std::log2(x))); }
float pow2_ceil(double x) { return (float)std::ldexp(1.0, (int)std::ceil(std::log2(x))); }

}  // namespace

bool tc_supported(int N, int Q, int d, int k) {
    return d >= 16 && d <= kTcMaxDim && k >= 1 && k <= kTcMaxK && N >= 32768 && Q >= 1;
}

bool tc_fp8_supported(int d) {
    const int d_pad = (d + 63) / 64 * 64, d_pad8 = (d + 127) / 128 * 128;
    return kind_fits(kTcFp8, d_pad, d_pad8);
}

size_t tc_ref_bytes(int N, int d) {
    const int d_pad = (d + 63) / 64 * 64, d_pad8 = (d + 127) / 128 * 128;
    const size_t lo = kind_fits(kTcBf16x3, d_pad, d_pad8) ? (size_t)N * d_pad * 2 : 0;
    const size_t f8 = kind_fits(kTcFp8, d_pad, d_pad8) ? (size_t)N * d_pad8 + (size_t)N * 32 : 0;
    const size_t ns = (size_t)(N + TC_SAMPLE_EVERY - 1) / TC_SAMPLE_EVERY;
    return (size_t)N * d_pad * 2 + (size_t)N * d_pad * 4 + (size_t)N * TC_NK * 2 +
           (size_t)d_pad * 4 + lo + f8 + ns * (d_pad + TC_NK) * 2 + 14 * 256;
}

static size_t fallback_bytes(int N, int Q, int d, int k, int num_sms) {
    const long long ldf = (Q + 3) / 4 * 4;
    return (size_t)d * ldf * 4 + (size_t)k * ldf * 8 + exact_scratch_bytes(N, Q, d, k, num_sms) +
           4 * 256;
}

size_t tc_scratch_bytes(int N, int Q, int d, int k, int num_sms) {
    TcPlan p = plan_tc(N, Q, d, k, num_sms);
    // the point sample's pass 1 may choose other splits: room for either
    p.splits1 = std::max(p.splits1, plan_tc(N, Q, d, k, num_sms, true).splits1);
    const size_t rows = (size_t)p.qtiles * TC_QT;
    size_t b = rows * p.d_pad * 2 * 2 + rows * p.d_pad8 + (size_t)Q * 4 * 10 + 64;
    b += (size_t)TP_LISTS * p.splits1 * Q * TC_KS * 4;
    b += (size_t)Q * p.cmax * 8;
    b += fallback_bytes(N, Q, d, k, num_sms);   // worst case: every query uncertified
    return b + 24 * 256;
}

int tc_prepare_ref(const TcRefView &v, const float *ref, int N, long long ldr, int d,
                   cudaStream_t st) {
    if (cudaMemsetAsync(v.rmax_bits, 0, 3 * 256, st) != cudaSuccess) return kErrCuda;
    if (v.state) *v.state = TcRefState{};
    const int n_tiles = (N + TP_BN - 1) / TP_BN;
    int rc = tc_center_from_tiles(v, ref, N, ldr, d, contiguous_tiles(n_tiles), kCenterStride,
                                  st);
    if (rc == kOk) rc = tc_prepare_ref_tiles(v, ref, N, ldr, d, 0, contiguous_tiles(n_tiles), st);
    if (rc != kOk || !v.sampB || !v.sampN) return rc;
    // the point sample of pass 1: every 16th point's rows
    const int ns = (N + TC_SAMPLE_EVERY - 1) / TC_SAMPLE_EVERY;
    const int d_pad = (d + 63) / 64 * 64;
    tc_sample_rows_kernel<<<(ns + 7) / 8, 256, 0, st>>>(v.refB, v.refN, ns, d_pad, v.sampB,
                                                        v.sampN);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrLaunch;
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
    tc_prep_ref_kernel<<<tiles.units * 2, 32 * TC_PREP_WARPS, 0, st>>>(
        ref, N, ldr, d, d_pad, tile0, tiles, v.center, v.refB, v.refT, v.refN, v.rmax_bits,
        v.absmax_bits);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrLaunch;
}

int tc_tile_points() { return TP_BN; }

TcRefView tc_carve_ref(void *mem, int N, int d, TcRefState *state) {
    const int d_pad = (d + 63) / 64 * 64, d_pad8 = (d + 127) / 128 * 128;
    Carve cv{static_cast<unsigned char *>(mem), 0, 0};
    TcRefView v;
    v.refB = cv.take<__nv_bfloat16>((size_t)N * d_pad);
    v.refT = cv.take<float>((size_t)N * d_pad);
    v.refN = cv.take<__nv_bfloat16>((size_t)N * TC_NK);
    // three words 256 bytes apart, cleared together by tc_prepare_ref
    v.rmax_bits = cv.take<unsigned>(64);
    v.absmax_bits = cv.take<unsigned>(64);
    v.resid8_bits = cv.take<unsigned>(64);
    v.center = cv.take<float>(d_pad);
    v.refBlo = kind_fits(kTcBf16x3, d_pad, d_pad8) ? cv.take<__nv_bfloat16>((size_t)N * d_pad)
                                                   : nullptr;
    const bool f8 = kind_fits(kTcFp8, d_pad, d_pad8);
    v.ref8 = f8 ? cv.take<unsigned char>((size_t)N * d_pad8) : nullptr;
    v.refN8 = f8 ? cv.take<unsigned char>((size_t)N * 32) : nullptr;
    const size_t ns = (size_t)(N + TC_SAMPLE_EVERY - 1) / TC_SAMPLE_EVERY;
    v.sampB = cv.take<__nv_bfloat16>(ns * d_pad);
    v.sampN = cv.take<__nv_bfloat16>(ns * TC_NK);
    v.state = state;
    if (state) *state = TcRefState{};
    return v;
}

namespace {

// The split-BF16 lo parts of the reference set, once per prepared set.
int ensure_ref_lo(const TcRun &r, cudaStream_t st) {
    TcRefState *s = r.R.state;
    if (!r.R.refBlo || !s) return kErrUnsupported;
    if (s->lo_ready) return kOk;
    const long long n = (long long)r.P.N * r.d_pad;
    tc_ref_lo_kernel<<<(unsigned)((n / 4 + 255) / 256), 256, 0, st>>>(r.R.refT, n, r.P.d, r.d_pad,
                                                                     r.R.center, r.R.refBlo);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    s->lo_ready = true;
    return kOk;
}

// The FP8 scales of the reference set, once per prepared set: reads back
// the set's largest |r - c| and ||r - c||^2 (one synchronisation) for the
// scale s_r = 2^floor(log2(448 / max|r - c|)) and the norm-step unit
// kappa = 2^ceil(log2(s_r max||r - c||^2 / 896)) (so the norm needs at most
// two saturated parts before the remainder).
int ensure_ref_f8_scale(const TcRun &r, cudaStream_t st, unsigned *host_tmp) {
    TcRefState *s = r.R.state;
    if (!r.R.ref8 || !s) return kErrUnsupported;
    if (s->f8_scaled) return kOk;
    if (cudaMemcpyAsync(host_tmp, r.R.rmax_bits, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(host_tmp + 1, r.R.absmax_bits, 4, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return kErrCuda;
    float r2, am;
    std::memcpy(&r2, host_tmp, 4);
    std::memcpy(&am, host_tmp + 1, 4);
    if (!(am > 0.f) || !std::isfinite(am) || !std::isfinite(r2)) return kErrUnsupported;
    s->absmax_r = am;
    s->r2max = r2;
    s->s_r = pow2_floor(448.0 / am);
    s->kappa = pow2_ceil(std::max(1e-30, (double)s->s_r * r2 / 896.0));
    s->resid8 = 0.f;
    s->f8_scaled = true;
    return kOk;
}

// The FP8 copy of the reference set (scales from ensure_ref_f8_scale),
// once per prepared set; reads back the norm split's largest residual.
int ensure_ref_f8(const TcRun &r, cudaStream_t st, unsigned *host_tmp) {
    TcRefState *s = r.R.state;
    if (!r.R.ref8 || !s) return kErrUnsupported;
    if (s->f8_ready) return kOk;
    int rc = ensure_ref_f8_scale(r, st, host_tmp);
    if (rc != kOk) return rc;
    if (cudaMemsetAsync(r.R.resid8_bits, 0, 4, st) != cudaSuccess) return kErrCuda;
    constexpr int W = 8;
    tc_pack_ref_f8_kernel<<<(r.P.N + W - 1) / W, W * 32, 0, st>>>(
        r.R.refT, r.P.N, r.P.d, r.d_pad, r.d_pad8, r.R.center, s->s_r, s->kappa, r.R.ref8,
        r.R.refN8, r.R.resid8_bits);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    if (cudaMemcpyAsync(host_tmp, r.R.resid8_bits, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return kErrCuda;
    std::memcpy(&s->resid8, host_tmp, 4);
    s->f8_ready = true;
    return kOk;
}

// Scan of the reference tiles [tile_base + tiles.tile(u)) for the Q queries
// of the operand copies qB (BF16 hi), qBlo (lo) or q8 (FP8), in `kind`.
// MODE 1 (emit) with thresholds thr, lists of stride cmax; MODE 0 (sample)
// into r.p1.
template <int MODE>
int launch_scan(const TcRun &r, cudaStream_t st, int kind, const __nv_bfloat16 *qB,
                const __nv_bfloat16 *qBlo, const unsigned char *q8, int Q, const float *thr,
                int cmax, int tile_base, const TileRuns &tiles, int n_splits) {
    const TcProblem &P = r.P;
    if (!kind_fits(kind, r.d_pad, r.d_pad8)) return kErrUnsupported;
    const TcOp op = tc_op(kind, r.d_pad, r.d_pad8);
    CUtensorMap tmA, tmA2, tmB, tmB2, tmN;
    bool ok;
    if (kind == kTcFp8) {
        ok = encode_u8_kmajor(&tmA, q8, Q, r.d_pad8) &&
             encode_u8_kmajor(&tmB, r.R.ref8, P.N, r.d_pad8) &&
             encode_norm_rows(&tmN, r.R.refN8, P.N, true);
        tmA2 = tmA;
        tmB2 = tmB;
    } else if (MODE == 0 && r.p1_every > 0) {
        // the point sample: rows 0, m, 2m, ... of the every-16th-point copy
        ok = encode_bf16_kmajor(&tmA, qB, Q, r.d_pad) &&
             encode_2d(&tmB, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, r.R.sampB, (uint64_t)r.d_pad,
                       (uint64_t)r.p1_rows, (uint64_t)r.p1_every * r.d_pad, TC_BK, TC_BM,
                       CU_TENSOR_MAP_SWIZZLE_128B) &&
             encode_2d(&tmN, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, r.R.sampN, (uint64_t)TC_NK,
                       (uint64_t)r.p1_rows, (uint64_t)r.p1_every * TC_NK, TC_NK, TC_BM,
                       CU_TENSOR_MAP_SWIZZLE_32B);
        tmA2 = tmA;
        tmB2 = tmB;
    } else {
        ok = encode_bf16_kmajor(&tmA, qB, Q, r.d_pad) &&
             encode_bf16_kmajor(&tmB, r.R.refB, P.N, r.d_pad) &&
             encode_norm_rows(&tmN, r.R.refN, P.N, false);
        if (kind == kTcBf16x3) {
            ok = ok && encode_bf16_kmajor(&tmA2, qBlo, Q, r.d_pad) &&
                 encode_bf16_kmajor(&tmB2, r.R.refBlo, P.N, r.d_pad);
        } else {
            tmA2 = tmA;
            tmB2 = tmB;
        }
    }
    if (!ok) return kErrTensorMap;
    TpArgs a;
    a.N = (MODE == 0 && r.p1_every > 0) ? r.p1_rows : P.N;
    a.Q = Q;
    a.kb = op.kb;
    a.ka = op.ka;
    a.stages = op.stages;
    a.items = op.items;
    a.tile_base = tile_base;
    a.tiles = tiles;
    a.n_splits = n_splits;
    a.thr = thr;
    a.thr_scale = kind == kTcFp8 ? r.scale : 1.f;
    if (kind == kTcFp8) {
        // c1 = s_q kappa, a power of two the e4m3 format holds exactly
        const unsigned char c1 = __nv_fp8_e4m3(r.s_q * r.R.state->kappa).__x;
        a.ones_word = 0x01010101u * c1;
    } else {
        a.ones_word = 0x3F803F80u;   // BF16 1.0, twice
    }
    a.p1 = r.p1;
    a.cand = r.cand;
    a.count = r.count;
    a.cmax = cmax;
    a.status = P.status;
    const dim3 grid(2 * ((Q + TC_QT - 1) / TC_QT), n_splits);
    auto go = [&](auto kern) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)TP_SMEM);
        if (e != cudaSuccess) return (int)kErrLaunch;
        kern<<<grid, TP_THREADS, TP_SMEM, st>>>(tmA, tmA2, tmB, tmB2, tmN, a);
        return cudaGetLastError() == cudaSuccess ? (int)kOk : (int)kErrLaunch;
    };
    switch (kind) {
        case kTcBf16x3: return go(knn_tc_pair_scan_kernel<MODE, kTcBf16x3>);
        case kTcFp8: return go(knn_tc_pair_scan_kernel<MODE, kTcFp8>);
        default: return go(knn_tc_pair_scan_kernel<MODE, kTcBf16>);
    }
}

// Emission scan of the reference tiles [tb, te).
int emit_scan(const TcRun &r, cudaStream_t st, int kind, int Q, const float *thr, int cmax,
              int tb, int te) {
    const int qtiles = (Q + TC_QT - 1) / TC_QT;
    // reference bytes a tile streams (operand rows + norm-step rows); a
    // split holds at most kSplitBytes of them: measured at 2^20 x 256 BF16
    // and 16384 queries, 15 splits of 36 MB read 0.93 GB per launch from
    // DRAM and 23 splits of 24 MB 0.63 GB (the set is 0.57 GB), in the same
    // time
    const size_t row = kind == kTcFp8 ? (size_t)r.d_pad8
                                      : (size_t)r.d_pad * 2 * (kind == kTcBf16x3 ? 2 : 1);
    const size_t tile_bytes = (size_t)TP_BN * (row + 32);
    const int max_tiles = (int)std::max<size_t>(1, kSplitBytes / tile_bytes);
    const int splits =
        choose_splits(qtiles, te - tb, 8, 2.0, std::max(1, r.P.num_sms / 2), max_tiles);
    return launch_scan<1>(r, st, kind, r.qB, r.qBlo, r.q8, Q, thr, cmax, tb,
                          contiguous_tiles(te - tb), splits);
}

TcBound run_bound(const TcRun &r, int kind) {
    const TcRefState *s = r.R.state;
    return bound_of(kind, r.P.d, r.d_pad, r.d_pad8, r.s_q, s ? s->s_r : 1.f, s ? s->resid8 : 0.f);
}

// Exact re-rank + certification of Q queries (tc_rerank_select_kernel,
// tc_rerank_gather_kernel, tc_rerank_certify_kernel) whose candidate lists
// (from a scan of `kind`) have stride cmax.
int rerank(const TcRun &r, cudaStream_t st, int kind, int Q, int cmax, const float *qry,
           long long ldq, const float *qn, const float *thr, const float *thr_raw,
           float *out_dist, int *out_idx, long long ld_out, int *fail, bool final_pass) {
    const TcProblem &P = r.P;
    if (cudaMemsetAsync(r.nfail, 0, 2 * sizeof(int), st) != cudaSuccess) return kErrCuda;
    int cpow = 32;
    while (cpow < cmax) cpow <<= 1;
    const size_t gsmem = tc_rr_gather_bytes(r.d_pad);
    const size_t csmem = (size_t)cpow * 8;
    RrBounds rb;
    rb.cur = run_bound(r, kind);
    rb.a_scale = kind == kTcFp8 ? 1.f / r.scale : 1.f;
    // the bound statistic runs in its own instantiation, only when asked for
    auto gather = P.bound_stat ? tc_rerank_gather_kernel<true> : tc_rerank_gather_kernel<false>;
    // one fixed limit for every launch, so that calls from several host
    // threads never lower it under each other
    if (gsmem > kRerankSmem || csmem > kRerankSmem ||
        cudaFuncSetAttribute(gather, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kRerankSmem) != cudaSuccess ||
        cudaFuncSetAttribute(tc_rerank_certify_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kRerankSmem) != cudaSuccess)
        return kErrLaunch;
    tc_rerank_select_kernel<<<Q, 32, 0, st>>>(r.cand, r.count, cmax, Q, P.k, qn, r.R.rmax_bits,
                                              thr, thr_raw, rb, r.d_pad, final_pass ? 1 : 0, fail,
                                              r.nfail, r.retry, r.retry_f, r.retry_s, r.cand_total,
                                              r.nsel);
    gather<<<Q, 32, gsmem, st>>>(r.R.refT, P.d, r.d_pad, qry, ldq, qn, r.R.rmax_bits, thr, rb,
                                 r.cand, r.nsel, cmax, Q, P.bound_stat);
    tc_rerank_certify_kernel<<<Q, 32, csmem, st>>>(r.cand, r.nsel, r.count, cmax, Q, P.k,
                                                   r.d_pad, qn, r.R.rmax_bits, thr, rb, out_dist,
                                                   out_idx, ld_out, fail, r.nfail, r.retry,
                                                   r.retry_f, r.retry_s);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrLaunch;
}

// FP8 query scale (reads back the batch's largest |q - c|): s_q =
// 2^floor(log2(min(224 / max|q - c|, 256 / kappa))), so that -2 s_q q and
// the ones value c1 = s_q kappa both fit e4m3.
int fp8_query_scale(TcRun &r, cudaStream_t st, unsigned *dev_absmax, unsigned *host_tmp) {
    if (cudaMemcpyAsync(host_tmp, dev_absmax, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return kErrCuda;
    float aq;
    std::memcpy(&aq, host_tmp, 4);
    const TcRefState *s = r.R.state;
    const double lim = std::min(aq > 0.f ? 224.0 / aq : 1e30, 256.0 / s->kappa);
    r.s_q = pow2_floor(lim);
    const double c1 = (double)r.s_q * s->kappa;
    if (!(c1 >= 1.0 / 512.0) || !std::isfinite(aq)) return kErrUnsupported;
    r.scale = r.s_q * s->s_r;
    return kOk;
}

}  // namespace

TileRuns tc_sample_runs(int N, int Q, int d, int k, int num_sms) {
    return plan_tc(N, Q, d, k, num_sms).sample;
}

int tc_run_begin(const TcProblem &P, const TcRefView &R, cudaStream_t st, TcRun &r) {
    if (!tc_supported(P.N, P.Q, P.d, P.k)) return kErrUnsupported;
    const bool points = P.point_sample && R.sampB && R.sampN;
    const TcPlan p = plan_tc(P.N, P.Q, P.d, P.k, P.num_sms, points);
    r.P = P;
    r.R = R;
    r.p1_rows = p.p1_rows;
    r.p1_every = p.p1_every;
    r.d_pad = p.d_pad;
    r.d_pad8 = p.d_pad8;
    r.qtiles = p.qtiles;
    r.n_tiles2 = p.n_tiles2;
    r.splits1 = p.splits1;
    r.sample = p.sample;
    r.cmax = p.cmax;
    r.kind = kTcBf16;
    r.s_q = 1.f;
    r.scale = 1.f;
    const bool fp8 = P.request == kTcReqFp8;
    if (fp8 && (!R.ref8 || !R.state || !P.host_tmp)) return kErrUnsupported;
    Carve cv{static_cast<unsigned char *>(P.scratch), 0, P.scratch_bytes};
    const size_t rows = (size_t)p.qtiles * TC_QT;
    r.qB = cv.take<__nv_bfloat16>(rows * p.d_pad);
    r.qBlo = cv.take<__nv_bfloat16>(rows * p.d_pad);
    r.q8 = cv.take<unsigned char>(rows * p.d_pad8);
    r.qn = cv.take<float>(P.Q);
    r.thr = cv.take<float>(P.Q);
    r.thr_raw = cv.take<float>(P.Q);
    r.retry = cv.take<float>(P.Q);
    r.retry_f = cv.take<float>(P.Q);
    r.retry_s = cv.take<float>(P.Q);
    r.count = cv.take<int>(P.Q);
    r.fail = cv.take<int>(P.Q);
    r.fail2 = cv.take<int>(P.Q);
    r.nsel = cv.take<int>(P.Q);
    r.nfail = cv.take<int>(4);
    r.nwide = cv.take<int>(4);   // [0] predicted overflows, [2] query max |q - c| bits
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

    // queries: norms (and their largest |q - c|) + BF16 K-major copy of -2 q
    if (cudaMemsetAsync(r.nwide, 0, 4 * sizeof(int), st) != cudaSuccess) return kErrCuda;
    tc_norms_kernel<<<(P.Q + 255) / 256, 256, 0, st>>>(
        P.qry, P.Q, P.ldq, P.d, R.center, r.qn, nullptr,
        fp8 ? reinterpret_cast<unsigned *>(r.nwide + 2) : nullptr);
    tc_pack_kernel<<<dim3((P.Q + 31) / 32, p.d_pad / 32), dim3(32, 8), 0, st>>>(
        P.qry, P.Q, P.ldq, P.d, p.d_pad, R.center, -2.0f, r.qB);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    r.want_fp8 = false;
    if (fp8) {
        // the reference set's and the queries' FP8 scales only: the sample
        // pass runs in BF16 and decides whether pass 2 runs in FP8, and the
        // FP8 copies are made then (tc_run_pass1)
        unsigned *host_tmp = reinterpret_cast<unsigned *>(P.host_tmp);
        int rc = ensure_ref_f8_scale(r, st, host_tmp);
        if (rc == kOk) rc = fp8_query_scale(r, st, reinterpret_cast<unsigned *>(r.nwide + 2), host_tmp);
        if (rc != kOk) return rc;
        r.want_fp8 = true;
    }
    if (P.timer) P.timer->mark(st, kPhaseTcPrepQuery);
    if (cudaMemsetAsync(r.cand_total, 0, sizeof(unsigned long long), st) != cudaSuccess)
        return kErrCuda;
    return kOk;
}

int tc_run_pass1(TcRun &r, cudaStream_t st) {
    const TcProblem &P = r.P;
    // the sample pass runs in BF16 for every request: its values are close
    // enough to the exact ones to set thresholds and to predict whether a
    // pass 2 of another kind would overflow its lists
    int rc = launch_scan<0>(r, st, kTcBf16, r.qB, r.qBlo, r.q8, P.Q, nullptr, r.cmax, 0, r.sample,
                            r.splits1);
    if (rc != kOk) return rc;
    if (P.timer) P.timer->mark(st, kPhaseTcPass1);
    // TP_LISTS lists (column ranges) per pair and split; resets the counts
    const bool lo_ok = kind_fits(kTcBf16x3, r.d_pad, r.d_pad8) && r.R.refBlo && r.R.state;
    const int force = P.force_kind;
    const bool forced = (force == kTcBf16) || (force == kTcBf16x3 && lo_ok) ||
                        (force == kTcFp8 && r.want_fp8);
    const bool probe = !forced && P.host_tmp && ((P.adaptive && lo_ok) || r.want_fp8);
    if (probe && cudaMemsetAsync(r.nwide, 0, 2 * sizeof(int), st) != cudaSuccess) return kErrCuda;
    const TcBound b16 = run_bound(r, kTcBf16);
    tc_threshold_kernel<<<(P.Q + 255) / 256, 256, 0, st>>>(
        r.p1, TP_LISTS * r.splits1, P.Q, r.qn, r.R.rmax_bits, b16, b16,
        r.want_fp8 ? run_bound(r, kTcFp8) : b16, r.thr, r.thr_raw, r.count,
        probe ? r.nwide : nullptr);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    r.kind = kTcBf16;
    int wide16 = 0, wide8 = 0;
    if (probe) {
        if ((rc = read_count(r.nwide, P.host_tmp, st, wide16, 2)) != kOk) return rc;
        wide8 = P.host_tmp[1];
    }
    if (forced) {
        // the caller's kind: predicted fit or not
        wide16 = force == kTcBf16x3 ? P.Q : 0;
        wide8 = force == kTcFp8 ? 0 : P.Q;
    }
    if (probe || forced) {
        if (r.want_fp8 && 2 * wide8 <= P.Q) {
            // FP8 pass 2: the FP8 copies (the prediction above took the
            // norm split's residual as 0: it only picks the kind), then
            // thresholds T + E_bf16 + E_fp8 (the sample value is a BF16 one)
            if ((rc = ensure_ref_f8(r, st, reinterpret_cast<unsigned *>(P.host_tmp))) != kOk)
                return rc;
            tc_pack_f8_kernel<<<dim3((P.Q + 31) / 32, r.d_pad8 / 32), dim3(32, 8), 0, st>>>(
                P.qry, P.Q, P.ldq, P.d, r.d_pad8, r.R.center, -2.0f * r.s_q, r.q8);
            tc_rethreshold_kernel<<<(P.Q + 255) / 256, 256, 0, st>>>(
                r.thr_raw, P.Q, r.qn, r.R.rmax_bits, run_bound(r, kTcFp8), b16, 1, r.thr);
            if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
            r.kind = kTcFp8;
        } else if ((P.adaptive || forced) && lo_ok && 2 * wide16 > P.Q) {
            // most lists expected to overflow in BF16: pass 2 runs in split
            // BF16 (thresholds re-derived from the sample)
            if ((rc = ensure_ref_lo(r, st)) != kOk) return rc;
            tc_pack_kernel<<<dim3((P.Q + 31) / 32, r.d_pad / 32), dim3(32, 8), 0, st>>>(
                P.qry, P.Q, P.ldq, P.d, r.d_pad, r.R.center, -2.0f, r.qB, r.qBlo);
            tc_rethreshold_kernel<<<(P.Q + 255) / 256, 256, 0, st>>>(
                r.thr_raw, P.Q, r.qn, r.R.rmax_bits, run_bound(r, kTcBf16x3), b16, 0, r.thr);
            if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
            r.kind = kTcBf16x3;
        }
    }
    if (P.timer) P.timer->mark(st, kPhaseTcThreshold);
    return kOk;
}

int tc_run_pass2(TcRun &r, int tile_begin, int tile_end, cudaStream_t st) {
    tile_end = std::min(tile_end, r.n_tiles2);
    if (tile_begin >= tile_end) return kOk;
    const int rc = emit_scan(r, st, r.kind, r.P.Q, r.thr, r.cmax, tile_begin, tile_end);
    if (rc == kOk && r.P.timer) r.P.timer->mark(st, kPhaseTcPass2);
    return rc;
}

int tc_run_rerank_piece(TcRun &r, cudaStream_t st) {
    const TcProblem &P = r.P;
    if (!r.pieces) {
        // the running lists take the exact-fallback scratch, which nothing
        // uses before the certification.  tc_scratch_bytes sizes that
        // scratch for the fallback's query copy (d * Q floats) and result
        // keys (k * Q), so Q * k keys plus Q flags always fit; the check
        // only guards a caller-sized scratch, for which the full re-rank
        // then runs in tc_run_finish instead
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
    const int kcap = P.k <= 32 ? 32 : (P.k <= 64 ? 64 : (P.k <= 128 ? 128 : 256));
    const size_t smem = (size_t)r.d_pad * 4 + (size_t)TC_RR_NBUF * TC_RR_BUF * 4 +
                        (size_t)(kcap + EX_CB) * 8;
    if (smem > kRerankSmem) return kErrUnsupported;
    auto go = [&](auto kern) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kRerankSmem) != cudaSuccess)
            return (int)kErrLaunch;
        kern<<<P.Q, 32, smem, st>>>(r.R.refT, P.d, r.d_pad, P.qry, P.ldq, r.cand, r.count, r.cmax,
                                    P.k, r.run_keys, r.done);
        return cudaGetLastError() == cudaSuccess ? (int)kOk : (int)kErrLaunch;
    };
    if (kcap == 32) return go(tc_rerank_piece_kernel<32>);
    if (kcap == 64) return go(tc_rerank_piece_kernel<64>);
    if (kcap == 128) return go(tc_rerank_piece_kernel<128>);
    return go(tc_rerank_piece_kernel<256>);
}

int tc_run_finish(TcRun &r, cudaStream_t st, int *host_stats) {
    const TcProblem &P = r.P;
    PhaseTimer *tm = P.timer;
    int *host_tmp = host_stats + 2;
    host_stats[0] = host_stats[1] = 0;
    host_stats[4] = host_stats[5] = 0;
    host_stats[6] = r.kind;
    host_stats[7] = -1;
    int rc = kOk;
    if (r.pieces) {
        // every candidate was re-ranked piece by piece: certify
        if (cudaMemsetAsync(r.nfail, 0, 2 * sizeof(int), st) != cudaSuccess) return kErrCuda;
        RrBounds rb;
        rb.cur = run_bound(r, r.kind);
        rb.a_scale = 1.f;
        constexpr int W = 4;
        tc_certify_pieces_kernel<<<(P.Q + W - 1) / W, W * 32, 0, st>>>(
            r.count, r.cmax, r.qn, r.R.rmax_bits, r.thr, r.thr_raw, rb, r.run_keys, P.Q, P.k,
            r.d_pad, P.out_dist, P.out_idx, P.ld_out, r.fail, r.nfail, r.retry, r.retry_f,
            r.retry_s, r.cand_total);
        if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    } else {
        rc = rerank(r, st, r.kind, P.Q, r.cmax, P.qry, P.ldq, r.qn, r.thr, r.thr_raw, P.out_dist,
                    P.out_idx, P.ld_out, r.fail, false);
    }
    if (rc != kOk) return rc;
    if (tm) tm->mark(st, kPhaseTcRerank);
    if (cudaMemcpyAsync(host_stats + 4, r.cand_total, sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return kErrCuda;
    int nf = 0;
    if ((rc = read_count(r.nfail, host_tmp, st, nf, 2)) != kOk) return rc;
    const int n_over = host_tmp[1];
    host_stats[0] = nf;
    if (nf == 0) return kOk;

    // second chance: the uncertified queries, compacted, scanned again with
    // thresholds that certify (list overflows excepted).  Kind: BF16 after
    // an FP8 scan, else the first scan's kind -- split BF16 instead of BF16
    // when most failures are overflowing lists (BF16 too coarse for them).
    const bool lo_ok = kind_fits(kTcBf16x3, r.d_pad, r.d_pad8) && r.R.refBlo && r.R.state;
    int kind2 = r.kind == kTcFp8 ? kTcBf16 : r.kind;
    if (kind2 == kTcBf16 && lo_ok && 2 * n_over > nf) kind2 = kTcBf16x3;
    host_stats[7] = kind2;
    if (kind2 == kTcBf16x3 && (rc = ensure_ref_lo(r, st)) != kOk) return rc;
    gather_queries_kernel<<<dim3((nf + 127) / 128, P.d), 128, 0, st>>>(P.qry, P.ldq, P.d, r.fail,
                                                                       nf, r.qsub, r.ldf);
    tc_norms_kernel<<<(nf + 255) / 256, 256, 0, st>>>(r.qsub, nf, r.ldf, P.d, r.R.center, r.qn,
                                                      nullptr);
    tc_pack_kernel<<<dim3((nf + 31) / 32, r.d_pad / 32), dim3(32, 8), 0, st>>>(
        r.qsub, nf, r.ldf, P.d, r.d_pad, r.R.center, -2.0f, r.qB,
        kind2 == kTcBf16x3 ? r.qBlo : nullptr);
    tc_retry_prep_kernel<<<(nf + 255) / 256, 256, 0, st>>>(
        r.fail, nf, r.retry, r.retry_f, r.retry_s, r.qn, r.R.rmax_bits, run_bound(r, kind2), r.thr,
        r.count);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    // the compacted queries share the whole list buffer (Q * cmax entries)
    const int cmax2 = (int)std::min<long long>(
        kTcCmaxRetry, std::max<long long>(r.cmax, (long long)P.Q * r.cmax / nf));
    if ((rc = emit_scan(r, st, kind2, nf, r.thr, cmax2, 0, r.n_tiles2)) != kOk) return rc;
    if (tm) tm->mark(st, kPhaseTcRetryScan);
    rc = rerank(r, st, kind2, nf, cmax2, r.qsub, r.ldf, r.qn, r.thr, nullptr, r.sd, r.si, r.ldf,
                r.fail2, true);
    if (rc != kOk) return rc;
    if (tm) tm->mark(st, kPhaseTcRetryRerank);
    int nf2 = 0;
    if ((rc = read_count(r.nfail, host_tmp, st, nf2)) != kOk) return rc;
    host_stats[1] = nf2;
    if (nf2 > 0) {
        // still uncertified (list overflow): the exact kernel answers them.
        // They are gathered once more (fail2 indexes the compacted batch)
        // into the candidate buffer, which nothing reads any more, when it
        // holds their queries and answers; else the exact kernel
        // recomputes the whole compacted batch.
        const int ld3 = (nf2 + 3) / 4 * 4;
        const size_t need = (size_t)ld3 * (P.d + 2 * (size_t)P.k) * 4;
        const bool narrow = nf2 < nf && need <= (size_t)P.Q * r.cmax * sizeof(unsigned long long);
        float *q3 = reinterpret_cast<float *>(r.cand);
        float *d3 = q3 + (size_t)P.d * ld3;
        int *i3 = reinterpret_cast<int *>(d3 + (size_t)P.k * ld3);
        if (narrow) {
            gather_queries_kernel<<<dim3((nf2 + 127) / 128, P.d), 128, 0, st>>>(
                r.qsub, r.ldf, P.d, r.fail2, nf2, q3, ld3);
            if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
        }
        const int nx = narrow ? nf2 : nf;
        const long long per_split = (long long)nx * std::min(P.k, 256) * 8;
        const int splits = (int)std::max<long long>(
            1, std::min<long long>(exact_plan_splits(P.N, nx, P.d, P.k, P.num_sms),
                                   (long long)(r.xcap / per_split)));
        ExactProblem x;
        x.ref = P.ref;
        x.N = P.N;
        x.ldr = P.ldr;
        x.qry = narrow ? q3 : r.qsub;
        x.Q = nx;
        x.ldq = narrow ? ld3 : r.ldf;
        x.d = P.d;
        x.k = P.k;
        x.out_dist = narrow ? d3 : r.sd;
        x.out_idx = narrow ? i3 : r.si;
        x.ld_out = narrow ? ld3 : r.ldf;
        x.scratch = r.xs;
        x.scratch_bytes = r.xcap;
        x.status = P.status;
        x.num_sms = P.num_sms;
        x.force_splits = splits;
        x.timer = nullptr;
        if ((rc = launch_exact(x, st)) != kOk) return rc;
        if (narrow) {
            scatter_results_kernel<<<dim3((nf2 + 127) / 128, P.k), 128, 0, st>>>(
                d3, i3, ld3, r.fail2, nf2, r.sd, r.si, r.ldf);
            if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
        }
    }
    scatter_results_kernel<<<dim3((nf + 127) / 128, P.k), 128, 0, st>>>(
        r.sd, r.si, r.ldf, r.fail, nf, P.out_dist, P.out_idx, P.ld_out);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;
    if (tm) tm->mark(st, kPhaseTcFallback);
    return kOk;
}

int tc_prepare_extras(const TcRefView &v, int N, int d, cudaStream_t st, int *host_tmp) {
    TcRun r;
    r.P = TcProblem{};
    r.P.N = N;
    r.P.d = d;
    r.R = v;
    r.d_pad = (d + 63) / 64 * 64;
    r.d_pad8 = (d + 127) / 128 * 128;
    int rc = v.refBlo ? ensure_ref_lo(r, st) : kOk;
    if (rc == kOk && v.ref8) rc = ensure_ref_f8(r, st, reinterpret_cast<unsigned *>(host_tmp));
    if (rc == kOk && cudaStreamSynchronize(st) != cudaSuccess) rc = kErrCuda;
    return rc;
}

int launch_tc(const TcProblem &P, const TcRefView &R, cudaStream_t st, int *host_stats) {
    TcRun r;
    TcProblem p = P;
    if (!p.host_tmp) p.host_tmp = host_stats + 2;
    int rc = tc_run_begin(p, R, st, r);
    if (rc == kOk) rc = tc_run_pass1(r, st);
    if (rc == kOk) rc = tc_run_pass2(r, 0, r.n_tiles2, st);
    if (rc == kOk) rc = tc_run_finish(r, st, host_stats);
    return rc;
}

}  // namespace knnb200
