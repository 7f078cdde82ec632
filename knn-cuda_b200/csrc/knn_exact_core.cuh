// knn_exact_core.cuh -- device building blocks of the fused exact FP32 k-NN
// kernels (single problem: knn_exact.cu; many problems in one persistent
// launch: knn_batched.cu).  See knn_exact.cu for the algorithm.
#pragma once

#include "knn_common.cuh"

namespace knnb200 {

constexpr int EX_BR = 256;       // reference points per tile
constexpr int EX_BD = 16;        // dimensions per pipeline stage
constexpr int EX_CB = 128;       // candidate slots per query (one half tile)
constexpr int EX_WARPS = 16;     // consumer warps
constexpr int EX_QPW = 4;        // queries per warp for k <= 128
constexpr int EX_QPW_K256 = 2;   // queries per warp for 128 < k <= 256
constexpr int EX_THREADS = (EX_WARPS + 1) * 32;
constexpr int EX_STAGES = 4;

template <int QPW, int KCAP>
struct ExCfg {
    static constexpr int BQ = QPW * EX_WARPS;
    // query slab of a stage: each query value stored twice, (q, q), so a
    // 64-bit shared load yields a ready packed operand
    static constexpr int Q_FLOATS = EX_BD * 2 * BQ;
    static constexpr int R_FLOATS = EX_BD * EX_BR;
    static constexpr int STAGE_FLOATS = Q_FLOATS + R_FLOATS;
    static constexpr int STAGE_BYTES = STAGE_FLOATS * 4;
    static constexpr int REGION = KCAP + EX_CB;   // keys per query: list + candidates
    static constexpr size_t LIST_BYTES = (size_t)BQ * REGION * 8;
    static constexpr size_t BAR_OFFSET = (size_t)EX_STAGES * STAGE_BYTES + LIST_BYTES;
    static constexpr size_t SMEM = 1024 + BAR_OFFSET + 2 * EX_STAGES * 8 + 16;
    static_assert(STAGE_BYTES % 1024 == 0, "stage alignment");
    static_assert(SMEM <= 232448, "shared memory per CTA");
    static_assert(KCAP % 32 == 0 && (KCAP & (KCAP - 1)) == 0, "KCAP power of two >= 32");
};

KNN_DI void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(EX_WARPS * 32) : "memory"); }

// Number of elements of the sorted array L[0..n) (n a power of two) below x.
template <int n>
KNN_DI int rank_pow2(const unsigned long long *L, unsigned long long x) {
    int pos = 0;
#pragma unroll
    for (int step = n / 2; step >= 1; step >>= 1)
        if (L[pos + step - 1] < x) pos += step;
    return pos + (L[pos] < x ? 1 : 0);
}

// Ascending bitonic sort of 128 keys held by one warp, four per lane
// (element e = b * 32 + lane in v[b]): lane partners by shuffle, register
// partners in place.
KNN_DI void warp_sort128(unsigned long long (&v)[4], int lane) {
#pragma unroll
    for (int size = 2; size <= 128; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= 32) {
                const int rs = stride >> 5;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    if (b & rs) continue;
                    const bool up = (((b << 5) | lane) & size) == 0;
                    const unsigned long long x = v[b], y = v[b | rs];
                    const bool sw = (x > y) == up;
                    v[b] = sw ? y : x;
                    v[b | rs] = sw ? x : y;
                }
            } else {
                const bool lower = (lane & stride) == 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const bool up = (((b << 5) | lane) & size) == 0;
                    const unsigned long long x = v[b];
                    const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, stride);
                    const unsigned long long mn = x < y ? x : y, mx = x < y ? y : x;
                    v[b] = (lower == up) ? mn : mx;
                }
            }
        }
    }
}

// Merge c (<= EX_CB) unsorted candidate keys (L[KCAP .. KCAP+c)) into the
// sorted list L[0..k) held by one warp.  The candidates are sorted in
// registers and written back sorted; then every key's final position is its
// index plus its rank in the other sorted array (binary search).  Keys are
// unique (distinct indices), so the positions form a permutation; positions
// >= k are dropped.
template <int KCAP>
KNN_DI void warp_merge(unsigned long long *L, int c, int k, int lane) {
    constexpr int LPL = KCAP / 32;
    constexpr int CPL = EX_CB / 32;
    static_assert(CPL == 4, "warp_sort128 holds four keys per lane");
    unsigned long long *C = L + KCAP;
    unsigned long long lv[LPL], cv[CPL];
#pragma unroll
    for (int b = 0; b < CPL; ++b) {
        const int t = b * 32 + lane;
        cv[b] = t < c ? C[t] : kKeyInf;
    }
    warp_sort128(cv, lane);
#pragma unroll
    for (int a = 0; a < LPL; ++a) lv[a] = L[a * 32 + lane];
    __syncwarp();
#pragma unroll
    for (int b = 0; b < CPL; ++b) C[b * 32 + lane] = cv[b];
    __syncwarp();
    int lp[LPL], cp[CPL];
#pragma unroll
    for (int a = 0; a < LPL; ++a) lp[a] = a * 32 + lane + rank_pow2<EX_CB>(C, lv[a]);
#pragma unroll
    for (int b = 0; b < CPL; ++b) cp[b] = b * 32 + lane + rank_pow2<KCAP>(L, cv[b]);
    __syncwarp();
#pragma unroll
    for (int a = 0; a < LPL; ++a)
        if (lp[a] < k) L[lp[a]] = lv[a];
#pragma unroll
    for (int b = 0; b < CPL; ++b)
        if (b * 32 + lane < c && cp[b] < k) L[cp[b]] = cv[b];
    __syncwarp();
}

// Buffer fill of query i (warp-uniform), one byte per query.
KNN_DI int nbuf_get(uint32_t nb, int i) { return (int)((nb >> (8 * i)) & 0xffu); }
KNN_DI uint32_t nbuf_set(uint32_t nb, int i, int v) {
    return (nb & ~(0xffu << (8 * i))) | ((uint32_t)v << (8 * i));
}

// Merge query i's buffered candidates into its list (whose k-th key is the
// query's threshold tau).
template <int QPW, int KCAP>
KNN_DI void flush_query(unsigned long long *wl, uint32_t &nb, int i, int k, int lane) {
    constexpr int REGION = KCAP + EX_CB;
    const int c = nbuf_get(nb, i);
    if (c > 0) {
        warp_merge<KCAP>(wl + i * REGION, c, k, lane);
        nb = nbuf_set(nb, i, 0);
    }
}

// Merge every query's buffered candidates (end of a reference range).
// (Loops over queries are not unrolled: one inlined copy of the merge.)
template <int QPW, int KCAP>
KNN_DI void flush_all(unsigned long long *wl, uint32_t &nb, int k, int lane) {
    static_assert(QPW <= 4 && EX_CB < 256, "buffer fills packed in one word");
#pragma unroll 1
    for (int i = 0; i < QPW; ++i) flush_query<QPW, KCAP>(wl, nb, i, k, lane);
}

// Filter one half tile (4 reference points per lane) against each query's
// threshold tau (the k-th key of its list) and append the survivors to the
// query's candidate buffer.  The buffer is merged into the list only when
// this half tile's survivors would not fit: tau then lags the candidates
// seen, so more points pass, but merges become rare (the gap between them
// grows geometrically as the list tightens) instead of one per half tile
// that holds any survivor.  nb packs the warp-uniform buffer fills.
// d2(i, j) gives the squared distance of query i to the lane's j-th point.
// With LB, only keys >= lb[i] are selected: pass p of a k > 256 problem keeps
// the 256 smallest keys above the ones earlier passes returned.
template <int QPW, int KCAP, bool LB, typename D2>
KNN_DI void select_half_lb(unsigned long long *wl, uint32_t &nb, D2 d2, uint32_t rbase, int N,
                           int k, int lane, const unsigned long long (&lb)[QPW]) {
    constexpr int REGION = KCAP + EX_CB;
    unsigned long long tau[QPW];
#pragma unroll
    for (int i = 0; i < QPW; ++i) tau[i] = wl[i * REGION + k - 1];
    uint32_t pm[QPW];
    bool any = false;
#pragma unroll
    for (int i = 0; i < QPW; ++i) {
        pm[i] = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t idx = rbase + j;
            const unsigned long long key = make_key(d2(i, j), idx);
            bool p = (idx < (uint32_t)N) && key < tau[i];
            if (LB) p = p && key >= lb[i];
            pm[i] |= (p ? 1u : 0u) << j;
            any |= p;
        }
    }
    if (!__any_sync(0xffffffffu, any)) return;
    const unsigned lt = (1u << lane) - 1u;
    // queries whose buffer cannot take this half tile's survivors: merge first
    uint32_t full_mask = 0;
#pragma unroll
    for (int i = 0; i < QPW; ++i) {
        const int m_i = (int)__reduce_add_sync(0xffffffffu, (unsigned)__popc(pm[i]));
        if (nbuf_get(nb, i) + m_i > EX_CB) full_mask |= 1u << i;
    }
    if (full_mask) {
        __syncwarp();
#pragma unroll 1
        for (int i = 0; i < QPW; ++i)
            if ((full_mask >> i) & 1u) flush_query<QPW, KCAP>(wl, nb, i, k, lane);
    }
#pragma unroll
    for (int i = 0; i < QPW; ++i) {
        if (__ballot_sync(0xffffffffu, pm[i] != 0) == 0) continue;
        unsigned long long *cb = wl + i * REGION + KCAP;
        int c = nbuf_get(nb, i);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const bool p = (pm[i] >> j) & 1u;
            const unsigned m = __ballot_sync(0xffffffffu, p);
            if (p) cb[c + __popc(m & lt)] = make_key(d2(i, j), rbase + j);
            c += __popc(m);
        }
        nb = nbuf_set(nb, i, c);
    }
    __syncwarp();
}

template <int QPW, int KCAP, typename D2>
KNN_DI void select_half(unsigned long long *wl, uint32_t &nb, D2 d2, uint32_t rbase, int N,
                        int k, int lane) {
    const unsigned long long none[QPW] = {};
    select_half_lb<QPW, KCAP, false>(wl, nb, d2, rbase, N, k, lane, none);
}


// Consume the n_dchunks pipeline stages of one reference tile: the lane's
// QPW x 8 block of squared distances accumulates sum_d (r_d - q_d)^2 with a
// rounded sub and a fused multiply-add per dimension, in increasing d (the
// order of the reference's compute_distances loop, code/knncuda.cu:77-80).
// `it` is the running stage counter of the CTA's ring.  Returns false (warp-
// uniformly) if a wait timed out or another warp aborted.
template <int QPW, int KCAP>
KNN_DI bool consume_ref_tile(f32x2_t (&acc)[QPW][4], const float *stages, uint64_t *full,
                             uint64_t *empty, volatile int *abort_flag, int &it, int n_dchunks,
                             int warp, int lane, int *status) {
    using C = ExCfg<QPW, KCAP>;
#pragma unroll
    for (int i = 0; i < QPW; ++i)
#pragma unroll
        for (int p = 0; p < 4; ++p) acc[i][p] = 0ull;
    for (int dc = 0; dc < n_dchunks; ++dc, ++it) {
        const int s = it % EX_STAGES;
        const bool got = mbar_wait(&full[s], (it / EX_STAGES) & 1);
        // warp-uniform decision: every lane leaves together or none does.
        // No per-stage check of the abort flag: when another warp gives up,
        // the producer stops refilling and this wait ends by its time limit.
        if (__any_sync(0xffffffffu, !got)) {
            if (lane == 0) {
                atomicMax(status, (int)kDevTimeoutFull);
                *abort_flag = 1;
            }
            return false;
        }
        const float *qs = stages + (size_t)s * C::STAGE_FLOATS + warp * 2 * QPW;
        const float *rs = stages + (size_t)s * C::STAGE_FLOATS + C::Q_FLOATS + lane * 4;
#pragma unroll
        for (int dd = 0; dd < EX_BD; ++dd) {
            // 16-byte loads straight into packed pairs (x, y), (z, w)
            const ulonglong2 ra = *reinterpret_cast<const ulonglong2 *>(rs + dd * EX_BR);
            const ulonglong2 rb = *reinterpret_cast<const ulonglong2 *>(rs + dd * EX_BR + 128);
            const f32x2_t r0 = ra.x, r1 = ra.y, r2 = rb.x, r3 = rb.y;
            const f32x2_t *qp = reinterpret_cast<const f32x2_t *>(qs + dd * 2 * C::BQ);
#pragma unroll
            for (int i = 0; i < QPW; ++i) {
                const f32x2_t qq = qp[i];   // (q_i, q_i)
                f32x2_t t;
                t = f2_sub(r0, qq); acc[i][0] = f2_fma(t, t, acc[i][0]);
                t = f2_sub(r1, qq); acc[i][1] = f2_fma(t, t, acc[i][1]);
                t = f2_sub(r2, qq); acc[i][2] = f2_fma(t, t, acc[i][2]);
                t = f2_sub(r3, qq); acc[i][3] = f2_fma(t, t, acc[i][3]);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
    return true;
}

// Select both halves of a consumed tile (reference points rt*256 + ...).
template <int QPW, int KCAP, bool LB = false>
KNN_DI void select_tile(unsigned long long *wl, uint32_t &nb, f32x2_t (&acc)[QPW][4], int rt,
                        int N, int k, int lane, const unsigned long long (&lb)[QPW]) {
    const uint32_t rb0 = (uint32_t)rt * EX_BR + lane * 4;
    select_half_lb<QPW, KCAP, LB>(
        wl, nb,
        [&](int i, int j) { return (j & 1) ? f2_hi(acc[i][j >> 1]) : f2_lo(acc[i][j >> 1]); },
        rb0, N, k, lane, lb);
    select_half_lb<QPW, KCAP, LB>(
        wl, nb,
        [&](int i, int j) {
            return (j & 1) ? f2_hi(acc[i][2 + (j >> 1)]) : f2_lo(acc[i][2 + (j >> 1)]);
        },
        rb0 + 128, N, k, lane, lb);
}
template <int QPW, int KCAP>
KNN_DI void select_tile(unsigned long long *wl, uint32_t &nb, f32x2_t (&acc)[QPW][4], int rt,
                        int N, int k, int lane) {
    const unsigned long long none[QPW] = {};
    select_tile<QPW, KCAP, false>(wl, nb, acc, rt, N, k, lane, none);
}

// Number of elements of sorted A[0..n) below x.
KNN_DI int rank_sorted(const unsigned long long *A, int n, unsigned long long x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (A[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

}  // namespace knnb200
