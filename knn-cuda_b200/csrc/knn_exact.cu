// knn_exact.cu -- fused exact FP32 k-NN (direct form) for sm_100a.
//
// Replaces the reference chain compute_distances (code/knncuda.cu:20-91) ->
// modified_insertion_sort (:143-189) -> compute_sqrt (:200-205) with ONE
// kernel: the ref_nb x query_nb distance matrix never reaches HBM.
//
//   * A CTA owns BQ queries (one query tile) and one contiguous slice
//     ("split") of the reference set.  Reference tiles of 256 points x 16
//     dimensions and the matching 16 x BQ query slab are brought into shared
//     memory by TMA (one producer warp, a 4-stage mbarrier ring).
//   * 16 consumer warps; warp w owns QPW queries, lane l owns the 8
//     reference points {4l..4l+3, 128+4l..128+4l+3} of each tile, so every
//     lane accumulates a QPW x 8 block of squared distances in registers as
//     sum_d (r_d - q_d)^2 with one rounding per sub and one fused
//     multiply-add per dimension, in increasing d -- the arithmetic and
//     order of the reference's compute_distances inner loop
//     (code/knncuda.cu:77-80), so squared distances are bit-identical to it.
//   * Selection is warp-local.  Each query keeps its k smallest
//     (distance, index) keys sorted in shared memory; the k-th key is the
//     threshold.  After each half tile the warp ballots the keys below it
//     into a 128-slot candidate buffer, which is merged into the list only
//     when it would overflow (a register bitonic sort of the buffer, then
//     every key placed at its index plus its rank in the other array).
//     Ordering by the 64-bit key (distance bits, index) reproduces the
//     reference's tie rule: equal distances keep the lower index
//     (code/knncuda.cu:172, :178).
//   * With one split the kernel writes sqrt(distance) and the index straight
//     into the k x query_nb output; with several splits it writes each
//     split's sorted keys to scratch and knn_merge_splits_kernel merges them.
//   * k > 256 (the reference's insertion sort has no limit on k,
//     code/knncuda.cu:143-189) runs in passes over the whole set: pass p
//     keeps the 256 smallest keys at or above a per-query lower bound (one
//     more than the last key of pass p - 1) and writes output rows
//     256 p .. 256 p + 255.  Keys are unique, so the passes together return
//     exactly the k smallest keys in order, with the same distances and tie
//     order as a single pass.
#include <algorithm>
#include <cstdio>

#include "knn_exact_core.cuh"
#include "knn_kernels.h"

namespace knnb200 {

template <int QPW, int KCAP, bool LB>
__global__ void __launch_bounds__(EX_THREADS, 1)
    knn_exact_kernel(const __grid_constant__ CUtensorMap tm_ref,
                     const __grid_constant__ CUtensorMap tm_qry, ExactArgs a) {
    using C = ExCfg<QPW, KCAP>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float *stages = reinterpret_cast<float *>(base);
    unsigned long long *lists =
        reinterpret_cast<unsigned long long *>(base + (size_t)EX_STAGES * C::STAGE_BYTES);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + C::BAR_OFFSET);
    uint64_t *empty = full + EX_STAGES;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + EX_STAGES);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qtile = blockIdx.x, split = blockIdx.y;
    const int t0 = (int)((long long)a.n_rtiles * split / a.n_splits);
    const int t1 = (int)((long long)a.n_rtiles * (split + 1) / a.n_splits);
    const int total = (t1 - t0) * a.n_dchunks;

    if (threadIdx.x == 0) {
        for (int s = 0; s < EX_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], EX_WARPS);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == EX_WARPS) {
        // ---------------- producer warp: one thread issues all TMA loads ----
        if (lane == 0) {
            prefetch_tensormap(&tm_ref);
            prefetch_tensormap(&tm_qry);
            int issued = 0;
            for (int it = 0; it < total; ++it) {
                const int s = it % EX_STAGES;
                if (it >= EX_STAGES && !mbar_wait(&empty[s], ((it / EX_STAGES) - 1) & 1)) {
                    atomicMax(a.status, (int)kDevTimeoutEmpty);
                    *abort_flag = 1;
                    break;
                }
                if (*abort_flag) break;
                float *qs = stages + (size_t)s * C::STAGE_FLOATS;
                float *rs = qs + C::Q_FLOATS;
                const int rt = t0 + it / a.n_dchunks, dc = it % a.n_dchunks;
                mbar_arrive_expect_tx(&full[s], C::STAGE_BYTES);
                tma_load_2d(qs, &tm_qry, &full[s], qtile * 2 * C::BQ, dc * EX_BD);
                tma_load_2d(rs, &tm_ref, &full[s], rt * EX_BR, dc * EX_BD);
                issued = it + 1;
            }
            // Never leave with copies in flight: wait for the last issued stages.
            for (int it = max(0, issued - EX_STAGES); it < issued; ++it)
                if (!mbar_wait(&full[it % EX_STAGES], (it / EX_STAGES) & 1))
                    atomicMax(a.status, (int)kDevTimeoutDrain);
        }
        return;
    }

    // -------------------- consumer warps ------------------------------------
    unsigned long long *wl = lists + (size_t)warp * QPW * C::REGION;
    for (int i = lane; i < QPW * C::REGION; i += 32) wl[i] = kKeyInf;
    __syncwarp();
    uint32_t nb = 0;   // candidate buffer fills
    unsigned long long lbk[QPW];
#pragma unroll
    for (int i = 0; i < QPW; ++i) {
        const int q = qtile * C::BQ + warp * QPW + i;
        lbk[i] = (LB && q < a.Q) ? a.lb[q] : 0ull;
    }

    int it = 0;
    for (int rt = t0; rt < t1; ++rt) {
        f32x2_t acc[QPW][4];
        if (!consume_ref_tile<QPW, KCAP>(acc, stages, full, empty, abort_flag, it, a.n_dchunks,
                                         warp, lane, a.status))
            break;
        select_tile<QPW, KCAP, LB>(wl, nb, acc, rt, a.N, a.k, lane, lbk);
    }
    flush_all<QPW, KCAP>(wl, nb, a.k, lane);

    consumer_sync();
    if (*abort_flag) return;

    const int q0 = qtile * C::BQ;
    if (a.n_splits == 1) {
        // Epilogue: sqrt and the reference's k x query_nb layout, coalesced
        // along queries.
        for (int e = threadIdx.x; e < a.k * C::BQ; e += EX_WARPS * 32) {
            const int j = e / C::BQ, qi = e - j * C::BQ, q = q0 + qi;
            if (q < a.Q) {
                const unsigned long long key = lists[(size_t)qi * C::REGION + j];
                a.out_dist[(size_t)(a.row0 + j) * a.ld_out + q] = sqrtf(key_dist2(key));
                a.out_idx[(size_t)(a.row0 + j) * a.ld_out + q] = key_index(key);
                if (a.lb_out && j == a.k - 1) a.lb_out[q] = key + 1;
            }
        }
    } else {
        for (int i = 0; i < QPW; ++i) {
            const int q = q0 + warp * QPW + i;
            if (q >= a.Q) break;
            unsigned long long *dst = a.part + ((size_t)split * a.Q + q) * a.k;
            for (int j = lane; j < a.k; j += 32) dst[j] = wl[i * C::REGION + j];
        }
    }
}

// Duplicate every query value into a (q, q) pair: dst[d][2i] = dst[d][2i+1]
// = src[d][i].
__global__ void dup_queries_kernel(const float *__restrict__ src, int Q, long long lds, int d,
                                   float2 *__restrict__ dst, long long ldd2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int dd = blockIdx.y;
    if (i < Q) {
        const float v = src[(size_t)dd * lds + i];
        dst[(size_t)dd * ldd2 + i] = make_float2(v, v);
    }
}


// Merge the per-split sorted key lists of each query (one warp per query).
// An element's output position is the sum of its ranks in every list.
__global__ void knn_merge_splits_kernel(const unsigned long long *__restrict__ part, int S,
                                        int Q, int k, float *__restrict__ out_dist,
                                        int *__restrict__ out_idx, long long ld_out, int row0,
                                        unsigned long long *__restrict__ lb_out) {
    extern __shared__ unsigned long long msm[];
    const int wpb = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * wpb + warp;
    if (q >= Q) return;
    unsigned long long *L = msm + (size_t)warp * S * k;
    for (int e = lane; e < S * k; e += 32) {
        const int t = e / k, j = e - t * k;
        L[e] = part[((size_t)t * Q + q) * k + j];
    }
    __syncwarp();
    for (int e = lane; e < S * k; e += 32) {
        const int t = e / k, j = e - t * k;
        const unsigned long long x = L[e];
        int pos = j;
        for (int u = 0; u < S && pos < k; ++u)
            if (u != t) pos += rank_sorted(L + (size_t)u * k, k, x);
        if (pos < k) {
            out_dist[(size_t)(row0 + pos) * ld_out + q] = sqrtf(key_dist2(x));
            out_idx[(size_t)(row0 + pos) * ld_out + q] = key_index(x);
            if (lb_out && pos == k - 1) lb_out[q] = x + 1;
        }
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kMergeSmemMax = 200u * 1024u;   // dynamic smem limit of the merge kernel

struct ExactShape {
    int qpw, kcap, bq, splits, n_rtiles, n_dchunks;
    size_t smem;
};

template <int QPW, int KCAP>
void shape_of(ExactShape &s) {
    using C = ExCfg<QPW, KCAP>;
    s.qpw = QPW;
    s.kcap = KCAP;
    s.bq = C::BQ;
    s.smem = C::SMEM;
}

// Ranks selected by one pass of the kernel: k <= 256 in one pass, larger k
// in passes of 256 (the last one may be shorter).
constexpr int kPassRanks = 256;

bool choose_shape(int N, int Q, int d, int k_all, int num_sms, ExactShape &s) {
    if (k_all < 1) return false;
    const int k = std::min(k_all, kPassRanks);
    if (k <= 32) shape_of<EX_QPW, 32>(s);
    else if (k <= 64) shape_of<EX_QPW, 64>(s);
    else if (k <= 128) shape_of<EX_QPW, 128>(s);
    else shape_of<EX_QPW_K256, 256>(s);
    s.n_rtiles = (N + EX_BR - 1) / EX_BR;
    s.n_dchunks = (d + EX_BD - 1) / EX_BD;
    const int qtiles = (Q + s.bq - 1) / s.bq;
    // Split the reference set so that the grid fills whole waves of one CTA
    // per SM.  Modelled time: waves x (tiles per split + fixed selection
    // warm-up cost of about 256/d tiles per split).
    const double warm = 256.0 / (s.n_dchunks * EX_BD);
    int best = 1;
    double best_t = 1e300;
    // up to 256 splits, while each query's merge input (splits * k keys) fits
    // one warp's shared-memory slab in the merge kernel
    int max_s = std::min(s.n_rtiles, std::min(256, (160 * 1024) / (8 * k)));
    // keep the per-split partial lists under 1 GiB of scratch
    const long long per_split = (long long)Q * k * 8;
    max_s = (int)std::max<long long>(1, std::min<long long>(max_s, (1ll << 30) / per_split));
    for (int S = 1; S <= max_s; ++S) {
        const long long ctas = (long long)qtiles * S;
        const long long waves = (ctas + num_sms - 1) / num_sms;
        const double t = (double)waves * ((double)s.n_rtiles / S + warm);
        if (t < best_t * 0.999) {
            best_t = t;
            best = S;
        }
    }
    s.splits = best;
    return true;
}

template <int QPW, int KCAP, bool LB = false>
cudaError_t launch_t(const CUtensorMap &mr, const CUtensorMap &mq, const ExactArgs &a,
                     int qtiles, cudaStream_t st) {
    using C = ExCfg<QPW, KCAP>;
    auto kern = knn_exact_kernel<QPW, KCAP, LB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)C::SMEM);
    if (e != cudaSuccess) return e;
    dim3 grid(qtiles, a.n_splits);
    kern<<<grid, EX_THREADS, C::SMEM, st>>>(mr, mq, a);
    return cudaGetLastError();
}

}  // namespace

// Row pitch (in float2) of the duplicated query copy.
static long long qdup_pitch2(int Q) { return ((long long)Q + 31) / 32 * 32; }

int launch_split_merge(const unsigned long long *part, int S, int Q, int k, float *out_dist,
                       int *out_idx, long long ld_out, cudaStream_t st, int row0,
                       unsigned long long *lb_out) {
    const size_t per_warp = (size_t)S * k * 8;
    const int wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (160u * 1024u) / per_warp));
    const size_t smem = per_warp * wpb;
    if (smem > kMergeSmemMax) return kErrUnsupported;
    // one fixed limit for every launch: calls from several host threads must
    // not lower it between another call's set and launch
    if (cudaFuncSetAttribute(knn_merge_splits_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kMergeSmemMax) != cudaSuccess)
        return kErrLaunch;
    knn_merge_splits_kernel<<<(Q + wpb - 1) / wpb, wpb * 32, smem, st>>>(
        part, S, Q, k, out_dist, out_idx, ld_out, row0, lb_out);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrLaunch;
}

// Scratch of the exact path: the (q, q)-duplicated queries, 256 bytes of
// alignment, the per-split key lists of one pass when the reference set is
// split, and for k > 256 the per-query lower-bound keys of the passes.
static size_t exact_need(const ExactShape &s, int Q, int d, int k, size_t *part_off,
                         size_t *lb_off) {
    const int kp = std::min(k, kPassRanks);
    const size_t dup = (size_t)d * qdup_pitch2(Q) * sizeof(float2);
    const size_t off = (dup + 255) & ~size_t(255);
    const size_t part = s.splits > 1 ? (size_t)s.splits * Q * kp * 8 : 0;
    const size_t lb = k > kPassRanks ? (size_t)Q * 8 : 0;
    if (part_off) *part_off = off;
    if (lb_off) *lb_off = off + part;
    return std::max(dup + 256, off) + part + lb;
}

size_t exact_scratch_bytes(int N, int Q, int d, int k, int num_sms) {
    if (lowdim_applies(N, Q, d, k)) return lowdim_scratch_bytes(N, Q, d, k, num_sms);
    ExactShape s;
    if (!choose_shape(N, Q, d, k, num_sms, s)) return 0;
    return exact_need(s, Q, d, k, nullptr, nullptr);
}

bool exact_supported_k(int k) { return k >= 1; }

int launch_exact(const ExactProblem &p, cudaStream_t st) {
    if (lowdim_applies(p.N, p.Q, p.d, p.k)) return launch_lowdim(p, st);
    ExactShape s;
    if (!choose_shape(p.N, p.Q, p.d, p.k, p.num_sms, s)) return kErrUnsupported;
    if (p.force_splits > 0) s.splits = std::min(p.force_splits, std::min(s.n_rtiles, 256));
    const long long ld2 = qdup_pitch2(p.Q);
    size_t part_off = 0, lb_off = 0;
    if (exact_need(s, p.Q, p.d, p.k, &part_off, &lb_off) > p.scratch_bytes) return kErrScratch;
    float2 *qdup = static_cast<float2 *>(p.scratch);
    unsigned char *sb = static_cast<unsigned char *>(p.scratch);
    unsigned long long *part = reinterpret_cast<unsigned long long *>(sb + part_off);
    unsigned long long *lb = reinterpret_cast<unsigned long long *>(sb + lb_off);
    dup_queries_kernel<<<dim3((p.Q + 255) / 256, p.d), 256, 0, st>>>(p.qry, p.Q, p.ldq, p.d, qdup,
                                                                   ld2);
    if (cudaGetLastError() != cudaSuccess) return kErrLaunch;

    CUtensorMap mr, mq;
    if (!encode_f32_2d(&mr, p.ref, (uint64_t)p.N, (uint64_t)p.d, (uint64_t)p.ldr, EX_BR, EX_BD))
        return kErrTensorMap;
    if (!encode_f32_2d(&mq, qdup, (uint64_t)(2 * p.Q), (uint64_t)p.d, (uint64_t)(2 * ld2),
                       2 * s.bq, EX_BD))
        return kErrTensorMap;

    ExactArgs a;
    a.N = p.N;
    a.Q = p.Q;
    a.d = p.d;
    a.n_rtiles = s.n_rtiles;
    a.n_splits = s.splits;
    a.n_dchunks = s.n_dchunks;
    a.out_dist = p.out_dist;
    a.out_idx = p.out_idx;
    a.ld_out = p.ld_out;
    a.part = part;
    a.status = p.status;
    a.lb = lb;
    const int qtiles = (p.Q + s.bq - 1) / s.bq;
    const bool multi = p.k > kPassRanks;
    // ranks [row0, row0 + a.k) per pass
    for (int row0 = 0; row0 < p.k; row0 += kPassRanks) {
        a.k = std::min(kPassRanks, p.k - row0);
        a.row0 = row0;
        a.lb_out = (multi && row0 + a.k < p.k) ? lb : nullptr;
        cudaError_t e;
        if (multi) {
            // pass 0 has no lower bound; every later pass starts above the
            // last key of the one before
            e = row0 == 0 ? launch_t<EX_QPW_K256, 256, false>(mr, mq, a, qtiles, st)
                          : launch_t<EX_QPW_K256, 256, true>(mr, mq, a, qtiles, st);
        } else {
            switch (s.kcap) {
                case 32: e = launch_t<EX_QPW, 32>(mr, mq, a, qtiles, st); break;
                case 64: e = launch_t<EX_QPW, 64>(mr, mq, a, qtiles, st); break;
                case 128: e = launch_t<EX_QPW, 128>(mr, mq, a, qtiles, st); break;
                default: e = launch_t<EX_QPW_K256, 256>(mr, mq, a, qtiles, st); break;
            }
        }
        if (e != cudaSuccess) return kErrLaunch;
        if (p.timer) p.timer->mark(st, kPhaseExactMain);
        if (s.splits > 1) {
            const int rc = launch_split_merge(a.part, s.splits, p.Q, a.k, p.out_dist, p.out_idx,
                                              p.ld_out, st, row0, a.lb_out);
            if (rc != kOk) return rc;
            if (p.timer) p.timer->mark(st, kPhaseExactMerge);
        }
    }
    return kOk;
}

int exact_plan_splits(int N, int Q, int d, int k, int num_sms) {
    if (lowdim_applies(N, Q, d, k)) return lowdim_plan_splits(N, Q, d, k, num_sms);
    ExactShape s;
    return choose_shape(N, Q, d, k, num_sms, s) ? s.splits : 0;
}

}  // namespace knnb200
