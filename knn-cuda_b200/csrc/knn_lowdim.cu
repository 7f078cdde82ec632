// knn_lowdim.cu -- exact FP32 k-NN for low dimension (d <= 4) and small k
// (k <= 16), e.g. 3-D point clouds.
//
// At d = 3 the distance of a pair costs three subtractions and three fused
// multiply-adds, so the work is dominated by issue, not by data: the tiled
// kernel's 16-dimension stages would waste 13/16 of its arithmetic.  Here
// every thread owns QPT queries (packed in pairs for sub.f32x2 / fma.f32x2)
// and their sorted top-k lists in registers; the CTA streams its range of
// reference points through a double-buffered shared-memory tile (each
// coordinate stored twice, (r, r), so a 64-bit load yields a packed operand)
// and every thread scans the tile in index order.
//
// Arithmetic: acc = fma(t0, t0, 0), acc = fma(t_i, t_i, acc) for i = 1..d-1,
// t_i = r_i - q_i -- the fused exact kernel's chain (its zero-padded
// dimensions add exact zeros), so distances are bit-identical to it.
// Selection: a candidate enters the list iff it is strictly smaller than the
// k-th distance, and shifts only past strictly larger entries; because each
// thread scans references in increasing index, equal distances keep the
// lower index first -- the reference's rule (code/knncuda.cu:172, :178).
#include <algorithm>

#include "knn_common.cuh"
#include "knn_kernels.h"

namespace knnb200 {

constexpr int LD_THREADS = 256;
constexpr int LD_TILE = 512;   // reference points per shared tile

template <int D, int K, int QPT>
__global__ void __launch_bounds__(LD_THREADS, 2)
    knn_lowdim_kernel(const float *__restrict__ ref, int N, long long ldr,
                      const float *__restrict__ qry, int Q, long long ldq, int k, int n_rtiles,
                      int n_splits, float *__restrict__ out_dist, int *__restrict__ out_idx,
                      long long ld_out, unsigned long long *__restrict__ part) {
    static_assert(QPT % 2 == 0, "queries are processed in pairs");
    __shared__ float2 tile[2][D][LD_TILE];
    const int tid = threadIdx.x;
    const int qtile = blockIdx.x, split = blockIdx.y;
    const int BQ = LD_THREADS * QPT;
    // thread's queries: q_base + tid + m * LD_THREADS (coalesced loads)
    f32x2_t qp[QPT / 2][D];
    int qid[QPT];
#pragma unroll
    for (int m = 0; m < QPT; ++m) qid[m] = qtile * BQ + tid + m * LD_THREADS;
#pragma unroll
    for (int pr = 0; pr < QPT / 2; ++pr)
#pragma unroll
        for (int dd = 0; dd < D; ++dd) {
            const int a = qid[2 * pr], b = qid[2 * pr + 1];
            const float va = a < Q ? qry[(size_t)dd * ldq + a] : 0.f;
            const float vb = b < Q ? qry[(size_t)dd * ldq + b] : 0.f;
            qp[pr][dd] = f2_pack(va, vb);
        }
    float ld[QPT][K];
    int li[QPT][K];
#pragma unroll
    for (int m = 0; m < QPT; ++m)
#pragma unroll
        for (int j = 0; j < K; ++j) {
            ld[m][j] = INFINITY;
            li[m][j] = -1;
        }

    // this CTA's reference range, in tiles of LD_TILE points
    const long long t0 = (long long)n_rtiles * split / n_splits;
    const long long t1 = (long long)n_rtiles * (split + 1) / n_splits;
    constexpr int PER = LD_TILE / LD_THREADS;   // points per thread per tile load
    float pre[D][PER];
    auto fetch = [&](long long t) {
#pragma unroll
        for (int dd = 0; dd < D; ++dd)
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const long long r = t * LD_TILE + u * LD_THREADS + tid;
                pre[dd][u] = r < N ? ref[(size_t)dd * ldr + r] : 0.f;
            }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int dd = 0; dd < D; ++dd)
#pragma unroll
            for (int u = 0; u < PER; ++u)
                tile[buf][dd][u * LD_THREADS + tid] = make_float2(pre[dd][u], pre[dd][u]);
    };
    if (t0 < t1) {
        fetch(t0);
        stash(0);
    }
    __syncthreads();
    for (long long t = t0; t < t1; ++t) {
        const int buf = (int)((t - t0) & 1);
        if (t + 1 < t1) fetch(t + 1);
        const int rbase = (int)(t * LD_TILE);
        const int valid = (int)std::min<long long>(LD_TILE, (long long)N - rbase);
        for (int j = 0; j < valid; ++j) {
            f32x2_t rr[D];
#pragma unroll
            for (int dd = 0; dd < D; ++dd)
                rr[dd] = *reinterpret_cast<const f32x2_t *>(&tile[buf][dd][j]);
#pragma unroll
            for (int pr = 0; pr < QPT / 2; ++pr) {
                f32x2_t tt = f2_sub(rr[0], qp[pr][0]);
                f32x2_t acc = f2_fma(tt, tt, 0ull);
#pragma unroll
                for (int dd = 1; dd < D; ++dd) {
                    tt = f2_sub(rr[dd], qp[pr][dd]);
                    acc = f2_fma(tt, tt, acc);
                }
                const float da = f2_lo(acc), db = f2_hi(acc);
                const int ma = 2 * pr, mb = 2 * pr + 1;
                if (da < ld[ma][K - 1] || db < ld[mb][K - 1]) {
                    const int id = rbase + j;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int m = h ? mb : ma;
                        const float v = h ? db : da;
                        if (v < ld[m][K - 1]) {
#pragma unroll
                            for (int i = K - 1; i > 0; --i) {
                                const bool past = v < ld[m][i - 1];
                                const bool here = v < ld[m][i];
                                ld[m][i] = past ? ld[m][i - 1] : (here ? v : ld[m][i]);
                                li[m][i] = past ? li[m][i - 1] : (here ? id : li[m][i]);
                            }
                            if (v < ld[m][0]) {
                                ld[m][0] = v;
                                li[m][0] = id;
                            }
                        }
                    }
                }
            }
        }
        if (t + 1 < t1) stash(buf ^ 1);
        __syncthreads();
    }

    // results (the first k of the K kept): sqrt into the k x Q layout, or
    // this split's sorted keys for the split merge
#pragma unroll
    for (int m = 0; m < QPT; ++m) {
        const int q = qid[m];
        if (q >= Q) continue;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (j >= k) break;
            if (n_splits == 1) {
                out_dist[(size_t)j * ld_out + q] = sqrtf(ld[m][j]);
                out_idx[(size_t)j * ld_out + q] = li[m][j];
            } else {
                part[((size_t)split * Q + q) * k + j] = make_key(ld[m][j], (uint32_t)li[m][j]);
            }
        }
    }
}

namespace {

struct LowdimShape {
    int kcap, qpt, bq, n_rtiles, splits;
};

bool lowdim_shape(int N, int Q, int d, int k, int num_sms, LowdimShape &s) {
    if (d < 1 || d > 4 || k < 1 || k > 16) return false;
    s.kcap = k <= 8 ? 8 : 16;
    s.qpt = s.kcap == 8 ? 4 : 2;
    s.bq = LD_THREADS * s.qpt;
    s.n_rtiles = (N + LD_TILE - 1) / LD_TILE;
    const int qtiles = (Q + s.bq - 1) / s.bq;
    // two CTAs per SM; splits fill whole waves, each CTA >= 8 tiles
    const int slots = 2 * num_sms;
    int best = 1;
    double best_t = 1e300;
    const int max_s = std::max(1, std::min({256, s.n_rtiles / 8, (160 * 1024) / (8 * k)}));
    for (int S = 1; S <= max_s; ++S) {
        const long long ctas = (long long)qtiles * S;
        const double t = (double)((ctas + slots - 1) / slots) * ((double)s.n_rtiles / S + 0.5);
        if (t < best_t * 0.999) {
            best_t = t;
            best = S;
        }
    }
    s.splits = best;
    return true;
}

template <int D, int K, int QPT>
cudaError_t launch_ld(const ExactProblem &p, const LowdimShape &s, unsigned long long *part,
                      cudaStream_t st) {
    dim3 grid((p.Q + s.bq - 1) / s.bq, s.splits);
    knn_lowdim_kernel<D, K, QPT><<<grid, LD_THREADS, 0, st>>>(
        p.ref, p.N, p.ldr, p.qry, p.Q, p.ldq, p.k, s.n_rtiles, s.splits, p.out_dist, p.out_idx,
        p.ld_out, part);
    return cudaGetLastError();
}

template <int K, int QPT>
cudaError_t launch_ld_d(const ExactProblem &p, const LowdimShape &s, unsigned long long *part,
                        cudaStream_t st) {
    switch (p.d) {
        case 1: return launch_ld<1, K, QPT>(p, s, part, st);
        case 2: return launch_ld<2, K, QPT>(p, s, part, st);
        case 3: return launch_ld<3, K, QPT>(p, s, part, st);
        default: return launch_ld<4, K, QPT>(p, s, part, st);
    }
}

}  // namespace

bool lowdim_applies(int N, int Q, int d, int k) {
    LowdimShape s;
    return lowdim_shape(N, Q, d, k, 148, s);
}

size_t lowdim_scratch_bytes(int N, int Q, int d, int k, int num_sms) {
    LowdimShape s;
    if (!lowdim_shape(N, Q, d, k, num_sms, s)) return 0;
    return s.splits > 1 ? (size_t)s.splits * Q * k * 8 : 0;
}

int lowdim_plan_splits(int N, int Q, int d, int k, int num_sms) {
    LowdimShape s;
    return lowdim_shape(N, Q, d, k, num_sms, s) ? s.splits : 0;
}

int launch_lowdim(const ExactProblem &p, cudaStream_t st) {
    LowdimShape s;
    if (!lowdim_shape(p.N, p.Q, p.d, p.k, p.num_sms, s)) return kErrUnsupported;
    if (p.force_splits > 0) s.splits = std::min(p.force_splits, std::min(s.n_rtiles, 256));
    const size_t need = s.splits > 1 ? (size_t)s.splits * p.Q * p.k * 8 : 0;
    if (need > p.scratch_bytes) return kErrScratch;
    unsigned long long *part = static_cast<unsigned long long *>(p.scratch);
    const cudaError_t e = s.kcap == 8 ? launch_ld_d<8, 4>(p, s, part, st)
                                      : launch_ld_d<16, 2>(p, s, part, st);
    if (e != cudaSuccess) return kErrLaunch;
    if (p.timer) p.timer->mark(st, kPhaseExactMain);
    if (s.splits > 1) {
        const int rc = launch_split_merge(part, s.splits, p.Q, p.k, p.out_dist, p.out_idx,
                                          p.ld_out, st);
        if (rc != kOk) return rc;
        if (p.timer) p.timer->mark(st, kPhaseExactMerge);
    }
    return kOk;
}

}  // namespace knnb200
