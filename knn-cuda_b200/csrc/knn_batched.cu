// knn_batched.cu -- many independent exact k-NN problems in one persistent
// launch fed by a device-side work queue.
//
// The reference solves one problem per call (code/knncuda.cu:271-278).  Here
// a plan holds up to thousands of problems of uneven ref_nb / query_nb / dim /
// k (device pointers, the reference's dim x n layouts).  Each problem is cut
// into work items (query tile of BQ queries x a contiguous range of reference
// tiles); items are ordered largest first and numbered.  One CTA per SM runs
// the fused exact pipeline of knn_exact.cu: its TMA producer warp pops the
// next item number off a global atomic counter, hands it to the 16 consumer
// warps through a double-buffered shared slot (mbarrier handshake), and
// streams that item's tiles through the shared stage ring; the consumers
// compute, select and write the item's result.  Problems cut into several
// reference ranges are finished by one batched split-merge kernel.
//
// A plan owns its tables (problem records, TMA descriptors, queue counter)
// and its scratch, so running it allocates nothing and synchronises nothing:
// it can be captured into a CUDA graph (knnb200_batched_graph_create).  The
// granularity of the work items (stages per item) is a tunable that
// knnb200_batched_autotune picks by timing candidate plans.
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <vector>

#include "../../include/knn_b200.h"
#include "knn_exact_core.cuh"
#include "knn_kernels.h"

namespace knnb200 {

struct BatchProb {
    int N, Q, d, k;
    int n_rtiles, n_splits, n_dchunks, qtiles;
    long long item_begin;     // first work item of this problem
    long long merge_begin;    // first merge task (one per query) or -1
    int row_begin;            // first row of the query-duplication pass
    const float *qry;
    long long ldq;
    float2 *qdup;
    long long ld2;
    float *out_dist;
    int *out_idx;
    long long ld_out;
    unsigned long long *part;   // [n_splits][Q][k] when n_splits > 1
};

struct ItemInfo {
    long long idx;
    int p, qtile, split;
};

// First index i in [0, n) with key(i) > x, minus one (records sorted by key).
template <typename F>
KNN_DI int find_record(int n, long long x, F key) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (key(mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Query duplication for every problem: one block per (problem, dimension) row.
__global__ void batched_dup_kernel(const BatchProb *__restrict__ probs, int n_probs,
                                   int n_rows) {
    const int row = blockIdx.x;
    if (row >= n_rows) return;
    const int p = find_record(n_probs, row, [&](int i) { return (long long)probs[i].row_begin; });
    const BatchProb P = probs[p];
    const int dd = row - P.row_begin;
    for (int i = threadIdx.x; i < P.Q; i += blockDim.x) {
        const float v = P.qry[(size_t)dd * P.ldq + i];
        P.qdup[(size_t)dd * P.ld2 + i] = make_float2(v, v);
    }
}

template <int QPW, int KCAP>
struct BatchCfg {
    using C = ExCfg<QPW, KCAP>;
    static constexpr size_t ITEM_OFFSET = C::BAR_OFFSET + 2 * EX_STAGES * 8 + 64;
    static constexpr size_t SMEM = 1024 + ITEM_OFFSET + 2 * sizeof(ItemInfo) + 4 * 8 + 64;
    static_assert(SMEM <= 232448, "shared memory per CTA");
};

template <int QPW, int KCAP>
__global__ void __launch_bounds__(EX_THREADS, 1)
    knn_exact_batched_kernel(const CUtensorMap *__restrict__ maps,
                             const BatchProb *__restrict__ probs, int n_probs, long long n_items,
                             unsigned long long *queue, int *status) {
    using C = ExCfg<QPW, KCAP>;
    using B = BatchCfg<QPW, KCAP>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float *stages = reinterpret_cast<float *>(base);
    unsigned long long *lists =
        reinterpret_cast<unsigned long long *>(base + (size_t)EX_STAGES * C::STAGE_BYTES);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + C::BAR_OFFSET);
    uint64_t *empty = full + EX_STAGES;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + EX_STAGES);
    ItemInfo *items = reinterpret_cast<ItemInfo *>(base + B::ITEM_OFFSET);
    uint64_t *item_full = reinterpret_cast<uint64_t *>(items + 2);
    uint64_t *item_empty = item_full + 2;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < EX_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], EX_WARPS);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(&item_full[s], 1);
            mbar_init(&item_empty[s], EX_WARPS);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == EX_WARPS) {
        // ---------------- producer: pops items, streams their tiles --------
        if (lane == 0) {
            int issued = 0, it = 0;
            for (int n = 0;; ++n) {
                const int slot = n & 1;
                if (n >= 2 && !mbar_wait(&item_empty[slot], ((n >> 1) - 1) & 1)) {
                    atomicMax(status, (int)kDevTimeoutEmpty);
                    *abort_flag = 1;
                    break;
                }
                ItemInfo inf;
                inf.idx = (long long)atomicAdd(queue, 1ull);
                inf.p = inf.qtile = inf.split = 0;
                if (inf.idx < n_items) {
                    inf.p = find_record(n_probs, inf.idx,
                                        [&](int i) { return probs[i].item_begin; });
                    const int li = (int)(inf.idx - probs[inf.p].item_begin);
                    inf.qtile = li % probs[inf.p].qtiles;
                    inf.split = li / probs[inf.p].qtiles;
                }
                items[slot] = inf;
                mbar_arrive(&item_full[slot]);
                if (inf.idx >= n_items || *abort_flag) break;
                const BatchProb &P = probs[inf.p];
                const CUtensorMap *mr = maps + 2 * inf.p;
                const CUtensorMap *mq = mr + 1;
                const int t0 = (int)((long long)P.n_rtiles * inf.split / P.n_splits);
                const int t1 = (int)((long long)P.n_rtiles * (inf.split + 1) / P.n_splits);
                bool ok = true;
                for (int rt = t0; rt < t1 && ok; ++rt)
                    for (int dc = 0; dc < P.n_dchunks; ++dc, ++it) {
                        const int s = it % EX_STAGES;
                        if (it >= EX_STAGES &&
                            !mbar_wait(&empty[s], ((it / EX_STAGES) - 1) & 1)) {
                            atomicMax(status, (int)kDevTimeoutEmpty);
                            *abort_flag = 1;
                            ok = false;
                            break;
                        }
                        if (*abort_flag) {
                            ok = false;
                            break;
                        }
                        float *qs = stages + (size_t)s * C::STAGE_FLOATS;
                        float *rs = qs + C::Q_FLOATS;
                        mbar_arrive_expect_tx(&full[s], C::STAGE_BYTES);
                        tma_load_2d(qs, mq, &full[s], inf.qtile * 2 * C::BQ, dc * EX_BD);
                        tma_load_2d(rs, mr, &full[s], rt * EX_BR, dc * EX_BD);
                        issued = it + 1;
                    }
                if (!ok) break;
            }
            for (int i = max(0, issued - EX_STAGES); i < issued; ++i)
                if (!mbar_wait(&full[i % EX_STAGES], (i / EX_STAGES) & 1))
                    atomicMax(status, (int)kDevTimeoutDrain);
        }
        return;
    }

    // -------------------- consumer warps ------------------------------------
    unsigned long long *wl = lists + (size_t)warp * QPW * C::REGION;
    int it = 0;
    for (int n = 0;; ++n) {
        const int slot = n & 1;
        const bool got = mbar_wait(&item_full[slot], (n >> 1) & 1);
        if (__any_sync(0xffffffffu, !got)) {
            if (lane == 0) {
                atomicMax(status, (int)kDevTimeoutFull);
                *abort_flag = 1;
            }
            break;
        }
        const ItemInfo inf = items[slot];
        __syncwarp();
        if (lane == 0) mbar_arrive(&item_empty[slot]);
        if (inf.idx >= n_items) break;
        const BatchProb P = probs[inf.p];
        for (int i = lane; i < QPW * C::REGION; i += 32) wl[i] = kKeyInf;
        __syncwarp();
        uint32_t nb = 0;   // candidate buffer fills
        const int t0 = (int)((long long)P.n_rtiles * inf.split / P.n_splits);
        const int t1 = (int)((long long)P.n_rtiles * (inf.split + 1) / P.n_splits);
        bool alive = true;
        for (int rt = t0; rt < t1; ++rt) {
            f32x2_t acc[QPW][4];
            if (!consume_ref_tile<QPW, KCAP>(acc, stages, full, empty, abort_flag, it,
                                             P.n_dchunks, warp, lane, status)) {
                alive = false;
                break;
            }
            select_tile<QPW, KCAP>(wl, nb, acc, rt, P.N, P.k, lane);
        }
        flush_all<QPW, KCAP>(wl, nb, P.k, lane);
        consumer_sync();
        if (!alive || *abort_flag) break;
        const int q0 = inf.qtile * C::BQ;
        if (P.n_splits == 1) {
            for (int e = threadIdx.x; e < P.k * C::BQ; e += EX_WARPS * 32) {
                const int j = e / C::BQ, qi = e - j * C::BQ, q = q0 + qi;
                if (q < P.Q) {
                    const unsigned long long key = lists[(size_t)qi * C::REGION + j];
                    P.out_dist[(size_t)j * P.ld_out + q] = sqrtf(key_dist2(key));
                    P.out_idx[(size_t)j * P.ld_out + q] = key_index(key);
                }
            }
        } else {
            for (int i = 0; i < QPW; ++i) {
                const int q = q0 + warp * QPW + i;
                if (q >= P.Q) break;
                unsigned long long *dst = P.part + ((size_t)inf.split * P.Q + q) * P.k;
                for (int j = lane; j < P.k; j += 32) dst[j] = wl[i * C::REGION + j];
            }
        }
        consumer_sync();   // lists are rewritten by the next item
    }
}

// Merge per-split lists of every split problem: one warp per (problem, query).
// mlist holds the record indices of the split problems, by merge_begin.
__global__ void batched_merge_kernel(const BatchProb *__restrict__ probs,
                                     const int *__restrict__ mlist, int n_split_probs,
                                     long long n_tasks, int slab_keys) {
    extern __shared__ unsigned long long msm[];
    const int wpb = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long task = (long long)blockIdx.x * wpb + warp;
    if (task >= n_tasks) return;
    const int m = find_record(n_split_probs, task,
                              [&](int i) { return probs[mlist[i]].merge_begin; });
    const BatchProb &P = probs[mlist[m]];
    const int q = (int)(task - P.merge_begin);
    const int S = P.n_splits, k = P.k;
    unsigned long long *L = msm + (size_t)warp * slab_keys;
    for (int e = lane; e < S * k; e += 32) {
        const int t = e / k, j = e - t * k;
        L[e] = P.part[((size_t)t * P.Q + q) * k + j];
    }
    __syncwarp();
    for (int e = lane; e < S * k; e += 32) {
        const int t = e / k, j = e - t * k;
        const unsigned long long x = L[e];
        int pos = j;
        for (int u = 0; u < S && pos < k; ++u)
            if (u != t) pos += rank_sorted(L + (size_t)u * k, k, x);
        if (pos < k) {
            P.out_dist[(size_t)pos * P.ld_out + q] = sqrtf(key_dist2(x));
            P.out_idx[(size_t)pos * P.ld_out + q] = key_index(x);
        }
    }
}

}  // namespace knnb200

using namespace knnb200;

namespace {

constexpr size_t kBatchMergeSmemMax = 200u * 1024u;

struct DevMem {
    void *ptr = nullptr;
    size_t bytes = 0;
    bool alloc(size_t n) {
        bytes = n;
        if (cudaMalloc(&ptr, n ? n : 256) != cudaSuccess) {
            cudaGetLastError();
            ptr = nullptr;
            return false;
        }
        return true;
    }
    ~DevMem() {
        if (ptr) cudaFree(ptr);
    }
};

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

}  // namespace

struct knnb200_batched_plan {
    int device = 0, num_sms = 148;
    int kcap = 32, qpw = 4, item_stages = 256;
    int count = 0, n_rows = 0, n_split_probs = 0;   // count: problems of the persistent launch
    std::vector<ExactProblem> lowdim;                // problems routed to the low-d kernel
    long long n_items = 0, n_tasks = 0;
    int merge_wpb = 1, slab_keys = 0;
    DevMem tables;      // BatchProb[count] | CUtensorMap[2*count] | counter, status | mlist
    DevMem scratch;     // qdup + parts
    BatchProb *probs = nullptr;
    CUtensorMap *maps = nullptr;
    unsigned long long *counter = nullptr;
    int *status = nullptr;
    int *mlist = nullptr;
};

namespace {

template <int QPW, int KCAP>
cudaError_t launch_batched_t(const knnb200_batched_plan *pl, cudaStream_t st) {
    using B = BatchCfg<QPW, KCAP>;
    auto kern = knn_exact_batched_kernel<QPW, KCAP>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)B::SMEM);
    if (e != cudaSuccess) return e;
    kern<<<pl->num_sms, EX_THREADS, B::SMEM, st>>>(pl->maps, pl->probs, pl->count, pl->n_items,
                                                   pl->counter, pl->status);
    return cudaGetLastError();
}

int validate(const knnb200_problem &q) {
    if (!q.ref || !q.query || !q.knn_dist || !q.knn_index) return KNNB200_EINVAL;
    if (q.ref_nb < 1 || q.query_nb < 1 || q.dim < 1 || q.k < 1 || q.k > q.ref_nb)
        return KNNB200_EINVAL;
    if (q.ref_ld < q.ref_nb || q.query_ld < q.query_nb || q.out_ld < q.query_nb)
        return KNNB200_EINVAL;
    if (q.ref_ld % 4 || (reinterpret_cast<uintptr_t>(q.ref) & 15)) return KNNB200_EINVAL;
    if (q.k > 256) return KNNB200_EUNSUPPORTED;
    return KNNB200_OK;
}

}  // namespace

extern "C" {

int knnb200_batched_plan_create_config(const knnb200_problem *all, int n_all,
                                       const knnb200_batched_config *cfg,
                                       knnb200_batched_plan **out) {
    if (!out) return KNNB200_EINVAL;
    *out = nullptr;
    if (!all || n_all < 1) return KNNB200_EINVAL;
    for (int i = 0; i < n_all; ++i) {
        const int rc = validate(all[i]);
        if (rc != KNNB200_OK) return rc;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return KNNB200_ENODEV;
    }
    const int item_stages = cfg && cfg->item_stages > 0 ? cfg->item_stages : 256;
    const int want_qpw = cfg ? cfg->queries_per_warp : 0;
    if (want_qpw != 0 && want_qpw != 2 && want_qpw != 4) return KNNB200_EINVAL;
    const bool route_lowdim = cfg && cfg->lowdim_kernel;
    knnb200_batched_plan *pl = new knnb200_batched_plan();
    cudaGetDevice(&pl->device);
    cudaDeviceGetAttribute(&pl->num_sms, cudaDevAttrMultiProcessorCount, pl->device);
    pl->item_stages = item_stages;
    // problem classes: d <= 4, k <= 16 to the low-d kernel (when asked),
    // the rest to the persistent launch
    std::vector<knnb200_problem> persist;
    std::vector<int> low_idx;
    for (int i = 0; i < n_all; ++i) {
        if (route_lowdim && lowdim_applies(all[i].ref_nb, all[i].query_nb, all[i].dim, all[i].k))
            low_idx.push_back(i);
        else
            persist.push_back(all[i]);
    }
    const knnb200_problem *in = persist.data();
    const int count = (int)persist.size();
    int kmax = 1;
    for (int i = 0; i < count; ++i) kmax = std::max(kmax, in[i].k);
    pl->kcap = kmax <= 32 ? 32 : kmax <= 64 ? 64 : kmax <= 128 ? 128 : 256;
    pl->qpw = pl->kcap == 256 ? EX_QPW_K256 : (want_qpw ? want_qpw : EX_QPW);
    const int bq = pl->qpw * EX_WARPS;

    // records, cut into items of about `item_stages` pipeline stages
    std::vector<BatchProb> recs(count);
    std::vector<double> cost(count);
    for (int i = 0; i < count; ++i) {
        const knnb200_problem &q = in[i];
        BatchProb &P = recs[i];
        P.N = q.ref_nb;
        P.Q = q.query_nb;
        P.d = q.dim;
        P.k = q.k;
        P.n_rtiles = (q.ref_nb + EX_BR - 1) / EX_BR;
        P.n_dchunks = (q.dim + EX_BD - 1) / EX_BD;
        P.qtiles = (q.query_nb + bq - 1) / bq;
        const long long stages = (long long)P.n_rtiles * P.n_dchunks;
        int S = (int)std::max<long long>(1, (stages + item_stages / 2) / item_stages);
        // split lists of one query must fit one merge warp's shared slab
        S = std::min({S, P.n_rtiles, 256, (int)(kBatchMergeSmemMax / (8ull * q.k))});
        P.n_splits = std::max(1, S);
        P.qry = q.query;
        P.ldq = q.query_ld;
        P.ld2 = round_up(q.query_nb, 32);
        P.out_dist = q.knn_dist;
        P.out_idx = q.knn_index;
        P.ld_out = q.out_ld;
        cost[i] = (double)stages / P.n_splits;
    }
    // largest items first: the tail of the persistent launch holds small items
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });

    // scratch: duplicated queries + per-split lists; then the low-d
    // problems' split lists
    size_t sbytes = 0;
    std::vector<size_t> dup_off(count), part_off(count), low_off(low_idx.size());
    for (int i = 0; i < count; ++i) {
        BatchProb &P = recs[i];
        dup_off[i] = sbytes;
        sbytes += round_up((long long)P.d * P.ld2 * sizeof(float2), 256);
        part_off[i] = sbytes;
        if (P.n_splits > 1) sbytes += round_up((long long)P.n_splits * P.Q * P.k * 8, 256);
    }
    for (size_t j = 0; j < low_idx.size(); ++j) {
        const knnb200_problem &q = all[low_idx[j]];
        low_off[j] = sbytes;
        sbytes += round_up((long long)lowdim_scratch_bytes(q.ref_nb, q.query_nb, q.dim, q.k,
                                                           pl->num_sms),
                           256);
    }
    const size_t tbytes = round_up((long long)count * sizeof(BatchProb), 64) +
                          (size_t)2 * count * sizeof(CUtensorMap) + 64 + (size_t)count * 4 + 256;
    if (!pl->scratch.alloc(sbytes) || !pl->tables.alloc(tbytes)) {
        delete pl;
        return KNNB200_ENOMEM;
    }
    unsigned char *tb = static_cast<unsigned char *>(pl->tables.ptr);
    pl->probs = reinterpret_cast<BatchProb *>(tb);
    pl->maps = reinterpret_cast<CUtensorMap *>(tb + round_up((long long)count * sizeof(BatchProb), 64));
    pl->counter = reinterpret_cast<unsigned long long *>(pl->maps + 2 * count);
    pl->status = reinterpret_cast<int *>(pl->counter + 4);   // counter and status: 64 bytes
    pl->mlist = reinterpret_cast<int *>(pl->counter + 8);

    std::vector<BatchProb> table(count);
    std::vector<CUtensorMap> maps(2 * count);
    std::vector<int> mlist;
    long long item = 0, task = 0;
    int row = 0, max_slab = 0;
    unsigned char *sb = static_cast<unsigned char *>(pl->scratch.ptr);
    for (int r = 0; r < count; ++r) {
        const int i = order[r];
        BatchProb P = recs[i];
        const knnb200_problem &q = in[i];
        P.qdup = reinterpret_cast<float2 *>(sb + dup_off[i]);
        P.part = P.n_splits > 1 ? reinterpret_cast<unsigned long long *>(sb + part_off[i]) : nullptr;
        P.item_begin = item;
        item += (long long)P.qtiles * P.n_splits;
        P.merge_begin = P.n_splits > 1 ? task : -1;
        if (P.n_splits > 1) {
            mlist.push_back(r);
            task += P.Q;
            max_slab = std::max(max_slab, P.n_splits * P.k);
        }
        P.row_begin = row;
        row += P.d;
        if (!encode_f32_2d(&maps[2 * r], q.ref, (uint64_t)P.N, (uint64_t)P.d, (uint64_t)q.ref_ld,
                           EX_BR, EX_BD) ||
            !encode_f32_2d(&maps[2 * r + 1], P.qdup, (uint64_t)(2 * P.Q), (uint64_t)P.d,
                           (uint64_t)(2 * P.ld2), 2 * bq, EX_BD)) {
            delete pl;
            return KNNB200_ETENSORMAP;
        }
        table[r] = P;
    }
    for (size_t j = 0; j < low_idx.size(); ++j) {
        const knnb200_problem &q = all[low_idx[j]];
        ExactProblem e;
        e.ref = q.ref;
        e.N = q.ref_nb;
        e.ldr = q.ref_ld;
        e.qry = q.query;
        e.Q = q.query_nb;
        e.ldq = q.query_ld;
        e.d = q.dim;
        e.k = q.k;
        e.out_dist = q.knn_dist;
        e.out_idx = q.knn_index;
        e.ld_out = q.out_ld;
        e.scratch = sb + low_off[j];
        e.scratch_bytes = (j + 1 < low_idx.size() ? low_off[j + 1] : sbytes) - low_off[j];
        e.status = pl->status;
        e.num_sms = pl->num_sms;
        e.force_splits = 0;
        e.timer = nullptr;
        pl->lowdim.push_back(e);
    }
    pl->count = count;
    pl->n_split_probs = (int)mlist.size();
    pl->n_items = item;
    pl->n_tasks = task;
    pl->n_rows = row;
    pl->slab_keys = max_slab;
    pl->merge_wpb = max_slab ? (int)std::max<size_t>(
                                   1, std::min<size_t>(8, kBatchMergeSmemMax / (8ull * max_slab)))
                             : 1;
    if ((count > 0 &&
         (cudaMemcpy(pl->probs, table.data(), count * sizeof(BatchProb),
                     cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(pl->maps, maps.data(), 2 * count * sizeof(CUtensorMap),
                     cudaMemcpyHostToDevice) != cudaSuccess)) ||
        (!mlist.empty() && cudaMemcpy(pl->mlist, mlist.data(), mlist.size() * sizeof(int),
                                      cudaMemcpyHostToDevice) != cudaSuccess)) {
        delete pl;
        return KNNB200_ECUDA;
    }
    *out = pl;
    return KNNB200_OK;
}

int knnb200_batched_plan_create(const knnb200_problem *in, int count, int item_stages,
                                knnb200_batched_plan **out) {
    const knnb200_batched_config c{item_stages, 0, 0};
    return knnb200_batched_plan_create_config(in, count, &c, out);
}

int knnb200_batched_plan_config(const knnb200_batched_plan *pl, knnb200_batched_config *cfg,
                                int *lowdim_problems) {
    if (!pl) return KNNB200_EINVAL;
    if (cfg) {
        cfg->item_stages = pl->item_stages;
        cfg->queries_per_warp = pl->qpw;
        cfg->lowdim_kernel = pl->lowdim.empty() ? 0 : 1;
    }
    if (lowdim_problems) *lowdim_problems = (int)pl->lowdim.size();
    return KNNB200_OK;
}

int knnb200_batched_run(knnb200_batched_plan *pl, void *stream) {
    if (!pl) return KNNB200_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // queue counter and status word (the first 64 bytes after the maps)
    if (cudaMemsetAsync(pl->counter, 0, 64, st) != cudaSuccess) return KNNB200_ECUDA;
    // low-d problems: one launch each (plus a split merge), no waits, so the
    // plan stays capturable
    for (const ExactProblem &e : pl->lowdim)
        if (launch_lowdim(e, st) != kOk) return KNNB200_ELAUNCH;
    if (pl->count == 0) return KNNB200_OK;
    batched_dup_kernel<<<pl->n_rows, 256, 0, st>>>(pl->probs, pl->count, pl->n_rows);
    if (cudaGetLastError() != cudaSuccess) return KNNB200_ELAUNCH;
    cudaError_t e;
    if (pl->kcap == 256) {
        e = launch_batched_t<EX_QPW_K256, 256>(pl, st);
    } else if (pl->qpw == 2) {
        switch (pl->kcap) {
            case 32: e = launch_batched_t<2, 32>(pl, st); break;
            case 64: e = launch_batched_t<2, 64>(pl, st); break;
            default: e = launch_batched_t<2, 128>(pl, st); break;
        }
    } else {
        switch (pl->kcap) {
            case 32: e = launch_batched_t<EX_QPW, 32>(pl, st); break;
            case 64: e = launch_batched_t<EX_QPW, 64>(pl, st); break;
            default: e = launch_batched_t<EX_QPW, 128>(pl, st); break;
        }
    }
    if (e != cudaSuccess) return KNNB200_ELAUNCH;
    if (pl->n_tasks > 0) {
        const size_t smem = (size_t)pl->merge_wpb * pl->slab_keys * 8;
        if (cudaFuncSetAttribute(batched_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kBatchMergeSmemMax) != cudaSuccess)
            return KNNB200_ELAUNCH;
        const long long blocks = (pl->n_tasks + pl->merge_wpb - 1) / pl->merge_wpb;
        batched_merge_kernel<<<(unsigned)blocks, pl->merge_wpb * 32, smem, st>>>(
            pl->probs, pl->mlist, pl->n_split_probs, pl->n_tasks, pl->slab_keys);
        if (cudaGetLastError() != cudaSuccess) return KNNB200_ELAUNCH;
    }
    return KNNB200_OK;
}

int knnb200_batched_status(knnb200_batched_plan *pl, void *stream) {
    if (!pl) return KNNB200_EINVAL;
    int s = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(&s, pl->status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return KNNB200_ECUDA;
    return s ? KNNB200_ETIMEOUT : KNNB200_OK;
}

long long knnb200_batched_items(const knnb200_batched_plan *pl) { return pl ? pl->n_items : 0; }

void knnb200_batched_plan_destroy(knnb200_batched_plan *pl) {
    if (!pl) return;
    cudaSetDevice(pl->device);
    delete pl;
}

int knnb200_batched_graph_create(knnb200_batched_plan *pl, void **graph_exec) {
    if (!pl || !graph_exec) return KNNB200_EINVAL;
    *graph_exec = nullptr;
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return KNNB200_ECUDA;
    cudaGraph_t g = nullptr;
    int rc = KNNB200_OK;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        rc = KNNB200_ECUDA;
    } else {
        rc = knnb200_batched_run(pl, cs);
        if (cudaStreamEndCapture(cs, &g) != cudaSuccess && rc == KNNB200_OK) rc = KNNB200_ECUDA;
    }
    cudaGraphExec_t ex = nullptr;
    if (rc == KNNB200_OK && cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) rc = KNNB200_ECUDA;
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    if (rc != KNNB200_OK) {
        cudaGetLastError();
        return rc;
    }
    *graph_exec = ex;
    return KNNB200_OK;
}

int knnb200_graph_launch(void *graph_exec, void *stream) {
    if (!graph_exec) return KNNB200_EINVAL;
    return cudaGraphLaunch(static_cast<cudaGraphExec_t>(graph_exec),
                           static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? KNNB200_OK
               : KNNB200_ECUDA;
}

void knnb200_graph_destroy(void *graph_exec) {
    if (graph_exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(graph_exec));
}

// Times one plan configuration: a warm-up run, then three.
static int time_config(const knnb200_problem *in, int count, const knnb200_batched_config &c,
                       cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, float *ms_out) {
    knnb200_batched_plan *pl = nullptr;
    int rc = knnb200_batched_plan_create_config(in, count, &c, &pl);
    if (rc != KNNB200_OK) return rc;
    float ms = 0.f;
    rc = knnb200_batched_run(pl, st);   // warm-up
    if (rc == KNNB200_OK) {
        cudaEventRecord(e0, st);
        for (int r = 0; r < 3 && rc == KNNB200_OK; ++r) rc = knnb200_batched_run(pl, st);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = KNNB200_ECUDA;
        cudaEventElapsedTime(&ms, e0, e1);
    }
    if (rc == KNNB200_OK) rc = knnb200_batched_status(pl, st);
    knnb200_batched_plan_destroy(pl);
    *ms_out = ms / 3;
    return rc;
}

int knnb200_batched_autotune_config(const knnb200_problem *in, int count, void *stream,
                                    knnb200_batched_config *best_cfg, float *best_ms) {
    if (!in || count < 1 || !best_cfg) return KNNB200_EINVAL;
    static const int stage_cands[] = {32, 64, 128, 256, 512, 1024, 2048};
    static const int qpw_cands[] = {4, 2};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    knnb200_batched_config bc{256, 4, 0};
    int rc = KNNB200_OK;
    // work-item size first (with the default tile shape), then the tile
    // shape and the low-d routing at the best size
    for (int c : stage_cands) {
        const knnb200_batched_config cfg{c, 4, 0};
        float ms = 0.f;
        if ((rc = time_config(in, count, cfg, st, e0, e1, &ms)) != KNNB200_OK) break;
        if (ms < best) {
            best = ms;
            bc = cfg;
        }
    }
    for (int qpw : qpw_cands) {
        for (int low = 0; low < 2 && rc == KNNB200_OK; ++low) {
            const knnb200_batched_config cfg{bc.item_stages, qpw, low};
            if (qpw == bc.queries_per_warp && low == bc.lowdim_kernel) continue;
            float ms = 0.f;
            if ((rc = time_config(in, count, cfg, st, e0, e1, &ms)) != KNNB200_OK) break;
            if (ms < best) {
                best = ms;
                bc = cfg;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != KNNB200_OK) return rc;
    *best_cfg = bc;
    if (best_ms) *best_ms = best;
    return KNNB200_OK;
}

int knnb200_batched_autotune(const knnb200_problem *in, int count, void *stream,
                             int *best_item_stages, float *best_ms) {
    if (!in || count < 1 || !best_item_stages) return KNNB200_EINVAL;
    static const int cands[] = {32, 64, 128, 256, 512, 1024, 2048};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int bestc = 256, rc = KNNB200_OK;
    for (int c : cands) {
        float ms = 0.f;
        if ((rc = time_config(in, count, knnb200_batched_config{c, 0, 0}, st, e0, e1, &ms)) !=
            KNNB200_OK)
            break;
        if (ms < best) {
            best = ms;
            bestc = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != KNNB200_OK) return rc;
    *best_item_stages = bestc;
    if (best_ms) *best_ms = best;
    return KNNB200_OK;
}

}  // extern "C"
