// knn_serve.cu -- resident reference sets and a continuous-batching server.
//
// The reference uploads the reference set on every call (code/knncuda.cu:341,
// :695), which dominates at large ref_nb.  A knnb200_refset keeps it on the
// device once -- the FP32 dim x N copy used by the exact kernel and, when the
// shape qualifies, the prepared tensor-core view (BF16 K-major copy, FP32
// point-major copy, norms) -- so queries pay only for themselves.
//
// knnb200_server runs a request loop over one refset: requests (host query
// sets of any size, any k) are queued; `slots` worker threads, each with its
// own stream and scratch, repeatedly form a batch from the head of the queue
// (up to max_batch_queries queries) and run it.  Batches are admitted only
// while the working memory of all batches in flight stays within the memory
// budget; a request that arrives while others are on the GPU joins the next
// batch a free slot forms, and batches of different slots overlap on the
// device.  A batch computes the top-k_max of all its queries; a request with
// k_i <= k_max receives the first k_i rows, which is exactly its own top-k_i
// (results are ordered by (distance, index)), so a request's answer does not
// depend on what it was batched with.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/knn_b200.h"
#include "knn_kernels.h"

namespace knnb200 {
namespace {

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    bool ensure(size_t need) {
        if (need <= bytes) return true;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        const size_t want = need + need / 8 + 256;
        if (cudaMalloc(&ptr, want) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        bytes = want;
        return true;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// Per-worker execution context: stream, scratch and staging buffers.
struct Slot {
    cudaStream_t stream = nullptr;
    DevBuf scratch, qry, dist, idx, status;
    int *host_stats = nullptr;   // pinned, 8 ints
    bool init(int device) {
        if (cudaSetDevice(device) != cudaSuccess) return false;
        if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return false;
        if (!status.ensure(sizeof(int))) return false;
        if (cudaMallocHost(reinterpret_cast<void **>(&host_stats), 8 * sizeof(int)) != cudaSuccess)
            return false;
        return true;
    }
    void destroy() {
        if (stream) cudaStreamSynchronize(stream);
        scratch.release();
        qry.release();
        dist.release();
        idx.release();
        status.release();
        if (host_stats) cudaFreeHost(host_stats);
        if (stream) cudaStreamDestroy(stream);
        host_stats = nullptr;
        stream = nullptr;
    }
};

int num_sms_of(int device) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return sms;
}

}  // namespace
}  // namespace knnb200

using namespace knnb200;

struct knnb200_refset {
    int device = 0;
    int N = 0, d = 0;
    long long ldr = 0;
    int num_sms = 148;
    DevBuf ref;          // [d][ldr] FP32
    DevBuf tcmem;        // prepared tensor-core view
    TcRefView tc{};
    TcRefState tc_state;
    bool has_tc = false;
    std::mutex mu;       // guards `slot` for knnb200_refset_knn
    Slot slot;
};

namespace {

bool use_tc_for(const knnb200_refset *rs, int method, int Q, int k) {
    return (method == KNNB200_METHOD_CUBLAS || method == KNNB200_METHOD_FP8) && rs->has_tc &&
           tc_supported(rs->N, Q, rs->d, k);
}

size_t scratch_need(const knnb200_refset *rs, int method, int Q, int k) {
    return use_tc_for(rs, method, Q, k) ? tc_scratch_bytes(rs->N, Q, rs->d, k, rs->num_sms)
                                        : exact_scratch_bytes(rs->N, Q, rs->d, k, rs->num_sms);
}

// Queue one k-NN of device-resident queries against the resident set on
// `st`, with the slot's scratch.  The tensor-core path synchronises `st` once.
int run_refset(knnb200_refset *rs, Slot &slot, const float *query, int Q, long long ldq, int k,
               int method, float *dist, int *idx, long long ld_out, cudaStream_t st) {
    if (!exact_supported_k(k)) return kErrUnsupported;
    if (!slot.scratch.ensure(scratch_need(rs, method, Q, k))) return kErrNoMemory;
    if (cudaMemsetAsync(slot.status.ptr, 0, sizeof(int), st) != cudaSuccess) return kErrCuda;
    if (use_tc_for(rs, method, Q, k)) {
        TcProblem t;
        t.ref = static_cast<const float *>(rs->ref.ptr);
        t.N = rs->N;
        t.ldr = rs->ldr;
        t.qry = query;
        t.Q = Q;
        t.ldq = ldq;
        t.d = rs->d;
        t.k = k;
        t.out_dist = dist;
        t.out_idx = idx;
        t.ld_out = ld_out;
        t.scratch = slot.scratch.ptr;
        t.scratch_bytes = slot.scratch.bytes;
        t.status = static_cast<int *>(slot.status.ptr);
        t.num_sms = rs->num_sms;
        t.timer = nullptr;
        t.request = (method == KNNB200_METHOD_FP8 && tc_fp8_supported(rs->d)) ? kTcReqFp8
                                                                             : kTcReqBf16;
        t.point_sample = true;   // the resident set was prepared as a whole
        return launch_tc(t, rs->tc, st, slot.host_stats);
    }
    ExactProblem p;
    p.ref = static_cast<const float *>(rs->ref.ptr);
    p.N = rs->N;
    p.ldr = rs->ldr;
    p.qry = query;
    p.Q = Q;
    p.ldq = ldq;
    p.d = rs->d;
    p.k = k;
    p.out_dist = dist;
    p.out_idx = idx;
    p.ld_out = ld_out;
    p.scratch = slot.scratch.ptr;
    p.scratch_bytes = slot.scratch.bytes;
    p.status = static_cast<int *>(slot.status.ptr);
    p.num_sms = rs->num_sms;
    p.force_splits = 0;
    p.timer = nullptr;
    return launch_exact(p, st);
}

// Device status word of a slot after its stream is synchronised.
int slot_status(Slot &slot, cudaStream_t st) {
    int s = 0;
    if (cudaMemcpyAsync(&s, slot.status.ptr, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return kErrCuda;
    return s ? kErrDeviceTimeout : kOk;
}

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

}  // namespace

extern "C" {

int knnb200_refset_create(const float *ref, int ref_nb, long long ref_ld, int dim, int on_device,
                          knnb200_refset **out) {
    if (!out) return KNNB200_EINVAL;
    *out = nullptr;
    if (!ref || ref_nb < 1 || dim < 1 || ref_ld < ref_nb) return KNNB200_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return KNNB200_ENODEV;
    }
    knnb200_refset *rs = new knnb200_refset();
    cudaGetDevice(&rs->device);
    rs->N = ref_nb;
    rs->d = dim;
    rs->ldr = round_up(ref_nb, 64);
    rs->num_sms = num_sms_of(rs->device);
    int rc = KNNB200_OK;
    if (!rs->slot.init(rs->device)) rc = KNNB200_ECUDA;
    if (rc == KNNB200_OK && !rs->ref.ensure((size_t)dim * rs->ldr * sizeof(float)))
        rc = KNNB200_ENOMEM;
    cudaStream_t st = rs->slot.stream;
    if (rc == KNNB200_OK &&
        cudaMemcpy2DAsync(rs->ref.ptr, rs->ldr * sizeof(float), ref, ref_ld * sizeof(float),
                          ref_nb * sizeof(float), dim,
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                          st) != cudaSuccess)
        rc = KNNB200_ECUDA;
    // the tensor-core view, when the shape qualifies for any k
    if (rc == KNNB200_OK && tc_supported(ref_nb, 1, dim, 1)) {
        if (!rs->tcmem.ensure(tc_ref_bytes(ref_nb, dim))) {
            rc = KNNB200_ENOMEM;
        } else {
            rs->tc = tc_carve_ref(rs->tcmem.ptr, ref_nb, dim, &rs->tc_state);
            // every copy prepared now: the server's slots share the set
            if (tc_prepare_ref(rs->tc, static_cast<const float *>(rs->ref.ptr), ref_nb, rs->ldr,
                               dim, st) != kOk ||
                tc_prepare_extras(rs->tc, ref_nb, dim, st, rs->slot.host_stats + 2) != kOk)
                rc = KNNB200_ELAUNCH;
            else
                rs->has_tc = true;
        }
    }
    if (rc == KNNB200_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = KNNB200_ECUDA;
    if (rc != KNNB200_OK) {
        cudaGetLastError();
        rs->slot.destroy();
        rs->ref.release();
        rs->tcmem.release();
        delete rs;
        return rc;
    }
    *out = rs;
    return KNNB200_OK;
}

void knnb200_refset_destroy(knnb200_refset *rs) {
    if (!rs) return;
    cudaSetDevice(rs->device);
    rs->slot.destroy();
    rs->ref.release();
    rs->tcmem.release();
    delete rs;
}

size_t knnb200_refset_device_bytes(const knnb200_refset *rs) {
    return rs ? rs->ref.bytes + rs->tcmem.bytes : 0;
}

int knnb200_refset_knn(knnb200_refset *rs, const float *query, int query_nb, long long query_ld,
                       int k, int method, float *knn_dist, int *knn_index, long long out_ld,
                       void *stream) {
    if (!rs || !query || !knn_dist || !knn_index) return KNNB200_EINVAL;
    if (query_nb < 1 || k < 1 || k > rs->N || query_ld < query_nb || out_ld < query_nb)
        return KNNB200_EINVAL;
    if (query_ld % 4 || (reinterpret_cast<uintptr_t>(query) & 15)) return KNNB200_EINVAL;
    if (method < KNNB200_METHOD_GLOBAL || method > KNNB200_METHOD_FP8) return KNNB200_EINVAL;
    std::lock_guard<std::mutex> lock(rs->mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // scratch of the refset's own slot: order this call after its previous one
    int rc = run_refset(rs, rs->slot, query, query_nb, query_ld, k, method, knn_dist, knn_index,
                        out_ld, st);
    if (rc != kOk) return rc;
    return slot_status(rs->slot, st);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Continuous-batching server
// ---------------------------------------------------------------------------
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    const float *query = nullptr;   // host, dim x qn
    int qn = 0, k = 0;
    float *dist = nullptr;          // host, k x qn
    int *idx = nullptr;
    Clock::time_point submitted, finished;
    int status = 0;
    bool done = false;
};

}  // namespace

struct knnb200_server {
    knnb200_refset *rs = nullptr;
    int method = 0;
    size_t budget = 0;
    int max_batch = 0;
    std::vector<Slot> slots;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::unordered_map<long long, Request *> live;
    size_t inflight = 0;
    int busy_slots = 0;
    bool stop = false;
    long long next_id = 1;
    std::vector<double> lat_ms;
    long long queries_done = 0, batches_done = 0;
    Clock::time_point t_first, t_last;
    bool any = false;
};

namespace {

// Slot buffers are sized at server creation for a full batch at this k
// (larger k grows them on first use).
constexpr int kPresizeK = 128;

size_t batch_bytes(const knnb200_server *s, int Q, int kmax) {
    const knnb200_refset *rs = s->rs;
    return (size_t)rs->d * round_up(Q, 64) * 4 + (size_t)kmax * Q * 8 +
           scratch_need(rs, s->method, Q, kmax);
}

void run_batch(knnb200_server *s, Slot &slot, std::vector<Request *> &batch) {
    knnb200_refset *rs = s->rs;
    int Q = 0, kmax = 0;
    for (Request *r : batch) {
        Q += r->qn;
        kmax = std::max(kmax, r->k);
    }
    const long long ldq = round_up(Q, 64);
    cudaStream_t st = slot.stream;
    int rc = kOk;
    if (!slot.qry.ensure((size_t)rs->d * ldq * 4) || !slot.dist.ensure((size_t)kmax * Q * 4) ||
        !slot.idx.ensure((size_t)kmax * Q * 4))
        rc = kErrNoMemory;
    float *qd = static_cast<float *>(slot.qry.ptr);
    float *dd = static_cast<float *>(slot.dist.ptr);
    int *id = static_cast<int *>(slot.idx.ptr);
    long long off = 0;
    for (Request *r : batch) {
        if (rc != kOk) break;
        if (cudaMemcpy2DAsync(qd + off, ldq * 4, r->query, (size_t)r->qn * 4, (size_t)r->qn * 4,
                              rs->d, cudaMemcpyHostToDevice, st) != cudaSuccess)
            rc = kErrCuda;
        off += r->qn;
    }
    if (rc == kOk)
        rc = run_refset(rs, slot, qd, Q, ldq, kmax, s->method, dd, id, Q, st);
    off = 0;
    for (Request *r : batch) {
        if (rc != kOk) break;
        if (cudaMemcpy2DAsync(r->dist, (size_t)r->qn * 4, dd + off, (size_t)Q * 4,
                              (size_t)r->qn * 4, r->k, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpy2DAsync(r->idx, (size_t)r->qn * 4, id + off, (size_t)Q * 4,
                              (size_t)r->qn * 4, r->k, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            rc = kErrCuda;
        off += r->qn;
    }
    if (rc == kOk) rc = slot_status(slot, st);
    if (rc != kOk) cudaGetLastError();
    const Clock::time_point now = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    for (Request *r : batch) {
        r->status = rc;
        r->finished = now;
        r->done = true;
        s->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - r->submitted).count());
        s->queries_done += r->qn;
    }
    s->batches_done += 1;
    s->t_last = now;
}

void worker_loop(knnb200_server *s, int w) {
    cudaSetDevice(s->rs->device);
    Slot &slot = s->slots[w];
    for (;;) {
        std::vector<Request *> batch;
        size_t need = 0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (s->stop && s->queue.empty()) return;
                if (!s->queue.empty()) {
                    // form a batch from the head of the queue
                    int Q = 0, kmax = 0;
                    size_t take = 0;
                    for (Request *r : s->queue) {
                        if (take > 0 && Q + r->qn > s->max_batch) break;
                        Q += r->qn;
                        kmax = std::max(kmax, r->k);
                        ++take;
                    }
                    need = batch_bytes(s, Q, kmax);
                    // memory admission: admit while the in-flight working set
                    // fits the budget (an idle server always admits one batch)
                    if (s->inflight == 0 || s->inflight + need <= s->budget) {
                        for (size_t i = 0; i < take; ++i) {
                            batch.push_back(s->queue.front());
                            s->queue.pop_front();
                        }
                        s->inflight += need;
                        s->busy_slots += 1;
                        break;
                    }
                }
                s->cv_work.wait(lk);
            }
        }
        run_batch(s, slot, batch);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->inflight -= need;
            s->busy_slots -= 1;
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

int knnb200_server_create(knnb200_refset *rs, int slots, size_t memory_budget_bytes,
                          int max_batch_queries, int method, knnb200_server **out) {
    if (!out) return KNNB200_EINVAL;
    *out = nullptr;
    if (!rs || slots < 1 || slots > 16 || max_batch_queries < 1) return KNNB200_EINVAL;
    if (method < KNNB200_METHOD_GLOBAL || method > KNNB200_METHOD_FP8) return KNNB200_EINVAL;
    knnb200_server *s = new knnb200_server();
    s->rs = rs;
    s->method = method;
    s->budget = memory_budget_bytes;
    s->max_batch = max_batch_queries;
    s->slots.resize(slots);
    for (int i = 0; i < slots; ++i)
        if (!s->slots[i].init(rs->device)) {
            for (int j = 0; j <= i; ++j) s->slots[j].destroy();
            delete s;
            return KNNB200_ECUDA;
        }
    // Size every slot for a full batch at k = kPresizeK now: growing a
    // buffer later frees device memory, which synchronises the whole device
    // and stalls every slot's batch in flight.
    const int kq = std::min(kPresizeK, rs->N);
    const long long ldq = round_up(max_batch_queries, 64);
    for (int i = 0; i < slots; ++i) {
        Slot &sl = s->slots[i];
        if (!sl.qry.ensure((size_t)rs->d * ldq * 4) ||
            !sl.dist.ensure((size_t)kq * max_batch_queries * 4) ||
            !sl.idx.ensure((size_t)kq * max_batch_queries * 4) ||
            !sl.scratch.ensure(scratch_need(rs, method, max_batch_queries, kq))) {
            for (int j = 0; j < slots; ++j) s->slots[j].destroy();
            delete s;
            return KNNB200_ENOMEM;
        }
    }
    for (int i = 0; i < slots; ++i) s->workers.emplace_back(worker_loop, s, i);
    *out = s;
    return KNNB200_OK;
}

long long knnb200_server_submit(knnb200_server *s, const float *query, int query_nb, int k,
                                float *knn_dist, int *knn_index) {
    if (!s || !query || !knn_dist || !knn_index || query_nb < 1 || k < 1 || k > s->rs->N ||
        !exact_supported_k(k))
        return -KNNB200_EINVAL;
    if (s->budget && batch_bytes(s, query_nb, k) > s->budget) return -KNNB200_ENOMEM;
    Request *r = new Request();
    r->query = query;
    r->qn = query_nb;
    r->k = k;
    r->dist = knn_dist;
    r->idx = knn_index;
    r->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete r;
            return -KNNB200_EINVAL;
        }
        r->id = s->next_id++;
        if (!s->any) {
            s->any = true;
            s->t_first = r->submitted;
        }
        s->live[r->id] = r;
        s->queue.push_back(r);
    }
    s->cv_work.notify_one();
    return r->id;
}

int knnb200_server_wait(knnb200_server *s, long long ticket, double *latency_ms) {
    if (!s) return KNNB200_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->live.find(ticket);
    if (it == s->live.end()) return KNNB200_EINVAL;
    Request *r = it->second;
    s->cv_done.wait(lk, [r]() { return r->done; });
    const int st = r->status;
    if (latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(r->finished - r->submitted).count();
    s->live.erase(it);
    delete r;
    return st;
}

int knnb200_server_stats(knnb200_server *s, double *p50_ms, double *p99_ms,
                         long long *queries_done, long long *batches_done, double *wall_seconds) {
    if (!s) return KNNB200_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&v](double p) {
        if (v.empty()) return 0.0;
        const size_t i = std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5));
        return v[i];
    };
    if (p50_ms) *p50_ms = pct(0.50);
    if (p99_ms) *p99_ms = pct(0.99);
    if (queries_done) *queries_done = s->queries_done;
    if (batches_done) *batches_done = s->batches_done;
    if (wall_seconds)
        *wall_seconds =
            s->any ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0.0;
    return KNNB200_OK;
}

void knnb200_server_destroy(knnb200_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    cudaSetDevice(s->rs->device);
    for (auto &sl : s->slots) sl.destroy();
    for (auto &kv : s->live) delete kv.second;
    delete s;
}

}  // extern "C"
