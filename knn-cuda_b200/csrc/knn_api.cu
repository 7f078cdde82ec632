// knn_api.cu -- host runtime and C ABI of libknnb200.so.
//
// Drop-in entry points knn_cuda_global / knn_cuda_texture / knn_cublas with
// the reference's signatures, C++ linkage and bool + "ERROR: ..." contract
// (code/knncuda.h:14-68; error convention e.g. code/knncuda.cu:290-293,
// :315-322), plus extern "C" aliases and a device-resident entry point.
//
// Where the reference allocates, copies and frees every buffer inside every
// call (code/knncuda.cu:311-314, :341-342, :409-412) -- including the
// ref_nb x query_nb FP32 distance matrix -- this runtime keeps a per-device
// workspace (grow-only device buffers, one stream, one status word) guarded
// by a mutex, so calls are thread-safe and no distance matrix exists.
#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include <cudaTypedefs.h>

#include "../../include/knn_b200.h"
#include "../../include/knncuda.h"
#include "knn_kernels.h"

namespace knnb200 {

// ---------------------------------------------------------------------------
// TMA descriptor encoding through the driver entry point (no -lcuda needed).
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

bool encode_2d(CUtensorMap *map, CUtensorMapDataType dtype, int elem_bytes, const void *base,
               uint64_t cols, uint64_t rows, uint64_t ld_elems, uint32_t box_cols,
               uint32_t box_rows, CUtensorMapSwizzle swizzle) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = get_encode_fn();
    if (!enc) return false;
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {ld_elems * (uint64_t)elem_bytes};
    cuuint32_t box[2] = {box_cols, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, dtype, 2, const_cast<void *>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// ---------------------------------------------------------------------------
// Per-device workspace.
// ---------------------------------------------------------------------------
namespace {

constexpr int kMaxDevices = 64;

struct Buffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    // Grow-only: keeps the allocation when it is large enough.
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

// A small pool of host threads for gathering pageable input into pinned
// staging buffers (memcpy of many rows at once).  run(n, fn) calls fn(i)
// for i in [0, n) on the pool and the calling thread, and returns when all
// are done.
class HostPool {
  public:
    explicit HostPool(int threads) {
        for (int t = 0; t < threads; ++t) workers_.emplace_back([this] { loop(); });
    }
    ~HostPool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (std::thread &t : workers_) t.join();
    }
    void run(int n, const std::function<void(int)> &fn) {
        {
            std::lock_guard<std::mutex> g(mu_);
            fn_ = &fn;
            n_ = n;
            next_ = 0;
            done_ = 0;
            ++gen_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> g(mu_);
        done_cv_.wait(g, [this] { return done_ == n_; });
        fn_ = nullptr;
    }

  private:
    void work() {
        for (;;) {
            int i;
            const std::function<void(int)> *fn;
            {
                std::lock_guard<std::mutex> g(mu_);
                if (!fn_ || next_ >= n_) return;
                i = next_++;
                fn = fn_;
            }
            (*fn)(i);
            std::lock_guard<std::mutex> g(mu_);
            if (++done_ == n_) done_cv_.notify_all();
        }
    }
    void loop() {
        long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)> *fn_ = nullptr;
    int n_ = 0, next_ = 0, done_ = 0;
    long long gen_ = 0;
    bool stop_ = false;
};

// Pinned staging of the streamed host entry for pageable input: two
// buffers; the host gathers a piece of the reference set into one while the
// other's copy is in flight.
constexpr size_t kStageBytes = 32u << 20;

// count floats from src to a 16-byte aligned dst with non-temporal stores:
// the staging buffer is read next by the copy engine, not by this core, so
// the stores skip the read-for-ownership of a cached write (with the copy
// engine reading the buffer meanwhile, the host's memory bandwidth is what
// bounds the gather).
static void stage_row(float *dst, const float *src, size_t count) {
#if defined(__SSE2__)
    if ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0) {
        size_t i = 0;
        for (; i + 16 <= count; i += 16) {
            const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i));
            const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i + 4));
            const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i + 8));
            const __m128i d = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i + 12));
            _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i), a);
            _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 4), b);
            _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 8), c);
            _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 12), d);
        }
        if (i < count) std::memcpy(dst + i, src + i, (count - i) * sizeof(float));
        _mm_sfence();   // the stores are visible before the copy is queued
        return;
    }
#endif
    std::memcpy(dst, src, count * sizeof(float));
}

// Host entry of knn_cublas on large sets: the reference set is copied in
// this many chunks (after the sample runs of the threshold pass), each
// chunk's prep and scan overlapping the copy of the next.  Relative chunk
// sizes: the last ones shrink so that little scanning is left once the last
// byte has landed (each chunk's scan still ends before the next chunk's
// copy: the scan runs about 2.5x faster than the copy).
constexpr int kStreamChunks = 8;
constexpr int kStreamWeights[kStreamChunks] = {8, 8, 8, 8, 6, 4, 2, 1};
constexpr int kStreamMinPoints = 1 << 18;

struct Workspace {
    std::mutex mu;
    bool init = false;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t last_done = nullptr;   // orders device-resident calls on this device
    Buffer ref, qry, dist, idx, scratch, status;
    Buffer tcref;                      // prepared reference set of the tensor-core path
    TcRefState tc_state;               // its host-side state
    Buffer bound;                      // re-rank bound check (test-only, off by default)
    bool bound_check = false;
    PhaseTimer timer;                  // optional per-phase device timing
    int *status_host = nullptr;        // pinned status word for the host path
    int *tc_stats = nullptr;           // pinned: [0] second-scan queries, [1] exact fallbacks
    cudaStream_t copy_stream = nullptr;          // host entry: reference copies
    cudaEvent_t copied[1 + kStreamChunks] = {};  // sample, then each chunk
    float *stage[2] = {nullptr, nullptr};        // pinned staging for pageable input
    cudaEvent_t stage_done[2] = {};              // the copy out of each stage has ended
    int stage_slot = 0;
    std::unique_ptr<HostPool> pool;              // gathers into the staging buffers

    // Staging buffers and the pool, on first use.
    bool ensure_staging() {
        if (stage[0]) return true;
        for (int i = 0; i < 2; ++i) {
            if (cudaMallocHost(reinterpret_cast<void **>(&stage[i]), kStageBytes) != cudaSuccess ||
                cudaEventCreateWithFlags(&stage_done[i], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                return false;
            }
        }
        const unsigned hc = std::thread::hardware_concurrency();
        pool.reset(new HostPool((int)std::max(1u, std::min(16u, hc ? hc : 4u)) - 1));
        return true;
    }

    bool setup(int dev) {
        if (init) return true;
        device = dev;
        if (cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return false;
        if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return false;
        if (cudaEventCreateWithFlags(&last_done, cudaEventDisableTiming) != cudaSuccess)
            return false;
        if (!status.ensure(sizeof(int))) return false;
        if (cudaMallocHost(reinterpret_cast<void **>(&status_host), sizeof(int)) != cudaSuccess)
            return false;
        if (cudaMallocHost(reinterpret_cast<void **>(&tc_stats), 8 * sizeof(int)) != cudaSuccess)
            return false;
        for (int i = 0; i < PhaseTimer::kMaxMarks; ++i)
            if (cudaEventCreate(&timer.ev[i]) != cudaSuccess) return false;
        if (cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking) != cudaSuccess)
            return false;
        for (cudaEvent_t &e : copied)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
        init = true;
        return true;
    }
};

Workspace g_ws[kMaxDevices];
int g_force_kind = -1;   // knnb200_set_tc_kind_override

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

bool valid_sizes(int ref_nb, int query_nb, int dim, int k) {
    return ref_nb >= 1 && query_nb >= 1 && dim >= 1 && k >= 1 && k <= ref_nb;
}

bool use_tc(int method, int N, int Q, int d, int k) {
    return (method == KNNB200_METHOD_CUBLAS || method == KNNB200_METHOD_FP8) &&
           tc_supported(N, Q, d, k);
}

size_t scratch_for(int method, int N, int Q, int d, int k, int num_sms) {
    if (use_tc(method, N, Q, d, k)) return tc_scratch_bytes(N, Q, d, k, num_sms);
    return exact_scratch_bytes(N, Q, d, k, num_sms);
}

// Queue the computation for one problem whose inputs are on the device.
// knn_cublas runs the tensor-core expansion path when the shape qualifies
// (it synchronises the stream once, to recompute uncertified queries);
// everything else runs the fused exact kernel.
// ref_prepared: the tensor-core view of this reference set is already in
// ws.tcref (a later query chunk of the same call).
int enqueue(Workspace &ws, const ExactProblem &p0, int method, cudaStream_t st,
            bool ref_prepared = false) {
    for (int i = 0; i < 8; ++i) ws.tc_stats[i] = 0;
    ws.tc_stats[6] = ws.tc_stats[7] = -1;
    if (!exact_supported_k(p0.k)) return kErrUnsupported;
    ExactProblem p = p0;
    p.timer = &ws.timer;
    ws.timer.begin(st);
    if (!use_tc(method, p.N, p.Q, p.d, p.k)) return launch_exact(p, st);
    if (!ws.tcref.ensure(tc_ref_bytes(p.N, p.d))) return kErrNoMemory;
    // a later chunk of the same call keeps the view (and its prepared copies)
    TcRefView v = tc_carve_ref(ws.tcref.ptr, p.N, p.d, ref_prepared ? nullptr : &ws.tc_state);
    v.state = &ws.tc_state;
    int rc = ref_prepared ? kOk : tc_prepare_ref(v, p.ref, p.N, p.ldr, p.d, st);
    if (rc != kOk) return rc;
    ws.timer.mark(st, kPhaseTcPrepRef);
    TcProblem t;
    t.ref = p.ref;
    t.N = p.N;
    t.ldr = p.ldr;
    t.qry = p.qry;
    t.Q = p.Q;
    t.ldq = p.ldq;
    t.d = p.d;
    t.k = p.k;
    t.out_dist = p.out_dist;
    t.out_idx = p.out_idx;
    t.ld_out = p.ld_out;
    t.scratch = p.scratch;
    t.scratch_bytes = p.scratch_bytes;
    t.status = p.status;
    t.num_sms = p.num_sms;
    t.timer = &ws.timer;
    t.request = (method == KNNB200_METHOD_FP8 && tc_fp8_supported(p.d)) ? kTcReqFp8 : kTcReqBf16;
    t.force_kind = g_force_kind;
    t.point_sample = true;   // the whole set is prepared before pass 1
    if (ws.bound_check) {
        if (cudaMemsetAsync(ws.bound.ptr, 0, 16, st) != cudaSuccess) return kErrCuda;
        t.bound_stat = static_cast<unsigned *>(ws.bound.ptr);
    }
    return launch_tc(t, v, st, ws.tc_stats);
}

// Calls fn(g0, g1) for each maximal range of tiles [g0, g1) of [tb, te)
// outside the runs of the sample pattern s.
template <class F>
int for_each_gap(const TileRuns &s, int tb, int te, F fn) {
    int t = tb;
    while (t < te) {
        const int r0 = (t / s.period) * s.period;   // first tile of this period's run
        if (t < r0 + s.run) {
            t = std::min(te, r0 + s.run);
            continue;
        }
        const int g1 = std::min(te, r0 + s.period);
        const int rc = fn(t, g1);
        if (rc != kOk) return rc;
        t = g1;
    }
    return kOk;
}

// knn_cublas from pinned host memory: the reference set streams in on the
// copy stream -- first the sample runs of the threshold pass (runs of
// consecutive 256-point tiles, one 2-D copy per run), then kStreamChunks
// contiguous chunks without those runs -- and the compute stream prepares
// and scans each piece once its copy has landed, so the copy of the set
// overlaps the threshold pass and the pass-2 scan of all but the last
// (smallest) chunk.  Every byte crosses the bus once.
int enqueue_tc_streamed(Workspace &ws, const ExactProblem &p, const float *ref_host,
                        bool pinned, cudaStream_t st) {
    for (int i = 0; i < 8; ++i) ws.tc_stats[i] = 0;
    ws.tc_stats[6] = ws.tc_stats[7] = -1;
    ws.timer.begin(st);
    if (!ws.tcref.ensure(tc_ref_bytes(p.N, p.d))) return kErrNoMemory;
    if (!pinned && !ws.ensure_staging()) return kErrNoMemory;
    const TcRefView rv = tc_carve_ref(ws.tcref.ptr, p.N, p.d, &ws.tc_state);
    float *ref_d = const_cast<float *>(p.ref);
    const int T = tc_tile_points();
    const int n_tiles = (p.N + T - 1) / T;
    const TileRuns sample = tc_sample_runs(p.N, p.Q, p.d, p.k, p.num_sms);
    const size_t fb = sizeof(float);
    cudaStream_t cs = ws.copy_stream;
    // points [c0, c0 + len) of every dimension from page-locked memory: one
    // 2-D copy
    auto copy_direct = [&](size_t c0, size_t len) -> int {
        return cudaMemcpy2DAsync(ref_d + c0, (size_t)p.ldr * fb, ref_host + c0, (size_t)p.N * fb,
                                 len * fb, p.d, cudaMemcpyHostToDevice, cs) == cudaSuccess
                   ? kOk
                   : kErrCuda;
    };
    // the same from pageable memory: through the staging buffers, at most
    // kStageBytes per piece; the host gathers the piece's rows (the pool
    // splits them) while the previous piece's copy is in flight
    auto copy_staged = [&](size_t c0, size_t len) -> int {
        const size_t cols = std::max<size_t>(1, kStageBytes / ((size_t)p.d * fb));
        for (size_t q0 = c0; q0 < c0 + len; q0 += cols) {
            const size_t n = std::min(cols, c0 + len - q0);
            const int slot = ws.stage_slot;
            ws.stage_slot ^= 1;
            if (cudaEventSynchronize(ws.stage_done[slot]) != cudaSuccess) return kErrCuda;
            float *dst = ws.stage[slot];
            const std::function<void(int)> rows = [&](int dd) {
                stage_row(dst + (size_t)dd * n, ref_host + (size_t)dd * p.N + q0, n);
            };
            ws.pool->run(p.d, rows);
            if (cudaMemcpy2DAsync(ref_d + q0, (size_t)p.ldr * fb, dst, n * fb, n * fb, p.d,
                                  cudaMemcpyHostToDevice, cs) != cudaSuccess ||
                cudaEventRecord(ws.stage_done[slot], cs) != cudaSuccess)
                return kErrCuda;
        }
        return kOk;
    };
    // points [t0 T, t1 T) of every dimension
    auto copy_tiles = [&](int t0, int t1) -> int {
        const size_t p0 = (size_t)t0 * T, p1 = std::min<size_t>(p.N, (size_t)t1 * T);
        if (p0 >= p1) return kOk;
        return pinned ? copy_direct(p0, p1 - p0) : copy_staged(p0, p1 - p0);
    };
    // the copies start after everything queued so far on the compute stream
    // (an earlier call may still read the reference buffer)
    if (cudaEventRecord(ws.last_done, st) != cudaSuccess ||
        cudaStreamWaitEvent(cs, ws.last_done, 0) != cudaSuccess)
        return kErrCuda;
    int rc = kOk;
    for (int t = 0; t < n_tiles && rc == kOk; t += sample.period)
        rc = copy_tiles(t, std::min(n_tiles, t + sample.run));
    if (rc != kOk) return rc;
    if (cudaEventRecord(ws.copied[0], cs) != cudaSuccess) return kErrCuda;
    int bound[kStreamChunks + 1], wsum = 0;
    for (int c = 0; c < kStreamChunks; ++c) wsum += kStreamWeights[c];
    bound[0] = 0;
    for (int c = 0, acc = 0; c < kStreamChunks; ++c) {
        acc += kStreamWeights[c];
        bound[c + 1] = (int)((long long)n_tiles * acc / wsum);
    }

    TcProblem t;
    t.ref = p.ref;
    t.N = p.N;
    t.ldr = p.ldr;
    t.qry = p.qry;
    t.Q = p.Q;
    t.ldq = p.ldq;
    t.d = p.d;
    t.k = p.k;
    t.out_dist = p.out_dist;
    t.out_idx = p.out_idx;
    t.ld_out = p.ld_out;
    t.scratch = p.scratch;
    t.scratch_bytes = p.scratch_bytes;
    t.status = p.status;
    t.num_sms = p.num_sms;
    t.timer = nullptr;
    t.host_tmp = ws.tc_stats + 2;
    t.adaptive = false;   // pass 2 starts before the whole set has arrived
    // the translation comes from every fourth sample tile; the query prep
    // (in tc_run_begin) needs it
    if (cudaStreamWaitEvent(st, ws.copied[0], 0) != cudaSuccess ||
        cudaMemsetAsync(rv.rmax_bits, 0, 3 * 256, st) != cudaSuccess)
        return kErrCuda;
    if ((rc = tc_center_from_tiles(rv, p.ref, p.N, p.ldr, p.d, sample, 4, st)) != kOk) return rc;
    TcRun run;
    if ((rc = tc_run_begin(t, rv, st, run)) != kOk ||
        (rc = tc_prepare_ref_tiles(rv, p.ref, p.N, p.ldr, p.d, 0, sample, st)) != kOk ||
        (rc = tc_run_pass1(run, st)) != kOk)
        return rc;
    auto prep_tiles = [&](int t0, int t1) {
        return tc_prepare_ref_tiles(rv, p.ref, p.N, p.ldr, p.d, t0, contiguous_tiles(t1 - t0), st);
    };
    // each chunk's copy, then its prep, scan and re-rank (queued behind the
    // copy's event), so the work of chunk c is on the device while the host
    // gathers chunk c + 1 (pageable input)
    for (int c = 0; c < kStreamChunks; ++c) {
        if ((rc = for_each_gap(sample, bound[c], bound[c + 1], copy_tiles)) != kOk) return rc;
        if (cudaEventRecord(ws.copied[1 + c], cs) != cudaSuccess ||
            cudaStreamWaitEvent(st, ws.copied[1 + c], 0) != cudaSuccess)
            return kErrCuda;
        if (bound[c] >= bound[c + 1]) continue;
        if ((rc = for_each_gap(sample, bound[c], bound[c + 1], prep_tiles)) != kOk ||
            (rc = tc_run_pass2(run, bound[c], bound[c + 1], st)) != kOk ||
            (rc = tc_run_rerank_piece(run, st)) != kOk)
            return rc;
    }
    return tc_run_finish(run, st, ws.tc_stats);
}

// Page-locked (or registered) host memory: only then do the copies run
// asynchronously and overlap the scans.
bool host_pinned(const void *ptr) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

int current_workspace(Workspace *&ws) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return kErrNoDevice;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= kMaxDevices) return kErrCuda;
    ws = &g_ws[dev];
    return kOk;
}

const char *method_name(int method) {
    switch (method) {
        case KNNB200_METHOD_GLOBAL: return "knn_cuda_global";
        case KNNB200_METHOD_TEXTURE: return "knn_cuda_texture";
        default: return "knn_cublas";
    }
}

// Query chunking by free memory (the legacy code's split of the query set
// by cuMemGetInfo, legacy/KNN.CUDA.with.indexes/knn_cuda_with_indexes.cu:
// 348-349, :406-444).  The memory a call may use is the device's free memory
// plus what this workspace already holds (its buffers are reallocated as
// needed), less a margin, and at most g_mem_cap when that is set (a host-side
// cap for tests).  Buffer::ensure over-allocates by 1/8, which the
// estimate includes.
size_t g_mem_cap = 0;
int g_last_chunks = 0;   // query chunks of the last host / device call
constexpr size_t kMemMargin = 64u << 20;

size_t grown(size_t b) { return b ? b + b / 8 + 256 : 0; }

size_t usable_memory(const Workspace &ws) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = 0;
    }
    const size_t held = ws.ref.bytes + ws.qry.bytes + ws.dist.bytes + ws.idx.bytes +
                        ws.scratch.bytes + ws.tcref.bytes;
    size_t avail = free_b + held;
    avail = avail > kMemMargin ? avail - kMemMargin : 0;
    return g_mem_cap ? std::min(avail, g_mem_cap) : avail;
}

// Largest query chunk (all of Q when it fits, else a multiple of 256) whose
// memory, per_chunk(qc) on top of `fixed`, fits the usable memory; 0 when
// not even one query fits.  When the whole call fits in what the workspace
// already holds (repeated calls of one shape) and no cap is set, the device
// is not asked for its free memory: cudaMemGetInfo costs a driver round
// trip on every call otherwise.
template <class F>
int plan_query_chunk(const Workspace &ws, int Q, size_t fixed, F per_chunk) {
    const size_t held = ws.ref.bytes + ws.qry.bytes + ws.dist.bytes + ws.idx.bytes +
                        ws.scratch.bytes + ws.tcref.bytes;
    if (!g_mem_cap && fixed + per_chunk(Q) <= held) return Q;
    const size_t avail = usable_memory(ws);
    auto fits = [&](int qc) { return fixed + per_chunk(qc) <= avail; };
    if (fits(Q)) return Q;
    int lo = 0, hi = Q;   // fits(lo) (or lo == 0), !fits(hi)
    while (hi - lo > 1) {
        const int mid = lo + (hi - lo) / 2;
        if (fits(mid)) lo = mid;
        else hi = mid;
    }
    if (lo >= 256) lo = lo / 256 * 256;
    return lo;
}

// Device bytes of one query chunk of the host entry: query copy, outputs,
// scratch.
size_t host_chunk_bytes(int method, int N, int qc, int d, int k, int num_sms) {
    return grown((size_t)d * round_up(qc, 64) * sizeof(float)) +
           2 * grown((size_t)k * qc * sizeof(float)) +
           grown(scratch_for(method, N, qc, d, k, num_sms));
}

// The body shared by the three host entry points.
bool host_entry(int method, const float *ref, int ref_nb, const float *query, int query_nb,
                int dim, int k, float *knn_dist, int *knn_index) {
    if (!ref || !query || !knn_dist || !knn_index) {
        std::printf("ERROR: %s: null pointer argument\n", method_name(method));
        return false;
    }
    if (!valid_sizes(ref_nb, query_nb, dim, k)) {
        std::printf("ERROR: %s: invalid sizes (ref_nb=%d query_nb=%d dim=%d k=%d; "
                    "need >= 1 and k <= ref_nb)\n",
                    method_name(method), ref_nb, query_nb, dim, k);
        return false;
    }
    Workspace *ws = nullptr;
    int rc = current_workspace(ws);
    if (rc == kErrNoDevice) {
        std::printf("ERROR: No CUDA device found\n");
        return false;
    }
    if (rc != kOk) {
        std::printf("ERROR: Cannot query the current CUDA device\n");
        return false;
    }
    std::lock_guard<std::mutex> lock(ws->mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (!ws->setup(dev)) {
        std::printf("ERROR: Cannot initialise the CUDA device\n");
        cudaGetLastError();
        return false;
    }
    const long long ldr = round_up(ref_nb, 64);
    const bool tc = use_tc(method, ref_nb, query_nb, dim, k);
    const size_t fixed = grown((size_t)dim * ldr * sizeof(float)) +
                         (tc ? grown(tc_ref_bytes(ref_nb, dim)) : 0);
    const int qc = plan_query_chunk(*ws, query_nb, fixed, [&](int c) {
        return host_chunk_bytes(method, ref_nb, c, dim, k, ws->num_sms);
    });
    if (qc < 1) {
        std::printf("ERROR: Memory allocation error\n");
        return false;
    }
    g_last_chunks = (query_nb + qc - 1) / qc;
    const long long ldq = round_up(qc, 64);
    const size_t out_elems = (size_t)k * qc;
    const size_t scratch = scratch_for(method, ref_nb, qc, dim, k, ws->num_sms);
    if (!ws->ref.ensure((size_t)dim * ldr * sizeof(float)) ||
        !ws->qry.ensure((size_t)dim * ldq * sizeof(float)) ||
        !ws->dist.ensure(out_elems * sizeof(float)) ||
        !ws->idx.ensure(out_elems * sizeof(int)) || !ws->scratch.ensure(scratch)) {
        std::printf("ERROR: Memory allocation error\n");
        return false;
    }
    cudaStream_t st = ws->stream;
    float *ref_d = static_cast<float *>(ws->ref.ptr);
    float *qry_d = static_cast<float *>(ws->qry.ptr);
    // the streamed reference copy serves a call that runs as one chunk;
    // page-locked input is copied directly, pageable input through the
    // pinned staging buffers
    const bool streamed = tc && qc == query_nb && ref_nb >= kStreamMinPoints;
    const bool pinned = streamed && host_pinned(ref);
    cudaError_t e0 = streamed ? cudaSuccess
                              : cudaMemcpy2DAsync(ref_d, ldr * sizeof(float), ref,
                                                  ref_nb * sizeof(float), ref_nb * sizeof(float),
                                                  dim, cudaMemcpyHostToDevice, st);
    cudaError_t e2 = cudaMemsetAsync(ws->status.ptr, 0, sizeof(int), st);
    if (e0 != cudaSuccess || e2 != cudaSuccess) {
        std::printf("ERROR: Unable to copy data from host to device\n");
        cudaGetLastError();
        return false;
    }
    long long stats[3] = {0, 0, 0};   // second scan, exact, candidates over the chunks
    for (int q0 = 0; q0 < query_nb; q0 += qc) {
        const int n = std::min(qc, query_nb - q0);
        if (cudaMemcpy2DAsync(qry_d, ldq * sizeof(float), query + q0, query_nb * sizeof(float),
                              n * sizeof(float), dim, cudaMemcpyHostToDevice,
                              st) != cudaSuccess) {
            std::printf("ERROR: Unable to copy data from host to device\n");
            cudaGetLastError();
            return false;
        }
        ExactProblem p;
        p.ref = ref_d;
        p.N = ref_nb;
        p.ldr = ldr;
        p.qry = qry_d;
        p.Q = n;
        p.ldq = ldq;
        p.d = dim;
        p.k = k;
        p.out_dist = static_cast<float *>(ws->dist.ptr);
        p.out_idx = static_cast<int *>(ws->idx.ptr);
        p.ld_out = n;
        p.scratch = ws->scratch.ptr;
        p.scratch_bytes = ws->scratch.bytes;
        p.status = static_cast<int *>(ws->status.ptr);
        p.num_sms = ws->num_sms;
        p.force_splits = 0;
        rc = streamed ? enqueue_tc_streamed(*ws, p, ref, pinned, st)
                      : enqueue(*ws, p, method, st, /*ref_prepared=*/q0 > 0);
        if (rc != kOk) {
            std::printf("ERROR: Unable to execute kernel (%s)\n", knnb200_status_string(rc));
            cudaGetLastError();
            return false;
        }
        stats[0] += ws->tc_stats[0];
        stats[1] += ws->tc_stats[1];
        stats[2] += *reinterpret_cast<const long long *>(ws->tc_stats + 4);
        e0 = cudaMemcpy2DAsync(knn_dist + q0, query_nb * sizeof(float), p.out_dist,
                               n * sizeof(float), n * sizeof(float), k, cudaMemcpyDeviceToHost,
                               st);
        cudaError_t e1 = cudaMemcpy2DAsync(knn_index + q0, query_nb * sizeof(int), p.out_idx,
                                           n * sizeof(int), n * sizeof(int), k,
                                           cudaMemcpyDeviceToHost, st);
        if (e0 != cudaSuccess || e1 != cudaSuccess) {
            std::printf("ERROR: Unable to copy data from device to host (%s)\n",
                        cudaGetErrorString(cudaGetLastError()));
            return false;
        }
    }
    ws->tc_stats[0] = (int)stats[0];
    ws->tc_stats[1] = (int)stats[1];
    *reinterpret_cast<long long *>(ws->tc_stats + 4) = stats[2];
    e2 = cudaMemcpyAsync(ws->status_host, ws->status.ptr, sizeof(int), cudaMemcpyDeviceToHost,
                         st);
    cudaError_t e3 = cudaStreamSynchronize(st);
    if (e2 != cudaSuccess || e3 != cudaSuccess) {
        std::printf("ERROR: Unable to copy data from device to host (%s)\n",
                    cudaGetErrorString(e3 != cudaSuccess ? e3 : cudaGetLastError()));
        cudaGetLastError();
        return false;
    }
    if (*ws->status_host != 0) {
        std::printf("ERROR: kernel wait timed out (device status %d)\n", *ws->status_host);
        return false;
    }
    return true;
}

}  // namespace
}  // namespace knnb200

using namespace knnb200;

// ---------------------------------------------------------------------------
// Drop-in entry points (C++ linkage, reference signatures).
// ---------------------------------------------------------------------------
bool knn_cuda_global(const float *ref, int ref_nb, const float *query, int query_nb, int dim,
                     int k, float *knn_dist, int *knn_index) {
    return host_entry(KNNB200_METHOD_GLOBAL, ref, ref_nb, query, query_nb, dim, k, knn_dist,
                      knn_index);
}

bool knn_cuda_texture(const float *ref, int ref_nb, const float *query, int query_nb, int dim,
                      int k, float *knn_dist, int *knn_index) {
    return host_entry(KNNB200_METHOD_TEXTURE, ref, ref_nb, query, query_nb, dim, k, knn_dist,
                      knn_index);
}

bool knn_cublas(const float *ref, int ref_nb, const float *query, int query_nb, int dim, int k,
                float *knn_dist, int *knn_index) {
    return host_entry(KNNB200_METHOD_CUBLAS, ref, ref_nb, query, query_nb, dim, k, knn_dist,
                      knn_index);
}

// ---------------------------------------------------------------------------
// C ABI.
// ---------------------------------------------------------------------------
extern "C" {

int knnb200_cuda_global(const float *ref, int ref_nb, const float *query, int query_nb,
                        int dim, int k, float *knn_dist, int *knn_index) {
    return knn_cuda_global(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index) ? 1 : 0;
}

int knnb200_cuda_texture(const float *ref, int ref_nb, const float *query, int query_nb,
                         int dim, int k, float *knn_dist, int *knn_index) {
    return knn_cuda_texture(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index) ? 1 : 0;
}

int knnb200_cublas(const float *ref, int ref_nb, const float *query, int query_nb, int dim,
                   int k, float *knn_dist, int *knn_index) {
    return knn_cublas(ref, ref_nb, query, query_nb, dim, k, knn_dist, knn_index) ? 1 : 0;
}

int knnb200_knn_device(const float *ref, int ref_nb, long long ref_ld, const float *query,
                       int query_nb, long long query_ld, int dim, int k, int method,
                       float *knn_dist, int *knn_index, long long out_ld, void *stream) {
    if (!ref || !query || !knn_dist || !knn_index) return KNNB200_EINVAL;
    if (!valid_sizes(ref_nb, query_nb, dim, k)) return KNNB200_EINVAL;
    if (method < KNNB200_METHOD_GLOBAL || method > KNNB200_METHOD_FP8) return KNNB200_EINVAL;
    if (ref_ld < ref_nb || query_ld < query_nb || out_ld < query_nb) return KNNB200_EINVAL;
    if (ref_ld % 4 || query_ld % 4) return KNNB200_EINVAL;
    if ((reinterpret_cast<uintptr_t>(ref) | reinterpret_cast<uintptr_t>(query)) & 15)
        return KNNB200_EINVAL;
    if (!exact_supported_k(k)) return KNNB200_EUNSUPPORTED;
    Workspace *ws = nullptr;
    int rc = current_workspace(ws);
    if (rc != kOk) return rc;
    std::lock_guard<std::mutex> lock(ws->mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (!ws->setup(dev)) return KNNB200_ECUDA;
    // inputs and outputs are the caller's: only the scratch (and the tensor
    // path's prepared reference set) grow with the call; queries that do not
    // fit in one go run in chunks (column offsets into the caller's arrays)
    const bool tc = use_tc(method, ref_nb, query_nb, dim, k);
    const int qc = plan_query_chunk(*ws, query_nb, tc ? grown(tc_ref_bytes(ref_nb, dim)) : 0,
                                    [&](int c) {
                                        return grown(scratch_for(method, ref_nb, c, dim, k,
                                                                 ws->num_sms));
                                    });
    if (qc < 1) return KNNB200_ENOMEM;
    g_last_chunks = (query_nb + qc - 1) / qc;
    if (!ws->scratch.ensure(scratch_for(method, ref_nb, qc, dim, k, ws->num_sms)))
        return KNNB200_ENOMEM;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Calls on one device share the workspace scratch: order them.
    if (cudaStreamWaitEvent(st, ws->last_done, 0) != cudaSuccess) return KNNB200_ECUDA;
    if (cudaMemsetAsync(ws->status.ptr, 0, sizeof(int), st) != cudaSuccess) return KNNB200_ECUDA;
    long long stats[3] = {0, 0, 0};
    for (int q0 = 0; q0 < query_nb && rc == kOk; q0 += qc) {
        ExactProblem p;
        p.ref = ref;
        p.N = ref_nb;
        p.ldr = ref_ld;
        p.qry = query + q0;
        p.Q = std::min(qc, query_nb - q0);
        p.ldq = query_ld;
        p.d = dim;
        p.k = k;
        p.out_dist = knn_dist + q0;
        p.out_idx = knn_index + q0;
        p.ld_out = out_ld;
        p.scratch = ws->scratch.ptr;
        p.scratch_bytes = ws->scratch.bytes;
        p.status = static_cast<int *>(ws->status.ptr);
        p.num_sms = ws->num_sms;
        p.force_splits = 0;
        rc = enqueue(*ws, p, method, st, /*ref_prepared=*/q0 > 0);
        stats[0] += ws->tc_stats[0];
        stats[1] += ws->tc_stats[1];
        stats[2] += *reinterpret_cast<const long long *>(ws->tc_stats + 4);
    }
    ws->tc_stats[0] = (int)stats[0];
    ws->tc_stats[1] = (int)stats[1];
    *reinterpret_cast<long long *>(ws->tc_stats + 4) = stats[2];
    if (cudaEventRecord(ws->last_done, st) != cudaSuccess && rc == kOk) rc = kErrCuda;
    return rc;
}

void knnb200_set_memory_cap(size_t bytes) {
    Workspace *ws = nullptr;
    if (current_workspace(ws) != kOk) return;
    std::lock_guard<std::mutex> lock(ws->mu);
    g_mem_cap = bytes;
}

int knnb200_last_query_chunks(void) { return g_last_chunks; }

size_t knnb200_call_bytes(int ref_nb, int query_nb, int dim, int k, int method, int host) {
    if (!valid_sizes(ref_nb, query_nb, dim, k)) return 0;
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    const bool tc = use_tc(method, ref_nb, query_nb, dim, k);
    const size_t tcb = tc ? grown(tc_ref_bytes(ref_nb, dim)) : 0;
    if (!host) return tcb + grown(scratch_for(method, ref_nb, query_nb, dim, k, sms));
    return grown((size_t)dim * round_up(ref_nb, 64) * sizeof(float)) + tcb +
           host_chunk_bytes(method, ref_nb, query_nb, dim, k, sms);
}

int knnb200_sync_status(void *stream) {
    Workspace *ws = nullptr;
    int rc = current_workspace(ws);
    if (rc != kOk) return rc;
    std::lock_guard<std::mutex> lock(ws->mu);
    if (!ws->init) return KNNB200_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(ws->status_host, ws->status.ptr, sizeof(int), cudaMemcpyDeviceToHost,
                        st) != cudaSuccess)
        return KNNB200_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return KNNB200_ECUDA;
    return *ws->status_host ? KNNB200_ETIMEOUT : KNNB200_OK;
}

size_t knnb200_scratch_bytes(int ref_nb, int query_nb, int dim, int k, int method) {
    if (!valid_sizes(ref_nb, query_nb, dim, k)) return 0;
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    return scratch_for(method, ref_nb, query_nb, dim, k, sms);
}

int knnb200_plan_splits(int ref_nb, int query_nb, int dim, int k) {
    if (!valid_sizes(ref_nb, query_nb, dim, k)) return 0;
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    return exact_plan_splits(ref_nb, query_nb, dim, k, sms);
}

void knnb200_release_workspace(void) {
    Workspace *ws = nullptr;
    if (current_workspace(ws) != kOk) return;
    std::lock_guard<std::mutex> lock(ws->mu);
    if (!ws->init) return;
    cudaStreamSynchronize(ws->stream);
    ws->ref.release();
    ws->qry.release();
    ws->dist.release();
    ws->idx.release();
    ws->scratch.release();
    ws->tcref.release();
}

const char *knnb200_status_string(int code) {
    switch (code) {
        case KNNB200_OK: return "ok";
        case KNNB200_EINVAL: return "invalid argument";
        case KNNB200_ENODEV: return "no CUDA device";
        case KNNB200_ENOMEM: return "device allocation failed";
        case KNNB200_ELAUNCH: return "kernel launch failed";
        case KNNB200_ETIMEOUT: return "device wait timed out";
        case KNNB200_ECUDA: return "CUDA runtime error";
        case KNNB200_EUNSUPPORTED: return "unsupported shape for this method";
        case KNNB200_ESCRATCH: return "scratch too small";
        case KNNB200_ETENSORMAP: return "TMA descriptor encoding failed";
        default: return "unknown";
    }
}

void knnb200_set_phase_timing(int enable) {
    Workspace *ws = nullptr;
    if (current_workspace(ws) != kOk) return;
    std::lock_guard<std::mutex> lock(ws->mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (!ws->setup(dev)) return;
    ws->timer.on = enable != 0;
    ws->timer.marks = 0;
}

int knnb200_last_phase_times(float *ms, int n) {
    if (!ms || n <= 0) return 0;
    for (int i = 0; i < n; ++i) ms[i] = -1.f;
    Workspace *ws = nullptr;
    if (current_workspace(ws) != kOk || !ws->init) return 0;
    std::lock_guard<std::mutex> lock(ws->mu);
    const PhaseTimer &t = ws->timer;
    if (t.marks < 2 || cudaEventSynchronize(t.ev[t.marks - 1]) != cudaSuccess) return 0;
    for (int i = 1; i < t.marks; ++i) {
        float x = 0.f;
        if (t.phase[i] < n && cudaEventElapsedTime(&x, t.ev[i - 1], t.ev[i]) == cudaSuccess)
            ms[t.phase[i]] = (ms[t.phase[i]] < 0.f ? 0.f : ms[t.phase[i]]) + x;
    }
    return kNumPhases;
}

void knnb200_last_tc_stats(long long *candidates, int *second_scan, int *exact) {
    if (candidates) *candidates = 0;
    if (second_scan) *second_scan = 0;
    if (exact) *exact = 0;
    Workspace *ws = nullptr;
    if (current_workspace(ws) != kOk || !ws->init) return;
    std::lock_guard<std::mutex> lock(ws->mu);
    if (candidates) *candidates = *reinterpret_cast<const long long *>(ws->tc_stats + 4);
    if (second_scan) *second_scan = ws->tc_stats[0];
    if (exact) *exact = ws->tc_stats[1];
}

int knnb200_set_bound_check(int enable) {
    Workspace *ws = nullptr;
    int rc = current_workspace(ws);
    if (rc != kOk) return rc;
    std::lock_guard<std::mutex> lock(ws->mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (!ws->setup(dev)) return KNNB200_ECUDA;
    if (enable) {
        if (!ws->bound.ensure(16)) return KNNB200_ENOMEM;
        if (cudaMemset(ws->bound.ptr, 0, 16) != cudaSuccess) return KNNB200_ECUDA;
    }
    ws->bound_check = enable != 0;
    return KNNB200_OK;
}

int knnb200_last_bound_check(double *max_ratio, long long *checked) {
    if (max_ratio) *max_ratio = 0.0;
    if (checked) *checked = 0;
    Workspace *ws = nullptr;
    int rc = current_workspace(ws);
    if (rc != kOk) return rc;
    std::lock_guard<std::mutex> lock(ws->mu);
    if (!ws->init || !ws->bound.ptr) return KNNB200_EINVAL;
    unsigned v[4] = {0, 0, 0, 0};
    // the call may have run on any stream (device entry): wait for all
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(v, ws->bound.ptr, 16, cudaMemcpyDeviceToHost) != cudaSuccess)
        return KNNB200_ECUDA;
    float r;
    std::memcpy(&r, &v[0], 4);
    if (max_ratio) *max_ratio = r;
    if (checked) *checked = (long long)v[2] | ((long long)v[3] << 32);
    return KNNB200_OK;
}

void knnb200_set_tc_kind_override(int kind) {
    g_force_kind = (kind >= 0 && kind <= 2) ? kind : -1;
}

void knnb200_last_tc_kinds(int *first, int *second) {
    if (first) *first = -1;
    if (second) *second = -1;
    Workspace *ws = nullptr;
    if (current_workspace(ws) != kOk || !ws->init) return;
    std::lock_guard<std::mutex> lock(ws->mu);
    if (first) *first = ws->tc_stats[6];
    if (second) *second = ws->tc_stats[7];
}

const char *knnb200_version(void) { return "knnb200 0.1.0 (sm_100a)"; }

}  // extern "C"
