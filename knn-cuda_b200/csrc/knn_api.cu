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
#include <cstdio>
#include <cstring>
#include <mutex>

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
    PhaseTimer timer;                  // optional per-phase device timing
    int *status_host = nullptr;        // pinned status word for the host path
    int *tc_stats = nullptr;           // pinned: [0] second-scan queries, [1] exact fallbacks
    cudaStream_t copy_stream = nullptr;          // host entry: reference copies
    cudaEvent_t copied[1 + kStreamChunks] = {};  // sample, then each chunk

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

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

bool valid_sizes(int ref_nb, int query_nb, int dim, int k) {
    return ref_nb >= 1 && query_nb >= 1 && dim >= 1 && k >= 1 && k <= ref_nb;
}

bool use_tc(int method, int N, int Q, int d, int k) {
    return method == KNNB200_METHOD_CUBLAS && tc_supported(N, Q, d, k);
}

size_t scratch_for(int method, int N, int Q, int d, int k, int num_sms) {
    if (use_tc(method, N, Q, d, k)) return tc_scratch_bytes(N, Q, d, k, num_sms);
    return exact_scratch_bytes(N, Q, d, k, num_sms);
}

// Queue the computation for one problem whose inputs are on the device.
// knn_cublas runs the tensor-core expansion path when the shape qualifies
// (it synchronises the stream once, to recompute uncertified queries);
// everything else runs the fused exact kernel.
int enqueue(Workspace &ws, const ExactProblem &p0, int method, cudaStream_t st) {
    for (int i = 0; i < 8; ++i) ws.tc_stats[i] = 0;
    if (!exact_supported_k(p0.k)) return kErrUnsupported;
    ExactProblem p = p0;
    p.timer = &ws.timer;
    ws.timer.begin(st);
    if (!use_tc(method, p.N, p.Q, p.d, p.k)) return launch_exact(p, st);
    if (!ws.tcref.ensure(tc_ref_bytes(p.N, p.d))) return kErrNoMemory;
    const TcRefView rv = tc_carve_ref(ws.tcref.ptr, p.N, p.d);
    int rc = tc_prepare_ref(rv, p.ref, p.N, p.ldr, p.d, st);
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
    return launch_tc(t, rv, st, ws.tc_stats);
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
                        cudaStream_t st) {
    for (int i = 0; i < 8; ++i) ws.tc_stats[i] = 0;
    ws.timer.begin(st);
    if (!ws.tcref.ensure(tc_ref_bytes(p.N, p.d))) return kErrNoMemory;
    const TcRefView rv = tc_carve_ref(ws.tcref.ptr, p.N, p.d);
    float *ref_d = const_cast<float *>(p.ref);
    const int T = tc_tile_points();
    const int n_tiles = (p.N + T - 1) / T;
    const TileRuns sample = tc_sample_runs(p.N, p.Q, p.d, p.k, p.num_sms);
    const size_t fb = sizeof(float);
    cudaStream_t cs = ws.copy_stream;
    // points [t0 T, t1 T) of every dimension, one 2-D copy
    auto copy_tiles = [&](int t0, int t1) -> int {
        const size_t p0 = (size_t)t0 * T, p1 = std::min<size_t>(p.N, (size_t)t1 * T);
        if (p0 >= p1) return kOk;
        return cudaMemcpy2DAsync(ref_d + p0, (size_t)p.ldr * fb, ref_host + p0, (size_t)p.N * fb,
                                 (p1 - p0) * fb, p.d, cudaMemcpyHostToDevice,
                                 cs) == cudaSuccess
                   ? kOk
                   : kErrCuda;
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
    for (int c = 0; c < kStreamChunks; ++c) {
        if ((rc = for_each_gap(sample, bound[c], bound[c + 1], copy_tiles)) != kOk) return rc;
        if (cudaEventRecord(ws.copied[1 + c], cs) != cudaSuccess) return kErrCuda;
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
    // the translation comes from every fourth sample tile; the query prep
    // (in tc_run_begin) needs it
    if (cudaStreamWaitEvent(st, ws.copied[0], 0) != cudaSuccess ||
        cudaMemsetAsync(rv.rmax_bits, 0, sizeof(unsigned), st) != cudaSuccess)
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
    for (int c = 0; c < kStreamChunks; ++c) {
        if (cudaStreamWaitEvent(st, ws.copied[1 + c], 0) != cudaSuccess) return kErrCuda;
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
    if (!exact_supported_k(k)) {
        std::printf("ERROR: %s: k=%d exceeds the supported maximum of 256\n",
                    method_name(method), k);
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
    const long long ldr = round_up(ref_nb, 64), ldq = round_up(query_nb, 64);
    const size_t out_elems = (size_t)k * query_nb;
    const size_t scratch = scratch_for(method, ref_nb, query_nb, dim, k, ws->num_sms);
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
    const bool streamed = use_tc(method, ref_nb, query_nb, dim, k) &&
                          ref_nb >= kStreamMinPoints && host_pinned(ref);
    cudaError_t e0 = streamed ? cudaSuccess
                              : cudaMemcpy2DAsync(ref_d, ldr * sizeof(float), ref,
                                                  ref_nb * sizeof(float), ref_nb * sizeof(float),
                                                  dim, cudaMemcpyHostToDevice, st);
    cudaError_t e1 = cudaMemcpy2DAsync(qry_d, ldq * sizeof(float), query,
                                       query_nb * sizeof(float), query_nb * sizeof(float), dim,
                                       cudaMemcpyHostToDevice, st);
    cudaError_t e2 = cudaMemsetAsync(ws->status.ptr, 0, sizeof(int), st);
    if (e0 != cudaSuccess || e1 != cudaSuccess || e2 != cudaSuccess) {
        std::printf("ERROR: Unable to copy data from host to device\n");
        cudaGetLastError();
        return false;
    }
    ExactProblem p;
    p.ref = ref_d;
    p.N = ref_nb;
    p.ldr = ldr;
    p.qry = qry_d;
    p.Q = query_nb;
    p.ldq = ldq;
    p.d = dim;
    p.k = k;
    p.out_dist = static_cast<float *>(ws->dist.ptr);
    p.out_idx = static_cast<int *>(ws->idx.ptr);
    p.ld_out = query_nb;
    p.scratch = ws->scratch.ptr;
    p.scratch_bytes = ws->scratch.bytes;
    p.status = static_cast<int *>(ws->status.ptr);
    p.num_sms = ws->num_sms;
    p.force_splits = 0;
    rc = streamed ? enqueue_tc_streamed(*ws, p, ref, st) : enqueue(*ws, p, method, st);
    if (rc != kOk) {
        std::printf("ERROR: Unable to execute kernel (%s)\n", knnb200_status_string(rc));
        cudaGetLastError();
        return false;
    }
    e0 = cudaMemcpyAsync(knn_dist, p.out_dist, out_elems * sizeof(float), cudaMemcpyDeviceToHost,
                         st);
    e1 = cudaMemcpyAsync(knn_index, p.out_idx, out_elems * sizeof(int), cudaMemcpyDeviceToHost,
                         st);
    e2 = cudaMemcpyAsync(ws->status_host, ws->status.ptr, sizeof(int), cudaMemcpyDeviceToHost,
                         st);
    cudaError_t e3 = cudaStreamSynchronize(st);
    if (e0 != cudaSuccess || e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
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
    if (method < KNNB200_METHOD_GLOBAL || method > KNNB200_METHOD_CUBLAS) return KNNB200_EINVAL;
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
    if (!ws->scratch.ensure(scratch_for(method, ref_nb, query_nb, dim, k, ws->num_sms)))
        return KNNB200_ENOMEM;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Calls on one device share the workspace scratch: order them.
    if (cudaStreamWaitEvent(st, ws->last_done, 0) != cudaSuccess) return KNNB200_ECUDA;
    if (cudaMemsetAsync(ws->status.ptr, 0, sizeof(int), st) != cudaSuccess) return KNNB200_ECUDA;
    ExactProblem p;
    p.ref = ref;
    p.N = ref_nb;
    p.ldr = ref_ld;
    p.qry = query;
    p.Q = query_nb;
    p.ldq = query_ld;
    p.d = dim;
    p.k = k;
    p.out_dist = knn_dist;
    p.out_idx = knn_index;
    p.ld_out = out_ld;
    p.scratch = ws->scratch.ptr;
    p.scratch_bytes = ws->scratch.bytes;
    p.status = static_cast<int *>(ws->status.ptr);
    p.num_sms = ws->num_sms;
    p.force_splits = 0;
    rc = enqueue(*ws, p, method, st);
    if (cudaEventRecord(ws->last_done, st) != cudaSuccess && rc == kOk) rc = kErrCuda;
    return rc;
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

const char *knnb200_version(void) { return "knnb200 0.1.0 (sm_100a)"; }

}  // extern "C"
