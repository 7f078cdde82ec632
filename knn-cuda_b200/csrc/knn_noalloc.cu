// knn_noalloc.cu -- the exact k-NN for callers that cannot allocate.
//
// Some callers may not call cudaMalloc at all: a host application whose
// device memory is handed out by its own pool allocator (so a foreign
// allocation can fail or fragment that pool), or a latency-bound loop where
// cudaMalloc / cudaFree are ruled out because they can stall the whole
// device.  For them this file provides knnb200_knn_device_noalloc: the same
// fused exact kernel and split merge as knnb200_knn_device, but the per-split
// partial result lists live in a statically sized device array owned by this
// library instead of the library's growable workspace, and the call creates
// no stream, event or buffer.
//
// Limits and sharing:
//   * the static area is 64 MiB of device memory, held on every GPU that
//     loads this library until the process exits;
//   * a call needs the exact path's whole scratch in it: the query set
//     duplicated into (q, q) pairs (dim * round_up(query_nb, 32) * 8 bytes),
//     256 bytes of alignment and, when the planner splits the reference set,
//     splits * query_nb * min(k, 256) * 8 bytes of per-split lists (for
//     k > 256 also query_nb * 8 bytes of lower-bound keys).  knnb200_scratch_bytes(...,
//     KNNB200_METHOD_GLOBAL) gives the exact figure; a call needing more
//     than the static area is rejected with KNNB200_ESCRATCH before anything
//     runs;
//   * the first call on a device looks up the area's device address
//     (cudaGetSymbolAddress, with that device current); make that first
//     call before any stream capture.  Every call waits for its own work
//     on `stream` (it reads the kernel's status word back) before it
//     returns;
//   * every call uses the same area and the same status word, and the area
//     keeps whatever the previous call left in it: each call overwrites the
//     lists it reads and clears the status word itself, but two calls whose
//     work overlaps on the GPU (for example on two streams, or from two host
//     threads) race on it and must be serialised by the caller.
#include <cstdio>
#include <mutex>

#include "../../include/knn_b200.h"
#include "knn_kernels.h"

namespace knnb200 {
namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;
constexpr int kNoAllocMaxDevices = 64;

// The static scratch area and status word.  In host code these names are
// only stand-ins for the device objects: the kernels must be given the
// device addresses from cudaGetSymbolAddress, which set_up() looks up once
// per device.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocScratchBytes / 8];
static __device__ int g_noalloc_status;

struct NoAllocDevice {
    std::mutex mu;
    bool ready = false;
    void *scratch = nullptr;
    int *status = nullptr;
    int num_sms = 0;
};

NoAllocDevice g_dev[kNoAllocMaxDevices];

// Looks up the device addresses once per device, with that device current.
// Only a successful lookup is kept: after a failure (reported to the caller)
// the next call on that device tries again.
cudaError_t set_up(int dev, NoAllocDevice *&out) {
    NoAllocDevice *d = &g_dev[dev];
    std::lock_guard<std::mutex> lock(d->mu);
    if (!d->ready) {
        void *scratch = nullptr, *status = nullptr;
        int sms = 0;
        cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&status, g_noalloc_status);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return e;
        }
        d->scratch = scratch;
        d->status = static_cast<int *>(status);
        d->num_sms = sms;
        d->ready = true;
    }
    out = d;
    return cudaSuccess;
}

}  // namespace
}  // namespace knnb200

extern "C" KNNB200_API int knnb200_knn_device_noalloc(const float *ref, int ref_nb,
                                                     long long ref_ld, const float *query,
                                                     int query_nb, long long query_ld, int dim,
                                                     int k, float *knn_dist, int *knn_index,
                                                     long long out_ld, void *stream) {
    using namespace knnb200;
    if (!ref || !query || !knn_dist || !knn_index) return KNNB200_EINVAL;
    if (ref_nb < 1 || query_nb < 1 || dim < 1 || k < 1 || k > ref_nb) return KNNB200_EINVAL;
    if (ref_ld < ref_nb || query_ld < query_nb || out_ld < query_nb) return KNNB200_EINVAL;
    if (ref_ld % 4 || query_ld % 4) return KNNB200_EINVAL;
    if ((reinterpret_cast<uintptr_t>(ref) | reinterpret_cast<uintptr_t>(query)) & 15)
        return KNNB200_EINVAL;
    if (!exact_supported_k(k)) return KNNB200_EUNSUPPORTED;
    int ndev = 0, dev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return KNNB200_ENODEV;
    }
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= kNoAllocMaxDevices) return KNNB200_ECUDA;
    NoAllocDevice *d = nullptr;
    const cudaError_t se = set_up(dev, d);
    if (se != cudaSuccess) {
        std::printf("ERROR: knnb200_knn_device_noalloc: cannot locate the static scratch (%s)\n",
                    cudaGetErrorString(se));
        return KNNB200_ECUDA;
    }
    const size_t need = exact_scratch_bytes(ref_nb, query_nb, dim, k, d->num_sms);
    if (need > kNoAllocScratchBytes) {
        std::printf("ERROR: knnb200_knn_device_noalloc: this shape needs %zu bytes of scratch; "
                    "the static maximum is %zu bytes\n",
                    need, kNoAllocScratchBytes);
        return KNNB200_ESCRATCH;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(d->status, 0, sizeof(int), st) != cudaSuccess) return KNNB200_ECUDA;
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
    p.scratch = d->scratch;
    p.scratch_bytes = kNoAllocScratchBytes;
    p.status = d->status;
    p.num_sms = d->num_sms;
    p.force_splits = 0;
    const int rc = launch_exact(p, st);
    if (rc != kOk) return rc;
    // The call returns once the results are in place, so that a kernel wait
    // that gave up can be reported without any extra allocation.
    int status = 0;
    if (cudaMemcpyAsync(&status, d->status, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return KNNB200_ECUDA;
    return status ? KNNB200_ETIMEOUT : KNNB200_OK;
}
