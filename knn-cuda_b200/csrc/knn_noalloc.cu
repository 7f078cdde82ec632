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
//   * a call needs splits * query_nb * k * 8 bytes of it (splits as chosen
//     by the kernel's planner; knnb200_plan_splits reports it), and a call
//     needing more is rejected with KNNB200_ESCRATCH before anything runs;
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
    std::once_flag once;
    cudaError_t err = cudaSuccess;
    void *scratch = nullptr;
    int *status = nullptr;
    int num_sms = 0;
};

NoAllocDevice g_dev[kNoAllocMaxDevices];

// Runs once per device, with that device current.
NoAllocDevice *set_up(int dev) {
    NoAllocDevice *d = &g_dev[dev];
    std::call_once(d->once, [d, dev]() {
        d->err = cudaGetSymbolAddress(&d->scratch, g_noalloc_scratch);
        if (d->err == cudaSuccess)
            d->err = cudaGetSymbolAddress(reinterpret_cast<void **>(&d->status),
                                          g_noalloc_status);
        if (d->err == cudaSuccess)
            d->err = cudaDeviceGetAttribute(&d->num_sms, cudaDevAttrMultiProcessorCount, dev);
    });
    return d;
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
    NoAllocDevice *d = set_up(dev);
    if (d->err != cudaSuccess) {
        std::printf("ERROR: knnb200_knn_device_noalloc: cannot locate the static scratch (%s)\n",
                    cudaGetErrorString(d->err));
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
