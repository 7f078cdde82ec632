// knn_probe.cu -- FP32 CUDA-core throughput calibration, and a self-test of
// the bounded waits every pipelined kernel relies on.
//
// The exact direct-form path is bound by FP32 CUDA-core issue, a peak that
// the measured copy-bandwidth / bf16-GEMM peaks do not cover, so the bench
// measures it on the same GPU and clocks: every thread runs 16 independent
// chains of packed FP32 fused multiply-adds (fma.rn.f32x2) and the kernel
// reports FLOP/s with 2 flops per multiply-add.
#include <cstdint>

#include "../../include/knn_b200.h"
#include "knn_common.cuh"

namespace knnb200 {

__global__ void __launch_bounds__(256) ffma_peak_kernel(float *out, int iters, float seed) {
    f32x2_t acc[16];
    const f32x2_t m = f2_pack(0.999999f, 0.999998f);
    const f32x2_t c = f2_pack(1e-7f, 2e-7f);
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = f2_pack(seed + i, seed - i);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] = f2_fma(acc[i], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 16; ++i) s += f2_lo(acc[i]) + f2_hi(acc[i]);
    if (s == 12345.678f) out[0] = s;   // keeps the chains live
}

// One warp waits on an mbarrier that nothing arrives on, through the same
// bounded wait as the pipelined kernels, with a short limit; on giving up it
// records the timeout in *status and returns normally.
__global__ void wait_timeout_selftest_kernel(int *status, unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncwarp();
    const bool got = mbar_wait(&bar, 0, limit_ns);
    if (threadIdx.x == 0) *status = got ? (int)kDevOk : (int)kDevTimeoutFull;
}

}  // namespace knnb200

extern "C" KNNB200_API int knnb200_selftest_wait_timeout(long long limit_ns, void *stream) {
    using namespace knnb200;
    if (limit_ns <= 0 || limit_ns > 1000000000ll) return KNNB200_EINVAL;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return KNNB200_ENODEV;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int *status = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void **>(&status), sizeof(int), st) != cudaSuccess)
        return KNNB200_ENOMEM;
    int h = -1;
    wait_timeout_selftest_kernel<<<1, 32, 0, st>>>(status, (unsigned long long)limit_ns);
    const bool ok = cudaGetLastError() == cudaSuccess &&
                    cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st) ==
                        cudaSuccess &&
                    cudaStreamSynchronize(st) == cudaSuccess;
    cudaFreeAsync(status, st);
    cudaStreamSynchronize(st);
    if (!ok) return KNNB200_ECUDA;
    return h == kDevOk ? KNNB200_OK : KNNB200_ETIMEOUT;
}

extern "C" KNNB200_API double knnb200_measure_fp32_peak(int iters, void *stream) {
    using namespace knnb200;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1.0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -1.0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float *out = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void **>(&out), sizeof(float), st) != cudaSuccess)
        return -1.0;
    const int blocks = sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    ffma_peak_kernel<<<blocks, threads, 0, st>>>(out, iters / 8 + 1, 1.0f);   // warm-up
    cudaEventRecord(e0, st);
    ffma_peak_kernel<<<blocks, threads, 0, st>>>(out, iters, 1.0f);
    cudaEventRecord(e1, st);
    float ms = 0.f;
    bool ok = cudaEventSynchronize(e1) == cudaSuccess &&
              cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms > 0.f;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(out, st);
    cudaStreamSynchronize(st);
    if (!ok) return -1.0;
    // 16 chains x 8 repeats x 2 lanes x 2 flops per iteration per thread
    const double flops = (double)blocks * threads * iters * 16.0 * 8.0 * 2.0 * 2.0;
    return flops / (ms * 1e-3);
}
