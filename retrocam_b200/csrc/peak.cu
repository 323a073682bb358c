// peak.cu -- FP32 FMA throughput microbenchmark, the denominator of the
// FP32 roofline fraction of the traversal kernels (their scene data is
// cache-resident, so issue rate rather than HBM bounds them).  Sixteen
// independent FMA chains per thread, every SM filled, timed with CUDA events.
#include <cuda_runtime.h>

#include "retrocam.h"

namespace {

constexpr int kChains = 16;

__global__ void __launch_bounds__(256) fma_kernel(float* out, int iters, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3f + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 12345.678f) out[0] = s;   // keeps the chains live
}

}  // namespace

extern "C" int rc_measure_fp32_peak(int device, double* tflops_out) {
    if (!tflops_out) return RC_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return RC_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float* out = nullptr;
    if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) return RC_ERR_OUT_OF_MEMORY;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    fma_kernel<<<blocks, threads>>>(out, 64, 0.999f, 1e-3f);   // warm-up
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        fma_kernel<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * kChains * (double)iters * blocks * threads;
        if (ms > 0.0f && flops / (ms * 1e9) > best) best = flops / (ms * 1e9);
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return RC_ERR_CUDA;
    *tflops_out = best;
    return RC_OK;
}
