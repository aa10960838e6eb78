// gqis_probe.cu - CUDA-core FMA throughput probes (FP64 DFMA, FP32 FFMA, packed FP32 FFMA2).
//
// The sweep kernels are bound by the FP32 / FP64 FMA pipes, which have no entry in the
// measured-peaks file of this machine; these probes measure them on the device that runs the
// sweep, so the roofline denominators are measured rather than nominal. Each thread runs
// eight independent FMA chains (enough ILP to hide the pipe latency) for `iters` iterations;
// the grid covers every SM several times over. Flops = 2 per FMA lane.
#include <cuda_runtime.h>
#include <stdint.h>

#include "gqis_b200.h"

namespace {

constexpr int kChains = 8;
constexpr int kBlock = 256;

__global__ void __launch_bounds__(kBlock) fma64_kernel(int iters, double* out) {
    double a[kChains];
    const double b = 0.999999 + 1e-9 * threadIdx.x, c = 1e-7;
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = 1.0 + k * 1e-3 + threadIdx.x * 1e-6;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    if (s == 123.456) out[blockIdx.x] = s;  // keeps the chains alive, never true in practice
}

__global__ void __launch_bounds__(kBlock) fma32_kernel(int iters, float* out) {
    float a[kChains];
    const float b = 0.999999f + 1e-9f * threadIdx.x, c = 1e-7f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = 1.0f + k * 1e-3f + threadIdx.x * 1e-6f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = fmaf(a[k], b, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    if (s == 123.456f) out[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kBlock) fma32x2_kernel(int iters, float* out) {
    float2 a[kChains];
    const float2 b = make_float2(0.999999f + 1e-9f * threadIdx.x, 0.9999995f);
    const float2 c = make_float2(1e-7f, 2e-7f);
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = make_float2(1.0f + k * 1e-3f, 1.5f + threadIdx.x * 1e-6f);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = __ffma2_rn(a[k], b, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k].x + a[k].y;
    if (s == 123.456f) out[blockIdx.x] = s;
}

}  // namespace

extern "C" {

// kind: 0 = FP64 DFMA, 1 = FP32 FFMA, 2 = packed FP32 FFMA2. On success *tflops holds the
// measured rate (best of `repeats` launches) in 1e12 flop/s.
__attribute__((visibility("default"))) int gqis_probe_fma(int kind, int iters, int repeats, double* tflops) {
    if (!tflops || iters < 1 || repeats < 1 || kind < 0 || kind > 2) return GQIS_ERR_INVALID;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GQIS_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return GQIS_ERR_CUDA;
    const int grid = sms * 16;
    void* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * grid) != cudaSuccess) return GQIS_ERR_CUDA;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    int rc = GQIS_OK;
    for (int r = 0; r <= repeats; ++r) {  // first launch is a warm-up
        cudaEventRecord(e0);
        if (kind == 0) fma64_kernel<<<grid, kBlock>>>(iters, (double*)out);
        else if (kind == 1) fma32_kernel<<<grid, kBlock>>>(iters, (float*)out);
        else fma32x2_kernel<<<grid, kBlock>>>(iters, (float*)out);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            rc = GQIS_ERR_CUDA;
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double lanes = (kind == 2) ? 2.0 : 1.0;
        const double flops = 2.0 * lanes * kChains * (double)iters * grid * kBlock;
        if (r > 0 && ms > 0.0f) best = fmax(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops = best;
    return rc;
}

}  // extern "C"
