// gqis_probe.cu - throughput probes: CUDA-core FMA (FP64 DFMA, FP32 FFMA, packed FP32 FFMA2) and
// the tcgen05 tensor-core MMA of kind::tf32 (the instruction of the tensor-core density-matrix kernel).
//
// The sweep kernels are bound by the FP32 / FP64 FMA pipes, which have no entry in the
// measured-peaks file of this machine; these probes measure them on the device that runs the
// sweep, so the roofline denominators are measured rather than nominal. Each thread runs
// eight independent FMA chains (enough ILP to hide the pipe latency) for `iters` iterations;
// the grid covers every SM several times over. Flops = 2 per FMA lane.
#include <cuda_runtime.h>
#include <stdint.h>

#include "gqis_b200.h"
#include "gqis_tcgen05.cuh"

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

// ---- tcgen05 kind::tf32 (KIND 0, K = 8) or kind::f16 (KIND 1, K = 16): one CTA per SM issues `iters` x 4
// MMAs of M = 128, N = 256 (A in tensor memory, B in shared memory, as the density-matrix kernel does)
// back to back and waits once. Both kinds read the same bytes per MMA (32 per row of A and of B).
constexpr int kTcN = 256, kTcKSteps = 4;
constexpr size_t kTcSmem = 120 * 1024;  // > half of the SM's shared memory: one CTA per SM

template <int KIND>
__global__ void __launch_bounds__(128, 1) tc_mma_kernel(int iters, float* out, int* status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    float* b = reinterpret_cast<float*>(smem);  // kTcKSteps x 256 rows x 8 TF32, K-major
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kTcKSteps * kTcN * 32);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kTcKSteps * kTcN * 32 + 8);
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int e = tid; e < kTcKSteps * kTcN * 8; e += blockDim.x) b[e] = (float)((e % 7) - 3) * 0.125f;
    gqtc::fence_proxy_async_smem();
    if (tid == 0) gqtc::mbar_init(bar, 1);
    if (warp == 0) {
        gqtc::tmem_alloc(slot, 512);
        gqtc::tmem_relinquish();
    }
    gqtc::fence_before_sync();
    __syncthreads();
    gqtc::fence_after_sync();
    const uint32_t tbase = *slot;
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = (float)((tid + i) % 5) * 0.25f;
#pragma unroll
    for (int kc = 0; kc < kTcKSteps; ++kc) gqtc::tmem_st8(tbase + lane_base + kTcN + 8 * kc, v);
    gqtc::tmem_wait_st();
    gqtc::fence_before_sync();
    __syncthreads();
    bool ok = true;
    if (tid == 0) {
        gqtc::fence_after_sync();
        const uint32_t idesc = KIND == 0 ? gqtc::idesc_tf32_m128(kTcN) : gqtc::idesc_f16_m128(kTcN);
        const uint32_t baddr = gqtc::smem_u32(b);
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int kc = 0; kc < kTcKSteps; ++kc) {
                const uint64_t bd = gqtc::smem_desc_kmajor(baddr + kc * kTcN * 32, 128, 256);
                if constexpr (KIND == 0)
                    gqtc::mma_tf32_ts(tbase, tbase + kTcN + 8 * kc, bd, idesc, (it | kc) ? 1u : 0u);
                else
                    gqtc::mma_f16_ts(tbase, tbase + kTcN + 8 * kc, bd, idesc, (it | kc) ? 1u : 0u);
            }
        }
        gqtc::mma_commit(bar);
        ok = gqtc::mbar_wait_bounded(bar, 0, 1u << 26);
        if (!ok) atomicExch(status, 1);
    }
    __syncthreads();
    gqtc::fence_after_sync();
    float d[8];
    gqtc::tmem_ld8(tbase + lane_base, d);
    gqtc::tmem_wait_ld();
    if (d[0] == 123.456f) out[blockIdx.x] = d[1];  // keeps the result alive, never true in practice
    gqtc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        gqtc::fence_after_sync();
        gqtc::tmem_dealloc(tbase, 512);
    }
}

// Measured dense tensor-core rate of kind KIND (best of `repeats` launches after a warm-up) in 1e12
// flop/s. GQIS_ERR_CUDA if an MMA chain did not signal completion within its bounded wait.
template <int KIND>
int probe_tc(int iters, int repeats, double* tflops) {
    if (!tflops || iters < 1 || repeats < 1) return GQIS_ERR_INVALID;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GQIS_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return GQIS_ERR_CUDA;
    if (cudaFuncSetAttribute(tc_mma_kernel<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem) != cudaSuccess)
        return GQIS_ERR_CUDA;
    void* out = nullptr;
    int* status = nullptr;
    if (cudaMalloc(&out, sizeof(float) * sms) != cudaSuccess) return GQIS_ERR_CUDA;
    if (cudaMalloc(&status, sizeof(int)) != cudaSuccess) {
        cudaFree(out);
        return GQIS_ERR_CUDA;
    }
    cudaMemset(status, 0, sizeof(int));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    int rc = GQIS_OK;
    for (int r = 0; r <= repeats; ++r) {
        cudaEventRecord(e0);
        tc_mma_kernel<KIND><<<sms, 128, kTcSmem>>>(iters, (float*)out, status);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            rc = GQIS_ERR_CUDA;
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 128.0 * kTcN * (KIND == 0 ? 8.0 : 16.0) * kTcKSteps * (double)iters * sms;
        if (r > 0 && ms > 0.0f) best = fmax(best, flops / (ms * 1e-3) / 1e12);
    }
    int host_status = 0;
    if (rc == GQIS_OK && cudaMemcpy(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = GQIS_ERR_CUDA;
    if (rc == GQIS_OK && host_status != 0) rc = GQIS_ERR_CUDA;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    cudaFree(status);
    *tflops = best;
    return rc;
}
}  // namespace

extern "C" {

// Measured dense TF32 (kind::tf32) / FP16 (kind::f16) tensor-core rate in 1e12 flop/s.
__attribute__((visibility("default"))) int gqis_probe_tc_tf32(int iters, int repeats, double* tflops) {
    return probe_tc<0>(iters, repeats, tflops);
}
__attribute__((visibility("default"))) int gqis_probe_tc_f16(int iters, int repeats, double* tflops) {
    return probe_tc<1>(iters, repeats, tflops);
}


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
