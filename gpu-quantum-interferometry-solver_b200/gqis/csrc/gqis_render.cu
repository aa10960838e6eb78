// gqis_render.cu - phase-space rasteriser: histogram of a point cloud, mean colour per pixel,
// and lookup-table colouring of the raster into an RGBA8 image (C ABI in include/gqis_render.h).
//
// The binning reads points in place (FP32 or FP64, any stride between points, so an odesolve_2D
// state trace on the device is binned without a gathered copy), rounds them to FP32 and applies
// the reference renderer's rules (Examples/fast_gpu_render.py:108-131). Colour sums are FP64
// atomics into L2, so the raster does not depend on the order of the atomics beyond FP64
// rounding; sub-histograms by CTA (`partitions`) spread the atomics of concentrated clouds.
// Coordinates and colours are computed with explicitly rounded operations (no contraction into
// FMA) in the order of the reference kernels, so the pixel of every point and the RGBA of every
// output pixel are those of the reference's arithmetic.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdint.h>

#include "gqis_b200.h"
#include "gqis_render.h"

namespace {

thread_local char g_render_error[512] = "";

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_render_error, sizeof(g_render_error), fmt, ap);
    va_end(ap);
    return code;
}

constexpr int kBlock = 256;

template <class T>
__global__ void __launch_bounds__(kBlock) phase_bin_kernel(const T* __restrict__ points, int64_t n, int64_t stride,
                                                           const float* __restrict__ colors, uint32_t* counts,
                                                           double* sums, int nx, int ny, int partitions, float xmin,
                                                           float ymin, float sx, float sy) {
    const size_t part = (size_t)(blockIdx.x % (unsigned)partitions) * (size_t)nx * (size_t)ny;
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
        const float x = (float)points[i * stride];
        const float v = (float)points[i * stride + 1];
        if (!isfinite(x) || !isfinite(v) || x < xmin || v < ymin) continue;
        const int ix = (int)__fmul_rn(__fsub_rn(x, xmin), sx);
        const int iy = (int)__fmul_rn(__fsub_rn(v, ymin), sy);
        if (ix >= 0 && ix < nx && iy >= 0 && iy < ny) {
            const size_t pixel = part + (size_t)iy * nx + ix;
            atomicAdd(counts + pixel, 1u);
            atomicAdd(sums + pixel, (double)colors[i]);
        }
    }
}

__global__ void __launch_bounds__(kBlock) phase_finalize_kernel(const uint32_t* __restrict__ counts,
                                                                const double* __restrict__ sums,
                                                                float* __restrict__ raster, int pixels,
                                                                int partitions) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= pixels) return;
    uint32_t count = 0;
    double sum = 0.0;
    for (int part = 0; part < partitions; ++part) {
        count += counts[(size_t)part * pixels + i];
        sum += sums[(size_t)part * pixels + i];
    }
    raster[i] = count ? (float)(sum / (double)count) : __int_as_float(0x7fc00000);
}

// Colour of raster pixel (x, y) clamped into the image: the table entry of its value scaled into
// [lo, lo + 1 / inv_range], or the last entry (empty pixels).
__device__ __forceinline__ float4 lut_colour(const float* __restrict__ src, const float4* __restrict__ lut, int x,
                                             int y, int nx, int ny, int ncolors, float lo, float inv_range) {
    x = max(0, min(nx - 1, x));
    y = max(0, min(ny - 1, y));
    const float value = src[y * nx + x];
    int index = ncolors;
    if (isfinite(value)) {
        const float u = fminf(1.0f, fmaxf(0.0f, __fmul_rn(__fsub_rn(value, lo), inv_range)));
        index = min(ncolors - 1, (int)__fmul_rn(u, (float)ncolors));
    }
    return lut[index];
}

__device__ __forceinline__ float lerp2(float a, float b, float d, float e, float fx, float fy) {
    // ((a + fx (b - a)) (1 - fy) + (d + fx (e - d)) fy), each operation rounded
    const float top = __fadd_rn(a, __fmul_rn(fx, __fsub_rn(b, a)));
    const float bot = __fadd_rn(d, __fmul_rn(fx, __fsub_rn(e, d)));
    return __fadd_rn(__fmul_rn(top, __fsub_rn(1.0f, fy)), __fmul_rn(bot, fy));
}

__device__ __forceinline__ unsigned char to_byte(float c) {
    return (unsigned char)__fadd_rn(__fmul_rn(255.0f, c), 0.5f);
}

__global__ void __launch_bounds__(kBlock) display_rgba_kernel(const float* __restrict__ src,
                                                              const float4* __restrict__ lut, uchar4* __restrict__ out,
                                                              int nx, int ny, int width, int height, int ncolors,
                                                              float lo, float inv_range, int linear, float u0, float u1,
                                                              float v0, float v1) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= width * height) return;
    const float du = __fdiv_rn(__fsub_rn(u1, u0), (float)width);
    const float dv = __fdiv_rn(__fsub_rn(v1, v0), (float)height);
    const float x = __fsub_rn(__fmul_rn(__fadd_rn(u0, __fmul_rn(__fadd_rn((float)(i % width), 0.5f), du)), (float)nx), 0.5f);
    const float y = __fsub_rn(__fmul_rn(__fadd_rn(v0, __fmul_rn(__fadd_rn((float)(i / width), 0.5f), dv)), (float)ny), 0.5f);
    float4 c;
    if (x < -0.5f || x > __fsub_rn((float)nx, 0.5f) || y < -0.5f || y > __fsub_rn((float)ny, 0.5f)) {
        c = lut[ncolors];  // outside the raster: background
    } else if (linear) {
        const int ix = (int)floorf(x), iy = (int)floorf(y);
        const float fx = __fsub_rn(x, (float)ix), fy = __fsub_rn(y, (float)iy);
        const float4 a = lut_colour(src, lut, ix, iy, nx, ny, ncolors, lo, inv_range);
        const float4 b = lut_colour(src, lut, ix + 1, iy, nx, ny, ncolors, lo, inv_range);
        const float4 d = lut_colour(src, lut, ix, iy + 1, nx, ny, ncolors, lo, inv_range);
        const float4 e = lut_colour(src, lut, ix + 1, iy + 1, nx, ny, ncolors, lo, inv_range);
        c = make_float4(lerp2(a.x, b.x, d.x, e.x, fx, fy), lerp2(a.y, b.y, d.y, e.y, fx, fy),
                        lerp2(a.z, b.z, d.z, e.z, fx, fy), lerp2(a.w, b.w, d.w, e.w, fx, fy));
    } else {
        c = lut_colour(src, lut, (int)floorf(__fadd_rn(x, 0.5f)), (int)floorf(__fadd_rn(y, 0.5f)), nx, ny, ncolors,
                       lo, inv_range);
    }
    out[i] = make_uchar4(to_byte(c.x), to_byte(c.y), to_byte(c.z), to_byte(c.w));
}

int launch_status(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(GQIS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return GQIS_OK;
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) const char* gqis_render_last_error(void) { return g_render_error; }

__attribute__((visibility("default"))) int gqis_phase_bin(const void* points, int points_type, int64_t n, int64_t stride,
                                                          const float* colors, uint32_t* counts, double* sums, int nx,
                                                          int ny, int partitions, float xmin, float ymin, float sx,
                                                          float sy, void* stream) {
    if (n < 0 || stride < 2 || nx < 1 || ny < 1 || partitions < 1)
        return fail(GQIS_ERR_INVALID, "invalid sizes (n %lld, stride %lld, %d x %d pixels, %d partitions)",
                    (long long)n, (long long)stride, nx, ny, partitions);
    if (points_type != GQIS_RENDER_F32 && points_type != GQIS_RENDER_F64)
        return fail(GQIS_ERR_INVALID, "points_type must be GQIS_RENDER_F32 or GQIS_RENDER_F64");
    if (n == 0) return GQIS_OK;
    if (!points || !colors || !counts || !sums) return fail(GQIS_ERR_INVALID, "NULL buffer");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return fail(GQIS_ERR_CUDA, "no CUDA device");
    const int64_t needed = (n + kBlock - 1) / kBlock;
    const int64_t cap = (int64_t)sms * 8;
    const unsigned grid = (unsigned)(needed < cap ? needed : cap);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (points_type == GQIS_RENDER_F32)
        phase_bin_kernel<float><<<grid, kBlock, 0, st>>>(static_cast<const float*>(points), n, stride, colors, counts,
                                                         sums, nx, ny, partitions, xmin, ymin, sx, sy);
    else
        phase_bin_kernel<double><<<grid, kBlock, 0, st>>>(static_cast<const double*>(points), n, stride, colors, counts,
                                                          sums, nx, ny, partitions, xmin, ymin, sx, sy);
    return launch_status("phase_bin_kernel");
}

__attribute__((visibility("default"))) int gqis_phase_finalize(const uint32_t* counts, const double* sums, float* raster,
                                                               int pixels, int partitions, void* stream) {
    if (pixels < 0 || partitions < 1) return fail(GQIS_ERR_INVALID, "invalid sizes");
    if (pixels == 0) return GQIS_OK;
    if (!counts || !sums || !raster) return fail(GQIS_ERR_INVALID, "NULL buffer");
    phase_finalize_kernel<<<(pixels + kBlock - 1) / kBlock, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(
        counts, sums, raster, pixels, partitions);
    return launch_status("phase_finalize_kernel");
}

__attribute__((visibility("default"))) int gqis_display_rgba(const float* raster, const float* lut, uint8_t* out, int nx,
                                                             int ny, int width, int height, int ncolors, float lo,
                                                             float inv_range, int linear, float u0, float u1, float v0,
                                                             float v1, void* stream) {
    if (nx < 1 || ny < 1 || width < 1 || height < 1 || ncolors < 1)
        return fail(GQIS_ERR_INVALID, "invalid sizes");
    if ((int64_t)width * height > 0x7fffffffLL) return fail(GQIS_ERR_TOO_LARGE, "output image too large");
    if (!raster || !lut || !out) return fail(GQIS_ERR_INVALID, "NULL buffer");
    if (((uintptr_t)lut & 15u) != 0 || ((uintptr_t)out & 3u) != 0)
        return fail(GQIS_ERR_INVALID, "lut must be 16-byte and out 4-byte aligned");
    const int total = width * height;
    display_rgba_kernel<<<(total + kBlock - 1) / kBlock, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(
        raster, reinterpret_cast<const float4*>(lut), reinterpret_cast<uchar4*>(out), nx, ny, width, height, ncolors,
        lo, inv_range, linear, u0, u1, v0, v1);
    return launch_status("display_rgba_kernel");
}

}  // extern "C"
