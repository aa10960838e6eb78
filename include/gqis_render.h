/* gqis_render.h - C ABI of the phase-space rasteriser library (libgqis_render.so).
 *
 * Replaces the three CUDA kernels the reference's phase-space renderer compiles with
 * cp.RawKernel (Examples/fast_gpu_render.py): phase_bin (:108-131), phase_finalize (:133-147)
 * and display_rgba (:258-300), and the host launch code around them (:185-235, :316-330).
 * Points can be read in place from an odesolve_2D state trace on the device (point stride),
 * so no gathered copy of the cloud is made. All calls enqueue on `stream` (a cudaStream_t,
 * NULL for the legacy stream) and return GQIS_OK or an error status; gqis_render_last_error()
 * describes the last failure of the calling thread.
 */
#ifndef GQIS_RENDER_H
#define GQIS_RENDER_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GQIS_RENDER_F32 0
#define GQIS_RENDER_F64 1

/* Histogram of n points into `partitions` sub-histograms of nx * ny pixels
 * (Examples/fast_gpu_render.py:108-131 and :201-228): point i is (p[i*stride], p[i*stride+1]) of
 * type points_type, rounded to FP32; it is skipped unless both are finite and x >= xmin, v >= ymin;
 * its pixel is ((int)((x - xmin) * sx), (int)((v - ymin) * sy)) when inside the image. counts[k]
 * (uint32) and sums[k] (FP64, the colour sums) must be zeroed by the caller (k < partitions*nx*ny);
 * the sub-histogram of a point is its CTA index modulo `partitions`. colors[i] is the point's colour. */
int gqis_phase_bin(const void* points, int points_type, int64_t n, int64_t stride, const float* colors,
                   uint32_t* counts, double* sums, int nx, int ny, int partitions, float xmin, float ymin,
                   float sx, float sy, void* stream);

/* raster[k] = sum / count over the partitions, NaN for empty pixels (:133-147). */
int gqis_phase_finalize(const uint32_t* counts, const double* sums, float* raster, int pixels, int partitions,
                        void* stream);

/* Colour a ny x nx raster into a height x width RGBA8 image through a lookup table of
 * ncolors + 1 RGBA float entries (the last one for empty pixels and the background), nearest or
 * bilinear (`linear`) sampling of the view [u0, u1] x [v0, v1] of the raster (:258-300). */
int gqis_display_rgba(const float* raster, const float* lut, uint8_t* out, int nx, int ny, int width, int height,
                      int ncolors, float lo, float inv_range, int linear, float u0, float u1, float v0, float v1,
                      void* stream);

const char* gqis_render_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GQIS_RENDER_H */
