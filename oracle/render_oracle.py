"""CPU oracle of the phase-space rasteriser (NumPy). Oracle infrastructure only: used by tests/.

Restates the reference renderer's kernels (Examples/fast_gpu_render.py):

* ``bin_raster``: phase_bin + phase_finalize (:108-147, launch :185-228): points rounded to FP32,
  skipped unless finite with x >= xmin and v >= vmin, pixel ((x - xmin) sx, (v - vmin) sy)
  truncated, FP32 scale factors nx / (xmax - xmin); the mean colour of each pixel with FP64 sums
  (the product's accumulation), NaN where empty;
* ``display_rgba``: display_rgba (:258-300): nearest or bilinear sampling of a view of the raster,
  table lookup of (value - lo) * inv_range with the last entry for empty pixels and the background,
  every operation rounded in FP32 as written.

Pinned against tests/golden/render_*.npz (the reference kernels run on the CPU by
tests/golden/make_render_golden.py): identical counts, means within the FP32 accumulation error of
the reference's sums, identical RGBA bytes.
"""

import numpy as np

F = np.float32


def bin_raster(points, colors, bins, x_range, v_range):
    """(ny, nx) FP32 mean-colour raster and (ny, nx) counts of a cloud of (x, v) points."""
    nx, ny = (int(b) for b in bins)
    xmin, xmax = (float(v) for v in x_range)
    ymin, ymax = (float(v) for v in v_range)
    p = np.asarray(points).reshape(-1, 2).astype(F)
    x, v = p[:, 0], p[:, 1]
    sx, sy = F(nx / (xmax - xmin)), F(ny / (ymax - ymin))
    with np.errstate(invalid="ignore", over="ignore"):
        ok = np.isfinite(x) & np.isfinite(v) & (x >= F(xmin)) & (v >= F(ymin))
        fx = (x[ok] - F(xmin)) * sx
        fy = (v[ok] - F(ymin)) * sy
    ix = np.where(fx < 2**31, fx, -1).astype(np.int64)
    iy = np.where(fy < 2**31, fy, -1).astype(np.int64)
    inside = (ix >= 0) & (ix < nx) & (iy >= 0) & (iy < ny)
    flat = iy[inside] * nx + ix[inside]
    col = np.asarray(colors, dtype=F)[ok][inside].astype(np.float64)
    counts = np.bincount(flat, minlength=nx * ny)
    sums = np.bincount(flat, weights=col, minlength=nx * ny)
    raster = np.full(nx * ny, np.nan, dtype=F)
    occ = counts > 0
    raster[occ] = (sums[occ] / counts[occ]).astype(F)
    return raster.reshape(ny, nx), counts.reshape(ny, nx)


def _lut_colour(raster, lut, x, y, lo, inv_range):
    ny, nx = raster.shape
    ncolors = len(lut) - 1
    x = np.clip(x, 0, nx - 1)
    y = np.clip(y, 0, ny - 1)
    value = raster[y, x]
    index = np.full(value.shape, ncolors, dtype=np.int64)
    fin = np.isfinite(value)
    u = np.minimum(F(1), np.maximum(F(0), (value[fin] - F(lo)) * F(inv_range)))
    index[fin] = np.minimum(ncolors - 1, (u * F(ncolors)).astype(np.int64))
    return lut[index]


def display_rgba(raster, lut, width, height, lo, inv_range, linear, view=(0.0, 1.0, 0.0, 1.0)):
    """(height, width, 4) uint8 image of a raster through an (ncolors + 1, 4) FP32 table."""
    raster = np.asarray(raster, dtype=F)
    lut = np.asarray(lut, dtype=F)
    ny, nx = raster.shape
    u0, u1, v0, v1 = (F(v) for v in view)
    i = np.arange(width * height)
    du = (u1 - u0) / F(width)
    dv = (v1 - v0) / F(height)
    x = (u0 + ((i % width).astype(F) + F(0.5)) * du) * F(nx) - F(0.5)
    y = (v0 + ((i // width).astype(F) + F(0.5)) * dv) * F(ny) - F(0.5)
    out = np.empty((width * height, 4), dtype=F)
    outside = (x < F(-0.5)) | (x > F(nx) - F(0.5)) | (y < F(-0.5)) | (y > F(ny) - F(0.5))
    out[outside] = lut[len(lut) - 1]
    inner = ~outside
    xi, yi = x[inner], y[inner]
    if linear:
        ix, iy = np.floor(xi).astype(np.int64), np.floor(yi).astype(np.int64)
        fx = (xi - ix.astype(F))[:, None]
        fy = (yi - iy.astype(F))[:, None]
        a = _lut_colour(raster, lut, ix, iy, lo, inv_range)
        b = _lut_colour(raster, lut, ix + 1, iy, lo, inv_range)
        d = _lut_colour(raster, lut, ix, iy + 1, lo, inv_range)
        e = _lut_colour(raster, lut, ix + 1, iy + 1, lo, inv_range)
        out[inner] = (a + fx * (b - a)) * (F(1) - fy) + (d + fx * (e - d)) * fy
    else:
        out[inner] = _lut_colour(raster, lut, np.floor(xi + F(0.5)).astype(np.int64),
                                 np.floor(yi + F(0.5)).astype(np.int64), lo, inv_range)
    return (F(255) * out + F(0.5)).astype(np.uint8).reshape(height, width, 4)
