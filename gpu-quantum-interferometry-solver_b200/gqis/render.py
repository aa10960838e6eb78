"""Phase-space rasteriser: a point cloud (e.g. the states of an ``odesolve_2D`` sweep) into a
mean-colour image on the GPU, and an image into display RGBA through a colour table.

Drop-in for the reference's ``PhaseRasterizer`` and ``GPUDisplayImage``
(Examples/fast_gpu_render.py:97-250, :251-330): same constructor arguments, the same
``render`` results (``(ny, nx)`` FP32 raster, NaN for empty pixels; ``(height, width, 4)`` uint8),
with the kernels of ``csrc/gqis_render.cu`` behind the C ABI of ``include/gqis_render.h``.
Differences:

* colour sums are FP64 (the reference's GPU kernel sums in FP32 in an arbitrary atomic order);
* ``render_trace`` bins one sample of an ``odesolve_2D`` state trace in place on the device, with
  no copy of the cloud;
* the colour table is an ``(ncolors + 1, 4)`` RGBA array (the last row for empty pixels and the
  background) instead of a Matplotlib colormap, which this package does not use;
* there is no CPU path: without a CUDA device the calls raise.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import native

_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        lib = native.load("gqis_render")
        P, I, L, Fl = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float
        lib.gqis_phase_bin.argtypes = [P, I, L, L, P, P, P, I, I, I, Fl, Fl, Fl, Fl, P]
        lib.gqis_phase_finalize.argtypes = [P, P, P, I, I, P]
        lib.gqis_display_rgba.argtypes = [P, P, P, I, I, I, I, I, Fl, Fl, I, Fl, Fl, Fl, Fl, P]
        for f in (lib.gqis_phase_bin, lib.gqis_phase_finalize, lib.gqis_display_rgba):
            f.restype = I
        lib.gqis_render_last_error.restype = ctypes.c_char_p
        _LIB = lib
    return _LIB


def _check(rc):
    if rc != 0:
        raise RuntimeError(f"gqis render kernel failed ({rc}): {_lib().gqis_render_last_error().decode()}")


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("The phase-space rasteriser needs a CUDA device (there is no CPU path).")
    return torch


class PhaseRasterizer:
    """Turn a cloud of (x, v) points into one ``(ny, nx)`` mean-colour image on the GPU.

    ``color_values``: one colour per point; ``x_range``, ``v_range``: the image extent;
    ``bins``: ``(nx, ny)``; ``partitions``: sub-histograms that spread the atomics of concentrated
    clouds (``histogram_partitions`` of the reference).
    """

    def __init__(self, color_values, *, x_range, v_range, bins, use_gpu=True, partitions=8):
        if not use_gpu:
            raise ValueError("gqis.render has no CPU path; use_gpu must be True.")
        torch = _torch()
        self.nx, self.ny = map(int, bins)
        self.xmin, self.xmax = map(float, x_range)
        self.ymin, self.ymax = map(float, v_range)
        self.partitions = int(partitions)
        if self.partitions < 1:
            raise ValueError("histogram_partitions must be positive.")
        if not (self.xmax > self.xmin and self.ymax > self.ymin) or self.nx < 1 or self.ny < 1:
            raise ValueError("x_range and v_range must be increasing and bins positive.")
        dev = torch.device("cuda", torch.cuda.current_device())
        colors = color_values if hasattr(color_values, "data_ptr") else np.asarray(color_values, dtype=np.float32)
        self._colors = torch.as_tensor(colors, dtype=torch.float32, device=dev).reshape(-1).contiguous()
        self._point_count = int(self._colors.numel())
        pixels = self.nx * self.ny
        self._counts = torch.empty(pixels * self.partitions, dtype=torch.int32, device=dev)
        self._sums = torch.empty(pixels * self.partitions, dtype=torch.float64, device=dev)
        self._raster = torch.empty((self.ny, self.nx), dtype=torch.float32, device=dev)
        self._upload = None
        self.use_gpu = True

    @property
    def backend_name(self) -> str:
        return "gqis B200 CUDA kernels"

    def _bin(self, base_ptr, points_type, n, stride, keepalive, return_device):
        torch = _torch()
        if n != self._point_count:
            raise ValueError("Phase-space point count changed between animation frames.")
        stream = torch.cuda.current_stream().cuda_stream
        self._counts.zero_()
        self._sums.zero_()
        sx = float(np.float32(self.nx / (self.xmax - self.xmin)))
        sy = float(np.float32(self.ny / (self.ymax - self.ymin)))
        lib = _lib()
        _check(lib.gqis_phase_bin(base_ptr, points_type, n, stride, self._colors.data_ptr(), self._counts.data_ptr(),
                                  self._sums.data_ptr(), self.nx, self.ny, self.partitions, self.xmin, self.ymin,
                                  sx, sy, stream))
        _check(lib.gqis_phase_finalize(self._counts.data_ptr(), self._sums.data_ptr(), self._raster.data_ptr(),
                                       self.nx * self.ny, self.partitions, stream))
        del keepalive
        if return_device:
            return self._raster  # reused by the next render: consume before rendering again
        return self._raster.cpu().numpy()

    def render(self, points, *, return_device=False):
        """``(ny, nx)`` FP32 image of ``points`` (``(n, 2)`` or any array of n pairs; host or CUDA;
        FP32 or FP64)."""
        torch = _torch()
        if hasattr(points, "data_ptr") and points.is_cuda:
            t = points.reshape(-1, 2)
            if t.dtype not in (torch.float32, torch.float64):
                t = t.to(torch.float32)
            t = t.contiguous()
        else:
            host = np.ascontiguousarray(np.asarray(points).reshape(-1, 2), dtype=np.float32)
            if self._upload is None or self._upload.shape[0] != len(host):
                self._upload = torch.empty((len(host), 2), dtype=torch.float32, device=self._raster.device)
            self._upload.copy_(torch.from_numpy(host))
            t = self._upload
        ptype = 1 if t.dtype == torch.float64 else 0
        return self._bin(t.data_ptr(), ptype, int(t.shape[0]), 2, t, return_device)

    def render_trace(self, trace, sample, *, components=(0, 1), return_device=False):
        """Image of sample ``sample`` of a state trace ``(..., num_trace, S)`` that lives on the
        device (``odesolve_2D(..., return_time_trace=True, return_device=True)``): binned in place."""
        torch = _torch()
        if not (hasattr(trace, "data_ptr") and trace.is_cuda and trace.is_contiguous()):
            raise ValueError("render_trace needs a contiguous CUDA tensor (return_device=True).")
        if trace.dtype not in (torch.float32, torch.float64):
            raise ValueError("trace must be FP32 or FP64")
        T, S = int(trace.shape[-2]), int(trace.shape[-1])
        cx, cv = components
        if not (0 <= sample < T) or cv != cx + 1 or not (0 <= cx and cv < S):
            raise ValueError("sample out of range, or components are not two adjacent state entries")
        n = int(trace.numel() // (T * S))
        base = trace.data_ptr() + (sample * S + cx) * trace.element_size()
        return self._bin(base, 1 if trace.dtype == torch.float64 else 0, n, T * S, trace, return_device)


class GPUDisplayImage:
    """Scale and colour a device raster into a display-sized RGBA8 image on the GPU.

    ``lut``: ``(ncolors + 1, 4)`` RGBA floats in [0, 1], the last row for empty pixels and the
    background; ``color_min``, ``color_max``: the colour range; ``interpolation``: "nearest" or
    "bilinear".
    """

    def __init__(self, lut, color_min, color_max, interpolation):
        if interpolation not in ("nearest", "bilinear"):
            raise ValueError("GPU display supports 'nearest' or 'bilinear'.")
        torch = _torch()
        table = np.asarray(lut, dtype=np.float32)
        if table.ndim != 2 or table.shape[1] != 4 or len(table) < 2:
            raise ValueError("lut must have shape (ncolors + 1, 4)")
        dev = torch.device("cuda", torch.cuda.current_device())
        self.lut = torch.as_tensor(table, device=dev).contiguous()
        self.ncolors = len(table) - 1
        self.lo = float(np.float32(color_min))
        self.inv_range = float(np.float32(1.0 / (color_max - color_min) if color_max > color_min else 0.0))
        self.linear = int(interpolation == "bilinear")
        self.shape = None
        self.device = None

    def render(self, raster, display_size, *, return_device=False):
        """``(height, width, 4)`` uint8 image; ``display_size`` = (width, height[, u0, u1, v0, v1])."""
        torch = _torch()
        width, height = int(display_size[0]), int(display_size[1])
        view = tuple(display_size[2:]) or (0.0, 1.0, 0.0, 1.0)
        shape = (height, width, 4)
        if shape != self.shape:
            self.device = torch.empty(shape, dtype=torch.uint8, device=self.lut.device)
            self.shape = shape
        src = raster if hasattr(raster, "data_ptr") else torch.as_tensor(np.asarray(raster, dtype=np.float32))
        src = src.to(device=self.lut.device, dtype=torch.float32).contiguous()
        ny, nx = int(src.shape[0]), int(src.shape[1])
        _check(_lib().gqis_display_rgba(src.data_ptr(), self.lut.data_ptr(), self.device.data_ptr(), nx, ny, width,
                                        height, self.ncolors, self.lo, self.inv_range, self.linear,
                                        *(float(v) for v in view), torch.cuda.current_stream().cuda_stream))
        if return_device:
            return self.device
        return self.device.cpu().numpy()
