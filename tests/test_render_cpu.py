"""CPU tests of the phase-space rasteriser: the NumPy oracle against the reference kernels' golden
outputs (tests/golden/make_render_golden.py), and the render library's C ABI: its symbols and its
argument checks."""

import ctypes
from pathlib import Path

import numpy as np
import pytest

import render_oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
ROOT = Path(__file__).resolve().parents[1]


def test_oracle_raster_matches_reference_kernels():
    g = np.load(GOLDEN / "render_raster.npz")
    raster, counts = render_oracle.bin_raster(g["points"], g["colors"], g["bins"], g["x_range"], g["v_range"])
    np.testing.assert_array_equal(counts, g["counts"])  # the binning rules are the reference's
    np.testing.assert_array_equal(np.isnan(raster), np.isnan(g["raster"]))
    occ = ~np.isnan(raster)
    # the reference sums colours in FP32 in point order, the oracle in FP64
    assert np.max(np.abs(raster[occ] - g["raster"][occ])) < 2e-4
    assert np.median(np.abs(raster[occ] - g["raster"][occ])) < 1e-7


def test_oracle_display_matches_reference_kernel():
    g = np.load(GOLDEN / "render_display.npz")
    lo, hi = g["color_range"]
    inv = np.float32(1.0 / (hi - lo))
    for k, ((w, h, linear), view) in enumerate(zip(g["cases"], g["views"])):
        img = render_oracle.display_rgba(g["raster"], g["lut"], int(w), int(h), np.float32(lo), inv, int(linear),
                                         tuple(float(v) for v in view))
        np.testing.assert_array_equal(img, g[f"image_{k}"], err_msg=f"case {k}")


def test_render_library_exports_the_header_symbols():
    import re
    from gqis import native
    lib = ctypes.CDLL(str(native.build("gqis_render")))  # nvcc builds it here; loading needs no GPU
    header = (ROOT / "include" / "gqis_render.h").read_text()
    names = re.findall(r"^(?:int|const char\*)\s+(gqis_\w+)\(", header, re.M)
    assert len(names) == 4
    for n in names:
        assert hasattr(lib, n), n


def test_render_library_rejects_invalid_arguments_before_any_cuda_call():
    """Every size, type, NULL and alignment check of the rasteriser's C ABI runs before it touches a
    device, and empty inputs return at once, so all of them are testable without a GPU."""
    import ctypes
    from gqis import native
    lib = ctypes.CDLL(str(native.build("gqis_render")))
    lib.gqis_render_last_error.restype = ctypes.c_char_p
    f, i, i64, p = ctypes.c_float, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p
    lib.gqis_phase_bin.argtypes = [p, i, i64, i64, p, p, p, i, i, i, f, f, f, f, p]
    lib.gqis_phase_finalize.argtypes = [p, p, p, i, i, p]
    lib.gqis_display_rgba.argtypes = [p, p, p, i, i, i, i, i, f, f, i, f, f, f, f, p]
    buf = ctypes.create_string_buffer(64)
    base = (ctypes.addressof(buf) + 15) // 16 * 16  # a 16-byte-aligned host address (never dereferenced)

    def bin_(points_type=0, n=4, stride=2, nx=8, ny=8, parts=2, ptr=base):
        return lib.gqis_phase_bin(ptr, points_type, n, stride, ptr, ptr, ptr, nx, ny, parts, 0, 0, 1, 1, None)

    def last():
        return lib.gqis_render_last_error()

    assert bin_(stride=1) == 1 and b"invalid sizes" in last()
    assert bin_(n=-1) == 1 and bin_(nx=0) == 1 and bin_(parts=0) == 1
    assert bin_(points_type=2) == 1 and b"points_type" in last()
    assert bin_(ptr=None) == 1 and b"NULL buffer" in last()
    assert bin_(n=0, ptr=None) == 0  # nothing to bin
    assert lib.gqis_phase_finalize(base, base, base, -1, 1, None) == 1
    assert lib.gqis_phase_finalize(base, base, base, 16, 0, None) == 1
    assert lib.gqis_phase_finalize(None, None, None, 0, 1, None) == 0
    assert lib.gqis_phase_finalize(None, base, base, 16, 1, None) == 1 and b"NULL buffer" in last()

    def display(width=4, height=4, lut=base, out=base, nx=8):
        return lib.gqis_display_rgba(base, lut, out, nx, 8, width, height, 16, 0, 1, 0, 0, 1, 0, 1, None)

    assert display(nx=0) == 1 and b"invalid sizes" in last()
    assert display(width=1 << 16, height=1 << 16) == 4 and b"too large" in last()
    assert display(lut=None) == 1 and b"NULL buffer" in last()
    assert display(lut=base + 4) == 1 and b"aligned" in last()
    assert display(out=base + 1) == 1 and b"aligned" in last()
