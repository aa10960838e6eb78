"""CPU tests of the phase-space rasteriser: the NumPy oracle against the reference kernels' golden
outputs (tests/golden/make_render_golden.py), and the render library's C ABI symbols."""

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
