"""Golden fixtures of the phase-space rasteriser from the reference's own kernels, on the CPU.

Run in the build container (needs the reference tree): ``python tests/golden/make_render_golden.py``.
The reference module Examples/fast_gpu_render.py is imported with small stand-ins for the Matplotlib
modules it imports (only names are needed; nothing of Matplotlib runs) and without CuPy. Its kernel
texts phase_bin, phase_finalize (PhaseRasterizer, :108-147) and display_rgba (GPUDisplayImage,
:258-300) are compiled by g++ through oracle/render_cpu_shim.h into oracle/_ref/librender_ref.so and
launched over every (block, thread) in launch order, so the fixtures hold the reference kernels'
arithmetic (FP32 sums in point order). Inputs are seeded; the fixtures are
tests/golden/render_raster.npz and tests/golden/render_display.npz.
"""

import ctypes
import importlib.util
import os
import subprocess
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REFERENCE = Path(os.environ.get("GQIS_REFERENCE_DIR", str(ROOT.parent / "reference")))
OUT = ROOT / "oracle" / "_ref"


def _stub_matplotlib():
    names = ["matplotlib", "matplotlib.pyplot", "matplotlib.animation", "matplotlib.colors", "matplotlib.cm",
             "matplotlib.artist"]
    for n in names:
        sys.modules.setdefault(n, types.ModuleType(n))
    anim = sys.modules["matplotlib.animation"]
    anim.FFMpegWriter = anim.FuncAnimation = object
    sys.modules["matplotlib.cm"].ScalarMappable = object
    sys.modules["matplotlib.artist"].Artist = object
    sys.modules["matplotlib"].colors = sys.modules["matplotlib.colors"]


def reference_kernels():
    _stub_matplotlib()
    sys.modules["cupy"] = None  # the module falls back to cp = None
    spec = importlib.util.spec_from_file_location("ref_fast_gpu_render", REFERENCE / "Examples" / "fast_gpu_render.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return (mod.PhaseRasterizer._BIN_KERNEL_SOURCE, mod.PhaseRasterizer._FINAL_KERNEL_SOURCE,
            mod.GPUDisplayImage._SOURCE)


DRIVER = r'''
extern "C" void run_bin(const float* points, const float* colors, unsigned* counts, float* weighted, int n, int nx,
                        int ny, int partitions, float xmin, float ymin, float sx, float sy) {
    const int threads = 256, blocks = (n + threads - 1) / threads;
    blockDim.x = threads;
    for (unsigned b = 0; b < (unsigned)blocks; ++b)
        for (unsigned t = 0; t < (unsigned)threads; ++t) {
            blockIdx.x = b; threadIdx.x = t;
            phase_bin(points, colors, counts, weighted, n, nx, ny, partitions, xmin, ymin, sx, sy);
        }
}
extern "C" void run_finalize(const unsigned* counts, const float* weighted, float* raster, int n, int partitions) {
    const int threads = 256, blocks = (n + threads - 1) / threads;
    blockDim.x = threads;
    for (unsigned b = 0; b < (unsigned)blocks; ++b)
        for (unsigned t = 0; t < (unsigned)threads; ++t) {
            blockIdx.x = b; threadIdx.x = t;
            phase_finalize(counts, weighted, raster, n, partitions);
        }
}
extern "C" void run_display(const float* src, const float* lut, unsigned char* out, int nx, int ny, int width,
                            int height, int ncolors, float lo, float inv_range, int linear, float u0, float u1,
                            float v0, float v1) {
    const int threads = 256, total = width * height, blocks = (total + threads - 1) / threads;
    blockDim.x = threads;
    for (unsigned b = 0; b < (unsigned)blocks; ++b)
        for (unsigned t = 0; t < (unsigned)threads; ++t) {
            blockIdx.x = b; threadIdx.x = t;
            display_rgba(src, (const float4*)lut, (uchar4*)out, nx, ny, width, height, ncolors, lo, inv_range, linear,
                         u0, u1, v0, v1);
        }
}
'''


def build():
    bin_src, fin_src, disp_src = reference_kernels()
    OUT.mkdir(parents=True, exist_ok=True)
    cpp = OUT / "render_ref.cpp"
    cpp.write_text('#include "render_cpu_shim.h"\n' + bin_src + "\n" + fin_src + "\n" + disp_src + "\n" + DRIVER)
    so = OUT / "librender_ref.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", f"-I{ROOT / 'oracle'}",
                    str(cpp), "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    P = ctypes.c_void_p
    lib.run_bin.argtypes = [P, P, P, P] + [ctypes.c_int] * 4 + [ctypes.c_float] * 4
    lib.run_finalize.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int]
    lib.run_display.argtypes = [P, P, P] + [ctypes.c_int] * 5 + [ctypes.c_float] * 2 + [ctypes.c_int] + [ctypes.c_float] * 4
    return lib


def point_cloud(seed=0, n=60_000):
    """Seeded cloud: a tight cluster, a spread over part of the image (the rest stays empty), points
    outside the range, on and just outside the range edges, and non-finite points."""
    rng = np.random.default_rng(seed)
    pts = np.concatenate([
        rng.normal([0.3, -0.4], [0.05, 0.08], size=(n // 2, 2)),
        rng.uniform([-1.5, -2.0], [1.0, 2.5], size=(n // 2 - 3000, 2)),
        rng.uniform([-2.5, -3.5], [2.5, 3.5], size=(2000, 2)),
        np.stack([np.full(250, -2.0), rng.uniform(-3, 3, 250)], 1),            # x = xmin exactly
        np.stack([rng.uniform(-2, 2, 250), np.full(250, 3.0)], 1),             # v = vmax (outside)
        np.stack([np.full(250, -2.0 - 1e-7), rng.uniform(-3, 3, 250)], 1),     # just below xmin
        np.stack([np.full(250, np.nan), rng.uniform(-3, 3, 250)], 1),
    ])
    pts[rng.integers(0, len(pts), 50), 1] = np.inf
    colors = rng.uniform(0.0, 1.0, size=len(pts)).astype(np.float32)
    return pts, colors


def lut(ncolors=33):
    """Seeded smooth RGBA table with an extra last entry for empty pixels."""
    t = np.linspace(0.0, 1.0, ncolors)
    rgba = np.stack([t, 0.5 + 0.5 * np.sin(3 * t), 1.0 - t, np.full(ncolors, 1.0)], 1)
    return np.vstack([rgba, [1.0, 1.0, 1.0, 1.0]]).astype(np.float32)


RASTER_CASE = dict(bins=(96, 64), x_range=(-2.0, 2.0), v_range=(-3.0, 3.0), partitions=8)
DISPLAY_CASES = [  # (width, height, linear, view)
    (160, 120, 0, (0.0, 1.0, 0.0, 1.0)),
    (200, 150, 1, (0.1, 0.9, 0.2, 0.8)),
    (123, 77, 1, (-0.2, 1.2, -0.1, 1.1)),
    (64, 64, 0, (0.25, 0.75, 0.0, 1.0)),
]
COLOR_RANGE = (0.1, 0.9)


def main():
    lib = build()
    pts, colors = point_cloud()
    nx, ny = RASTER_CASE["bins"]
    (xmin, xmax), (ymin, ymax) = RASTER_CASE["x_range"], RASTER_CASE["v_range"]
    parts = RASTER_CASE["partitions"]
    p32 = np.ascontiguousarray(pts, dtype=np.float32)
    counts = np.zeros(parts * nx * ny, dtype=np.uint32)
    weighted = np.zeros(parts * nx * ny, dtype=np.float32)
    sx, sy = np.float32(nx / (xmax - xmin)), np.float32(ny / (ymax - ymin))
    lib.run_bin(p32.ctypes.data, colors.ctypes.data, counts.ctypes.data, weighted.ctypes.data, len(p32), nx, ny, parts,
                xmin, ymin, float(sx), float(sy))
    raster = np.empty(nx * ny, dtype=np.float32)
    lib.run_finalize(counts.ctypes.data, weighted.ctypes.data, raster.ctypes.data, nx * ny, parts)
    total_counts = counts.reshape(parts, -1).sum(0).reshape(ny, nx)
    np.savez_compressed(HERE / "render_raster.npz", points=pts, colors=colors, bins=np.array(RASTER_CASE["bins"]),
                        x_range=np.array(RASTER_CASE["x_range"]), v_range=np.array(RASTER_CASE["v_range"]),
                        partitions=parts, counts=total_counts.astype(np.uint32), raster=raster.reshape(ny, nx))
    table = lut()
    lo, hi = COLOR_RANGE
    inv = np.float32(1.0 / (hi - lo))
    images = {}
    for k, (w, h, linear, view) in enumerate(DISPLAY_CASES):
        out = np.zeros((h, w, 4), dtype=np.uint8)
        lib.run_display(raster.ctypes.data, table.ctypes.data, out.ctypes.data, nx, ny, w, h, len(table) - 1,
                        float(np.float32(lo)), float(inv), linear, *view)
        images[f"image_{k}"] = out
    np.savez_compressed(HERE / "render_display.npz", raster=raster.reshape(ny, nx), lut=table,
                        color_range=np.array(COLOR_RANGE), cases=np.array([c[:3] for c in DISPLAY_CASES]),
                        views=np.array([c[3] for c in DISPLAY_CASES], dtype=np.float32), **images)
    print("raster: %d occupied pixels of %d; display cases: %d" % (int((total_counts > 0).sum()), nx * ny,
                                                                   len(DISPLAY_CASES)))


if __name__ == "__main__":
    main()
