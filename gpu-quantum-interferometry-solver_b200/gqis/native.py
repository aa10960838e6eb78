"""The package's fixed native libraries (built in-tree by nvcc for sm_100a).

* ``libgqis_probe.so``  - FMA-pipe and TF32 / FP16 tensor-core throughput probes (roofline denominators);
* ``libgqis_render.so`` - phase-space rasteriser kernels (``gqis.render``);
* ``libgqis_serve.so``  - native sweep server for C/C++ hosts (``include/gqis_serve.h``).

Model modules (one per model variant) are built separately by ``engine``.
"""

from __future__ import annotations

import ctypes
import hashlib
import subprocess
from pathlib import Path

from .engine import ARCH_FLAGS, CSRC_DIR, INCLUDE_DIR, PACKAGE_DIR, nvcc_path

BUILD_DIR = PACKAGE_DIR / "_build"
LIBS = {"gqis_probe": ["gqis_probe.cu"], "gqis_render": ["gqis_render.cu"], "gqis_serve": ["gqis_serve.cu"]}
LINK = {"gqis_serve": ["-ldl"]}
_loaded: dict = {}


def _digest(sources):
    h = hashlib.sha256()
    for p in sorted(CSRC_DIR.glob("*.cuh")) + sorted(INCLUDE_DIR.glob("*.h")) + [CSRC_DIR / s for s in sources]:
        h.update(p.name.encode())
        h.update(p.read_bytes())
    return h.hexdigest()[:16]


def lib_path(name) -> Path:
    """In-tree path of the fixed library ``lib<name>.so``."""
    return BUILD_DIR / f"lib{name}.so"


def build(name, force=False) -> Path:
    """Compile one fixed library if its sources changed; returns the .so path."""
    sources = LIBS[name]
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    out = lib_path(name)
    stamp = BUILD_DIR / f"lib{name}.digest"
    digest = _digest(sources)
    if out.exists() and stamp.exists() and stamp.read_text() == digest and not force:
        return out
    cmd = [nvcc_path(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", f"-I{CSRC_DIR}", f"-I{INCLUDE_DIR}",
           *[str(CSRC_DIR / s) for s in sources], "-o", str(out) + ".tmp", "-lcuda", *LINK.get(name, [])]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for lib{name}.so:\n{proc.stderr[-6000:]}")
    Path(str(out) + ".tmp").replace(out)
    stamp.write_text(digest)
    return out


def load(name):
    """Load a fixed library; it must have been built (``__graft_entry__.build()``)."""
    if name in _loaded:
        return _loaded[name]
    path = lib_path(name)
    if not path.exists():
        path = build(name)
    lib = ctypes.CDLL(str(path))
    _loaded[name] = lib
    return lib


def probe_fma_tflops(kind, iters=4096, repeats=3):
    """Measured FMA throughput in TFLOP/s: kind 0 FP64, 1 FP32, 2 packed FP32."""
    lib = load("gqis_probe")
    lib.gqis_probe_fma.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.gqis_probe_fma.restype = ctypes.c_int
    out = ctypes.c_double()
    rc = lib.gqis_probe_fma(int(kind), int(iters), int(repeats), ctypes.byref(out))
    if rc != 0:
        raise RuntimeError(f"gqis_probe_fma failed with status {rc}")
    return out.value


def _probe_tc(symbol, iters, repeats):
    lib = load("gqis_probe")
    fn = getattr(lib, symbol)
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    fn.restype = ctypes.c_int
    out = ctypes.c_double()
    rc = fn(int(iters), int(repeats), ctypes.byref(out))
    if rc != 0:
        raise RuntimeError(f"{symbol} failed with status {rc}")
    return out.value


def probe_tc_tf32_tflops(iters=4096, repeats=3):
    """Measured dense TF32 tensor-core rate in TFLOP/s (tcgen05 kind::tf32, M=128, N=256, K=8)."""
    return _probe_tc("gqis_probe_tc_tf32", iters, repeats)


def probe_tc_f16_tflops(iters=4096, repeats=3):
    """Measured dense FP16 tensor-core rate in TFLOP/s (tcgen05 kind::f16, M=128, N=256, K=16), the
    instruction of the density-matrix tensor-core kernel."""
    return _probe_tc("gqis_probe_tc_f16", iters, repeats)
