"""Run the captured reference kernels of ``oracle/_ref`` (see ``ref_capture.py``).

Oracle infrastructure: used by tests, golden-fixture generation and bench.py's reference arm
only. ``run_case(name, device="cpu" | "gpu")`` returns the outputs in the reference API's
shapes: ``result`` and, for trace cases, ``trace`` and ``trace_t``.
"""

from __future__ import annotations

import ctypes
import json
import time
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parent / "_ref"

_C_DTYPES = {"float64": np.float64, "float32": np.float32, "complex128": np.complex128,
             "complex64": np.complex64, "int32": np.int32}


def available(name, device="cpu"):
    return (REF_DIR / f"{name}.json").exists() and (REF_DIR / f"{name}_{device}.so").exists()


def meta(name):
    return json.loads((REF_DIR / f"{name}.json").read_text())


def _buffers(m):
    inputs = np.load(REF_DIR / f"{m['name']}_inputs.npz")
    bufs = []
    for arg in m["args"]:
        if arg["kind"] != "array":
            continue
        dt = _C_DTYPES[arg["dtype"]]
        if arg.get("output"):
            bufs.append(np.zeros(arg["shape"], dtype=dt))
        else:
            bufs.append(np.ascontiguousarray(inputs[arg["key"]]).astype(dt, copy=False))
    return bufs


def _assemble(m, bufs):
    arrays = [a for a in m["args"] if a["kind"] == "array"]
    got = {a.get("param"): b for a, b in zip(arrays, bufs)}
    out = {"result": got["results"]}
    if "time_trace_results" in got:
        out["trace"] = got["time_trace_results"]
        out["trace_t"] = np.asarray(m["trace_t"])
    if "adaptive_steps" in got:
        out["adaptive_steps"] = got["adaptive_steps"]
    return out


def run_case(name, device="cpu", repeats=1):
    """Run a captured reference kernel; returns (outputs, seconds per run)."""
    m = meta(name)
    lib = ctypes.CDLL(str(REF_DIR / f"{name}_{device}.so"))
    lib.ref_launch.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]
    lib.ref_launch.restype = ctypes.c_int
    bufs = _buffers(m)
    if device == "cpu":
        ptrs = (ctypes.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
        t0 = time.perf_counter()
        for _ in range(repeats):
            for b, a in zip(bufs, [a for a in m["args"] if a["kind"] == "array"]):
                if a.get("output"):
                    b[...] = 0
            rc = lib.ref_launch(ptrs, None)
        dt = (time.perf_counter() - t0) / repeats
        if rc:
            raise RuntimeError(f"reference CPU kernel {name} returned {rc}")
        return _assemble(m, bufs), dt
    import torch
    dev = [torch.as_tensor(b).cuda() if b.dtype != np.complex128 and b.dtype != np.complex64
           else torch.view_as_real(torch.as_tensor(b)).cuda() for b in bufs]
    ptrs = (ctypes.c_void_p * len(dev))(*[t.data_ptr() for t in dev])
    stream = torch.cuda.current_stream()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(repeats):
        rc = lib.ref_launch(ptrs, ctypes.c_void_p(stream.cuda_stream))
        if rc:
            raise RuntimeError(f"reference GPU kernel {name} launch failed: cudaError {rc}")
    stop.record(stream)
    stop.synchronize()
    dt = start.elapsed_time(stop) / 1000.0 / repeats
    host = []
    for t, b in zip(dev, bufs):
        a = t.cpu().numpy()
        if np.iscomplexobj(b):
            a = a[..., 0] + 1j * a[..., 1]
            a = a.astype(b.dtype)
        host.append(a)
    return _assemble(m, host), dt
