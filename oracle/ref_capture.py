"""Recipe: capture the reference's own generated kernels and build them as oracles.

Oracle infrastructure only (used by tests/, ``__graft_entry__.build()`` and the CPU baseline of
bench.py; never by the product path). Needs the reference source tree, so it runs only in the
build container; its outputs go to ``oracle/_ref/`` (git-ignored) and travel with the tree.

For every case of ``oracle/ref_cases.py``:

1. a child process imports the reference ``gqis`` package from the reference tree with the
   recording CuPy stand-in of ``oracle/refstub`` and calls ``mesolve_2D`` / ``odesolve_2D``;
   the stand-in records the generated CUDA source and the launch arguments
   (reference ``gqis/solver.py:2237-2340``);
2. the source is compiled (a) with nvcc for sm_100a plus a generated host launcher into
   ``<case>_gpu.so`` and (b) with g++ through ``ref_cpu_shim.h`` into ``<case>_cpu.so``
   (OpenMP over the points), both exporting ``int ref_launch(void** buffers, void* stream)``;
3. ``<case>.json`` records the kernel parameters, the input arrays (``<case>.npz``) and the
   output shapes.

Usage: ``python oracle/ref_capture.py [--reference DIR] [--cases a,b] [--jobs N]``
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# the reference checkout beside this repository unless --reference or GQIS_REFERENCE_DIR names another
DEFAULT_REFERENCE = Path(os.environ.get("GQIS_REFERENCE_DIR", str(HERE.parents[1] / "reference")))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
OUTPUT_PARAMS = ("results", "time_trace_results", "adaptive_steps")


# ------------------------------------------------------------------ child: capture
def _child(reference, names, out):
    sys.path.insert(0, str(HERE / "refstub"))
    sys.path.insert(0, str(reference))
    sys.path.insert(0, str(HERE))
    import cupy  # the recording stand-in
    import gqis
    import ref_cases
    all_cases = ref_cases.cases()
    for name in names:
        case = all_cases[name]
        cupy.RECORDS.clear()
        fn = getattr(gqis, case["api"])
        kwargs = dict(case["kwargs"])
        if case["api"] == "mesolve_2D":
            kwargs["ignore_non_finite_output"] = True
        result = fn(*case["args"], **kwargs)
        rec = cupy.RECORDS[-1]
        params = kernel_params(rec["code"])
        arrays, scalars = {}, []
        for k, (a, (_ctype, _ptr, pname)) in enumerate(zip(rec["args"], params)):
            if isinstance(a, np.ndarray):
                output = pname in OUTPUT_PARAMS
                if not output:
                    arrays[f"arg{k}"] = a
                scalars.append({"kind": "array", "key": f"arg{k}", "dtype": str(a.dtype), "shape": list(a.shape),
                                "param": pname, "output": output})
            elif isinstance(a, (np.floating, float)) and not isinstance(a, (bool, np.bool_)):
                dt = "float32" if isinstance(a, np.float32) else "float64"
                scalars.append({"kind": "scalar", "dtype": dt, "value": float(a)})
            else:
                scalars.append({"kind": "scalar", "dtype": "int", "value": int(a)})
        shapes = []
        outs = result if isinstance(result, tuple) else (result,)
        for o in outs:
            if isinstance(o, np.ndarray):
                shapes.append({"shape": list(o.shape), "dtype": str(o.dtype)})
            else:
                shapes.append(None)
        trace_t = outs[2].tolist() if isinstance(result, tuple) and len(outs) >= 3 else None
        (out / f"{name}.cu").write_text(rec["code"])
        np.savez(out / f"{name}_inputs.npz", **arrays)
        meta = {"name": name, "grid": rec["grid"], "block": rec["block"], "args": scalars,
                "api": case["api"], "outputs": shapes, "trace_t": trace_t, "cpu": bool(case.get("cpu"))}
        (out / f"{name}.json").write_text(json.dumps(meta, indent=1))


# ------------------------------------------------------------------ parent: build
_PARAM = re.compile(r"^\s*(const\s+)?([A-Za-z_][\w]*)\s*(\*?)\s*(?:__restrict__\s*)?([A-Za-z_]\w*)\s*$")


def kernel_params(code):
    """(type, is_pointer, name) of every parameter of time_evolution_kernel."""
    start = code.index("time_evolution_kernel(") + len("time_evolution_kernel(")
    depth, end = 1, start
    while depth:
        depth += {"(": 1, ")": -1}.get(code[end], 0)
        end += 1
    body = re.sub(r"//[^\n]*", "", code[start:end - 1])
    params = []
    for part in body.split(","):
        part = " ".join(part.split())
        if not part:
            continue
        m = re.match(r"^(?:const\s+)?(\w+)\s*(\*)?\s*(?:__restrict__\s+)?(\w+)$", part)
        if not m:
            raise ValueError(f"cannot parse kernel parameter '{part}'")
        params.append((m.group(1), bool(m.group(2)), m.group(3)))
    return params


def launcher(meta, code, gpu):
    params = kernel_params(code)
    if len(params) != len(meta["args"]):
        raise ValueError(f"{meta['name']}: {len(params)} kernel parameters, {len(meta['args'])} captured")
    call, nbuf = [], 0
    for (ctype, ptr, _name), arg in zip(params, meta["args"]):
        if ptr:
            call.append(f"({ctype}*)bufs[{nbuf}]")
            nbuf += 1
        elif ctype == "float":
            call.append(f"(float){np.float32(arg['value']).item()!r}")
        elif ctype == "double":
            call.append(f"{float(arg['value'])!r}")
        else:
            call.append(f"({ctype}){int(arg['value'])}")
    gx, gy = meta["grid"][0], meta["grid"][1]
    bx, by = meta["block"][0], meta["block"][1]
    args = ", ".join(call)
    if gpu:
        return (f'#include "{meta["name"]}.cu"\n#include <cuda_runtime.h>\n'
                'extern "C" int ref_launch(void** bufs, void* stream) {\n'
                f"  dim3 grid({gx}, {gy}), block({bx}, {by});\n"
                f"  time_evolution_kernel<<<grid, block, 0, (cudaStream_t)stream>>>({args});\n"
                "  return (int)cudaGetLastError();\n}\n")
    return ('#include "ref_cpu_shim.h"\n'
            f'#include "{meta["name"]}.cu"\n'
            'extern "C" int ref_launch(void** bufs, void* stream) {\n'
            "  (void)stream;\n"
            f"  const long total = (long){gx} * {gy} * {bx} * {by};\n"
            "  #pragma omp parallel for schedule(dynamic, 64)\n"
            "  for (long k = 0; k < total; ++k) {\n"
            f"    long r = k; const unsigned tx = r % {bx}; r /= {bx}; const unsigned ty = r % {by}; r /= {by};\n"
            f"    const unsigned gxi = r % {gx}; r /= {gx}; const unsigned gyi = (unsigned)r;\n"
            f"    blockDim.x = {bx}; blockDim.y = {by}; blockDim.z = 1;\n"
            "    threadIdx.x = tx; threadIdx.y = ty; threadIdx.z = 0;\n"
            "    blockIdx.x = gxi; blockIdx.y = gyi; blockIdx.z = 0;\n"
            f"    time_evolution_kernel({args});\n"
            "  }\n  return 0;\n}\n")


def build_case(name, out):
    meta = json.loads((out / f"{name}.json").read_text())
    code = (out / f"{name}.cu").read_text()
    built = []
    gpu_src = out / f"{name}_gpu_launch.cu"
    gpu_src.write_text(launcher(meta, code, gpu=True))
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-shared", "-Xcompiler", "-fPIC",
           f"-I{out}", str(gpu_src), "-o", str(out / f"{name}_gpu.so")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {name}:\n{r.stderr[-3000:]}")
    built.append(f"{name}_gpu.so")
    cpu_src = out / f"{name}_cpu_launch.cpp"
    cpu_src.write_text(launcher(meta, code, gpu=False))
    cmd = ["g++", "-O2", "-fopenmp", "-ffp-contract=off", "-shared", "-fPIC", "-std=c++17", f"-I{HERE}",
           f"-I{out}", "-w", str(cpu_src), "-o", str(out / f"{name}_cpu.so")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed for {name}:\n{r.stderr[-3000:]}")
    built.append(f"{name}_cpu.so")
    return built


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=os.environ.get("GQIS_REFERENCE_DIR", str(DEFAULT_REFERENCE)))
    ap.add_argument("--cases", default="")
    ap.add_argument("--jobs", type=int, default=max(1, (os.cpu_count() or 2)))
    ap.add_argument("--child", action="store_true")
    ap.add_argument("--out", default=str(OUT))
    a = ap.parse_args(argv)
    out = Path(a.out)
    reference = Path(a.reference)
    sys.path.insert(0, str(HERE))
    if a.child:
        _child(reference, a.cases.split(","), out)
        return 0
    if not (reference / "gqis" / "solver.py").exists():
        print(f"ref_capture: reference tree not found at {reference}; nothing to build")
        return 0
    import ref_cases
    names = a.cases.split(",") if a.cases else list(ref_cases.cases())
    out.mkdir(parents=True, exist_ok=True)
    env = dict(os.environ, PYTHONPATH="")
    subprocess.run([sys.executable, str(Path(__file__).resolve()), "--child", "--reference", str(reference),
                    "--out", str(out), "--cases", ",".join(names)], check=True, env=env)
    with cf.ThreadPoolExecutor(max_workers=a.jobs) as pool:
        for built in pool.map(lambda n: build_case(n, out), names):
            print("built", *built)
    return 0


if __name__ == "__main__":
    sys.exit(main())
