"""Generate the golden fixtures of tests/golden from the reference's own kernels.

Each fixture ``<case>.npz`` holds the output of the reference GQIS kernel for one case of
``oracle/ref_cases.py``: the CUDA source that the reference package generates for that case
(captured by ``oracle/ref_capture.py`` with the recording CuPy stand-in) compiled for the CPU
through ``oracle/ref_cpu_shim.h`` and run over all points in FP64. Long traces are stored with
a sample stride (``trace_stride`` in the file) to keep the fixtures small.

Run in the build container, where the reference tree exists:

    python oracle/ref_capture.py && python tests/golden/make_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))

import ref_cases  # noqa: E402
import ref_kernels  # noqa: E402

TRACE_STRIDE = {"duffing_tsit5a_trace": 4, "duffing_rk4_observable_trace": 5}


def main():
    out_dir = Path(__file__).resolve().parent
    for name, case in ref_cases.cases().items():
        if not case.get("cpu"):
            continue
        if not ref_kernels.available(name, "cpu"):
            raise SystemExit(f"{name}: run oracle/ref_capture.py first")
        out, seconds = ref_kernels.run_case(name, "cpu")
        payload = {"result": out["result"]}
        stride = TRACE_STRIDE.get(name, 1)
        if "trace" in out:
            payload["trace"] = out["trace"][:, :, ::stride]
            payload["trace_t"] = out["trace_t"][::stride]
            payload["trace_stride"] = np.array(stride)
        if "adaptive_steps" in out:
            payload["adaptive_steps"] = out["adaptive_steps"]
        np.savez_compressed(out_dir / f"{name}.npz", **payload)
        print(f"{name}: {seconds:.2f} s", {k: v.shape for k, v in payload.items()})


if __name__ == "__main__":
    main()
