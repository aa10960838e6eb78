"""Model modules: generate the translation unit, build it with nvcc for sm_100a, load it.

This replaces the reference's NVRTC path (``cp.RawKernel(code, "time_evolution_kernel")``,
``gqis/solver.py:2237-2241``). A module is one model variant - emitted model struct, integrator,
precision form, output and trace mode - compiled into a shared library that exports the C ABI
of ``include/gqis_b200.h``. Modules are cached on disk by the hash of their source and of the
CUDA templates, so a later process (or another machine with the same tree) loads them without
compiling. There is no fallback: if nvcc or the GPU is missing the call fails loudly.
"""

from __future__ import annotations

import ctypes
import hashlib
import os
import re
import shutil
import subprocess
import tempfile
import threading
from pathlib import Path

from . import emit
from .cuda_solvers import tableau_source

PACKAGE_DIR = Path(__file__).resolve().parent
CSRC_DIR = PACKAGE_DIR / "csrc"
INCLUDE_DIR = PACKAGE_DIR.parent.parent / "include"
ARCH_FLAGS = ("-gencode", "arch=compute_100a,code=sm_100a")

FORMS = {"fp64": 0, "fp32": 1}
OUTPUT_MODES = {"mean": 0, "final": 1, "final_rho": 2, "mean_state": 3}
TRACE_MODES = {None: 0, "observable": 1, "state": 2}
FORM_TYPES = {"fp64": "FormFP64", "fp32": "FormFP32"}

_LOADED: dict = {}
_LOCK = threading.Lock()


def cache_dir() -> Path:
    """Where built modules live: ``$GQIS_CACHE_DIR``, else ``_build/modules`` in the package."""
    env = os.environ.get("GQIS_CACHE_DIR")
    path = Path(env) if env else PACKAGE_DIR / "_build" / "modules"
    try:
        path.mkdir(parents=True, exist_ok=True)
        probe = path / ".write_probe"
        probe.touch()
        probe.unlink()
    except OSError:
        path = Path.home() / ".cache" / "gqis_b200" / "modules"
        path.mkdir(parents=True, exist_ok=True)
    return path


def nvcc_path() -> str:
    for cand in (os.environ.get("GQIS_NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc was not found: the B200 sweep engine compiles every model with nvcc "
                       "(set GQIS_NVCC or put CUDA's bin directory on PATH).")


_INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)
_DIGESTS: dict = {}


def _header_path(name: str):
    for base in (CSRC_DIR, INCLUDE_DIR):
        if (base / name).exists():
            return base / name
    return None


def templates_digest(source: str) -> str:
    """Hash of the headers ``source`` includes from csrc/ and include/, followed transitively.

    A module's cache key depends only on the templates it is built from, so a change to one
    integrator header leaves modules of the other integrators valid.
    """
    names, todo = set(), _INCLUDE_RE.findall(source)
    while todo:
        name = todo.pop()
        if name in names:
            continue
        names.add(name)
        path = _header_path(name)
        if path is not None:
            todo.extend(_INCLUDE_RE.findall(path.read_text()))
    key = tuple(sorted(names))
    digest = _DIGESTS.get(key)
    if digest is None:
        h = hashlib.sha256()
        for name in key:
            path = _header_path(name)
            h.update(name.encode())
            h.update(path.read_bytes() if path is not None else b"<system>")
        digest = _DIGESTS[key] = h.hexdigest()
    return digest


PACKED_MAX_STATE = 15  # two points' RK4 registers (5 vectors of S each) stay below 255 per thread
_PACKED_UNSUPPORTED = re.compile(r"[?<>!=&|]")  # comparisons / conditionals have no packed form


def packed_pairs(frag, spec, form):
    """Whether a reduced-form module runs two points per thread in packed FP32 arithmetic.

    Classical RK4 in the FP32 form with a small state (measured on the four-level model, S = 15:
    515 vs 562 ms per 2048^2 x 8000 sweep; the FMA pipe is busy 78% instead of 70% because the
    packed instructions free issue slots for the FP64 drive and bookkeeping instructions). The
    emitted RHS and observable must be plain arithmetic (no comparisons or conditionals)."""
    if frag.get("matrix") or form != "fp32" or spec.name != "rk4" or frag["state_size"] > PACKED_MAX_STATE:
        return False
    lines = list(frag["rhs_lines"]) + [frag["obs_re"], frag["obs_im"]]
    return not any(_PACKED_UNSUPPORTED.search(ln.split("=", 1)[1] if "=" in ln else ln) for ln in lines)


def module_source(frag, spec, form, output_mode, trace_mode, unroll=False, extra_code="", defines=None):
    """Complete translation unit of one model variant (``extra_code`` goes into ``gqmodel``)."""
    model = emit.model_source(frag)
    model_hash = int(hashlib.sha256(model.encode()).hexdigest()[:16], 16)
    lines = [
        "// Model module generated by gqis (B200 sweep engine). Do not edit.",
        '#include "gqis_common.cuh"',
        "namespace gqmodel {",
        model,
        tableau_source(spec),
        extra_code,
        "}  // namespace gqmodel",
        "#define GQ_MODEL gqmodel::Model",
        f"#define GQ_FORM {FORM_TYPES[form]}",
        f"#define GQ_SOLVER {spec.template}",
        f"#define GQ_SOLVER_ID {spec.solver_id}",
        f"#define GQ_ADAPTIVE {1 if spec.adaptive else 0}",
        f"#define GQ_OUT {OUTPUT_MODES[output_mode]}",
        f"#define GQ_TRACE {TRACE_MODES[trace_mode]}",
        f"#define GQ_MODEL_HASH 0x{model_hash:016x}ULL",
        *[f"#define {k} {v}" for k, v in (defines or {}).items()],
        *([] if not packed_pairs(frag, spec, form) else
          ["#ifndef GQ_PACK2", "#define GQ_PACK2 1  // two points per thread, packed FP32", "#endif"]),
        '#include "gqis_module.cuh"',
        "",
    ]
    return "\n".join(lines)


class ModelModule:
    """A loaded model module (ctypes handle of its shared library)."""

    def __init__(self, path: Path):
        from . import abi
        self.path = Path(path)
        self.lib = ctypes.CDLL(str(self.path))
        abi.bind_module(self.lib)
        self._info = None

    def info(self):
        """The module's ``gqis_model_info`` (state size, solver, output mode, launch shape), read once."""
        from . import abi
        if self._info is None:
            info = abi.ModelInfo()
            rc = self.lib.gqis_model_info_get(ctypes.byref(info))
            abi.check(rc, self.lib)
            self._info = info
        return self._info

    def launch(self, desc, stream_handle):
        """``gqis_sweep_launch`` of a filled descriptor on a CUDA stream handle; raises on a non-OK
        status with the module's error text."""
        from . import abi
        rc = self.lib.gqis_sweep_launch(ctypes.byref(desc), ctypes.c_void_p(stream_handle))
        abi.check(rc, self.lib)


def include_dirs_digest(flags) -> str:
    """Hash of the header files in the ``-I`` directories of ``flags`` (a caller's own template
    directory, ``kernel_template_file``): a module built from edited headers gets a new cache key."""
    h = hashlib.sha256()
    for flag in flags:
        if not flag.startswith("-I"):
            continue
        root = Path(flag[2:])
        if not root.is_dir():
            continue
        for path in sorted(root.iterdir()):
            if path.is_file() and path.suffix in (".cuh", ".h", ".hpp", ".hh", ".inc", ".cu"):
                h.update(path.name.encode() + b"\0")
                h.update(path.read_bytes())
    return h.hexdigest()


def build_module(source: str, *, extra_flags=(), quiet=True) -> Path:
    """Compile ``source`` into a cached shared library; returns its path."""
    flags = tuple(extra_flags)
    key = hashlib.sha256((source + "\0" + templates_digest(source) + "\0" + " ".join(flags) + "\0" +
                          include_dirs_digest(flags)).encode()).hexdigest()[:24]
    out_dir = cache_dir()
    so_path = out_dir / f"gqis_model_{key}.so"
    if so_path.exists():
        return so_path
    nvcc = nvcc_path()
    with tempfile.TemporaryDirectory(prefix="gqis_build_", dir=out_dir) as tmp:
        cu = Path(tmp) / f"gqis_model_{key}.cu"
        cu.write_text(source)
        tmp_so = Path(tmp) / so_path.name
        # a caller's include directories (kernel_template_file) are searched before the packaged ones
        includes = [f for f in flags if f.startswith("-I")]
        others = [f for f in flags if not f.startswith("-I")]
        cmd = [nvcc, *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", "-Xptxas", "-v", "--expt-relaxed-constexpr",
               *includes, f"-I{CSRC_DIR}", f"-I{INCLUDE_DIR}", *others, str(cu), "-o", str(tmp_so)]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed for a model module ({cu.name}):\n{proc.stderr[-6000:]}")
        (out_dir / f"gqis_model_{key}.cu").write_text(source)
        (out_dir / f"gqis_model_{key}.ptxas.txt").write_text(proc.stderr)
        os.replace(tmp_so, so_path)  # atomic: concurrent builders of the same key agree
    return so_path


def load_module(source: str, *, extra_flags=()) -> ModelModule:
    """Build (or find) and load the module of ``source``; loaded modules are kept per process."""
    path = build_module(source, extra_flags=extra_flags)
    with _LOCK:
        mod = _LOADED.get(str(path))
        if mod is None:
            mod = ModelModule(path)
            _LOADED[str(path)] = mod
    return mod
