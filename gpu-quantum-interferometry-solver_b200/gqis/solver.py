"""``mesolve_2D`` and the shared sweep engine (drop-in for ``gqis/solver.py`` of GQIS).

Call path of one sweep (reference ``gqis/solver.py:1712-2391``):

1. validate the call (uniform ``tlist`` from zero, warmup, trace stride/offset);
2. prepare and optimise the RHS (``rhs.compile_rhs``, cached);
3. emit the model struct (``emit.emit_model``) and build the model module for the chosen
   integrator, precision form, output and trace mode (``engine``, cached in memory and on disk);
4. upload sweep axes, constants and initial states into torch CUDA tensors, launch through the
   C ABI on the current torch stream, time the launch with CUDA events;
5. check the outputs for non-finite values and return NumPy arrays (or CUDA tensors with
   ``return_device=True``).

``calibrate_timesteps`` wraps the call in the step-size search of ``gqis/solver.py:928-1341``.
The precision form is chosen by ``precision`` (``"fp64"`` or ``"fp32"``); by default it follows
``fp64``. The FP32 form keeps time, drive phase and the running averages in FP64.
"""

from __future__ import annotations

import os
import sys
import time
from contextlib import contextmanager
from dataclasses import dataclass, field

import numpy as np

from ._options import OPTION_GROUPS, apply_option_groups
from .cuda_solvers import counts_steps, get_solver_spec
from .lindblad import build_independent_rho, build_reduced_lindblad_rhs, rho_matrix_to_independent_exprs
from .rhs import _RHS_CODE_CACHE, CompiledRHS, compile_rhs as _compile_rhs_impl, runtime_const_values
from . import calibration, emit

__all__ = ["mesolve_2D", "compile_lindblad_rhs", "CompiledRHS", "build_independent_rho",
           "build_reduced_lindblad_rhs", "rho_matrix_to_independent_exprs"]

_KERNEL_CACHE: dict = {}
_TIMESTEP_CALIBRATION_CACHE: dict = {}

TIMESTEP_CALIBRATION_DEFAULTS = calibration.DEFAULTS
TIMESTEP_CALIBRATION_ODE_DEFAULTS = calibration.ODE_DEFAULTS

PRECISIONS = ("fp64", "fp32")
MATRIX_FORM_FROM = 8  # rhs_form="auto" switches to the density-matrix kernels from this dimension
# (measured at N = 8, 4096 points x 2000 RK4 steps: FP64 51 ms vs 110 ms for the reduced form; FP32 on
# the tensor cores 11 ms vs 65 ms; the reduced form stays faster at N = 4)


@contextmanager
def _nvtx(name):
    """An NVTX range around a stage of a call (seen by Nsight Systems and Nsight Compute), when torch
    has a CUDA device; otherwise nothing."""
    try:
        import torch
        on = torch.cuda.is_available()
    except ImportError:
        on = False
    if on:
        torch.cuda.nvtx.range_push(name)
    try:
        yield
    finally:
        if on:
            torch.cuda.nvtx.range_pop()


def _compile_rhs(*args, **kwargs):
    """Indirection so tests can count symbolic preparations."""
    with _nvtx("gqis.compile_rhs"):
        return _compile_rhs_impl(*args, **kwargs)


def compile_lindblad_rhs(H, Drive, Col_Ops, mean_operator, sweep_symbols, *, const_values=None,
                         runtime_consts=None, keep_symbolic_consts=None, auto_runtime_consts=False,
                         rho0=None, pre_expand=True, collect_rho=False, factor_terms=False,
                         cse_batch_size=None, cse_simplify=False, hoist_rho_independent=True,
                         RHSreuse=True, symbolic_workers="auto", max_symbolic_workers=None):
    """Prepare and optimise a Lindblad RHS without device code (``gqis/solver.py:1592-1627``).

    ``mesolve_2D(compiled, tlist=..., var_arrays=...)`` then starts from code emission.
    """
    sweep_symbols = tuple(sweep_symbols)
    if not 1 <= len(sweep_symbols) <= 2:
        raise ValueError("sweep_symbols must contain one or two symbols.")
    compiled, _ = _compile_rhs(
        H, Drive, Col_Ops, mean_operator, sweep_symbols=sweep_symbols, const_values=const_values,
        runtime_consts=runtime_consts, keep_symbolic_consts=keep_symbolic_consts,
        auto_runtime_consts=auto_runtime_consts, rho0=rho0, pre_expand=pre_expand,
        collect_rho=collect_rho, factor_terms=factor_terms, cse_batch_size=cse_batch_size,
        cse_simplify=cse_simplify, hoist_rho_independent=hoist_rho_independent, reuse=RHSreuse,
        symbolic_workers=symbolic_workers, max_symbolic_workers=max_symbolic_workers)
    return compiled


# ----------------------------------------------------------------------------------------
# device seam
# ----------------------------------------------------------------------------------------

@dataclass
class SweepLaunch:
    """Everything one kernel launch needs; ``_device_run`` is the only code touching the GPU."""

    entry: dict                 # kernel-cache entry: source text, loaded module
    form: str
    output_mode: str
    trace_mode: object
    state_size: int
    par_x: object
    par_y: object
    consts: list
    rho0: object
    num_steps: int
    warmup_steps: int
    dt: float
    t_in: float
    trace_stride: int = 1
    trace_offset: int = 0
    num_trace: int = 0
    solver_params: tuple = ()
    adaptive: bool = False
    count_steps: bool = False
    return_device: bool = False
    collect_timing: bool = False
    extra: dict = field(default_factory=dict)


def _load_kernel(entry):
    """Build (nvcc, disk-cached) and load the module of a kernel-cache entry."""
    if entry.get("module") is None:
        from . import engine
        with _nvtx("gqis.build_module"):
            entry["module"] = engine.load_module(entry["source"], extra_flags=entry.get("flags", ()))
    return entry["module"]


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("The B200 sweep engine needs a CUDA device; none is visible "
                           "(there is no CPU fallback).")
    return torch


def _as_device(torch, values, dtype, device):
    if isinstance(values, torch.Tensor):
        return values.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(np.asarray(values)), dtype=dtype).to(device)


def _device_buffers(launch: SweepLaunch, point_begin=0, point_count=None):
    """Upload inputs and allocate outputs on the current device; returns ``(desc, tensors)``."""
    from . import abi
    torch = _torch()
    device = torch.device("cuda", torch.cuda.current_device())
    real = torch.float64 if launch.form == "fp64" else torch.float32
    px = _as_device(torch, launch.par_x, torch.float64, device)
    py = _as_device(torch, launch.par_y, torch.float64, device)
    total = int(px.numel()) * int(py.numel())
    npts = total - point_begin if point_count is None else int(point_count)
    consts = (torch.tensor(launch.consts, dtype=torch.float64, device=device) if launch.consts else None)
    rho0 = None
    if launch.rho0 is not None:
        rho0 = _as_device(torch, launch.rho0, real, device).reshape(total, launch.state_size)
        rho0 = rho0[point_begin:point_begin + npts].contiguous()
    width = 2 if launch.output_mode in ("mean", "final") else launch.state_size
    results = torch.empty((npts, width), dtype=real, device=device)
    trace = None
    if launch.trace_mode is not None:
        tw = 2 if launch.trace_mode == "observable" else launch.state_size
        trace = torch.zeros((npts, launch.num_trace, tw), dtype=real, device=device)
    counts = torch.zeros((npts, 2), dtype=torch.int32, device=device) if launch.count_steps else None
    counter = torch.zeros(1, dtype=torch.int32, device=device) if launch.adaptive else None

    desc = abi.SweepDesc()
    desc.abi_version = abi.ABI_VERSION
    desc.num_x, desc.num_y = int(px.numel()), int(py.numel())
    desc.num_steps, desc.warmup_steps = int(launch.num_steps), int(launch.warmup_steps)
    desc.trace_stride, desc.trace_offset = int(launch.trace_stride), int(launch.trace_offset)
    desc.num_trace = int(launch.num_trace)
    desc.point_begin, desc.point_count = int(point_begin), npts
    desc.dt, desc.t_in = float(launch.dt), float(launch.t_in)
    desc.par_x, desc.par_y = px.data_ptr(), py.data_ptr()
    desc.consts = consts.data_ptr() if consts is not None else None
    desc.rho0 = rho0.data_ptr() if rho0 is not None else None
    desc.results = results.data_ptr()
    desc.trace = trace.data_ptr() if trace is not None else None
    desc.step_counts = counts.data_ptr() if counts is not None else None
    desc.work_counter = counter.data_ptr() if counter is not None else None
    for k, v in enumerate(launch.solver_params[:8]):
        desc.solver_params[k] = float(v)
    tensors = {"par_x": px, "par_y": py, "consts": consts, "rho0": rho0, "results": results,
               "trace": trace, "step_counts": counts, "work_counter": counter}
    return desc, tensors


def _device_run_many(launches):
    """Run several sweeps and wait for all of them; returns ``[(results, trace, step_counts, 0.0), ...]``.

    Used by the batched calibration search, whose candidate resolutions are small launches of one
    module whose results are only needed together: sweeps of the same module go out as one
    ``gqis_sweep_launch_batch`` grid (up to ``abi.BATCH_MAX`` per grid, one shared work counter for
    the adaptive kernels). The density-matrix modules, which have no batch launch, get one launch
    each on its own stream.
    """
    from . import abi
    torch = _torch()
    current = torch.cuda.current_stream()
    prepared = [(launch, _load_kernel(launch.entry), *_device_buffers(launch)) for launch in launches]
    groups = {}
    for k, (launch, module, desc, buf) in enumerate(prepared):
        groups.setdefault(str(module.path), []).append(k)
    for members in groups.values():
        module = prepared[members[0]][1]
        if prepared[members[0]][0].entry["frag"].get("matrix"):
            for k in members:
                stream = torch.cuda.Stream()
                stream.wait_stream(current)  # inputs were uploaded on the current stream
                module.launch(prepared[k][2], stream.cuda_stream)
            continue
        for start in range(0, len(members), abi.BATCH_MAX):
            part = members[start:start + abi.BATCH_MAX]
            descs = (abi.SweepDesc * len(part))(*[prepared[k][2] for k in part])
            counter = torch.zeros(1, dtype=torch.int32, device=current.device)
            rc = module.lib.gqis_sweep_launch_batch(descs, len(part), counter.data_ptr(), current.cuda_stream)
            abi.check(rc, module.lib)
            prepared[part[0]][3]["batch_counter"] = counter  # kept alive until the sync below
    torch.cuda.synchronize()
    return [(buf["results"], buf["trace"], buf["step_counts"], 0.0) for _, _, _, buf in prepared]


def _with_steps(launch, steps, duration, warmup_time):
    """The fixed-step launch ``launch`` with ``steps`` uniform steps over ``duration``."""
    import dataclasses
    warmup_time = float(warmup_time or 0.0)
    warm = steps if warmup_time >= 1.0 else int(np.floor(warmup_time * steps))
    return dataclasses.replace(launch, num_steps=int(steps), dt=float(duration) / steps,
                               warmup_steps=max(0, min(int(steps), warm)))


def _calibration_map(launch, results):
    """Device results of one calibration launch as the map ``mesolve_2D`` would return."""
    res = results.cpu().numpy() if hasattr(results, "cpu") else np.asarray(results)
    nx, ny = len(launch.par_x), len(launch.par_y)
    if launch.output_mode in ("mean", "final"):
        out = (res[:, 0] + 1j * res[:, 1]).reshape(nx, ny)
        return out.astype(np.complex128 if launch.form == "fp64" else np.complex64, copy=False)
    return res.reshape(nx, ny, launch.state_size)


def _device_run(launch: SweepLaunch):
    """Build/load the module, upload inputs, launch and return output tensors on the device.

    Returns ``(results, trace, step_counts, gpu_seconds)``; ``results`` has shape (P, 2) or
    (P, S), ``trace`` (P, num_trace, 2 or S), ``step_counts`` (P, 2) int32 or None.
    """
    torch = _torch()
    module = _load_kernel(launch.entry)
    desc, buf = _device_buffers(launch)
    stream = torch.cuda.current_stream()
    gpu_s = 0.0
    if launch.collect_timing:
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
    module.launch(desc, stream.cuda_stream)
    if launch.collect_timing:
        stop.record(stream)
        stop.synchronize()
        gpu_s = start.elapsed_time(stop) / 1000.0
    return buf["results"], buf["trace"], buf["step_counts"], gpu_s


class PreparedSweep:
    """A sweep set up once and launched many times on device-resident buffers.

    ``prepare_sweep("mesolve_2D", *args, **kwargs)`` runs the front end and module build of the
    call, uploads its inputs and allocates its outputs; ``launch()`` then only enqueues the kernel
    on the current stream (used by bench.py, the serving loop and the parity tests).
    ``point_begin`` / ``point_count`` restrict it to a slice of the flattened grid (sharding).
    """

    def __init__(self, launch: SweepLaunch, point_begin=0, point_count=None):
        self.launch_spec = launch
        self.module = _load_kernel(launch.entry)
        self.desc, self.tensors = _device_buffers(launch, point_begin, point_count)
        self.points = int(self.desc.point_count)
        self.steps = int(launch.num_steps)
        frag = launch.entry["frag"]
        self.state_size = frag["state_size"]
        self.matrix = bool(frag.get("matrix"))
        self.rhs_flops = None if self.matrix else emit.count_rhs_flops(frag)
        self.drive_flops = None if self.matrix else emit.count_drive_flops(frag)
        self.solver = launch.entry["spec"].name

    @property
    def results(self):
        return self.tensors["results"]

    def reset(self):
        if self.tensors["work_counter"] is not None:
            self.tensors["work_counter"].zero_()

    def launch(self, stream=None):
        import torch
        self.reset()
        st = stream if stream is not None else torch.cuda.current_stream()
        self.module.launch(self.desc, st.cuda_stream)

    def flops_per_point_step(self):
        """Algorithmic flops per point and RK4 step: 4 RHS + stage updates + 2 drive sets + <O>."""
        if self.matrix:
            return self.launch_spec.entry["frag"]["flops_per_point_step"]
        S = self.state_size
        return 4 * self.rhs_flops + 13 * S + 2 * self.drive_flops + 4


def prepare_sweep(api, *args, point_begin=0, point_count=None, **kwargs):
    """Set up a sweep for repeated device-resident launches (see :class:`PreparedSweep`)."""
    holder = {}
    kwargs["_prepare_only"] = holder
    if api in ("odesolve_2D", "odesolve"):
        from .gqis_ode_api import odesolve_2D
        odesolve_2D(*args, **kwargs)
    else:
        mesolve_2D(*args, **kwargs)
    return PreparedSweep(holder["launch"], point_begin, point_count)


def _to_output(tensor, return_device):
    if tensor is None:
        return None
    if return_device:
        return tensor
    with _nvtx("gqis.copy_out"):
        return tensor.cpu().numpy()


def _all_finite(x):
    if hasattr(x, "isfinite") and not isinstance(x, np.ndarray):
        import torch
        return bool(torch.isfinite(x).all())
    return bool(np.all(np.isfinite(x)))


def _beep():
    print("\a", end="", flush=True)


def _save_kernel(path_or_flag, source):
    if not path_or_flag:
        return None
    if isinstance(path_or_flag, str) and path_or_flag.strip():
        path = os.path.abspath(path_or_flag)
    else:
        main = getattr(sys.modules.get("__main__"), "__file__", None)
        path = (os.path.join(os.path.dirname(os.path.abspath(main)),
                             os.path.splitext(os.path.basename(main))[0] + "_Kernel.cu")
                if main else os.path.abspath("Generated_Kernel.cu"))
    with open(path, "w", encoding="utf-8", newline="\n") as f:
        f.write(source)
    return path


def _print_timings(api_name, info, mode):
    ode = {"miss": "new ODE", "hit": "reused ODE", "provided": "compiled ODE"}[info["cached_rhs"]]
    kernel = "new kernel" if info["cached_kernel"] == "miss" else "reused kernel"
    prep, gpu, total = info["rhs_stage_s"], info["gpu_kernel_s"], info["total_s"]

    def show(s):
        return f"{s * 1e3:.1f} ms" if s < 1.0 else f"{s:.2f} s"

    if mode != "full":
        print(f"{api_name}: preparation {show(prep)} ({ode}, {kernel}), GPU {show(gpu)}, total {show(total)}")
        return
    stages = [("symbolic ODE", info["ode_prepare_s"]), ("optimization", info["ode_optimize_s"]),
              ("CUDA code", info["code_emit_s"]), ("kernel build", info["kernel_build_s"])]
    stages.append(("setup", max(0.0, prep - sum(s for _, s in stages))))
    print(f"{api_name} timings ({info['solver']}, {info['precision']}):")
    print(f"  {'preparation':<16}{show(prep):>10}   {ode}, {kernel}")
    for name, s in stages:
        print(f"    {name:<14}{show(s):>10}")
    print(f"  {'GPU calculation':<16}{show(gpu):>10}")
    print(f"  {'other':<16}{show(max(0.0, total - prep - gpu)):>10}   transfer and checks")
    print(f"  {'total':<16}{show(total):>10}")


# ----------------------------------------------------------------------------------------
# public entry point
# ----------------------------------------------------------------------------------------

def prebuild(api, *args, source_only=False, **kwargs):
    """Compile the model module a ``mesolve_2D`` / ``odesolve_2D`` call would use, without a GPU.

    Returns the path of the cached shared library, so a later process (or the same tree on
    another machine) loads it without running nvcc; ``source_only=True`` returns
    ``(source, nvcc_flags)`` instead, for parallel builds.
    """
    mode = "source" if source_only else True
    kwargs.pop("calibrate_timesteps", None)
    if api in ("odesolve_2D", "odesolve"):
        from .gqis_ode_api import odesolve_2D
        return odesolve_2D(*args, _prebuild_only=mode, **kwargs)
    return mesolve_2D(*args, _prebuild_only=mode, **kwargs)


def mesolve_2D(H, Drive=None, Col_Ops=None, mean_operator=None, tlist=None,
               var_arrays=None, const_values=None, kernel_template_file=None, *,
               RHSreuse=True, runtime_consts=None, keep_symbolic_consts=None,
               auto_runtime_consts=False, output_mode="mean", solver="rk4",
               solver_frequency=None, adaptive_options=None, unroll=False, fp64=False,
               precision=None, pre_expand=True, collect_rho=False, factor_terms=False,
               cse_batch_size=None, cse_simplify=False, hoist_rho_independent=True,
               symbolic_workers="auto", max_symbolic_workers=None,
               nvrtc_options=(), timings=False, return_timing_info=False, warmup_time=0.0,
               rho0=None, rho0_var_arrays=None, rho0_values=None,
               return_time_trace=False, time_trace_every=None,
               time_trace_samples_per_period=None, solver_samples_per_period=None,
               Actual_Kernel_Save=False, beep_on_error=False, ignore_non_finite_output=False,
               t_in=0.0, return_device=False, calibrate_timesteps=None, consts=None, initial=None,
               output=None, solver_options=None, codegen=None, diagnostics=None, rhs_form="auto",
               _prebuild_only=False, _prepare_only=None):
    args = dict(locals())
    groups = {name: args.pop(name) for name in OPTION_GROUPS}
    args, _ = apply_option_groups(mesolve_2D, args, groups)
    if args["output_mode"] not in {"mean", "final", "final_rho"}:
        raise ValueError("output_mode must be 'mean', 'final', or 'final_rho'.")
    if isinstance(H, CompiledRHS):
        if H.kind != "lindblad":
            raise ValueError("This CompiledRHS comes from compile_ode_rhs; pass it to odesolve_2D.")
        args.update(H=None, compiled_rhs=H)
    return _solve_symbolic_system(**args)


def _resolve_precision(precision, fp64):
    if precision is None:
        return "fp64" if fp64 else "fp32"
    p = str(precision).lower()
    if p not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS} or None.")
    return p


def _check_sweep_arrays_nonempty(var_arrays):
    """Reject a sweep array without values: its grid has zero points, which the launch rejects
    (the module's descriptor check), so say so before any derivation or compile."""
    for sym, arr in (var_arrays or {}).items():
        if (arr.numel() if hasattr(arr, "numel") else np.size(arr)) == 0:
            raise ValueError(f"The sweep array of {sym} is empty; every sweep array needs at least one value.")


def _solve_symbolic_system(H, Drive, Col_Ops, mean_operator, tlist,
                           var_arrays=None, const_values=None, kernel_template_file=None, *,
                           RHSreuse=True, runtime_consts=None, keep_symbolic_consts=None,
                           auto_runtime_consts=False, output_mode="mean", solver="rk4",
                           solver_frequency=None, adaptive_options=None, unroll=False,
                           fp64=False, precision=None,
                           pre_expand=True, collect_rho=False, factor_terms=False,
                           cse_batch_size=None, cse_simplify=False, hoist_rho_independent=True,
                           symbolic_workers="auto", max_symbolic_workers=None,
                           nvrtc_options=(), timings=False, return_timing_info=False, warmup_time=0.0,
                           rho0=None, rho0_var_arrays=None, rho0_values=None,
                           return_time_trace=False, time_trace_every=None,
                           time_trace_samples_per_period=None, solver_samples_per_period=None,
                           Actual_Kernel_Save=False, beep_on_error=False, ignore_non_finite_output=False,
                           t_in=0.0, return_device=False, calibrate_timesteps=None, compiled_rhs=None,
                           _ode_size=None, _state_trace=False, _time_trace_offset=0, _prebuild_only=False,
                           _prepare_only=None, rhs_form="auto"):
    """Solve a Lindblad master equation (or, through ``odesolve_2D``, a real ODE) on a 1-D or 2-D
    parameter sweep, one independent time integration per point on the GPU.

    Arguments, defaults and return shapes are those of the reference ``mesolve_2D``
    (``gqis/solver.py:1739-1900``):

    * result ``(num_X, num_Y)`` complex for ``"mean"`` / ``"final"``; ``(num_X, num_Y, N*N-1)``
      real for ``"final_rho"`` (and ``"mean_state"`` from ``odesolve_2D``);
    * with ``return_time_trace`` the tuple ``(result, trace, trace_t)``; with
      ``return_timing_info`` the timing dict is appended;
    * ``return_device=True`` returns torch CUDA tensors instead of NumPy arrays.

    Additions of this engine: ``precision`` (``"fp64"`` or ``"fp32"``; default from ``fp64``),
    the adaptive ``"dop853a"`` solver, ``kernel_template_file``, which here names an extra
    include directory (or a file in it) searched before the packaged CUDA templates, and
    ``rhs_form``: ``"reduced"`` (the reference's N*N-1 real equations), ``"matrix"`` (the
    density-matrix kernel of ``matrix_form`` on the CUDA cores; fixed-step RK4, outputs
    ``mean``/``final``/``final_rho`` and the observable time trace), ``"matrix_tc"`` (the same on the tensor
    cores, split-FP16 operands with FP32 accumulation; FP32 form, padded N of 8, 16, 32 or 64) or
    ``"auto"`` (matrix from N = 8 on where it applies, on the tensor cores for FP32 sweeps the
    tensor-core kernel can run).
    """
    if (calibrate_timesteps is not None and calibrate_timesteps is not False and not _prebuild_only
            and _prepare_only is None):
        return _solve_with_timestep_calibration(dict(locals()))
    valid_modes = {"mean", "final", "final_rho", "mean_state"}
    if output_mode not in valid_modes:
        raise ValueError(f"Unsupported output_mode '{output_mode}'. Use one of: {sorted(valid_modes)}")
    if not isinstance(unroll, (bool, np.bool_)):
        raise ValueError("unroll must be True or False.")
    unroll = bool(unroll)
    template_dir = None
    if kernel_template_file is not None:
        if not os.path.exists(kernel_template_file):
            raise FileNotFoundError(f"CUDA kernel template was not found: {kernel_template_file}")
        template_dir = (os.path.abspath(kernel_template_file) if os.path.isdir(kernel_template_file)
                        else os.path.dirname(os.path.abspath(kernel_template_file)))
    form = _resolve_precision(precision, fp64)
    t_in = float(t_in)
    if not np.isfinite(t_in):
        raise ValueError("t_in must be finite.")

    var_arrays = {} if var_arrays is None else dict(var_arrays)
    for sym, arr in (rho0_var_arrays or {}).items():
        if sym in var_arrays:
            raise ValueError(f"Symbol {sym} is present in both var_arrays and rho0_var_arrays.")
        var_arrays[sym] = arr
    const_values = {} if const_values is None else const_values
    if rho0 is not None and rho0_values is not None:
        raise ValueError("Use either rho0 or rho0_values, not both.")
    uses_rho0_values = rho0_values is not None
    if not var_arrays:
        raise ValueError("var_arrays or rho0_var_arrays must contain at least one sweep array (ParX).")
    if len(var_arrays) > 2:
        raise ValueError("Only 2 total sweep arrays are supported across var_arrays and rho0_var_arrays.")
    _check_sweep_arrays_nonempty(var_arrays)
    if compiled_rhs is None:
        if H is None or Drive is None or Col_Ops is None or mean_operator is None:
            raise TypeError("Give H, Drive, Col_Ops and mean_operator, or a CompiledRHS.")
    else:
        if any(x is not None for x in (H, Drive, Col_Ops, mean_operator)):
            raise ValueError("With a CompiledRHS, do not pass the model (H, Drive, Col_Ops, "
                             "mean_operator) again.")
        if const_values or keep_symbolic_consts is not None or auto_runtime_consts or rho0 is not None:
            raise ValueError("const_values, keep_symbolic_consts, auto_runtime_consts and rho0 are "
                             "fixed when the RHS is compiled; give values of constants kept "
                             "symbolic through runtime_consts.")
        if tuple(var_arrays) != compiled_rhs.sweep_symbols:
            raise ValueError(f"The sweep arrays must be for {compiled_rhs.sweep_symbols}, in the "
                             "order given when the RHS was compiled.")

    # ---- time grid (gqis/solver.py:1951-2010)
    if tlist is None:
        raise ValueError("tlist is required for fixed-step integration.")
    n_t = int(len(tlist))
    if n_t < 2:
        raise ValueError("tlist must contain at least two time samples.")
    t_raw = np.asarray(tlist.cpu() if hasattr(tlist, "cpu") else tlist)
    t_host = np.asarray(t_raw, dtype=np.float64)
    if t_host.ndim != 1 or not np.all(np.isfinite(t_host)):
        raise ValueError("tlist must be a finite one-dimensional array.")
    diffs = np.diff(t_host)
    if np.any(diffs <= 0.0):
        raise ValueError("tlist must be strictly increasing.")
    in_dtype = t_raw.dtype if np.issubdtype(t_raw.dtype, np.floating) else np.dtype(np.float64)
    tol = 8.0 * np.finfo(in_dtype).eps * max(1.0, float(np.max(np.abs(t_host))))
    dt_host = float((t_host[-1] - t_host[0]) / (n_t - 1))
    spec = get_solver_spec(solver, frequency=solver_frequency, step_size=dt_host,
                           adaptive_options=adaptive_options, fp64=form == "fp64")
    if not np.isclose(t_host[0], 0.0, rtol=0.0, atol=tol):
        raise ValueError("tlist must begin at zero; the CUDA kernel derives stage times from the step index.")
    if not np.allclose(diffs, dt_host, rtol=1.0e-6, atol=tol):
        raise ValueError("tlist must be uniformly spaced because the GPU solver uses one fixed dt.")
    num_steps = n_t - 1
    warmup_time = float(warmup_time)
    if warmup_time < 0.0 or warmup_time > 1.0:
        raise ValueError("warmup_time must be within [0, 1].")
    warmup_steps = num_steps if warmup_time >= 1.0 else int(np.floor(warmup_time * num_steps))
    warmup_steps = max(0, min(num_steps, warmup_steps))
    return_time_trace = bool(return_time_trace)
    if time_trace_every is not None and time_trace_samples_per_period is not None:
        raise ValueError("Use either time_trace_every or time_trace_samples_per_period, not both.")
    if time_trace_samples_per_period is not None:
        if solver_samples_per_period is None:
            raise ValueError("solver_samples_per_period is required when "
                             "time_trace_samples_per_period is used.")
        sspp, tspp = int(solver_samples_per_period), int(time_trace_samples_per_period)
        if sspp <= 0 or tspp <= 0:
            raise ValueError("solver_samples_per_period and time_trace_samples_per_period must be positive.")
        stride = max(1, int(round(sspp / tspp)))
    elif time_trace_every is not None:
        stride = int(time_trace_every)
        if stride <= 0:
            raise ValueError("time_trace_every must be a positive integer.")
    else:
        stride = 1
    offset = int(_time_trace_offset)
    num_trace = int(np.ceil((num_steps - offset) / stride)) if return_time_trace else 0

    mode = output_mode
    if output_mode == "mean" and warmup_steps >= num_steps:
        mode = "final"
    if output_mode == "mean_state" and warmup_steps >= num_steps:
        mode = "final_rho"

    if timings not in (False, None, True, "compact", "full"):
        raise ValueError("timings must be False, True, 'compact' or 'full'.")
    collect = bool(timings or return_timing_info)
    t_total = time.time()

    if rhs_form not in ("auto", "reduced", "matrix", "matrix_tc"):
        raise ValueError("rhs_form must be 'auto', 'reduced', 'matrix' or 'matrix_tc'.")
    matrix_ok = (compiled_rhs is None and _ode_size is None and spec.name == "rk4" and not _state_trace
                 and mode in ("mean", "final", "final_rho"))
    if rhs_form in ("matrix", "matrix_tc") and not matrix_ok:
        raise ValueError(f"rhs_form='{rhs_form}' needs a Lindblad model given symbolically, solver='rk4' "
                         "and output_mode 'mean', 'final' or 'final_rho'.")
    use_matrix = rhs_form in ("matrix", "matrix_tc") or (rhs_form == "auto" and matrix_ok and H is not None
                                                         and H.shape[0] >= MATRIX_FORM_FROM)
    tensor_cores = rhs_form == "matrix_tc"

    # ---- 1) symbolic preparation
    if use_matrix:
        from . import matrix_form
        with _nvtx("gqis.compile_matrix_model"):
            compiled, rhs_status = matrix_form.compile_matrix_model(
                H, Drive, Col_Ops, mean_operator, sweep_symbols=tuple(var_arrays), const_values=const_values,
                runtime_consts=runtime_consts, keep_symbolic_consts=keep_symbolic_consts,
                auto_runtime_consts=auto_runtime_consts, rho0=rho0, reuse=RHSreuse,
                tensor_cores=form == "fp32" and rhs_form in ("auto", "matrix_tc"))
        if rhs_form == "auto" and not matrix_form.tensor_core_blockers(compiled, form):
            tensor_cores = True  # FP32 sweeps from N = 8 run on the tensor cores
    elif compiled_rhs is None:
        compiled, rhs_status = _compile_rhs(
            H, Drive, Col_Ops, mean_operator, sweep_symbols=tuple(var_arrays), const_values=const_values,
            runtime_consts=runtime_consts, keep_symbolic_consts=keep_symbolic_consts,
            auto_runtime_consts=auto_runtime_consts, rho0=rho0, ode_size=_ode_size,
            pre_expand=pre_expand, collect_rho=collect_rho, factor_terms=factor_terms,
            cse_batch_size=cse_batch_size, cse_simplify=cse_simplify,
            hoist_rho_independent=hoist_rho_independent, reuse=RHSreuse,
            symbolic_workers=symbolic_workers, max_symbolic_workers=max_symbolic_workers)
    else:
        compiled, rhs_status = compiled_rhs, "provided"
    if use_matrix:
        stages = {"ode_prepare_s": time.time() - t_total, "ode_optimize_s": 0.0}
    else:
        stages = (dict(compiled.timings) if rhs_status == "miss" else {"ode_prepare_s": 0.0, "ode_optimize_s": 0.0})
    const_vals = runtime_const_values(compiled, runtime_consts, const_values,
                                      use_defaults=compiled_rhs is not None)

    # ---- 2) model emission
    t0 = time.time()
    ekey = ("b200", bool(uses_rho0_values))
    if use_matrix:
        frag = {"matrix": True, "state_size": compiled.state_size,
                "used_const_indices": tuple(range(len(const_vals))),
                "flops_per_point_step": matrix_form.flops_per_point_step(compiled), "dimension": compiled.Np,
                "tensor_cores": tensor_cores,
                "tensor_flops_per_point_step": matrix_form.tensor_flops_per_point_step(compiled),
                "algorithmic_flops_per_point_step": matrix_form.algorithmic_flops_per_point_step(compiled)}
        stages["emit_s"] = 0.0
    elif RHSreuse and ekey in compiled.emitted:
        frag, stages["emit_s"] = compiled.emitted[ekey], 0.0
    else:
        with _nvtx("gqis.emit"):
            frag = emit.emit_model(compiled, uses_rho0_values)
        if RHSreuse:
            compiled.emitted[ekey] = frag
        stages["emit_s"] = time.time() - t0
    codegen_s = stages["ode_prepare_s"] + stages["ode_optimize_s"] + stages["emit_s"]

    # ---- 3) module (kernel) for this variant
    trace_mode = ("state" if _state_trace else "observable") if return_time_trace else None
    count = spec.adaptive and counts_steps(adaptive_options)
    flags = tuple([nvrtc_options] if isinstance(nvrtc_options, str) else nvrtc_options)
    if template_dir:
        flags = (f"-I{template_dir}",) + flags
    tmtime = os.path.getmtime(kernel_template_file) if kernel_template_file else None
    kkey = ("b200_kernel_v1", compiled.cache_key, bool(uses_rho0_values), mode, spec.name, unroll,
            form, trace_mode, flags, tmtime, use_matrix, tensor_cores)
    kernel_status = "miss"
    t_build = time.time()
    entry = _KERNEL_CACHE.get(kkey) if RHSreuse else None
    if entry is None:
        from . import engine
        source = (matrix_form.module_source(compiled, form, mode, bool(uses_rho0_values), tensor_cores,
                                            trace=trace_mode == "observable")
                  if use_matrix
                  else engine.module_source(frag, spec, form, mode, trace_mode, unroll))
        # `unroll` (the reference's "#pragma unroll on the solver's vector loops", gqis/solver.py:1821)
        # is validated and reported but builds the same module: the templates unroll every loop over
        # the state, which is what keeps the state in registers.
        entry = {"source": source,
                 "module": None, "flags": flags,
                 "frag": frag, "spec": spec, "compiled": compiled}
        if RHSreuse:
            _KERNEL_CACHE[kkey] = entry
    else:
        kernel_status = "hit"
    saved = _save_kernel(Actual_Kernel_Save, entry["source"])
    if _prebuild_only:  # build the module for later processes; no device is touched
        if _prebuild_only == "source":
            return entry["source"], entry["flags"]
        from . import engine
        return engine.build_module(entry["source"], extra_flags=entry["flags"])

    # ---- 4) inputs and launch
    axes = list(var_arrays.values())

    def host_axis(a):
        return a if hasattr(a, "data_ptr") else np.asarray(a, dtype=np.float64).reshape(-1)

    par_x = host_axis(axes[0])
    par_y = host_axis(axes[1]) if len(axes) > 1 else np.zeros(1)
    nx, ny = int(len(par_x)), int(len(par_y))
    rho0_arr = None
    if uses_rho0_values:
        shape = tuple(rho0_values.shape) if hasattr(rho0_values, "shape") else np.shape(rho0_values)
        S = compiled.state_size
        if not (shape == (nx, ny, S) or (shape == (nx, S) and ny == 1)):
            raise ValueError(f"rho0_values must have shape ({nx}, {ny}, {S}) or ({nx}, {S}) "
                             f"when num_Y=1; got {tuple(shape)}.")
        rho0_arr = rho0_values if hasattr(rho0_values, "data_ptr") else np.asarray(rho0_values, dtype=np.float64)
    used = frag["used_const_indices"]
    consts_eff = [const_vals[i] for i in used] if used else []
    if spec.adaptive:
        params = tuple(spec.parameters)
    elif spec.parameters:
        params = tuple(spec.parameters)
    else:
        params = ()
    launch = SweepLaunch(entry=entry, form=form, output_mode=mode, trace_mode=trace_mode,
                         state_size=compiled.state_size, par_x=par_x, par_y=par_y, consts=consts_eff,
                         rho0=rho0_arr, num_steps=num_steps, warmup_steps=warmup_steps, dt=dt_host,
                         t_in=t_in, trace_stride=stride, trace_offset=offset, num_trace=num_trace,
                         solver_params=params, adaptive=spec.adaptive, count_steps=count,
                         return_device=bool(return_device), collect_timing=collect)
    if _prepare_only is not None:
        _prepare_only["launch"] = launch
        return None
    _load_kernel(entry)
    stage_build = time.time() - t_build
    rhs_stage_s = time.time() - t_total
    with _nvtx("gqis.sweep"):
        results, trace, counts, gpu_s = _device_run(launch)

    # ---- 5) outputs
    cplx = mode in ("mean", "final")
    S = compiled.state_size

    def shape_result(x):
        if x is None:
            return None
        if hasattr(x, "reshape") and not isinstance(x, np.ndarray):
            import torch
            if cplx:
                return torch.view_as_complex(x.reshape(nx, ny, 2).contiguous())
            return x.reshape(nx, ny, S)
        x = np.asarray(x)
        if cplx:
            x = x.reshape(nx, ny, 2)
            return x[..., 0] + 1j * x[..., 1]
        return x.reshape(nx, ny, S)

    def shape_trace(x):
        if x is None:
            return None
        if hasattr(x, "reshape") and not isinstance(x, np.ndarray):
            import torch
            if trace_mode == "observable":
                return torch.view_as_complex(x.reshape(nx, ny, num_trace, 2).contiguous())
            return x.reshape(nx, ny, num_trace, S)
        x = np.asarray(x)
        if trace_mode == "observable":
            x = x.reshape(nx, ny, num_trace, 2)
            return x[..., 0] + 1j * x[..., 1]
        return x.reshape(nx, ny, num_trace, S)

    res = shape_result(results)
    tr = shape_trace(trace) if return_time_trace else None
    # finite checks on the device, before any host copy (a reduction instead of a host pass)
    finite_res = _all_finite(res)
    finite_tr = _all_finite(tr) if return_time_trace else True
    if not return_device:
        res = _to_output(res, False) if not isinstance(res, np.ndarray) else res
        tr = _to_output(tr, False) if (tr is not None and not isinstance(tr, np.ndarray)) else tr
    if cplx and isinstance(res, np.ndarray):
        res = res.astype(np.complex128 if form == "fp64" else np.complex64, copy=False)
        if tr is not None and trace_mode == "observable":
            tr = tr.astype(np.complex128 if form == "fp64" else np.complex64, copy=False)
    if not finite_res and not ignore_non_finite_output:
        if beep_on_error:
            _beep()
        raise RuntimeError("Non-finite values detected in mesolve_2D output. Try reducing dt "
                           "(increase time samples) or check model parameters/RHS.")
    if return_time_trace and not finite_tr and not ignore_non_finite_output:
        if beep_on_error:
            _beep()
        raise RuntimeError("Non-finite values detected in mesolve_2D time trace. Try reducing dt "
                           "(increase time samples) or check model parameters/RHS.")

    info = None
    if collect:
        info = {"rhs_stage_s": rhs_stage_s, "gpu_kernel_s": gpu_s, "rhs_codegen_s": codegen_s,
                "total_s": time.time() - t_total, "ode_prepare_s": stages["ode_prepare_s"],
                "ode_optimize_s": stages["ode_optimize_s"], "code_emit_s": stages["emit_s"],
                "kernel_build_s": stage_build, "cached_rhs": rhs_status, "cached_kernel": kernel_status,
                "solver": spec.name, "solver_frequency": solver_frequency, "unroll": unroll,
                "precision": form,
                "rhs_form": ("matrix_tc" if tensor_cores else "matrix") if use_matrix else "reduced",
                "rhs_flops": None if use_matrix else emit.count_rhs_flops(frag)}
        module = entry.get("module")
        if hasattr(module, "info"):
            mi = module.info()
            info.update(registers_per_thread=mi.registers_per_thread, ctas_per_sm=mi.ctas_per_sm,
                        module_path=str(module.path))
        if counts is not None:
            c = counts if isinstance(counts, np.ndarray) else counts.cpu().numpy()
            c = c.reshape(nx, ny, 2)
            info["adaptive_steps"] = {"accepted": c[..., 0], "rejected": c[..., 1]}
    if timings:
        _print_timings("mesolve_2D" if _ode_size is None else "odesolve_2D", info, timings)
    if saved:
        print(f"Generated kernel saved to: {saved}")
    if return_time_trace:
        steps = np.arange(num_trace, dtype=np.float64 if form == "fp64" else np.float32) * stride
        trace_t = t_in + (steps + 1.0 + offset) * dt_host
        out = (res, tr, trace_t)
        return (*out, info) if return_timing_info else out
    if return_timing_info:
        return res, info
    return res




# ----------------------------------------------------------------------------------------
# calibrate_timesteps (reference gqis/solver.py:928-1341): implemented in calibration.py. These
# module-level names are the hooks the search calls through (and that tests replace).
# ----------------------------------------------------------------------------------------

def _timestep_calibration_settings(value, ode=False):
    """Validated ``calibrate_timesteps`` settings merged with the defaults."""
    return calibration.Settings.from_request(value, ode=ode)


def _undersampled_arguments(args, stride):
    """The call on every ``stride``-th point of each sweep axis (axis ends kept), and whether that
    is the whole grid."""
    return calibration.test_grid_arguments(args, stride)


def _calibrate_timestep(args, settings, base_steps, duration):
    """Coarsest resolution whose undersampled map meets the limits (report dict)."""
    return calibration.calibrate(args, settings, base_steps, duration)


def _solve_with_timestep_calibration(args):
    """Pick a uniform step (or adaptive tolerance) on a subgrid, then run the full sweep."""
    return calibration.solve_calibrated(args)


mesolve_2D.__doc__ = _solve_symbolic_system.__doc__
