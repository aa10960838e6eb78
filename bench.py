#!/usr/bin/env python
"""Benchmark: points*steps/s of the four-level interferogram sweep on B200.

Workload (the configuration the headline metric is quoted on): N = 4 Lindblad model, 2048 x 2048
grid of (eps, A), RK4 with 8000 steps over t in [0, 400], time-averaged <|3><3|> map. One bench
"step" is one full sweep of that grid. The headline ``value`` is the FP32 form (FP32 state and
RHS, FP64 time / drive phase / compensated average) with device-resident inputs; the plain FP64
form is timed beside it on the same GPU and the FP32 map's max-abs error against it is reported.

Multi-GPU (torchrun): weak scaling - rank r sweeps its own 2048 x 2048 tile (rows r*2048 ..
of a (2048 N) x 2048 grid); no collective on the data path, timings are the max over ranks.

``--impl reference`` times the reference's own kernel code on the host CPU cores (the CUDA
source that GQIS generates for this model, compiled for the CPU with OpenMP; falls back to
the NumPy oracle) on a strided sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "gpu-quantum-interferometry-solver_b200"))

METRIC = "points*steps/s (RK4, four-level Lindblad sweep); FP32 form vs plain FP64 at <=1e-6 max-abs err"
UNIT = "points*steps/s"
SIDE, NSTEPS, DURATION = 2048, 8000, 400.0


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index):
        self.index, self.proc, self.lines = index, None, []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _flush_l2(torch, buf):
    buf.add_(1)  # 256 MiB write: larger than the 126 MB L2


def time_launches(torch, sweep, steps, warmup, flush):
    """Per-launch CUDA-event times (ms) of ``steps`` launches after ``warmup`` launches."""
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        sweep.launch(stream)
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        _flush_l2(torch, flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sweep.launch(stream)
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    return times


def _max_over_ranks(torch, value, ws):
    from gqis.shard import max_over_ranks
    return max_over_ranks(value) if ws > 1 else value


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


CPU_SAMPLE = "c2_fp64_mean_sub128"  # 128 x 128 strided subgrid of the 2048^2 grid, 8000 steps


def cpu_reference(steps=1, sample=CPU_SAMPLE):
    """Reference kernel (GQIS-generated CUDA source compiled for the CPU) on host cores."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import ref_kernels
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    if ref_kernels.available(sample, "cpu"):
        meta = ref_kernels.meta(sample)
        shape = meta["outputs"][0]["shape"]
        points = shape[0] * shape[1]
        nsteps = [a for a in meta["args"] if a["kind"] == "scalar"][4]["value"]
        times = []
        for _ in range(steps):
            _, dt = ref_kernels.run_case(sample, "cpu")
            times.append(dt)
        return {"kind": "reference", "points": points, "steps": nsteps, "times": times, "cores": cores,
                "sample": f"{shape[0]}x{shape[1]} strided subgrid of the 2048x2048 grid, {nsteps} RK4 steps, "
                          "reference GQIS FP64 kernel source compiled for the CPU (OpenMP)"}
    import numpy as np
    import lindblad_oracle
    sys.path.insert(0, str(ROOT / "gpu-quantum-interferometry-solver_b200"))
    from gqis import workloads
    w = workloads.four_level(side=16, steps=800, duration=40.0)
    model = lindblad_oracle.from_workload(w)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        lindblad_oracle.rk4_sweep(model, w["tlist"])
        times.append(time.perf_counter() - t0)
    return {"kind": "port", "points": 256, "steps": 800, "times": times, "cores": 1,
            "sample": "16x16 strided subgrid, 800 RK4 steps, NumPy density-matrix oracle (one core)"}


def four_level_config(side, nsteps, ws):
    """The four-level workload's ``config``, shared by both arms (the reference arm times a sample of it)."""
    return {"workload": f"four-level Lindblad interferogram, {side}x{side} (eps, A) grid per GPU, "
                        f"RK4 {nsteps} steps on [0, {DURATION * nsteps / NSTEPS:g}], mean <|3><3|>",
            "points_per_gpu": side * side, "rk4_steps": nsteps, "parallelism": f"sweep shards x{ws}"}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    ref = cpu_reference(steps=args.warmup + args.steps)
    times = ref["times"][args.warmup:]
    per = [ref["points"] * ref["steps"] / t for t in times]
    value = statistics.median(per)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": four_level_config(args.side, args.nsteps, args.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref["cores"], "kind": ref["kind"],
                             "sample": ref["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def _traffic_from_profiles():
    p = ROOT / "profiles" / "roofline_inputs.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            return {}
    return {}


def run_ours(args):
    import numpy as np
    import torch
    ws, rank, local = _dist()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    import gqis
    from gqis import native, solver, workloads

    side, nsteps = args.side, args.nsteps
    from gqis.shard import weak_axis
    w = workloads.four_level(side=None, steps=nsteps, duration=DURATION * nsteps / NSTEPS, full=side * ws)
    eps, A = w["symbols"]
    eps_axis = weak_axis(w["var_arrays"][eps], ws, rank)  # this rank's 2048-row tile of the eps axis
    a_axis = np.linspace(0.0, 5.0, side)
    call = dict(var_arrays={eps: eps_axis, A: a_axis}, const_values={})
    model = (w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"])
    # the FP32 form's kernel: two points per thread in packed f32x2 arithmetic (the default for this
    # model), or one point per thread (--fp32-kernel scalar, for comparison)
    kernel_flags = ("-DGQ_PACK2=0",) if args.fp32_kernel == "scalar" else ()
    fp32 = solver.prepare_sweep("mesolve_2D", *model, **call, precision="fp32", nvrtc_options=kernel_flags)
    fp64 = solver.prepare_sweep("mesolve_2D", *model, **call, precision="fp64")
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    points, ksteps = fp32.points, fp32.steps

    peaks = {}
    if rank == 0:
        for kind, name in ((0, "fp64"), (1, "fp32"), (2, "fp32x2")):
            peaks[name] = native.probe_fma_tflops(kind)

    # ---- plain FP64 (timed first, its map is the accuracy reference of the FP32 form)
    _barrier(ws)
    t64 = time_launches(torch, fp64, args.steps, args.warmup, flush)
    ms64 = _max_over_ranks(torch, float(np.mean(t64)), ws)
    ref_map = fp64.results.clone()

    # ---- headline: FP32 form
    _barrier(ws)
    sampler = ClockSampler(local).start()
    torch.cuda.synchronize()
    t32 = time_launches(torch, fp32, args.steps, args.warmup, flush)
    clocks = sampler.stop()
    ms32 = _max_over_ranks(torch, float(np.mean(t32)), ws)
    err = float((fp32.results.double() - ref_map).abs().max().item())
    err = _max_over_ranks(torch, err, ws)

    # ---- end to end through the public API (host arrays in, NumPy map out)
    e2e_ms = []
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        out = gqis.mesolve_2D(*model, **call, fp64=False, nvrtc_options=kernel_flags)
        b.record()
        b.synchronize()
        if k >= args.warmup:
            e2e_ms.append(a.elapsed_time(b))
    e2e = _max_over_ranks(torch, float(np.mean(e2e_ms)), ws)
    h2d = (len(eps_axis) + len(a_axis)) * 8
    d2h = int(out.size) * out.itemsize

    flops_ps = fp32.flops_per_point_step()
    total_units = points * ksteps * ws
    value = total_units / (ms32 / 1e3)
    line = None
    if rank == 0:
        achieved = points * ksteps * flops_ps / (float(np.mean(t32)) / 1e3) / 1e12
        measured = _traffic_from_profiles()
        traffic = measured.get("fp32_dram_bytes_per_launch")
        lat = sorted(t32)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(four_level_config(side, ksteps, ws),
                           l2="flushed (256 MiB write) between timed launches",
                           form="FP32 state/RHS, FP64 time + drive phase + compensated average",
                           fp32_kernel=("two points per thread, packed f32x2" if args.fp32_kernel == "packed"
                                        else "one point per thread")),
            "plain_fp64": {"value": total_units / (ms64 / 1e3), "ms_per_step": ms64},
            "speedup_vs_plain_fp64": ms64 / ms32,
            "max_abs_err_vs_fp64": err,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peaks.get("fp32"), "unit": "TFLOP/s",
                         "frac": achieved / peaks["fp32"] if peaks.get("fp32") else None,
                         "traffic": traffic, "traffic_source": measured.get("fp32_traffic_source"),
                         "peak_source": "measured FFMA probe (gqis_probe_fma) in this run",
                         "flops_per_point_step": flops_ps},
            "peaks_measured_tflops": peaks,
            "clocks": clocks,
            "e2e": {"value": total_units / (e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e},
            "gpu_launches": args.steps,
        }
        if ws == 1 and not args.no_cpu_baseline:
            ref = cpu_reference(steps=1)
            line["cpu_baseline"] = {"value": ref["points"] * ref["steps"] / ref["times"][0], "unit": UNIT,
                                    "cores": ref["cores"], "kind": ref["kind"], "sample": ref["sample"]}
        if ws == 1 and args.reference_gpu and side == SIDE and nsteps == NSTEPS:
            line["reference_kernel_gpu"] = reference_gpu_kernels(ref_map)
    if ws == 1 and not args.headline_only:
        # the other configurations on the same GPU, after the headline measurement: C4 (Hilbert-space
        # scaling on the tensor cores), C3 (adaptive Duffing) and C5 (serving)
        del fp32, fp64
        torch.cuda.empty_cache()
        sys.path.insert(0, str(ROOT / "oracle"))
        sampler = ClockSampler(local).start()
        hpeaks = {"fp64": peaks["fp64"], "fp32": peaks["fp32"], "f16_tensor": native.probe_tc_f16_tflops()}
        t_sub = time.perf_counter()
        line["hilbert"] = {"workload": HILBERT_WORKLOAD.format(steps=2000), "l2": "flushed between timed launches",
                           "measured_peaks_tflops": hpeaks,
                           "per_dimension": hilbert_rows(torch, (8, 16, 32, 64), 2000, flush, hpeaks)}
        line["duffing"] = {"workload": DUFFING_WORKLOAD.format(side=1024, solver="dop853a | tsit5a"),
                           "per_solver": duffing_rows(torch, flush, 1024, 2, 1)}
        del flush
        torch.cuda.empty_cache()
        line["serving"] = serving_summary(torch, args.sub_requests, args.rate, args.seed)
        line["other_configs_wall_s"] = time.perf_counter() - t_sub
        line["other_configs_clocks"] = sampler.stop()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))
    return 0


def reference_gpu_kernels(fp64_map):
    """The reference's own generated kernels for this workload, compiled for sm_100a, same GPU,
    with each map's max-abs difference from our plain FP64 map (which equals the reference FP64
    kernel's map to 1e-10)."""
    import numpy as np
    sys.path.insert(0, str(ROOT / "oracle"))
    import ref_kernels
    ours = fp64_map[:, 0].cpu().numpy().reshape(SIDE, SIDE)
    out = {}
    for form, case in (("fp64", "c2_fp64_mean_full"), ("fp32", "c2_fp32_mean_full")):
        if not ref_kernels.available(case, "gpu"):
            out[form] = None
            continue
        res, _ = ref_kernels.run_case(case, "gpu")
        _, dt = ref_kernels.run_case(case, "gpu", repeats=2)
        err = float(np.max(np.abs(res["result"].real - ours)))
        out[form] = {"ms_per_sweep": dt * 1e3, "value": SIDE * SIDE * NSTEPS / dt, "max_abs_diff_vs_our_fp64": err}
    return out


DUFFING_OPTIONS = {"step_rtol": 1e-8, "step_atol": 1e-10, "max_substeps": 2000, "count_steps": True}


def duffing_rows(torch, flush, side, reps, warmup, solvers=("dop853a", "tsit5a"), reference_gpu=True,
                 static_schedule=False):
    """Config C3 per adaptive solver: the 1024^2 Duffing sweep (FP64, rtol 1e-8, atol 1e-10, final
    state + 512-sample trace), accepted/rejected steps, and the final states on a 16 x 16 subgrid
    against the C oracle of the same method and a tight-tolerance DOP853 reference; plus the
    reference's own generated tsit5a kernel on the same GPU (final state, no trace)."""
    import numpy as np
    import ode_oracle
    from gqis import solver, workloads
    d = workloads.duffing(side=None, full=side)
    model = (d["rhs"], d["states"], None, d["tlist"])
    idx = np.round(np.linspace(0, side - 1, 16)).astype(int)
    F, W = (np.asarray(v)[idx] for v in d["var_arrays"].values())
    y0 = d["y0_values"][np.ix_(idx, idx)]
    tight, _, _ = ode_oracle.sweep("dop853a", F, W, y0, d["tlist"], rtol=1e-13, atol=1e-15,
                                   max_substeps=200000, want_trace=False)
    tight2, _, _ = ode_oracle.sweep("dop853a", F, W, y0, d["tlist"], rtol=1e-12, atol=1e-14,
                                    max_substeps=200000, want_trace=False)
    chaotic = np.max(np.abs(tight - tight2), axis=-1) > 1e-4  # points the tight references disagree on
    rows = {}
    for name in solvers:
        call = dict(var_arrays=d["var_arrays"], y0_values=d["y0_values"], solver=name, fp64=True,
                    return_time_trace=True, adaptive_options=DUFFING_OPTIONS)
        sweep = solver.prepare_sweep("odesolve_2D", *model, **call)
        ms = float(np.mean(time_launches(torch, sweep, reps, warmup, flush)))
        counts = sweep.tensors["step_counts"].cpu().numpy().astype(np.int64)
        acc, rej = int(counts[:, 0].sum()), int(counts[:, 1].sum())
        trace_bytes = sweep.tensors["trace"].numel() * sweep.tensors["trace"].element_size()
        final = sweep.results.cpu().numpy().reshape(side, side, 2)[np.ix_(idx, idx)]
        same, _, _ = ode_oracle.sweep(name, F, W, y0, d["tlist"], rtol=1e-8, atol=1e-10, max_substeps=2000,
                                      want_trace=False)
        err_true = np.max(np.abs(final - tight), axis=-1)
        row = {"ms": ms, "accepted_steps": acc, "rejected_steps": rej,
               "points_accepted_steps_per_s": acc / (ms / 1e3),
               "trace_bytes_per_launch": trace_bytes, "trace_write_gbs": trace_bytes / (ms / 1e3) / 1e9,
               "subgrid_16x16_max_abs_vs_same_method_c_oracle": float(np.max(np.abs(final - same))),
               "subgrid_16x16_max_abs_vs_tight_dop853_nonchaotic":
                   float(err_true[~chaotic].max()) if (~chaotic).any() else None,
               "chaotic_points_of_256": int(chaotic.sum())}
        if static_schedule:
            static = solver.prepare_sweep("odesolve_2D", *model, **call, nvrtc_options=("-DGQ_STATIC_SCHEDULE=1",))
            row["static_schedule_ms"] = float(np.mean(time_launches(torch, static, 1, 1, flush)))
            row["static_schedule_results_identical"] = bool(torch.equal(static.results, sweep.results))
            row["work_stealing_speedup"] = row["static_schedule_ms"] / ms
            del static
        rows[name] = row
        del sweep
    if reference_gpu and "tsit5a" in solvers and side == 1024:
        rows["reference_tsit5a_kernel_gpu"] = reference_tsit5a_gpu(torch, model, d, DUFFING_OPTIONS, flush)
    return rows


def run_duffing(args):
    """Config C3: adaptive sweep of the driven Duffing oscillator with a 512-sample state trace."""
    import torch
    torch.cuda.set_device(0)
    sys.path.insert(0, str(ROOT / "oracle"))
    side = args.side if args.side != SIDE else 1024
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    sampler = ClockSampler(0).start()
    rows = duffing_rows(torch, flush, side, args.steps, args.warmup, solvers=(args.solver,),
                        reference_gpu=args.reference_gpu, static_schedule=True)
    clocks = sampler.stop()
    row = rows[args.solver]
    line = {
        "metric": "points*accepted-steps/s (adaptive Duffing sweep, FP64, rtol 1e-8, atol 1e-10)",
        "value": row["points_accepted_steps_per_s"], "unit": "points*accepted-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": row["ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": DUFFING_WORKLOAD.format(side=side, solver=args.solver),
                   "l2": "flushed (256 MiB write) between timed launches"},
        **row, "clocks": clocks, "gpu_launches": args.steps,
    }
    if "reference_tsit5a_kernel_gpu" in rows:
        line["reference_kernel_gpu"] = rows["reference_tsit5a_kernel_gpu"]
    print(json.dumps(line))
    return 0


DUFFING_WORKLOAD = ("driven Duffing x''+0.1x'+x+x^3=F cos(W t), {side}x{side} (F, W) grid, t in [0, 500], "
                    "{solver}, state trace 512 samples + final state")


def reference_tsit5a_gpu(torch, model, d, opts, flush):
    """The reference's own generated tsit5a kernel for the Duffing sweep (1024^2, final state, no
    trace), compiled for sm_100a, against our Tsit5A on the same call without the trace."""
    import numpy as np
    sys.path.insert(0, str(ROOT / "oracle"))
    import ref_kernels
    from gqis import solver
    case = "duffing_tsit5a_full_final"
    if not ref_kernels.available(case, "gpu"):
        return None
    call = dict(var_arrays=d["var_arrays"], y0_values=d["y0_values"], solver="tsit5a", fp64=True,
                adaptive_options={k: v for k, v in opts.items() if k != "count_steps"})
    ours = solver.prepare_sweep("odesolve_2D", *model, **call)
    ms = float(np.mean(time_launches(torch, ours, 2, 1, flush)))
    mine = ours.results.cpu().numpy()
    ref_kernels.run_case(case, "gpu")
    res, dt = ref_kernels.run_case(case, "gpu", repeats=2)
    ref = np.asarray(res["result"]).reshape(mine.shape)
    return {"reference_ms": dt * 1e3, "ours_ms_without_trace": ms, "speedup": dt * 1e3 / ms,
            "max_abs_diff": float(np.max(np.abs(mine - ref))),
            "points_differing_by_more_than_1e-6": int(np.sum(np.max(np.abs(mine - ref), axis=-1) > 1e-6))}


def run_two_level(args):
    """The two-level model at the size of the reference's published two-level benchmark (RK4, 2048^2
    points, 10,240 steps): our FP32 form and plain FP64 form, and the reference's own generated FP32 and
    FP64 kernels for the same call compiled for sm_100a (``oracle/_ref``), on the same GPU."""
    import numpy as np
    import torch
    torch.cuda.set_device(0)
    sys.path.insert(0, str(ROOT / "oracle"))
    import ref_kernels
    from gqis import solver, workloads
    w = workloads.two_level(full=2048, steps=10240, duration=512.0)
    model = (w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"])
    call = dict(var_arrays=w["var_arrays"], const_values=w["const_values"])
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    units = 2048 * 2048 * 10240
    sampler = ClockSampler(0).start()
    rows, maps = {}, {}
    for form in ("fp64", "fp32"):
        sw = solver.prepare_sweep("mesolve_2D", *model, **call, precision=form)
        ms = float(np.mean(time_launches(torch, sw, args.steps, args.warmup, flush)))
        maps[f"ours_{form}"] = sw.results.double().cpu().numpy()[:, 0].reshape(2048, 2048)
        rows[f"ours_{form}"] = {"ms": ms, "points_steps_per_s": units / (ms / 1e3)}
        del sw
    for form in ("fp64", "fp32"):
        case = f"c1_big_{form}_mean"
        if not ref_kernels.available(case, "gpu"):
            continue
        ref_kernels.run_case(case, "gpu")
        res, dt = ref_kernels.run_case(case, "gpu", repeats=args.steps)
        maps[f"reference_{form}"] = np.asarray(res["result"]).real.reshape(2048, 2048)
        rows[f"reference_{form}"] = {"ms": dt * 1e3, "points_steps_per_s": units / dt}
    clocks = sampler.stop()
    for key in rows:
        rows[key]["max_abs_vs_our_fp64"] = float(np.max(np.abs(maps[key] - maps["ours_fp64"])))
    line = {
        "metric": "points*steps/s (RK4, two-level Lindblad sweep at the reference's published benchmark size)",
        "value": rows["ours_fp32"]["points_steps_per_s"], "unit": "points*steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": rows["ours_fp32"]["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "two-level driven qubit (H = eps/2 sz + 1/2 sx + A cos(pi t) sz, sqrt(0.01) s-, "
                               "sqrt(0.01) sz), 2048 x 2048 (eps, A), 10,240 RK4 steps of dt 0.05, mean <|1><1|>",
                   "l2": "flushed (256 MiB write) between timed launches"},
        "forms": rows, "reference_published_rtx3080_fp32": 1.19e11, "clocks": clocks,
    }
    print(json.dumps(line))
    return 0


def hilbert_rows(torch, dims, hsteps, flush, peaks, *, tc_reps=3, fp64_reps=1, cuda_fp32=False, only=()):
    """Config C4 per dimension N: the tensor-core FP32 form against the plain FP64 density-matrix
    form on the full 64 x 64 map (both timed), the FP64 form pinned to the FP64 NumPy oracle on 4
    points, and the tensor-core kernel's roofline by the algorithmic count (16 N^3 per product
    pair, no split passes) and by the MMAs it issues (three split-FP16 passes). ``only``: names of
    the forms to run (e.g. "matrix_tc_fp32"); the comparisons with a form that did not run are left out."""
    import numpy as np
    import lindblad_oracle
    from gqis import solver, workloads
    points = 64 * 64
    rows = {}
    for N in dims:
        w = workloads.n_level(N, side=64, steps=hsteps, duration=100.0 * hsteps / 2000)
        model = (w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"])
        forms = [("matrix_tc", "fp32", tc_reps, 1), ("matrix", "fp64", fp64_reps, 1 if N < 64 else 0)]
        if cuda_fp32:
            forms.append(("matrix", "fp32", tc_reps, 1))
        if only:
            forms = [f for f in forms if f"{f[0]}_{f[1]}" in only]
        row, maps = {}, {}
        for rhs_form, prec, reps, warm in forms:
            sweep = solver.prepare_sweep("mesolve_2D", *model, var_arrays=w["var_arrays"], precision=prec,
                                         rhs_form=rhs_form)
            ms = float(np.mean(time_launches(torch, sweep, reps, warm, flush)))
            frag = sweep.launch_spec.entry["frag"]
            algo = frag["algorithmic_flops_per_point_step"] * points * hsteps / (ms / 1e3) / 1e12
            entry = {"ms": ms, "points_steps_per_s": points * hsteps / (ms / 1e3), "timed_launches": reps,
                     "warmup_launches": warm, "algorithmic_tflops": algo}
            if rhs_form == "matrix_tc":
                mma = frag["tensor_flops_per_point_step"] * points * hsteps / (ms / 1e3) / 1e12
                entry.update(mma_tflops=mma, frac_mma_of_measured_f16=mma / peaks["f16_tensor"],
                             frac_algorithmic_of_measured_f16=algo / peaks["f16_tensor"])
            else:
                entry["frac_algorithmic_of_measured_fma"] = algo / peaks[prec]
            row[f"{rhs_form}_{prec}"] = entry
            maps[(rhs_form, prec)] = sweep.results.double().cpu().numpy()
            del sweep
        eps, A = w["symbols"]
        idx = np.array([0, 21, 42, 63])
        sub = {eps: np.asarray(w["var_arrays"][eps])[idx[:2]], A: np.asarray(w["var_arrays"][A])[idx[2:]]}
        ref = lindblad_oracle.rk4_sweep(lindblad_oracle.from_workload(w, sub), w["tlist"]).reshape(-1)
        sel = (idx[:2][:, None] * 64 + idx[2:][None, :]).reshape(-1)
        full64 = maps.get(("matrix", "fp64"))
        for (rhs_form, prec), m in maps.items():
            got = m[sel, 0] + 1j * m[sel, 1]
            row[f"{rhs_form}_{prec}"]["max_abs_vs_fp64_oracle_4pts"] = float(np.max(np.abs(got - ref)))
            if prec == "fp32" and full64 is not None:
                row[f"{rhs_form}_{prec}"]["max_abs_vs_fp64_form_full_map"] = float(np.max(np.abs(m - full64)))
        if "matrix_fp64" in row and "matrix_tc_fp32" in row:
            row["tensor_core_speedup_vs_fp64"] = row["matrix_fp64"]["ms"] / row["matrix_tc_fp32"]["ms"]
        rows[str(N)] = row
    return rows


def run_hilbert(args):
    """Config C4: Hilbert-space scaling of the density-matrix kernel, N in {8, 16, 32, 64}, 64 x 64
    (eps, A) points, 2000 RK4 steps on [0, 100]; FP64 and FP32 forms, error vs the FP64 oracle."""
    import torch
    torch.cuda.set_device(0)
    sys.path.insert(0, str(ROOT / "oracle"))
    from gqis import native
    peaks = {"fp64": native.probe_fma_tflops(0), "fp32": native.probe_fma_tflops(1),
             "f16_tensor": native.probe_tc_f16_tflops()}
    dims = tuple(int(n) for n in args.dims.split(","))
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    sampler = ClockSampler(0).start()
    only = tuple(f for f in args.forms.split(",") if f)
    rows = hilbert_rows(torch, dims, args.hsteps, flush, peaks, tc_reps=max(1, args.steps // 2),
                        cuda_fp32=True, only=only)
    clocks = sampler.stop()
    hk = "16" if "16" in rows else str(dims[0])
    if "matrix_tc_fp32" not in rows[hk]:
        print(json.dumps({"per_dimension": rows, "measured_fma_peaks_tflops": peaks, "clocks": clocks}))
        return 0
    head = rows[hk]["matrix_tc_fp32"]
    line = {
        "metric": "points*steps/s (RK4 density-matrix sweep, N-level scaling model; tensor-core split-FP16 "
                  "form, N=16 headline)",
        "value": head["points_steps_per_s"], "unit": "points*steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": 1, "ms_per_step": head["ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": HILBERT_WORKLOAD.format(steps=args.hsteps), "dims": list(dims),
                   "l2": "flushed (256 MiB write) between timed launches"},
        "per_dimension": rows,
        "roofline": {"bound": "tensor", "achieved": head["algorithmic_tflops"], "peak": peaks["f16_tensor"],
                     "unit": "TFLOP/s", "frac": head["frac_algorithmic_of_measured_f16"], "traffic": None,
                     "peak_source": "tcgen05 kind::f16 probe (gqis_probe_tc_f16), same run",
                     "kernel": f"matrix_tc_kernel N={hk}", "mma_tflops": head["mma_tflops"],
                     "frac_mma": head["frac_mma_of_measured_f16"]},
        "measured_fma_peaks_tflops": peaks, "clocks": clocks,
    }
    print(json.dumps(line))
    return 0


HILBERT_WORKLOAD = ("N-level model: H0 seeded GUE-like + eps diag(0..N-1) + A cos(t) X; N-1 lowering ops at rate "
                    "0.01, N dephasing ops at rate 0.005; 64x64 (eps, A) grid, {steps} RK4 steps of dt 0.05, "
                    "mean <|N-1><N-1|>")


def run_render(args):
    """Phase-space rasteriser: a 2048^2-point cloud resident on the device binned into a
    512 x 512 mean-colour image each frame, then coloured into a 1920 x 1080 RGBA frame."""
    import numpy as np
    import torch
    torch.cuda.set_device(0)
    sys.path.insert(0, str(ROOT / "oracle"))
    import render_oracle
    from gqis.render import GPUDisplayImage, PhaseRasterizer
    n = 2048 * 2048
    gen = torch.Generator(device="cuda").manual_seed(args.seed)
    cluster = torch.randn((n // 2, 2), generator=gen, device="cuda", dtype=torch.float64) * 0.15
    ang = torch.rand(n - n // 2, generator=gen, device="cuda", dtype=torch.float64) * 6.283185307179586
    rad = 1.2 + 0.1 * torch.randn(n - n // 2, generator=gen, device="cuda", dtype=torch.float64)
    ring = torch.stack([rad * torch.cos(ang), 1.5 * rad * torch.sin(ang)], 1)
    points = torch.cat([cluster, ring]).contiguous()          # FP64, like an odesolve_2D state
    colors = torch.rand(n, generator=gen, device="cuda", dtype=torch.float32)
    r = PhaseRasterizer(colors, x_range=(-2.0, 2.0), v_range=(-2.5, 2.5), bins=(512, 512), partitions=8)
    ncol = 256
    t = np.linspace(0, 1, ncol)
    lut = np.vstack([np.stack([t, t ** 2, 1 - t, np.ones(ncol)], 1), [1, 1, 1, 1]]).astype(np.float32)
    disp = GPUDisplayImage(lut, 0.0, 1.0, "bilinear")
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        disp.render(r.render(points, return_device=True), (1920, 1080), return_device=True)
    torch.cuda.synchronize()
    sampler = ClockSampler(0).start()
    tb, td = [], []
    for _ in range(args.steps):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(stream)
        raster = r.render(points, return_device=True)
        b.record(stream)
        disp.render(raster, (1920, 1080), return_device=True)
        c.record(stream)
        c.synchronize()
        tb.append(a.elapsed_time(b))
        td.append(b.elapsed_time(c))
    clocks = sampler.stop()
    ms_bin, ms_disp = float(np.mean(tb)), float(np.mean(td))
    # end to end: host FP32 points uploaded each frame, the raster read back
    host = points.float().cpu().numpy()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        img = r.render(host)
    e2e_ms = (time.perf_counter() - t0) / args.steps * 1e3
    # correctness: the frame against the oracle
    ref, _ = render_oracle.bin_raster(host, colors.cpu().numpy(), (512, 512), (-2.0, 2.0), (-2.5, 2.5))
    same_empty = bool(np.array_equal(np.isnan(img), np.isnan(ref)))
    occ = ~np.isnan(ref)
    max_rel = float(np.max(np.abs(img[occ] - ref[occ]) / np.abs(ref[occ])))
    t1 = time.perf_counter()
    render_oracle.bin_raster(host[: n // 8], colors.cpu().numpy()[: n // 8], (512, 512), (-2.0, 2.0), (-2.5, 2.5))
    cpu_pts_s = (n // 8) / (time.perf_counter() - t1)
    algo_bytes = n * (16 + 4)  # FP64 (x, v) and FP32 colour per point
    line = {
        "metric": "phase-space rasteriser: points binned per second (2048^2 FP64 points -> 512x512 image)",
        "value": n / (ms_bin / 1e3), "unit": "points/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_bin + ms_disp, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (coordinates), f64 (colour sums)", "data": "synthetic",
        "config": {"workload": "4,194,304 (x, v) FP64 points resident on the device (cluster + ring), 512x512 bins, "
                               "8 partitions, 1920x1080 bilinear RGBA display frame", "l2": "inputs (84 MB) not flushed"},
        "bin_ms": ms_bin, "display_ms": ms_disp,
        "roofline": {"bound": "hbm", "achieved": algo_bytes / (ms_bin / 1e3) / 1e9, "peak": 6550.1, "unit": "GB/s",
                     "frac": algo_bytes / (ms_bin / 1e3) / 1e9 / 6550.1, "traffic": None,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs",
                     "note": "bin + finalize time; algorithmic bytes 20 per point (x, v FP64 + colour FP32)"},
        "e2e": {"value": n / (e2e_ms / 1e3), "unit": "points/s", "h2d_bytes_per_step": n * 8,
                "d2h_bytes_per_step": 512 * 512 * 4},
        "cpu_baseline": {"value": cpu_pts_s, "unit": "points/s", "cores": 1, "kind": "port",
                         "sample": f"{n // 8} points through the NumPy oracle"},
        "check_vs_oracle": {"same_empty_pixels": same_empty, "max_rel_diff": max_rel},
        "clocks": clocks, "gpu_launches": 3 * args.steps,
    }
    print(json.dumps(line))
    return 0


def run_fit(args):
    """Gradients of a time-averaged map (fit step): the checkpointed RK4 adjoint of a 256 x 256
    two-level map, 4000 steps, d<O>avg / d(Gamma1, Gamma_phi, Delta), against the plain FP64 forward
    sweep of the same map and central differences."""
    import numpy as np
    import torch
    torch.cuda.set_device(0)
    sys.path.insert(0, str(ROOT / "oracle"))
    import gqis
    from gqis import adjoint, solver
    from gqis.workloads import qubit_fit_model
    fit_args, fit_kwargs, params = qubit_fit_model(side=(256, 256), steps=4000, duration=200.0)
    params = list(params[:3])
    prob = adjoint.Problem(*fit_args, **fit_kwargs, params=params)
    fwd = solver.prepare_sweep("mesolve_2D", *fit_args, **fit_kwargs, fp64=True)
    stream = torch.cuda.current_stream()

    def timed(fn, k):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        out = []
        for _ in range(k):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return float(np.mean(out))
    sampler = ClockSampler(0).start()
    ms_adj = timed(lambda: prob.run(), args.steps)
    ms_fwd = timed(lambda: fwd.launch(stream), args.steps)
    clocks = sampler.stop()
    mean, grad = (x.cpu().numpy() for x in prob.run())
    torch.cuda.synchronize()
    plain = fwd.results[:, 0].double().cpu().numpy().reshape(256, 256)
    sel = np.round(np.linspace(0, 255, 16)).astype(int)
    es, As = list(fit_kwargs["var_arrays"])
    sub = dict(fit_kwargs, var_arrays={es: fit_kwargs["var_arrays"][es][sel], As: fit_kwargs["var_arrays"][As][sel]})
    errs = []
    for m, prm in enumerate(params):
        up, dn = dict(sub["runtime_consts"]), dict(sub["runtime_consts"])
        up[prm] += 1e-6
        dn[prm] -= 1e-6
        fd = (gqis.mesolve_2D(*fit_args, **dict(sub, runtime_consts=up), fp64=True).real
              - gqis.mesolve_2D(*fit_args, **dict(sub, runtime_consts=dn), fp64=True).real) / 2e-6
        errs.append(float(np.max(np.abs(grad[np.ix_(sel, sel)][..., m] - fd)) / np.max(np.abs(fd))))
    units = 256 * 256 * 4000
    line = {
        "metric": "gradient throughput: points*steps/s of the checkpointed RK4 adjoint (mean map + 3 parameter gradients)",
        "value": units / (ms_adj / 1e3), "unit": "points*steps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_adj, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "two-level driven qubit, 256x256 (eps, A) map, 4000 RK4 steps on [0, 200], "
                               "params Gamma1, Gamma_phi, Delta (runtime constants), checkpoint every "
                               f"{prob.checkpoint_every} steps", "l2": "not flushed (inputs are a few KB)"},
        "forward_fp64_ms": ms_fwd, "adjoint_over_forward": ms_adj / ms_fwd,
        "scratch_bytes": prob.scratch_bytes,
        "mean_vs_plain_fp64_max_abs": float(np.max(np.abs(mean - plain))),
        "grad_vs_central_fd_max_rel": dict(zip([str(p) for p in params], errs)),
        "clocks": clocks, "gpu_launches": args.steps,
    }
    print(json.dumps(line))
    return 0


def _central_difference_check(fit_args, fit_kwargs, params, grad, side=256, samples=16, h=1e-6):
    """Max relative error of adjoint gradients against FP64 central differences on a strided subgrid."""
    import numpy as np
    import gqis
    sel = np.round(np.linspace(0, side - 1, samples)).astype(int)
    es, As = list(fit_kwargs["var_arrays"])
    sub = dict(fit_kwargs, var_arrays={es: fit_kwargs["var_arrays"][es][sel], As: fit_kwargs["var_arrays"][As][sel]})
    errs = []
    for m, prm in enumerate(params):
        up, dn = dict(sub["runtime_consts"]), dict(sub["runtime_consts"])
        up[prm] += h
        dn[prm] -= h
        fd = (gqis.mesolve_2D(*fit_args, **dict(sub, runtime_consts=up), fp64=True).real
              - gqis.mesolve_2D(*fit_args, **dict(sub, runtime_consts=dn), fp64=True).real) / (2 * h)
        errs.append(float(np.max(np.abs(grad[np.ix_(sel, sel)][..., m] - fd)) / np.max(np.abs(fd))))
    return errs


SERVING_DIMS = (2, 4, 8, 16)


def serving_summary(torch, requests, rate, seed, one_by_one=("fp32", "fp64"), fit_check=True):
    """Config C5: a seeded Poisson stream of mixed-N, mixed-size sweep requests (FP32 form) and fit
    requests (checkpointed FP64 adjoint) through the continuous-batching server; latency p50/p99
    and aggregate points*steps/s, against the same requests run one by one through the public API
    in the same form (what batching alone buys) and on the plain FP64 path."""
    import numpy as np
    import gqis
    from gqis import adjoint
    from gqis.serving import SweepServer
    from gqis.workloads import SERVING_SIDES, qubit_fit_model, serving_model
    rng = np.random.default_rng(seed)
    reqs, t = [], 0.0
    for _ in range(requests):
        t += rng.exponential(1.0 / rate)
        if rng.random() < 0.2:
            reqs.append((t, "fit", 256))
        else:
            N = int(rng.choice(SERVING_DIMS))
            sides = SERVING_SIDES if N < 16 else tuple(x for x in SERVING_SIDES if x <= 512)
            reqs.append((t, N, int(rng.choice(sides))))
    models = {}
    for _, N, side in reqs:
        if N != "fit" and (N, side) not in models:
            models[(N, side)] = serving_model(N, side)
    fit_args, fit_kwargs, fit_params = qubit_fit_model(side=(256, 256), steps=4000, duration=200.0)
    fit_params = list(fit_params[:3])
    for N in SERVING_DIMS:  # warm the caches (symbolic model, module load) before timing
        a, kw = serving_model(N, 64)
        for form in ("fp32",) + tuple(f for f in one_by_one if f != "fp32"):
            gqis.mesolve_2D(*a, **kw, precision=form)
    adjoint.module_source(*fit_args, **fit_kwargs, params=fit_params)

    def steps_of(N, side):
        return 4000 if N == "fit" else len(models[(N, side)][0][4]) - 1
    point_steps = sum(side * side * steps_of(N, side) for _, N, side in reqs)
    futs = []
    with SweepServer(streams=4, chunk_points=1 << 15, max_inflight=16) as srv:
        t0 = time.perf_counter()
        for arrival, N, side in reqs:
            delay = t0 + arrival - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            if N == "fit":
                futs.append(srv.submit_fit(*fit_args, **fit_kwargs, params=fit_params))
            else:
                a, kw = models[(N, side)]
                futs.append(srv.submit("mesolve_2D", *a, **kw, precision="fp32"))
        outs = [f.result(900) for f in futs]
        t_end = max(f.finished_at for f in futs)
        stats = dict(srv.stats)
    lat = np.array([f.latency for f in futs]) * 1e3
    served = point_steps / (t_end - t0)
    baselines = {}
    for form in one_by_one:  # the same requests one by one through the public API
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _, N, side in reqs:
            if N == "fit":
                adjoint.mean_gradient(*fit_args, **fit_kwargs, params=fit_params)
            else:
                a, kw = models[(N, side)]
                gqis.mesolve_2D(*a, **kw, precision=form)
        torch.cuda.synchronize()
        rate_seq = point_steps / (time.perf_counter() - t1)
        baselines[f"one_by_one_{form}"] = {"value": rate_seq, "served_speedup": served / rate_seq}
    fit_idx = [k for k, (_, N, _) in enumerate(reqs) if N == "fit"]
    check = None
    if fit_check and fit_idx:
        errs = _central_difference_check(fit_args, fit_kwargs, fit_params, outs[fit_idx[0]]["grad"])
        check = {"params": [str(p) for p in fit_params], "max_rel_err_vs_central_fd": errs}
    return {"value": served, "unit": "points*steps/s",
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            **baselines, "requests": requests, "fit_requests": len(fit_idx), "total_point_steps": point_steps,
            "workload": SERVING_WORKLOAD.format(requests=requests, rate=rate, dims=SERVING_DIMS, sides=SERVING_SIDES),
            "server": "4 streams, 32768-point chunks, <= 16 admitted requests, memory budget 50% free",
            "server_stats": stats, "fit_gradient_check": check}


SERVING_WORKLOAD = ("{requests} seeded requests, Poisson rate {rate}/s; 80% sweeps (N uniform in {dims}, grid side "
                    "uniform in {sides} (N = 16: up to 512), mean <O> maps, RK4, FP32 form; N = 8 and 16 on the "
                    "tensor-core density-matrix kernel), 20% fits (d<O>avg/d(Gamma1, Gamma_phi, Delta), 256x256 "
                    "two-level map, 4000 RK4 steps, checkpointed adjoint, FP64)")


def run_serving(args):
    """Config C5 (sweeps): Poisson stream of mixed-N, mixed-size sweep requests through the
    continuous-batching server (FP32 form), against the same requests one by one."""
    import torch
    torch.cuda.set_device(0)
    sys.path.insert(0, str(ROOT / "oracle"))
    summary = serving_summary(torch, args.requests, args.rate, args.seed)
    lat = summary["latency_ms"]
    line = {
        "metric": "sweep serving: aggregate points*steps/s and latency (Poisson 50/s, N in {2,4,8,16}, 20% fits)",
        "value": summary["value"], "unit": "points*steps/s", "n_gpus": 1, "steps": args.requests,
        "warmup": len(SERVING_DIMS), "ms_per_step": lat["p50"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": summary["workload"], "server": summary["server"]}, **summary,
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--side", type=int, default=SIDE)
    ap.add_argument("--nsteps", type=int, default=NSTEPS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp32-kernel", default="packed", choices=("packed", "scalar"),
                    help="four_level: the FP32 form's kernel (two points per thread, or one)")
    ap.add_argument("--reference-gpu", action="store_true",
                    help="also time the reference's generated kernels on this GPU")
    ap.add_argument("--requests", type=int, default=48, help="serving: number of requests")
    ap.add_argument("--sub-requests", type=int, default=24,
                    help="requests of the serving sub-object of the headline line")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the C3/C4/C5 sub-objects of the headline line")
    ap.add_argument("--rate", type=float, default=50.0, help="serving: Poisson arrival rate (1/s)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--dims", default="8,16,32,64", help="hilbert: Hilbert-space dimensions")
    ap.add_argument("--forms", default="", help="hilbert: comma list of forms to run (e.g. matrix_tc_fp32); all if empty")
    ap.add_argument("--hsteps", type=int, default=2000, help="hilbert: RK4 steps (t spans 100 * hsteps / 2000)")
    ap.add_argument("--workload", default="four_level",
                    choices=("four_level", "two_level", "duffing", "serving", "hilbert", "render", "fit"),
                    help="four_level: the headline RK4 interferogram; duffing: the adaptive ODE sweep")
    ap.add_argument("--solver", default="dop853a", help="adaptive solver of --workload duffing")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "duffing":
        return run_duffing(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "two_level":
        return run_two_level(args)
    if args.workload == "hilbert":
        return run_hilbert(args)
    if args.workload == "render":
        return run_render(args)
    if args.workload == "fit":
        return run_fit(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
