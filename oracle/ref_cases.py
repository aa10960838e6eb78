"""Parity cases shared by the reference capture recipe, the golden fixtures and the GPU tests.

Each case is a dict ``{"api": "mesolve_2D" | "odesolve_2D", "args": [...], "kwargs": {...}}``
built from the synthetic workloads (loaded by file path, so this module also works next to the
reference package). ``cpu`` marks cases small enough for the CPU build of the reference kernel
(golden fixtures); the others run only on the GPU.
"""

from __future__ import annotations

import importlib.util
from pathlib import Path

import numpy as np
import sympy as sp

_WORKLOADS = Path(__file__).resolve().parents[1] / "gpu-quantum-interferometry-solver_b200" / "gqis" / "workloads.py"


def workloads():
    spec = importlib.util.spec_from_file_location("gqis_b200_workloads", _WORKLOADS)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


FIXED_SOLVERS = ("rk4", "lserk4", "lserk4f", "dp5", "ab5", "anas5", "tsit5", "alshina6", "dop853")


def _lindblad(w, **kw):
    args = [w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"]]
    kwargs = {"var_arrays": w["var_arrays"], "const_values": w["const_values"]}
    kwargs.update(kw)
    return {"api": "mesolve_2D", "args": args, "kwargs": kwargs}


def small_qubit():
    """8 x 6 driven qubit over 400 steps: the per-solver and output-mode cases."""
    W = workloads()
    w = W.two_level(side=None)
    eps, A = w["symbols"]
    w["var_arrays"] = {eps: np.linspace(-3.0, 3.0, 8), A: np.linspace(0.0, 2.0, 6)}
    w["tlist"] = np.linspace(0.0, 20.0, 401)
    return w


def cases():
    W = workloads()
    out = {}
    out["c1_fp64_mean"] = dict(_lindblad(W.two_level(), fp64=True), cpu=True)
    out["c1_fp32_mean"] = dict(_lindblad(W.two_level(), fp64=False), cpu=True)
    out["c2_fp64_mean_sub32"] = dict(_lindblad(W.four_level(side=32), fp64=True), cpu=True)
    out["c2_fp64_mean_sub64"] = dict(_lindblad(W.four_level(side=64), fp64=True), cpu=False)
    out["c2_fp64_mean_sub128"] = dict(_lindblad(W.four_level(side=128), fp64=True), cpu=False)
    out["c2_fp64_mean_sub256"] = dict(_lindblad(W.four_level(side=256), fp64=True), cpu=False)
    out["c2_fp64_mean_full"] = dict(_lindblad(W.four_level(), fp64=True), cpu=False)
    out["c2_fp32_mean_full"] = dict(_lindblad(W.four_level(), fp64=False), cpu=False)
    for name in FIXED_SOLVERS:
        out[f"qubit_{name}_final_rho"] = dict(_lindblad(small_qubit(), fp64=True, solver=name,
                                                        output_mode="final_rho", solver_frequency=np.pi),
                                              cpu=True)
    out["qubit_rk4_final"] = dict(_lindblad(small_qubit(), fp64=True, output_mode="final"), cpu=True)
    out["qubit_rk4_mean_warmup_trace"] = dict(
        _lindblad(small_qubit(), fp64=True, warmup_time=0.3, return_time_trace=True, time_trace_every=7),
        cpu=True)
    out["qubit_rk4_t_in"] = dict(_lindblad(small_qubit(), fp64=True, t_in=3.25), cpu=True)
    q = small_qubit()
    delta = [s for s in q["const_values"]][0]
    out["qubit_rk4_runtime_const"] = dict(_lindblad(q, fp64=True, keep_symbolic_consts=[delta]), cpu=True)
    q = small_qubit()
    rng = np.random.default_rng(3)
    vec = rng.normal(size=(8, 6, 3)) * 0.2
    vec[..., 0] = rng.uniform(0.2, 0.8, size=(8, 6))
    out["qubit_rk4_rho0_values"] = dict(_lindblad(q, fp64=True, rho0_values=vec, output_mode="final_rho"),
                                        cpu=True)
    out["qubit_tsit5a_mean"] = dict(_lindblad(small_qubit(), fp64=True, solver="tsit5a",
                                              adaptive_options={"step_rtol": 1e-9, "step_atol": 1e-9,
                                                                "max_substeps": 2000, "count_steps": True}),
                                    cpu=True)
    d = W.duffing(side=12)
    x, v = d["states"]
    out["duffing_tsit5a_trace"] = {
        "api": "odesolve_2D", "args": [d["rhs"], d["states"], None, d["tlist"]],
        "kwargs": {"var_arrays": d["var_arrays"], "y0_values": d["y0_values"], "solver": "tsit5a", "fp64": True,
                   "return_time_trace": True,
                   "adaptive_options": {"step_rtol": 1e-8, "step_atol": 1e-10, "max_substeps": 4000}},
        "cpu": True}
    # the two-level model at the size of the reference's published two-level benchmark (2048^2 points,
    # 10,240 RK4 steps): timing on the GPU
    big = W.two_level(full=2048, steps=10240, duration=512.0)
    out["c1_big_fp64_mean"] = dict(_lindblad(big, fp64=True), cpu=False)
    out["c1_big_fp32_mean"] = dict(_lindblad(big, fp64=False), cpu=False)
    d_full = W.duffing(side=None)  # config C3 at full size (1024^2), final state: timing on the GPU
    out["duffing_tsit5a_full_final"] = {
        "api": "odesolve_2D", "args": [d_full["rhs"], d_full["states"], None, d_full["tlist"]],
        "kwargs": {"var_arrays": d_full["var_arrays"], "y0_values": d_full["y0_values"], "solver": "tsit5a",
                   "fp64": True,
                   "adaptive_options": {"step_rtol": 1e-8, "step_atol": 1e-10, "max_substeps": 2000}},
        "cpu": False}
    out["duffing_rk4_observable_trace"] = {
        "api": "odesolve_2D", "args": [d["rhs"], d["states"], None, np.linspace(0.0, 50.0, 5001)],
        "kwargs": {"var_arrays": d["var_arrays"], "y0_values": d["y0_values"], "fp64": True,
                   "observable": x**2 + sp.I * v, "return_time_trace": True, "time_trace_every": 10},
        "cpu": True}
    out["duffing_rk4_mean_state"] = {
        "api": "odesolve_2D", "args": [d["rhs"], d["states"], None, np.linspace(0.0, 50.0, 5001)],
        "kwargs": {"var_arrays": d["var_arrays"], "y0_values": d["y0_values"], "fp64": True,
                   "output_mode": "mean"},
        "cpu": True}
    return out
