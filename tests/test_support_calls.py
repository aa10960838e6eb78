"""Model-module variants used by GPU tests beyond the reference cases (prebuilt by build()).

Not a test module itself: ``__graft_entry__.build()`` imports ``calls()`` so that the GPU box
loads these modules instead of compiling them.
"""

import numpy as np

import ref_cases

ADAPTIVE_OPTIONS = {"step_rtol": 1e-8, "step_atol": 1e-10, "max_substeps": 4000, "count_steps": True}


def duffing_case(side=8, solver="dop853a", **extra):
    d = ref_cases.workloads().duffing(side=side)
    kwargs = dict(var_arrays=d["var_arrays"], y0_values=d["y0_values"], solver=solver, fp64=True,
                  return_time_trace=True, adaptive_options=dict(ADAPTIVE_OPTIONS))
    kwargs.update(extra)
    return d, (d["rhs"], d["states"], None, d["tlist"]), kwargs


def calls():
    out = []
    for solver in ("dop853a", "tsit5a"):
        for extra in ({}, {"nvrtc_options": ("-DGQ_STATIC_SCHEDULE=1",)}):
            _, args, kwargs = duffing_case(solver=solver, **extra)
            out.append(("odesolve_2D", args, kwargs))
    return out
