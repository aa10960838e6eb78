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


SERVING_SIDES = (64, 128, 256, 512, 1024)


def serving_model(N, side):
    """(args, kwargs) of one serving request: the Lindblad model of dimension N on a side^2 grid."""
    W = ref_cases.workloads()
    if N == 2:
        w = W.two_level()
    elif N == 4:
        w = W.four_level(full=side)
    else:
        w = W.n_level(N, side=side)
    eps, A = w["symbols"]
    var = {eps: np.linspace(float(np.min(w["var_arrays"][eps])), float(np.max(w["var_arrays"][eps])), side),
           A: np.linspace(float(np.min(w["var_arrays"][A])), float(np.max(w["var_arrays"][A])), side)}
    return ((w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"]),
            {"var_arrays": var, "const_values": w["const_values"]})


def calls():
    out = []
    for N in (2, 4, 8):
        args, kwargs = serving_model(N, 64)
        for form in ("fp32", "fp64"):
            out.append(("mesolve_2D", args, dict(kwargs, precision=form)))
    for solver in ("dop853a", "tsit5a"):
        for extra in ({}, {"nvrtc_options": ("-DGQ_STATIC_SCHEDULE=1",)}):
            _, args, kwargs = duffing_case(solver=solver, **extra)
            out.append(("odesolve_2D", args, kwargs))
    return out
