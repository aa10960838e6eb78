"""The benchmark configurations at their full sizes on the GPU.

The other GPU tests pin each kernel on small grids; these run the Hilbert-space scaling model
(64 x 64 points, 2000 RK4 steps) and the adaptive Duffing sweep (1024 x 1024 points, t in
[0, 500]) exactly as the benchmark does and check them at that size:

* tensor-core density-matrix kernel (split-FP16 MMAs, FP32 state) against the plain FP64
  density-matrix form on the whole 4096-point map, <= 1e-6 max-abs; the FP64 form itself against
  the NumPy FP64 oracle on 4 points, <= 1e-11;
* Tsit5A against the reference's own generated tsit5a kernel for the same call, compiled for
  sm_100a (when ``oracle/_ref`` holds it): final states within 1e-6 on every point (adaptive
  accept/reject decisions near err = 1 may flip under a different rounding order);
* DOP853A against the C oracle of the same method and tolerances on a 16 x 16 strided subgrid
  (<= 1e-6: 100x the step tolerance, the bar of the small-grid adaptive tests).
"""

import numpy as np
import pytest

import lindblad_oracle
import ode_oracle
import ref_kernels

ADAPTIVE = {"step_rtol": 1e-8, "step_atol": 1e-10, "max_substeps": 2000}


def _hilbert(N):
    from gqis import workloads
    w = workloads.n_level(N, side=64, steps=2000, duration=100.0)
    return w, (w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"])


@pytest.mark.gpu
@pytest.mark.parametrize("N", [16, 64])
def test_hilbert_config_tensor_cores_against_fp64_on_the_full_map(N):
    import gqis
    w, model = _hilbert(N)
    tc, info = gqis.mesolve_2D(*model, var_arrays=w["var_arrays"], precision="fp32", rhs_form="matrix_tc",
                               return_timing_info=True)
    assert info["rhs_form"] == "matrix_tc"
    fp64 = gqis.mesolve_2D(*model, var_arrays=w["var_arrays"], precision="fp64", rhs_form="matrix")
    assert tc.shape == fp64.shape == (64, 64)
    err = float(np.max(np.abs(tc - fp64)))
    assert err <= 1e-6, f"N={N}: tensor-core map max-abs {err:.3e} from the FP64 form"
    eps, A = w["symbols"]
    idx = np.array([0, 21, 42, 63])
    sub = {eps: np.asarray(w["var_arrays"][eps])[idx[:2]], A: np.asarray(w["var_arrays"][A])[idx[2:]]}
    ref = lindblad_oracle.rk4_sweep(lindblad_oracle.from_workload(w, sub), w["tlist"])
    got = fp64[np.ix_(idx[:2], idx[2:])]
    assert np.max(np.abs(ref)) > 1e-6
    assert float(np.max(np.abs(got - ref))) <= 1e-11


def _duffing(solver, **extra):
    from gqis import workloads
    d = workloads.duffing(side=None)
    kwargs = dict(var_arrays=d["var_arrays"], y0_values=d["y0_values"], solver=solver, fp64=True,
                  adaptive_options=dict(ADAPTIVE))
    kwargs.update(extra)
    return d, (d["rhs"], d["states"], None, d["tlist"]), kwargs


@pytest.mark.gpu
def test_duffing_config_tsit5a_matches_the_reference_kernel():
    import gqis
    case = "duffing_tsit5a_full_final"
    if not ref_kernels.available(case, "gpu"):
        pytest.skip("oracle/_ref was not built (reference tree absent when build() ran)")
    d, args, kwargs = _duffing("tsit5a")
    ours = gqis.odesolve_2D(*args, **kwargs)
    ref, _ = ref_kernels.run_case(case, "gpu")
    ref = np.asarray(ref["result"]).reshape(ours.shape)
    diff = np.max(np.abs(ours - ref), axis=-1)
    assert ours.shape == (1024, 1024, 2)
    assert float(diff.max()) <= 1e-6, f"max |ours - reference| {diff.max():.3e}"
    assert float(np.median(diff)) <= 1e-9


@pytest.mark.gpu
def test_duffing_config_dop853a_matches_the_c_oracle_on_a_subgrid():
    import gqis
    import torch
    d, args, kwargs = _duffing("dop853a", return_time_trace=True, return_device=True)
    final, trace, _ = gqis.odesolve_2D(*args, **kwargs)  # the 8.6 GB trace stays on the device
    assert tuple(final.shape) == (1024, 1024, 2) and tuple(trace.shape) == (1024, 1024, 512, 2)
    idx = np.round(np.linspace(0, 1023, 16)).astype(int)
    sel = torch.as_tensor(idx, device=final.device)
    final_sub = final[sel][:, sel].cpu().numpy()
    trace_sub = trace[sel][:, sel].cpu().numpy()
    del trace
    F, W = (np.asarray(v)[idx] for v in d["var_arrays"].values())
    y0 = d["y0_values"][np.ix_(idx, idx)]
    o_final, o_trace, _ = ode_oracle.sweep("dop853a", F, W, y0, d["tlist"], rtol=1e-8, atol=1e-10,
                                           max_substeps=2000)
    assert float(np.max(np.abs(final_sub - o_final))) <= 1e-6
    assert float(np.max(np.abs(trace_sub - o_trace))) <= 1e-6
