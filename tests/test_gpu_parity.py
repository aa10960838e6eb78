"""GPU parity: the sm_100a sweep kernels against the reference's own kernels and the oracles.

* golden fixtures (tests/golden, made by running the reference's generated kernel source on
  the CPU) - the plain FP64 form must agree to 1e-10 relative to the map's largest magnitude;
* the FP32 form must agree with the FP64 oracle to 1e-6 max-abs (the precision target);
* when ``oracle/_ref`` holds the reference kernels built for sm_100a, the full four-level
  interferogram (2048 x 2048, 8000 RK4 steps) is compared on the GPU as well.
"""

import numpy as np
import pytest

import ref_cases
import ref_kernels

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"
CASES = ref_cases.cases()
CPU_CASES = [n for n, c in CASES.items() if c.get("cpu")]

# Adaptive cases take tolerance-level decisions (accept / reject near err = 1) that rounding can
# flip; their parity bar is the step tolerance, not 1e-10.
ADAPTIVE_TOL = {"qubit_tsit5a_mean": 1e-9, "duffing_tsit5a_trace": 1e-6}


def _run(case, **override):
    import gqis
    kwargs = dict(case["kwargs"])
    kwargs.update(override)
    return getattr(gqis, case["api"])(*case["args"], **kwargs)


def _scaled_err(got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("name", CPU_CASES)
def test_fp64_matches_reference_kernel(name):
    case = CASES[name]
    golden = np.load(GOLDEN / f"{name}.npz")
    if not case["kwargs"].get("fp64", False):
        pytest.skip("FP32 reference case: covered by test_fp32_form_accuracy")
    out = _run(case)
    result = out[0] if isinstance(out, tuple) else out
    tol = ADAPTIVE_TOL.get(name, 1e-10)
    err = _scaled_err(result, golden["result"])
    assert err <= tol, f"{name}: scaled max error {err:.3e} > {tol:g}"
    if "trace" in golden:
        stride = int(golden["trace_stride"])
        trace, times = out[1], out[2]
        terr = _scaled_err(trace[:, :, ::stride], golden["trace"])
        assert terr <= tol, f"{name}: trace error {terr:.3e}"
        np.testing.assert_allclose(times[::stride], golden["trace_t"], rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1_fp64_mean", "c2_fp64_mean_sub32", "qubit_rk4_final_rho",
                                  "qubit_rk4_mean_warmup_trace", "duffing_rk4_observable_trace"])
def test_fp32_form_accuracy(name):
    """FP32 state and RHS with FP64 time, phase and averages: <= 1e-6 max-abs vs FP64."""
    case = CASES[name]
    golden = np.load(GOLDEN / f"{name}.npz")
    out = _run(case, fp64=False)
    result = out[0] if isinstance(out, tuple) else out
    err = float(np.max(np.abs(np.asarray(result) - golden["result"])))
    scale = max(1.0, float(np.max(np.abs(golden["result"]))))
    assert err <= 1e-6 * scale, f"{name}: FP32 form max-abs error {err:.3e}"


@pytest.mark.gpu
def test_reference_fp32_kernel_is_less_accurate_than_fp32_form():
    """Context for the precision form: the reference's FP32 kernel drifts more on the same map."""
    case = CASES["c1_fp64_mean"]
    ours = np.asarray(_run(case, fp64=False))
    ref32 = np.load(GOLDEN / "c1_fp32_mean.npz")["result"]
    ref64 = np.load(GOLDEN / "c1_fp64_mean.npz")["result"]
    assert np.max(np.abs(ours - ref64)) <= np.max(np.abs(ref32 - ref64))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c2_fp64_mean_sub256", "c2_fp64_mean_full"])
def test_full_size_against_reference_kernel_on_gpu(name):
    if not ref_kernels.available(name, "gpu"):
        pytest.skip("oracle/_ref was not built (reference tree absent when build() ran)")
    ref, _ = ref_kernels.run_case(name, "gpu")
    out = _run(CASES[name])
    err = _scaled_err(out, ref["result"])
    assert err <= 1e-10, f"{name}: scaled max error {err:.3e}"


@pytest.mark.gpu
def test_adaptive_step_counts_match_reference():
    golden = np.load(GOLDEN / "qubit_tsit5a_mean.npz")
    out, info = _run(CASES["qubit_tsit5a_mean"], return_timing_info=True)
    acc = info["adaptive_steps"]["accepted"]
    ref_acc = golden["adaptive_steps"][..., 0]
    assert np.mean(acc == ref_acc) >= 0.9
    assert np.max(np.abs(acc - ref_acc)) <= 2


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c2_fp64_mean_sub32", "qubit_rk4_mean_warmup_trace", "qubit_rk4_final_rho"])
def test_packed_pairs_match_the_one_point_kernel(name):
    """Small FP32 RK4 models run two points per thread in packed f32x2 arithmetic. The map equals
    the one-point-per-thread FP32 kernel's to FP32 rounding, and each point's result is bit for bit
    the same whichever neighbour shares its thread (chunks that start at odd points, odd counts)."""
    import torch
    from pathlib import Path
    from gqis import solver
    case = CASES[name]
    kw = dict(case["kwargs"], fp64=False)
    packed = solver.prepare_sweep(case["api"], *case["args"], **kw)
    assert "#define GQ_PACK2 1" in Path(str(packed.module.path).replace(".so", ".cu")).read_text()
    single = solver.prepare_sweep(case["api"], *case["args"], **kw, nvrtc_options=("-DGQ_PACK2=0",))
    packed.launch()
    single.launch()
    torch.cuda.synchronize()
    a, b = packed.results.double().cpu().numpy(), single.results.double().cpu().numpy()
    scale = max(1.0, float(np.max(np.abs(b))))
    assert float(np.max(np.abs(a - b))) <= 1e-6 * scale
    trace = packed.tensors.get("trace")
    n = packed.points
    for begin in (1, 7):
        part = solver.prepare_sweep(case["api"], *case["args"], **kw, point_begin=begin, point_count=n - begin - 2)
        part.launch()
        torch.cuda.synchronize()
        assert torch.equal(part.results, packed.results[begin:n - 2])
        if trace is not None:
            assert torch.equal(part.tensors["trace"], trace[begin:n - 2])
