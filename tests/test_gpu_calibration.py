"""calibrate_timesteps on the GPU: the batched search (candidate resolutions launched together on
separate streams) accepts the same step count, and returns the same map, as the one-at-a-time search
of the reference (gqis/solver.py:1066-1216)."""

import numpy as np
import pytest

import ref_cases


def _calibrated(case, batch_levels, **extra):
    import gqis
    from gqis import solver
    solver._TIMESTEP_CALIBRATION_CACHE.clear()
    kwargs = dict(case["kwargs"])
    kwargs.update(extra)
    settings = dict(rms_atol=1e-4, max_atol=1e-3, sample_stride=8, batch_levels=batch_levels)
    res, info = gqis.mesolve_2D(*case["args"], **kwargs, calibrate_timesteps=settings, return_timing_info=True)
    return res, info["timestep_calibration"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1_fp64_mean", "qubit_rk4_final"])
def test_batched_calibration_matches_one_at_a_time(name):
    case = ref_cases.cases()[name]
    steps = len(case["args"][4]) - 1
    tl = np.linspace(0.0, float(case["args"][4][-1]), steps // 8 + 1)  # coarse but stable: several refinements
    case = dict(case, args=tuple(case["args"][:4]) + (tl,))
    res1, info1 = _calibrated(case, 1)
    res3, info3 = _calibrated(case, 3)
    assert info1["steps"] == info3["steps"]
    d1, d3 = info1["details"], info3["details"]
    assert d1["status"] == d3["status"] == "converged"
    assert len(d1["tested"]) >= 2
    assert [t["steps"] for t in d1["tested"]] == [t["steps"] for t in d3["tested"]]
    assert [t["rms"] for t in d1["tested"]] == [t["rms"] for t in d3["tested"]]
    np.testing.assert_array_equal(res1, res3)


# ---- the reference's calibration tests (tests/test_gpu_solver.py:131-266): each calibrated run is
# checked against a fine-step reference map, not against another search mode.

from test_support_calls import CAL_PERIOD, calibration_oscillator_call, calibration_qubit_call  # noqa: E402

LIMITS = dict(rms_atol=1e-3, max_atol=1e-2, sample_stride=2)


def _within(result, reference, rms_limit, max_limit):
    error = np.abs(np.asarray(result) - np.asarray(reference))
    rms, worst = float(np.sqrt(np.mean(error ** 2))), float(error.max())
    assert rms <= rms_limit and worst <= max_limit, f"RMS {rms:.2e} (limit {rms_limit:g}), max {worst:.2e}"


def _qubit(steps_per_period, **options):
    import gqis
    args, kwargs = calibration_qubit_call(steps_per_period, **options)
    return gqis.mesolve_2D(*args, **kwargs)


@pytest.mark.gpu
def test_calibrated_timestep_meets_limits_against_fine_reference():
    """A too-coarse start (64 steps per period over 30 periods, 64 x 64 points) is refined until the
    map meets its limits against a 2048-steps-per-period run."""
    from gqis import solver
    wide = dict(periods=30, side=64, span=10.0)
    solver._TIMESTEP_CALIBRATION_CACHE.clear()
    reference = np.abs(_qubit(2048, **wide))
    result, timing = _qubit(64, **wide, calibrate_timesteps=dict(rms_atol=1e-3, max_atol=1e-2, sample_stride=8),
                            return_timing_info=True)
    assert timing["timestep_calibration"]["steps"] > 30 * 64  # the coarse start was refined
    _within(np.abs(result), reference, 1e-3, 1e-2)


@pytest.mark.gpu
@pytest.mark.parametrize("solver_name", ("rk4", "tsit5a"))
@pytest.mark.parametrize("output_mode", ("mean", "final", "final_rho"))
def test_calibration_meets_limits_for_every_lindblad_output(solver_name, output_mode):
    """The calibrated step count (rk4) or step tolerances (tsit5a) meet the limits for each output."""
    from gqis import solver
    solver._TIMESTEP_CALIBRATION_CACHE.clear()
    reference = _qubit(2048, output_mode=output_mode)
    result = _qubit(8, output_mode=output_mode, solver=solver_name, calibrate_timesteps=LIMITS)
    _within(result, reference, LIMITS["rms_atol"], LIMITS["max_atol"])


@pytest.mark.gpu
@pytest.mark.parametrize("solver_name", ("rk4", "tsit5a"))
def test_calibration_keeps_trace_sample_times(solver_name):
    """A calibrated trace is sampled at the times of the supplied grid and meets the limits there."""
    from gqis import solver
    solver._TIMESTEP_CALIBRATION_CACHE.clear()
    common = dict(output_mode="final", solver=solver_name, return_time_trace=True, time_trace_every=8)
    _, _, plain_times = _qubit(8, **common, ignore_non_finite_output=True)  # only its sample times are used
    result, trace, times, timing = _qubit(8, **common, calibrate_timesteps=LIMITS, return_timing_info=True)
    np.testing.assert_allclose(times, plain_times, rtol=1e-6)
    np.testing.assert_allclose(times, (np.arange(len(times)) * 8 + 1) * CAL_PERIOD / 8, rtol=1e-6)
    if solver_name == "rk4":
        assert timing["timestep_calibration"]["steps"] > 80  # the grid was refined
    reference, reference_trace, reference_times = _qubit(2048, output_mode="final", return_time_trace=True)
    picked = np.searchsorted(reference_times, times - 1e-6 * CAL_PERIOD)
    np.testing.assert_allclose(reference_times[picked], times, rtol=1e-5)
    _within(result, reference, LIMITS["rms_atol"], LIMITS["max_atol"])
    _within(trace, reference_trace[:, :, picked], LIMITS["rms_atol"], LIMITS["max_atol"])


@pytest.mark.gpu
@pytest.mark.parametrize("solver_name", ("rk4", "tsit5a"))
@pytest.mark.parametrize("output", ("final", "mean", "observable", "trace"))
def test_calibration_meets_limits_for_ode_outputs(solver_name, output):
    """odesolve_2D calibration for final and mean states, an observable and a state trace."""
    import gqis
    from gqis import solver
    if solver_name == "tsit5a" and output == "mean":
        pytest.skip("tsit5a averages with the trapezoidal rule over its own steps; on a coarse tlist that "
                    "quadrature error is not controlled by the step tolerance (as in the reference)")
    options = {"observable": dict(observable=True), "mean": dict(output_mode="mean"),
               "trace": dict(return_time_trace=True, time_trace_every=8), "final": {}}[output]
    limits = dict(rms_atol=1e-4, max_atol=1e-3, sample_stride=2)

    def run(steps, **extra):
        args, kwargs = calibration_oscillator_call(steps, **extra)
        return gqis.odesolve_2D(*args, **kwargs)
    solver._TIMESTEP_CALIBRATION_CACHE.clear()
    result = run(64, solver=solver_name, calibrate_timesteps=limits, **options)
    if output == "trace":
        _, trace, times = result
        _, fine_trace, fine_times = run(16384, return_time_trace=True)
        picked = np.searchsorted(fine_times, times - 1e-6)
        np.testing.assert_allclose(fine_times[picked], times, rtol=1e-5)
        _within(trace, fine_trace[:, :, picked], limits["rms_atol"], limits["max_atol"])
    elif output == "mean":  # reference: the exact time integral of a fine trace (trapezoid, from y0)
        _, fine_trace, fine_times = run(16384, return_time_trace=True)
        start = np.broadcast_to([1.0, 0.0], fine_trace.shape[:2] + (1, 2))
        states = np.concatenate([start, fine_trace], axis=2)
        reference = np.trapezoid(states, np.concatenate([[0.0], fine_times]), axis=2) / 20.0
        _within(result, reference, limits["rms_atol"], limits["max_atol"])
    else:
        _within(result, run(16384, **options), limits["rms_atol"], limits["max_atol"])
