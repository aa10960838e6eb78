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
