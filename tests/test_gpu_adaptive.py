"""Adaptive sweeps on the GPU: DOP853A / Tsit5A against the C oracle, schedule independence."""

import numpy as np
import pytest

import ode_oracle
from test_support_calls import duffing_case


def _run(args, kwargs):
    import gqis
    return gqis.odesolve_2D(*args, **kwargs)


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["dop853a", "tsit5a"])
def test_adaptive_duffing_matches_c_oracle(solver):
    """Same method, tolerances and output times as the C oracle (FP64): equal to rounding, except
    where rounding flips an accept/reject decision; the bar is 100x the step tolerance."""
    d, args, kwargs = duffing_case(solver=solver)
    final, trace, _, info = _run(args, dict(kwargs, return_timing_info=True))
    F, W = d["var_arrays"].values()
    o_final, o_trace, o_counts = ode_oracle.sweep(solver, F, W, d["y0_values"], d["tlist"], rtol=1e-8,
                                                  atol=1e-10, max_substeps=4000)
    assert np.max(np.abs(final - o_final)) < 1e-6
    assert np.max(np.abs(trace - o_trace)) < 1e-6
    same = info["adaptive_steps"]["accepted"] == o_counts[..., 0]
    assert same.mean() > 0.9


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["dop853a", "tsit5a"])
def test_work_stealing_results_do_not_depend_on_the_schedule(solver):
    """Each point's result is the same alone (static one-point-per-thread schedule) and in the mix
    (lanes refilled from the shared counter): bit for bit."""
    _, args, kwargs = duffing_case(solver=solver)
    stolen = _run(args, kwargs)
    static = _run(args, dict(kwargs, nvrtc_options=("-DGQ_STATIC_SCHEDULE=1",)))
    np.testing.assert_array_equal(stolen[0], static[0])
    np.testing.assert_array_equal(stolen[1], static[1])


@pytest.mark.gpu
def test_point_alone_equals_point_in_the_sweep():
    d, args, kwargs = duffing_case(solver="dop853a")
    full = _run(args, kwargs)[0]
    F, W = d["var_arrays"].values()
    (fs, ws) = list(d["var_arrays"])
    i, j = 5, 2
    alone_kwargs = dict(kwargs, var_arrays={fs: np.asarray(F)[i:i + 1], ws: np.asarray(W)[j:j + 1]},
                        y0_values=d["y0_values"][i:i + 1, j:j + 1])
    alone = _run(args, alone_kwargs)[0]
    np.testing.assert_array_equal(alone[0, 0], full[i, j])
