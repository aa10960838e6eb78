"""Failures made on the host, checked on the GPU (no device fault, trap or hang is involved): an
adaptive substep cap too small for the tolerance marks points NaN and the call raises; a NaN sweep
parameter poisons only its own points."""

import numpy as np
import pytest

import ref_cases
from test_support_calls import duffing_case


@pytest.mark.gpu
def test_adaptive_substep_cap_marks_points_nan_and_raises():
    import gqis
    _, args, kwargs = duffing_case(solver="tsit5a")
    kwargs = dict(kwargs, adaptive_options=dict(kwargs["adaptive_options"], max_substeps=1))
    with pytest.raises(RuntimeError, match="Non-finite"):
        gqis.odesolve_2D(*args, **kwargs)
    out = gqis.odesolve_2D(*args, **kwargs, ignore_non_finite_output=True)
    final = out[0] if isinstance(out, tuple) else out
    assert np.isnan(np.asarray(final, dtype=np.float64)).any()


@pytest.mark.gpu
def test_nan_parameter_poisons_only_its_points():
    import gqis
    case = ref_cases.cases()["c2_fp64_mean_sub32"]
    clean = gqis.mesolve_2D(*case["args"], **case["kwargs"])
    va = dict(case["kwargs"]["var_arrays"])
    first = list(va)[0]
    axis = np.array(va[first], dtype=np.float64)
    axis[5] = np.nan
    va[first] = axis
    bad = dict(case["kwargs"], var_arrays=va)
    with pytest.raises(RuntimeError, match="Non-finite"):
        gqis.mesolve_2D(*case["args"], **bad)
    out = gqis.mesolve_2D(*case["args"], **bad, ignore_non_finite_output=True)
    assert np.isnan(out[5].real).all()
    np.testing.assert_array_equal(np.delete(out, 5, axis=0), np.delete(clean, 5, axis=0))


@pytest.mark.gpu
def test_tensor_core_mma_wait_that_runs_out_marks_the_tile_nan_and_raises():
    """The tensor-core kernel's waits for its MMAs are bounded. A build whose in-loop poll limit is 0
    (no wait can succeed; the final wait for the MMA in flight keeps its full limit) takes the
    give-up path on every tile: the CTA stops integrating, waits for the MMA it issued, writes NaN
    for its points and frees its tensor memory. The call then raises like any non-finite map, and
    the same process runs the ordinary kernel correctly afterwards."""
    import gqis
    from test_support_calls import GIVE_UP, hilbert_model
    _, args, kwargs = hilbert_model(16)
    common = dict(kwargs, precision="fp32", rhs_form="matrix_tc")
    with pytest.raises(RuntimeError, match="Non-finite"):
        gqis.mesolve_2D(*args, **common, nvrtc_options=GIVE_UP)
    lost = gqis.mesolve_2D(*args, **common, nvrtc_options=GIVE_UP, ignore_non_finite_output=True)
    assert np.isnan(np.asarray(lost).real).all()
    good = gqis.mesolve_2D(*args, **common)
    assert np.isfinite(good).all()
    reference = gqis.mesolve_2D(*args, **dict(kwargs, precision="fp64", rhs_form="matrix"))
    assert float(np.max(np.abs(good - reference))) <= 5e-6
