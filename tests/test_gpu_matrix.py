"""GPU tests of the density-matrix (matrix-form) kernel, csrc/gqis_matrix.cuh.

* FP64 against the reduced-form kernel on the same N = 8 model (two independent derivations of
  one master equation): 1e-12 max-abs;
* FP64 against the matrix-form CPU oracle (oracle/lindblad_oracle.py) at N = 16, 32, 64:
  1e-11 max-abs on <O> maps whose entries are O(1e-5 .. 1);
* the FP32 form against the same oracle: 2e-6 max-abs;
* final_rho in the reduced layout, and rho0_values read back from it (a run split in two
  equals the run in one piece);
* rhs_form="auto" picks the matrix form from N = 8 on (tensor cores for FP32);
* the tensor-core kernel (split-FP16 tcgen05 MMAs, FP32 accumulation and state) against the same
  oracle at N = 8, 16, 32: 5e-6 max-abs, and within 5e-6 of the CUDA-core FP32 form; final_rho
  through it as well. The grids leave the last tile of points partly empty.
"""

import numpy as np
import pytest

import lindblad_oracle
from test_support_calls import MATRIX_DIMS, TENSOR_DIMS, hilbert_model, serving_model


def _oracle(w, kwargs, output_mode="mean", rho0=None, t_in=0.0):
    model = lindblad_oracle.from_workload(w, kwargs["var_arrays"])
    return lindblad_oracle.rk4_sweep(model, w["tlist"], output_mode=output_mode, rho0=rho0, t_in=t_in)


@pytest.mark.gpu
def test_matrix_form_matches_reduced_form_n8():
    import gqis
    args, kwargs = serving_model(8, 6)
    tl = np.linspace(0.0, 5.0, 101)
    args = args[:4] + (tl,)
    red = gqis.mesolve_2D(*args, **kwargs, fp64=True, rhs_form="reduced")
    mat = gqis.mesolve_2D(*args, **kwargs, fp64=True, rhs_form="matrix")
    assert np.max(np.abs(mat - red)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("N", MATRIX_DIMS)
def test_matrix_form_fp64_vs_oracle(N):
    import gqis
    w, args, kwargs = hilbert_model(N)
    got, info = gqis.mesolve_2D(*args, **kwargs, fp64=True, rhs_form="matrix", return_timing_info=True)
    assert info["rhs_form"] == "matrix"
    ref = _oracle(w, kwargs)
    assert np.max(np.abs(ref)) > 1e-5  # a non-trivial map (the top level fills slowly at N = 64)
    err = float(np.max(np.abs(got - ref)))
    assert err <= 1e-11, f"N={N}: FP64 matrix form max-abs error {err:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("N", MATRIX_DIMS)
def test_matrix_form_fp32_accuracy(N):
    import gqis
    w, args, kwargs = hilbert_model(N)
    got = gqis.mesolve_2D(*args, **kwargs, precision="fp32", rhs_form="matrix")
    err = float(np.max(np.abs(got - _oracle(w, kwargs))))
    assert err <= 2e-6, f"N={N}: FP32 matrix form max-abs error {err:.3e}"


@pytest.mark.gpu
def test_matrix_form_final_rho_and_rho0_values_continuation():
    import gqis
    w, args, kwargs = hilbert_model(16)
    full = gqis.mesolve_2D(*args, **kwargs, fp64=True, rhs_form="matrix", output_mode="final_rho")
    ref = _oracle(w, kwargs, output_mode="final_rho")
    assert full.shape == (4, 3, 255)
    assert np.max(np.abs(full - ref)) <= 1e-11
    tl = w["tlist"]
    half = len(tl) // 2
    first = gqis.mesolve_2D(*args[:4], tl[:half + 1], **kwargs, fp64=True, rhs_form="matrix",
                            output_mode="final_rho")
    second = gqis.mesolve_2D(*args[:4], tl[:len(tl) - half], **kwargs, fp64=True, rhs_form="matrix",
                             output_mode="final_rho", rho0_values=first, t_in=float(tl[half]))
    assert np.max(np.abs(second - full)) <= 1e-12


@pytest.mark.gpu
def test_auto_picks_reduced_below_n8_and_matrix_from_n8():
    import gqis
    args4, kwargs4 = serving_model(4, 8)
    _, info = gqis.mesolve_2D(*args4, **kwargs4, precision="fp32", return_timing_info=True)
    assert info["rhs_form"] == "reduced"
    w, args, kwargs = hilbert_model(8)
    _, info = gqis.mesolve_2D(*args, **kwargs, precision="fp32", return_timing_info=True)
    assert info["rhs_form"] == "matrix_tc"
    _, info = gqis.mesolve_2D(*args, **kwargs, precision="fp64", return_timing_info=True)
    assert info["rhs_form"] == "matrix"


@pytest.mark.gpu
@pytest.mark.parametrize("N", TENSOR_DIMS)
def test_tensor_core_form_vs_oracle(N):
    import gqis
    w, args, kwargs = hilbert_model(N)
    got, info = gqis.mesolve_2D(*args, **kwargs, precision="fp32", rhs_form="matrix_tc", return_timing_info=True)
    assert info["rhs_form"] == "matrix_tc"
    ref = _oracle(w, kwargs)
    err = float(np.max(np.abs(got - ref)))
    cuda = gqis.mesolve_2D(*args, **kwargs, precision="fp32", rhs_form="matrix")
    assert err <= 5e-6, f"N={N}: tensor-core form max-abs error {err:.3e}"
    assert float(np.max(np.abs(got - cuda))) <= 5e-6


@pytest.mark.gpu
@pytest.mark.parametrize("N", [16, 64])
def test_tensor_core_form_final_rho(N):
    """The final state in the reduced layout; at N = 64 each CTA of the cluster writes its half of the rows."""
    import gqis
    w, args, kwargs = hilbert_model(N)
    got = gqis.mesolve_2D(*args, **kwargs, precision="fp32", rhs_form="matrix_tc", output_mode="final_rho")
    ref = _oracle(w, kwargs, output_mode="final_rho")
    assert got.shape == ref.shape
    assert float(np.max(np.abs(got - ref))) <= 5e-6


@pytest.mark.gpu
@pytest.mark.parametrize("form,tc", [("fp64", False), ("fp32", False), ("fp32", True)])
def test_matrix_forms_with_runtime_rates_one_axis_and_rho0(form, tc):
    """Runtime-constant collapse rates and Hamiltonian terms (the fit model), a one-axis sweep, a
    numeric initial state and the `final` output, through the matrix kernels, against the reduced
    form (FP64) of the same call."""
    import sympy as sp
    import gqis
    from test_support_calls import qubit_fit_model
    args, kwargs, (G1, Gp, D, A) = qubit_fit_model(side=(9, 5), steps=200, duration=10.0)
    rho0 = sp.Matrix([[0.7, 0.2 - 0.1j], [0.2 + 0.1j, 0.3]])
    eps = list(kwargs["var_arrays"])[0]
    one_axis = dict(kwargs, var_arrays={eps: kwargs["var_arrays"][eps]}, rho0=rho0)
    args1 = (args[0], args[1].subs(A, 0.8)) + args[2:]  # the drive amplitude fixed: one swept axis (eps)
    for mode in ("mean", "final"):
        ref = gqis.mesolve_2D(*args1, **one_axis, output_mode=mode, fp64=True, rhs_form="reduced")
        got = gqis.mesolve_2D(*args1, **one_axis, output_mode=mode, precision=form,
                              rhs_form="matrix_tc" if tc else "matrix")
        assert got.shape == ref.shape == (9, 1)
        tol = 1e-12 if form == "fp64" else 2e-6
        assert float(np.max(np.abs(got - ref))) <= tol, (mode, float(np.max(np.abs(got - ref))))


@pytest.mark.gpu
@pytest.mark.parametrize("form,rhs_form,tol", [("fp64", "matrix", 1e-12), ("fp32", "matrix", 2e-6),
                                               ("fp32", "matrix_tc", 2e-6)])
def test_matrix_forms_record_the_observable_trace(form, rhs_form, tol):
    """return_time_trace through the density-matrix kernels: the same samples (every k-th step) as the
    reduced form's trace (FP64), and the same final map."""
    import gqis
    args, kwargs = serving_model(8, 6)
    args = args[:4] + (np.linspace(0.0, 5.0, 101),)
    ref_map, ref_tr, ref_t = gqis.mesolve_2D(*args, **kwargs, fp64=True, rhs_form="reduced",
                                             return_time_trace=True, time_trace_every=7)
    got_map, got_tr, got_t = gqis.mesolve_2D(*args, **kwargs, precision=form, rhs_form=rhs_form,
                                             return_time_trace=True, time_trace_every=7)
    assert got_tr.shape == ref_tr.shape == (6, 6, 15)
    np.testing.assert_allclose(got_t, ref_t, rtol=1e-6)
    assert float(np.max(np.abs(got_tr - ref_tr))) <= tol
    assert float(np.max(np.abs(got_map - ref_map))) <= tol


@pytest.mark.gpu
def test_two_cta_tensor_core_kernel_records_the_trace():
    """N = 64 runs on a cluster of two CTAs per tile whose point sums meet through distributed shared
    memory: its observable trace (every 9th step) against the FP64 CUDA-core matrix form."""
    import gqis
    w, args, kwargs = hilbert_model(64)
    trace = dict(kwargs, return_time_trace=True, time_trace_every=9)
    ref_map, ref_tr, ref_t = gqis.mesolve_2D(*args, **trace, fp64=True, rhs_form="matrix")
    got_map, got_tr, got_t = gqis.mesolve_2D(*args, **trace, precision="fp32", rhs_form="matrix_tc")
    assert got_tr.shape == ref_tr.shape and got_tr.shape[2] == 12
    np.testing.assert_allclose(got_t, ref_t, rtol=1e-6)
    assert float(np.max(np.abs(ref_tr))) > 1e-4  # the top level's population grows to ~1e-3 by t = 5
    assert float(np.max(np.abs(got_tr - ref_tr))) <= 5e-6
    assert float(np.max(np.abs(got_map - ref_map))) <= 5e-6


@pytest.mark.gpu
def test_dimension_40_runs_on_the_tensor_cores_padded_to_64():
    """A model of dimension 33 .. 48 pads to 64 for the tensor-core kernel (its rows and columns past
    N stay zero), while the FP64 CUDA-core form keeps the 48-wide tile: both equal the oracle."""
    import gqis
    w, args, kwargs = hilbert_model(40)
    tc, info = gqis.mesolve_2D(*args, **kwargs, precision="fp32", return_timing_info=True)
    assert info["rhs_form"] == "matrix_tc"
    fp64 = gqis.mesolve_2D(*args, **kwargs, fp64=True, rhs_form="matrix")
    ref = _oracle(w, kwargs)
    assert float(np.max(np.abs(fp64 - ref))) <= 1e-11
    assert float(np.max(np.abs(tc - ref))) <= 2e-6


@pytest.mark.gpu
def test_tensor_core_split_fp16_keeps_entries_far_below_a_terms_largest():
    """The split-FP16 operands are scaled per operator term by the term's largest entry: level energies
    up to 45.5 share Heff0 with couplings of 2e-3 and decay terms of 5e-5 (below the smallest normal
    FP16 number unscaled), and the drive operator holds 1 beside 3e-4. The decay terms move the driven
    population (level 1) by more than 1e-4; the tensor-core form matches the FP64 form there to 2e-6,
    and the population fed only by the small couplings (level 2) to 1% of its size."""
    import gqis
    from test_support_calls import wide_range_model

    def run(level, tc, decay=True):
        args, kwargs = wide_range_model(level, decay)
        form = dict(precision="fp32", rhs_form="matrix_tc") if tc else dict(fp64=True, rhs_form="matrix")
        return gqis.mesolve_2D(*args, **kwargs, **form)

    ref1 = run(1, False)
    assert np.max(np.abs(ref1)) > 0.05  # the resonant drive moves level 1
    assert float(np.max(np.abs(ref1 - run(1, False, decay=False)))) > 1e-4  # the decay terms matter
    assert float(np.max(np.abs(run(1, True) - ref1))) <= 2e-6
    ref2 = run(2, False)
    assert 1e-8 < float(np.max(np.abs(ref2))) < 1e-3  # fed by the small couplings only
    assert float(np.max(np.abs(run(2, True) - ref2))) <= 1e-2 * float(np.max(np.abs(ref2)))


@pytest.mark.gpu
def test_tensor_core_diagonal_terms_in_the_epilogue():
    """Three dense drive operators and a diagonal term at N = 20 (padded to 32) need 320 MMA columns,
    so the tensor-core kernel adds the diagonal term in its epilogue from each point's sums, which
    all threads form in shared memory while the MMA runs: the map equals the FP64 form to 5e-6."""
    import gqis
    from gqis import matrix_form
    from test_support_calls import epilogue_diagonal_model
    args, kwargs = epilogue_diagonal_model()
    mm, _ = matrix_form.compile_matrix_model(*args[:4], sweep_symbols=tuple(kwargs["var_arrays"]))
    assert (mm.num_dense, mm.num_diag) == (3, 1) and not matrix_form.diag_in_mma(mm)
    ref = gqis.mesolve_2D(*args, **kwargs, fp64=True, rhs_form="matrix")
    got = gqis.mesolve_2D(*args, **kwargs, precision="fp32", rhs_form="matrix_tc")
    assert np.max(np.abs(ref)) > 1e-6
    assert float(np.max(np.abs(got - ref))) <= 5e-6


@pytest.mark.gpu
@pytest.mark.parametrize("N", [16, 64])
def test_tensor_core_form_with_an_offdiagonal_observable(N):
    """An observable with coherences (the kernel's general observable path; a diagonal observable is
    read only by the threads that hold diagonal elements): the tensor-core map equals the FP64 form
    to 5e-6, one CTA per tile (N = 16) and on two-CTA clusters (N = 64)."""
    import gqis
    from gqis import matrix_form
    from test_support_calls import offdiagonal_observable_model
    args, kwargs = offdiagonal_observable_model(N)
    ref = gqis.mesolve_2D(*args, **kwargs, fp64=True, rhs_form="matrix")
    got = gqis.mesolve_2D(*args, **kwargs, precision="fp32", rhs_form="matrix_tc")
    assert np.max(np.abs(ref.imag)) > 1e-6 or np.max(np.abs(ref.real)) > 1e-3  # a non-trivial map
    assert float(np.max(np.abs(got - ref))) <= 5e-6
