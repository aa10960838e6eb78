"""CPU tests of the matrix-form decomposition (gqis/matrix_form.py), no GPU.

The kernel's RHS is restated here in NumPy from the decomposed operator data (Heff0, dense and
diagonal terms, element-wise and listed jump terms) and compared with the matrix-form oracle's
RHS, d rho/dt = -i[H, rho] + sum_L (L rho L^dag - 1/2 {L^dag L, rho}), on random Hermitian
states: this pins the decomposition the module is generated from.
"""

import numpy as np
import pytest
import sympy as sp

import lindblad_oracle
from gqis import matrix_form
from gqis.rhs import runtime_const_values


def kernel_rhs(mm, X, Y, t, consts, rho):
    """The RHS of csrc/gqis_matrix.cuh on one padded state, from the module's data."""
    H, c = matrix_form.dense_operators(mm, X, Y, t, consts)
    K = H @ rho
    out = -1j * (K - K.conj().T) + mm.wjump * rho
    flat, src = out.reshape(-1), rho.reshape(-1)
    for dst, s, coef, rate in mm.jumps:
        flat[dst] += coef * (c[rate] if rate >= 0 else 1.0) * src[s]
    return out


def random_state(N, Np, rng):
    G = rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))
    rho = G @ G.conj().T
    rho /= np.trace(rho)
    out = np.zeros((Np, Np), dtype=complex)
    out[:N, :N] = rho
    return out


def _compare(mm, oracle, consts, rng, N):
    oracle.superop = False  # the oracle's explicit matrix RHS
    P = oracle.H_static.shape[0]
    for p in (0, P - 1):
        X = float(oracle.params[0][p])
        Y = float(oracle.params[1][p]) if len(oracle.params) > 1 else 0.0
        for t in (0.0, 0.37, 2.5):
            rho = random_state(N, mm.Np, rng)
            H = oracle.hamiltonian(t)
            ref = oracle.rhs(H[p:p + 1], rho[None, :N, :N])[0]
            got = kernel_rhs(mm, X, Y, t, consts, rho)
            assert np.max(np.abs(got[:N, :N] - ref)) < 1e-12
            assert np.all(got[N:, :] == 0) and np.all(got[:, N:] == 0)


def test_n_level_decomposition_matches_oracle_rhs():
    from gqis import workloads
    rng = np.random.default_rng(1)
    for N in (8, 16):
        w = workloads.n_level(N, side=3)
        mm, _ = matrix_form.compile_matrix_model(w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"],
                                                 sweep_symbols=tuple(w["var_arrays"]))
        assert (mm.num_dense, mm.num_diag) == (1, 1)  # A cos(t) X dense, eps diag(0..N-1) diagonal
        assert len(mm.jumps) == N - 1                 # lowering: rho_kk -> (k-1, k-1)
        oracle = lindblad_oracle.from_workload(w, {k: v[:2] for k, v in w["var_arrays"].items()})
        _compare(mm, oracle, [], rng, N)


def test_runtime_constant_rates_and_hamiltonian_terms():
    eps, A, D, Drive, t, G1, Gp = sp.symbols("eps A Delta Drive t Gamma1 Gammaphi", real=True)
    sz, sx, sm = sp.Matrix([[1, 0], [0, -1]]), sp.Matrix([[0, 1], [1, 0]]), sp.Matrix([[0, 1], [0, 0]])
    H = eps / 2 * sz + D / 2 * sx + Drive * sz
    col = [sp.sqrt(G1) * sm, sp.sqrt(Gp / 2) * sz]
    var = {eps: np.array([-1.0, 0.5]), A: np.array([0.2, 1.5])}
    rc = {G1: 0.013, Gp: 0.021, D: 0.9}
    mm, _ = matrix_form.compile_matrix_model(H, A * sp.cos(sp.pi * t), col, sp.diag(0, 1),
                                             sweep_symbols=tuple(var), runtime_consts=rc)
    assert any(r >= 0 for _, _, _, r in mm.jumps)  # the Gamma1 jump term carries its runtime rate
    consts = runtime_const_values(mm, rc, {}, use_defaults=True)
    oracle = lindblad_oracle.MatrixModel(H, A * sp.cos(sp.pi * t), col, sp.diag(0, 1), var, const_values=rc)
    _compare(mm, oracle, consts, np.random.default_rng(2), 2)


def test_padding_and_tiles():
    assert [matrix_form.padded_dimension(n) for n in (2, 8, 9, 16, 17, 33, 64)] == [8, 8, 16, 16, 32, 48, 64]
    for Np in (8, 16, 32, 48, 64):
        TR, TC, threads = matrix_form.tile_shape(Np)
        assert threads % 32 == 0 and threads <= 1024 and Np % TR == 0 and Np % TC == 0
    with pytest.raises(ValueError):
        matrix_form.padded_dimension(65)


def test_unsupported_models_are_rejected():
    a, b, eps = sp.symbols("a b eps", real=True)
    H = sp.diag(eps, 0, 0)
    two_factor = [a * sp.Matrix([[0, 1, 0], [0, 0, 0], [0, 0, 0]]) + b * sp.Matrix([[0, 0, 0], [0, 0, 1], [0, 0, 0]])]
    with pytest.raises(ValueError, match="scalar times a numeric"):
        matrix_form.compile_matrix_model(H, 0, two_factor, sp.eye(3), sweep_symbols=(eps,),
                                         runtime_consts={a: 0.1, b: 0.2}, reuse=False)
    with pytest.raises(ValueError, match="numeric mean operator"):
        matrix_form.compile_matrix_model(H, 0, [], sp.diag(eps, 0, 0), sweep_symbols=(eps,), reuse=False)


def test_emitted_source_shape():
    from gqis import workloads
    w = workloads.n_level(16, side=2)
    mm, _ = matrix_form.compile_matrix_model(w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"],
                                             sweep_symbols=tuple(w["var_arrays"]))
    src = matrix_form.module_source(mm, "fp32", "mean", False)
    assert "#define GQ_MATRIX 1" in src and "using mreal = float;" in src
    assert "c[0] = ParY*gq::cos(t);" in src and "c[1] = ParX;" in src
    assert "TR = 2, TC = 2, THREADS = 64;" in src
    with pytest.raises(ValueError):
        matrix_form.module_source(mm, "fp64", "mean_state", False)


def test_tensor_core_jump_lists_of_a_dephased_qubit():
    """sigma_z dephasing at a runtime rate acts element-wise on the coherences: those terms read the
    thread's own element; relaxation feeds the ground population from the excited one."""
    from gqis.rhs import runtime_const_values  # noqa: F401  (model preparation path)
    eps, A, D, Drive, t, G1, Gp = sp.symbols("eps A Delta Drive t Gamma1 Gammaphi", real=True)
    sz, sx, sm = sp.Matrix([[1, 0], [0, -1]]), sp.Matrix([[0, 1], [1, 0]]), sp.Matrix([[0, 1], [0, 0]])
    mm, _ = matrix_form.compile_matrix_model(eps / 2 * sz + D / 2 * sx + Drive * sz, A * sp.cos(t),
                                             [sp.sqrt(G1) * sm, sp.sqrt(Gp / 2) * sz], sp.diag(0, 1),
                                             sweep_symbols=(eps, A), runtime_consts={G1: 0.01, Gp: 0.02, D: 1.0},
                                             reuse=False)
    lists, own = matrix_form.tensor_core_jump_lists(mm)
    assert own
    col1 = lists[1][0]  # column 1: rows 0 and 1
    assert any(e == 0 and a == -1 and r >= 0 for e, a, c, r in col1)  # coherence (0, 1): own element, rate
    assert any(e == 1 and a == 1 for e, a, c, r in col1)               # population (1, 1) from itself
    assert any(e == 0 and a == 1 for e, a, c, r in lists[0][0])        # (0, 0) fed by rho_11 (relaxation)
    assert matrix_form.tensor_core_blockers(mm, "fp32") == []


def test_tensor_core_shape_of_the_two_cta_kernel():
    """N = 64 splits each tile's rows over a cluster of two CTAs: half the B columns per CTA, and the
    shared memory (B in two FP16 parts, transposed K, exchange buffer) fits one CTA up to the widest
    MMA (256 columns: three dense operators, the diagonal one then in the epilogue); more dense
    operators exceed one MMA."""
    from types import SimpleNamespace
    import numpy as np

    def fake(Np, dense, diag):
        return SimpleNamespace(Np=Np, num_dense=dense, num_diag=diag, coef_exprs=[0] * (dense + diag),
                               jumps=[], wjump=np.zeros((Np, Np)))
    cl, nh, nmma, smem = matrix_form.tensor_core_shape(fake(64, 1, 1))
    assert (cl, nh, nmma) == (2, 32, 192) and smem <= matrix_form.SMEM_LIMIT  # diagonal on the MMA
    assert matrix_form.tensor_core_blockers(fake(64, 1, 1), "fp32") == []
    assert matrix_form.tensor_core_shape(fake(32, 1, 1))[:3] == (1, 32, 192)  # diagonal on the MMA
    assert matrix_form.tensor_core_shape(fake(32, 3, 1))[:3] == (1, 32, 256)  # 320 columns: in the epilogue
    assert matrix_form.tensor_core_shape(fake(16, 1, 1))[:3] == (1, 16, 96)   # diagonal on the MMA
    assert matrix_form.tensor_core_blockers(fake(64, 3, 1), "fp32") == []  # 2 x 32 x 4 = 256 columns
    cl, nh, nmma, smem = matrix_form.tensor_core_shape(fake(64, 3, 1))
    assert nmma == 256 and smem <= matrix_form.SMEM_LIMIT
    assert "exceed one MMA" in matrix_form.tensor_core_blockers(fake(64, 4, 1), "fp32")[0]
    assert matrix_form.tensor_core_blockers(fake(32, 3, 1), "fp32") == []  # 2 x 32 x 4 = 256 columns
    assert "exceed one MMA" in matrix_form.tensor_core_blockers(fake(32, 4, 1), "fp32")[0]
    assert "padded dimension 48" in matrix_form.tensor_core_blockers(fake(48, 1, 1), "fp32")[0]


def test_tensor_core_module_flags_a_diagonal_observable():
    """The tensor-core kernel reads a diagonal observable only in the threads that hold diagonal
    elements (kObsDiagonal); an observable with coherences takes the general path."""
    from gqis import workloads
    w = workloads.n_level(16, side=2)
    for O, diagonal in ((w["mean_operator"], True), (w["mean_operator"] + sp.Matrix(16, 16, lambda i, j: 1 if abs(i - j) == 1 else 0), False)):
        mm, _ = matrix_form.compile_matrix_model(w["H"], w["Drive"], w["Col_Ops"], O,
                                                 sweep_symbols=tuple(w["var_arrays"]), reuse=False)
        src = matrix_form.module_source(mm, "fp32", "mean", False, tensor_cores=True)
        assert f"kObsDiagonal = {'true' if diagonal else 'false'};" in src
