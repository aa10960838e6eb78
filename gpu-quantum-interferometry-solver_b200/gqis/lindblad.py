"""Symbolic Lindblad master equation in the reduced real layout.

A density matrix of dimension N is Hermitian with unit trace, so it is carried as
``S = N*N - 1`` real numbers (the layout of ``gqis/solver.py:202-250``, which the
generated kernels, ``rho0_values`` and ``final_rho`` outputs all share):

* ``rho[0] .. rho[N-2]``: the populations rho_00 .. rho_{N-2,N-2};
* then, for each upper-triangle element (i < j) in row-major order, its real part
  followed by its imaginary part.

rho_{N-1,N-1} is ``1 - sum(populations)``, and the lower triangle is the conjugate.
The right-hand side is

    d rho / dt = -i [H, rho] + sum_L ( L rho L^dag - 1/2 {L^dag L, rho} )

(``gqis/solver.py:452-457``), split into real and imaginary parts of the independent
elements. The sequence of SymPy transformations (expand, substitute the last
population, take real/imaginary parts, simplify coefficient by coefficient) follows
``gqis/solver.py:340-493`` step for step, because it decides the printed floating
literals and therefore the last bits of every generated kernel.
"""

from __future__ import annotations

import os

import numpy as np
import sympy as sp

HALF = sp.Float(0.5)  # the reference builds the anticommutator with a Float 1/2
PARALLEL_FROM_DIMENSION = 10  # "auto" symbolic workers start at this Hilbert dimension


def _pair_slot(N, i, j):
    """Position of the upper-triangle pair (i < j) among all N*(N-1)/2 pairs, row-major."""
    return i * N - (i * (i + 1)) // 2 + (j - i - 1)


def reduced_symbols(size):
    """The real state symbols ``rho[0] .. rho[size-1]`` used in generated code."""
    return [sp.Symbol(f"rho[{k}]", real=True) for k in range(size)]


def build_independent_rho(N):
    """Density matrix of dimension ``N`` written in the reduced real symbols.

    Returns ``(rho, meta)``: ``rho`` is an N x N SymPy matrix and ``meta`` holds
    ``N``, ``rho_syms``, ``num_diag``, ``num_coherences`` and ``vec_len``
    (the fields of ``gqis/solver.py:202-258``).
    """
    N = int(N)
    n_pop = N - 1
    n_pairs = N * (N - 1) // 2
    size = n_pop + 2 * n_pairs
    syms = reduced_symbols(size)
    last_pop = 1 - sum(syms[:n_pop])

    entries = {}
    for i in range(N):
        entries[(i, i)] = syms[i] if i < n_pop else last_pop
        for j in range(i + 1, N):
            k = n_pop + 2 * _pair_slot(N, i, j)
            upper = syms[k] + sp.I * syms[k + 1]
            entries[(i, j)] = upper
            entries[(j, i)] = sp.conjugate(upper)
    rho = sp.Matrix(N, N, lambda i, j: entries[(i, j)])
    meta = {"N": N, "rho_syms": syms, "num_diag": n_pop, "num_coherences": n_pairs,
            "vec_len": size}
    return rho, meta


def rho_matrix_to_independent_exprs(rho0):
    """Reduced real vector of an initial density matrix (or a reduced vector as given).

    A square matrix gives its first N-1 populations and then (Re, Im) of the upper
    triangle; an iterable of length N*N-1 is taken as already reduced
    (``gqis/solver.py:261-290``).
    """
    if isinstance(rho0, sp.MatrixBase):
        rows, cols = rho0.shape
        if rows != cols:
            raise ValueError("rho0 matrix must be square.")
        out = [sp.simplify(sp.re(rho0[i, i])) for i in range(rows - 1)]
        for i in range(rows):
            for j in range(i + 1, rows):
                out.append(sp.simplify(sp.re(rho0[i, j])))
                out.append(sp.simplify(sp.im(rho0[i, j])))
        return out
    values = list(rho0)
    N = int(round(np.sqrt(len(values) + 1)))
    if N * N - 1 != len(values):
        raise ValueError("rho0 reduced vector length must match N*N-1.")
    return [sp.simplify(sp.sympify(v)) for v in values]


def simplify_affine(expr, states):
    """Simplify each state coefficient of an affine expression on its own.

    A whole-expression ``simplify`` would put drive-dependent terms over a common
    denominator and cost an extra multiplication per term in every RHS evaluation.
    Non-affine expressions are simplified as a whole (``gqis/solver.py:325-337``).
    """
    parts = sp.collect(sp.expand(expr), states, evaluate=False)
    if any(key != 1 and key not in states for key in parts):
        return sp.simplify(expr)
    terms = []
    for key, coeff in parts.items():
        terms.append((coeff if coeff.is_number else sp.simplify(coeff)) * key)
    return sp.Add(*terms)


def _finish(expr, pre_expand):
    return sp.expand(expr) if pre_expand else expr


def _element_equations(N, H, Col_Ops, rows, pre_expand, collect_rho):
    """Equations of the density-matrix rows ``rows`` (one symbolic worker's share).

    Element (i, j) is built from row i of H, rho and the collapse terms exactly as the
    whole-matrix form does, so the equations are identical to ``_whole_matrix_equations``.
    Returns ``{(i, j): [re] or [re, im]}``.
    """
    rho, meta = build_independent_rho(N)
    states = meta["rho_syms"]
    last_pop = 1 - sum(rho[k, k] for k in range(N - 1))
    ops = [(L, L.H, L.H * L) for L in Col_Ops]
    out = {}
    for i in rows:
        H_row, rho_row = H[i, :], rho[i, :]
        L_rho_rows = [L[i, :] * rho for L, _, _ in ops]
        for j in range(i, N):
            val = -sp.I * ((H_row * rho[:, j])[0] - (rho_row * H[:, j])[0])
            diss = sp.Integer(0)
            for (L, Ld, LdL), L_rho_row in zip(ops, L_rho_rows):
                diss += ((L_rho_row * Ld[:, j])[0]
                         - HALF * ((LdL[i, :] * rho[:, j])[0] + (rho_row * LdL[:, j])[0]))
            val = _finish(val + diss, pre_expand)
            val = _finish(val.subs(rho[N - 1, N - 1], last_pop), pre_expand)
            pieces = [sp.re(val)] if i == j else [sp.re(val), sp.im(val)]
            pieces = [simplify_affine(_finish(p, pre_expand), states) for p in pieces]
            if collect_rho:
                pieces = [sp.collect(p, states) for p in pieces]
            out[(i, j)] = pieces
    return out


def _worker_count(N, symbolic_workers, max_symbolic_workers):
    """Processes for the row-parallel derivation: at most one per row (N - 1)."""
    if max_symbolic_workers is None:
        max_symbolic_workers = max(1, (os.cpu_count() or 2) // 2)
    if int(max_symbolic_workers) < 1:
        raise ValueError("max_symbolic_workers must be a positive integer or None.")
    if symbolic_workers in (None, "auto"):
        n = int(max_symbolic_workers) if N >= PARALLEL_FROM_DIMENSION else 1
    elif isinstance(symbolic_workers, str) or int(symbolic_workers) < 1:
        raise ValueError('symbolic_workers must be "auto" or a positive integer.')
    else:
        n = int(symbolic_workers)
    return max(1, min(n, N - 1))


def build_reduced_lindblad_rhs(N, H, Col_Ops, mean_operator, *, pre_expand=False,
                               collect_rho=False, factor_terms=False, symbolic_workers=1,
                               max_symbolic_workers=None):
    """Real ODE of the reduced density vector and the observable's real/imag parts.

    Returns ``(drho_eqs, mean_re, mean_im, meta)`` with ``len(drho_eqs) == N*N - 1``
    (interface of ``gqis/solver.py:399-493``). ``symbolic_workers > 1`` derives
    the rows in separate processes (spawned, so it is safe after CUDA use); the
    equations are identical either way.
    """
    N = int(N)
    rho, meta = build_independent_rho(N)
    states = meta["rho_syms"]
    mean_val = sp.simplify(sp.Trace(mean_operator * rho))
    mean_re = sp.simplify(sp.re(mean_val))
    mean_im = sp.simplify(sp.im(mean_val))

    workers = _worker_count(N, symbolic_workers, max_symbolic_workers)
    if workers > 1 and not factor_terms:
        import multiprocessing
        from concurrent.futures import ProcessPoolExecutor
        shares = [list(range(w, N - 1, workers)) for w in range(workers)]
        shares = [s for s in shares if s]
        ctx = multiprocessing.get_context("spawn")
        elements = {}
        with ProcessPoolExecutor(max_workers=len(shares), mp_context=ctx) as pool:
            jobs = [pool.submit(_element_equations, N, H, list(Col_Ops), share, pre_expand,
                                collect_rho) for share in shares]
            for job in jobs:
                elements.update(job.result())
        eqs = [elements[(i, i)][0] for i in range(N - 1)]
        for i in range(N - 1):
            for j in range(i + 1, N):
                eqs.extend(elements[(i, j)])
        return eqs, mean_re, mean_im, meta

    # Commutator and dissipator are summed separately and then added, as in the reference:
    # SymPy merges Float coefficients in summation order, so the order is kept.
    commutator = -sp.I * (H * rho - rho * H)
    dissipator = sp.zeros(N)
    for L in Col_Ops:
        Ld = L.H
        LdL = Ld * L
        dissipator += L * rho * Ld - HALF * (LdL * rho + rho * LdL)
    full = commutator + dissipator
    if pre_expand:
        full = sp.expand(full)
    if factor_terms:
        full = sp.factor_terms(full, clear=True)
    last_pop = 1 - sum(rho[k, k] for k in range(N - 1))
    full = full.subs(rho[N - 1, N - 1], last_pop)
    if pre_expand:
        full = sp.expand(full)
    if factor_terms:
        full = sp.factor_terms(full, clear=True)

    eqs = [_finish(sp.re(full[i, i]), pre_expand) for i in range(N - 1)]
    for i in range(N):
        for j in range(i + 1, N):
            eqs.append(_finish(sp.re(full[i, j]), pre_expand))
            eqs.append(_finish(sp.im(full[i, j]), pre_expand))
    eqs = [simplify_affine(_finish(e, pre_expand), states) for e in eqs]
    if factor_terms:
        eqs = [sp.factor_terms(e, clear=True) for e in eqs]
    if collect_rho:
        eqs = [sp.collect(e, states) for e in eqs]
    return eqs, mean_re, mean_im, meta
