"""Density-matrix ("matrix form") Lindblad sweeps for larger Hilbert spaces.

The reduced real form (``lindblad.py``, the reference's only form, ``gqis/solver.py:340-493``)
derives N*N-1 scalar equations with SymPy; from N ~ 16 on that derivation takes minutes and the
equations no longer fit a thread's registers. The matrix form keeps the model as numeric
operators instead:

    H(t) = sum_s f_s(t, X, Y, consts) * M_s       (affine split of every H entry)
    L_k  = g_k(X, Y, consts) * Lhat_k              (one scalar factor per collapse operator)
    d rho/dt = -i (H_eff rho - rho H_eff^dag) + sum_k |g_k|^2 Lhat_k rho Lhat_k^dag,
    H_eff = H - i/2 sum_k |g_k|^2 Lhat_k^dag Lhat_k,

which is the same master equation (``gqis/solver.py:452-457``). Terms whose factor is a number
are folded into one constant matrix ``Heff0``; factors that depend on the sweep parameters,
the drives or runtime constants become coefficient functions evaluated in FP64 on the GPU at
each stage time. Diagonal operators are kept as vectors. The jump terms ``Lhat rho Lhat^dag``
of sparse collapse operators become an element-wise coefficient matrix (constant rates, source
element = destination element) and a CSR list of the remaining (destination, source,
coefficient, rate) terms.

Floats in H are rounded to ten significant digits before the split, the convention of the
reference's code printer (``gqis/solver.py:166-170``); coefficient functions are printed by
the same printer as the reduced form's model code.

The CUDA kernels are ``csrc/gqis_matrix.cuh`` (CUDA cores, one CTA per parameter point) and
``csrc/gqis_matrix_tc.cuh`` (tensor cores, one CTA per 128 / N points). The dimension is padded
with inert levels to the kernel's tile (8, 16, 32, 48 or 64); padded levels have zero operators
and zero population and stay exactly zero.
"""

from __future__ import annotations

import os

import hashlib
from dataclasses import dataclass, field

import numpy as np
import sympy as sp

from . import emit
from .rhs import PARAM_NAMES, prepare_model

MAX_DIM = 64
MAX_JUMP_TERMS_PER_ELEMENT = 8
_CACHE: dict = {}


@dataclass(eq=False)
class MatrixModel:
    """Numeric operator decomposition of a Lindblad model (input of the matrix-form module)."""

    kind: str
    N: int                      # Hilbert-space dimension of the model
    Np: int                     # padded dimension of the kernel tile
    state_size: int             # N*N - 1 (reduced layout of final_rho / rho0_values)
    sweep_symbols: tuple
    runtime_const_syms: tuple   # Const_arr order (the base runtime constants)
    base_runtime_syms: tuple
    derived_const_exprs: tuple
    const_values: dict          # defaults of the runtime constants
    coef_exprs: tuple           # FP64 coefficient functions: dense terms, diagonal terms, jump rates
    heff0: np.ndarray           # (Np, Np) complex
    dense: tuple                # ND (Np, Np) complex matrices
    diag: tuple                 # NG (Np,) complex vectors
    wjump: np.ndarray           # (Np, Np) complex element-wise jump coefficients (constant rates)
    jumps: tuple                # (dst, src, coef, rate) with flat indices dst = i*Np + j
    obs: np.ndarray             # (Np, Np) complex mean operator
    rho0: np.ndarray            # (Np, Np) complex initial state
    cache_key: tuple
    emitted: dict = field(default_factory=dict, repr=False)

    @property
    def num_dense(self):
        return len(self.dense)

    @property
    def num_diag(self):
        return len(self.diag)


def padded_dimension(N):
    """Kernel tile dimension for a model of dimension ``N`` (error above ``MAX_DIM``)."""
    if N < 2:
        raise ValueError("the matrix form needs a Hilbert-space dimension of at least 2")
    Np = 8 if N <= 8 else -(-N // 16) * 16
    if Np > MAX_DIM:
        raise ValueError(f"the matrix form supports dimensions up to {MAX_DIM}; this model has {N}")
    return Np


def tile_shape(Np):
    """(TR, TC, threads): each thread owns a TR x TC block of rho; threads = Np^2/(TR*TC)."""
    TR, TC = {8: (1, 1), 16: (2, 2), 32: (2, 2), 48: (2, 4), 64: (2, 4)}[Np]
    return TR, TC, (Np // TR) * (Np // TC)


def _round10(expr):
    """Exact constants evaluated and every Float rounded to 10 significant digits: the values the
    code printer writes (``emit._ModelPrinter``, the reference convention gqis/solver.py:166-170)."""
    expr = emit._evaluate_constants(sp.sympify(expr))
    return expr.xreplace({f: sp.Float(float(f"{float(f):.9e}")) for f in expr.atoms(sp.Float)})


def _numeric(expr, what):
    expr = emit._evaluate_constants(sp.sympify(expr))
    if expr.free_symbols:
        raise ValueError(f"the matrix form needs a numeric {what}; it depends on "
                         f"{sorted(map(str, expr.free_symbols))}")
    return complex(expr)


def _split_terms(M, variables):
    """Affine split of a symbolic matrix: ``{factor: complex ndarray}`` with ``factor`` free of
    numbers (``1`` for the constant part) and every entry = sum factor * coefficient."""
    n = M.shape[0]
    groups = {}
    for i in range(n):
        for j in range(M.shape[1]):
            e = sp.expand(emit._evaluate_constants(sp.sympify(M[i, j])))
            if e == 0:
                continue
            for term in sp.Add.make_args(e):
                coeff, factor = term.as_independent(*variables, as_Add=False)
                if not coeff.is_number:
                    raise ValueError(f"cannot split the term {term} into a number and a factor")
                mat = groups.setdefault(factor, np.zeros((n, M.shape[1]), dtype=np.complex128))
                mat[i, j] += complex(coeff)
    return groups


def _drive_table(Drive):
    """Drive placeholder name -> expression (one ``Drive`` or the reference's dict form)."""
    if isinstance(Drive, dict):
        return {str(k): sp.sympify(v) for k, v in Drive.items()}
    return {"Drive": sp.sympify(Drive)}


def _positive_copy(expr):
    return expr.xreplace({s: sp.Symbol(str(s), positive=True) for s in expr.free_symbols})


def tile_dimension(N, tensor_cores=False):
    """Padded dimension of the kernel tile: :func:`padded_dimension`, except that a tensor-core
    sweep of a model of dimension 33 .. 48 pads to 64 (the tcgen05 kernel takes 8, 16, 32 or 64 and
    the padded rows and columns stay exactly zero)."""
    Np = padded_dimension(N)
    return 64 if tensor_cores and Np == 48 else Np


def decompose(model, sweep_symbols, cache_key, tile=None):
    """:class:`MatrixModel` of a model prepared by :func:`gqis.rhs.prepare_model` (``tile``: the padded
    dimension, :func:`padded_dimension` when None)."""
    N = int(model["N"])
    Np = padded_dimension(N) if tile is None else int(tile)
    # Constant-only subexpressions that prepare_model named (ConstExpr_k, x__sqrt ...) are put
    # back: the split below needs sqrt(G)/2 and -sqrt(G)/2 to share the factor sqrt(G).
    base = tuple(model["base_runtime_syms"])
    derived = dict(zip(model["runtime_const_syms"][len(base):], model["derived_const_exprs"]))

    def undo(e):
        return e.xreplace(derived) if derived else e

    H = undo(model["H"]).applyfunc(_round10)
    col_ops = [undo(L) for L in model["Col_Ops"]]
    Dm = model["Drive"]
    drives = _drive_table({k: undo(sp.sympify(v)) for k, v in Dm.items()} if isinstance(Dm, dict)
                          else undo(sp.sympify(Dm)))
    variables = set(H.free_symbols)
    for L in col_ops:
        variables |= L.free_symbols
    variables = sorted(variables, key=str)

    def with_drives(expr):
        table = {s: drives[str(s)] for s in expr.free_symbols if str(s) in drives}
        return expr.xreplace(table) if table else expr

    def pad(m):
        out = np.zeros((Np, Np), dtype=np.complex128)
        out[:m.shape[0], :m.shape[1]] = m
        return out

    terms = {}  # factor -> (Np, Np) matrix of H_eff
    for factor, mat in _split_terms(H, variables).items():
        terms[factor] = terms.get(factor, 0) + pad(mat)

    wjump = np.zeros((Np, Np), dtype=np.complex128)
    jump_terms = {}  # (dst, src, rate factor) -> coefficient
    for k, L in enumerate(col_ops):
        parts = _split_terms(L, variables)
        if not parts:
            continue
        if len(parts) != 1:
            raise ValueError(f"the matrix form needs each collapse operator to be a scalar times a numeric "
                             f"matrix; operator {k} has the factors {[str(f) for f in parts]}")
        (g, Lhat), = parts.items()
        g = with_drives(g)
        rate = sp.expand(_positive_copy(g * sp.conjugate(g)))
        rate = rate.xreplace({s: sp.Symbol(str(s), real=True) for s in rate.free_symbols})
        if rate.has(sp.conjugate) or rate.has(sp.Abs):
            raise ValueError(f"cannot form the rate |g|^2 of collapse operator {k} (factor {g})")
        Lh = pad(Lhat)
        key = sp.Integer(1) if rate == 1 else rate
        terms[key] = terms.get(key, 0) + (-0.5j) * (Lh.conj().T @ Lh)
        nz = list(zip(*np.nonzero(Lh)))
        if len(nz) ** 2 > MAX_JUMP_TERMS_PER_ELEMENT * Np * Np:
            raise ValueError(f"collapse operator {k} is too dense for the matrix form's jump list")
        for (i, a) in nz:
            for (j, b) in nz:
                coef = Lh[i, a] * np.conj(Lh[j, b])
                dst, src = i * Np + j, a * Np + b
                if key == 1 and dst == src:
                    wjump[i, j] += coef
                else:
                    jump_terms[(dst, src, key)] = jump_terms.get((dst, src, key), 0) + coef

    heff0 = terms.pop(sp.Integer(1), np.zeros((Np, Np), dtype=np.complex128))
    dense, diag, coef_exprs = [], [], []
    diag_items = []
    for factor, mat in sorted(terms.items(), key=lambda kv: str(kv[0])):
        if not np.any(mat):
            continue
        off = mat - np.diag(np.diag(mat))
        if np.any(off):
            dense.append(mat)
            coef_exprs.append(with_drives(factor))
        else:
            diag_items.append((factor, np.diag(mat).copy()))
    for factor, vec in diag_items:
        diag.append(vec)
        coef_exprs.append(with_drives(factor))
    rate_index = {}
    jumps = []
    for (dst, src, key), coef in sorted(jump_terms.items(), key=lambda kv: (kv[0][0], kv[0][1], str(kv[0][2]))):
        if coef == 0:
            continue
        if key == 1:
            r = -1
        else:
            if key not in rate_index:
                rate_index[key] = len(coef_exprs)
                coef_exprs.append(with_drives(key))
            r = rate_index[key]
        jumps.append((dst, src, complex(coef), r))

    O = undo(model["mean_operator"])
    obs = pad(np.array([[_numeric(O[i, j], "mean operator") for j in range(N)] for i in range(N)]))
    rho0 = np.zeros((Np, Np), dtype=np.complex128)
    if model["rho0_exprs"] is None:
        rho0[0, 0] = 1.0
    else:
        vals = [_numeric(undo(e), "rho0") for e in model["rho0_exprs"]]
        pops = [v.real for v in vals[:N - 1]]
        for i, v in enumerate(pops):
            rho0[i, i] = v
        rho0[N - 1, N - 1] = 1.0 - sum(pops)
        slot = N - 1
        for i in range(N):
            for j in range(i + 1, N):
                rho0[i, j] = vals[slot].real + 1j * vals[slot + 1].real
                rho0[j, i] = np.conj(rho0[i, j])
                slot += 2

    allowed_names = set(PARAM_NAMES) | {str(s) for s in base} | {"t"}
    for e in coef_exprs:
        bad = {str(s) for s in e.free_symbols} - allowed_names
        if bad:
            raise ValueError(f"a coefficient of the matrix form depends on unknown symbols {sorted(bad)}")

    return MatrixModel(
        kind="lindblad_matrix", N=N, Np=Np, state_size=N * N - 1, sweep_symbols=tuple(sweep_symbols),
        runtime_const_syms=base, base_runtime_syms=base, derived_const_exprs=(), const_values=dict(model["defaults"]),
        coef_exprs=tuple(coef_exprs), heff0=heff0, dense=tuple(dense), diag=tuple(diag), wjump=wjump,
        jumps=tuple(jumps), obs=obs, rho0=rho0, cache_key=cache_key)


def compile_matrix_model(H, Drive, Col_Ops, mean_operator, *, sweep_symbols, const_values=None,
                         runtime_consts=None, keep_symbolic_consts=None, auto_runtime_consts=False,
                         rho0=None, reuse=True, tensor_cores=False):
    """Prepare a model for the matrix form; returns ``(MatrixModel, "hit" | "miss")``.
    ``tensor_cores``: pad for the tensor-core kernel (:func:`tile_dimension`)."""
    model = prepare_model(H, Drive, Col_Ops, mean_operator, sweep_symbols=tuple(sweep_symbols),
                          const_values=const_values, runtime_consts=runtime_consts,
                          keep_symbolic_consts=keep_symbolic_consts, auto_runtime_consts=auto_runtime_consts,
                          rho0=rho0, ode_size=None)
    Dm = model["Drive"]
    drive_key = (tuple((str(k), sp.srepr(v)) for k, v in Dm.items()) if isinstance(Dm, dict) else sp.srepr(Dm))
    key = ("b200_matrix_v1", model["N"], sp.srepr(model["H"]), drive_key,
           tuple(sp.srepr(L) for L in model["Col_Ops"]), sp.srepr(model["mean_operator"]),
           tuple(str(s) for s in model["runtime_const_syms"]),
           None if model["rho0_exprs"] is None else tuple(sp.srepr(e) for e in model["rho0_exprs"]))
    tile = tile_dimension(int(model["N"]), tensor_cores)
    if tile != padded_dimension(int(model["N"])):
        key = key + (("tile", tile),)
    if reuse and key in _CACHE:
        return _CACHE[key], "hit"
    mm = _disk_load(key) if reuse else None
    if mm is None:
        mm = decompose(model, sweep_symbols, key, tile)
        if reuse:
            _disk_store(key, mm)
    if reuse:
        _CACHE[key] = mm
    return mm, "miss"


# Decomposing a dense model takes seconds (N = 64: ~18 s) and would repeat in every process;
# decomposed models are pickled next to the model modules like prepared reduced-form RHS objects
# (GQIS_DISK_CACHE=0 disables both).
def _disk_load(key):
    import pickle
    from .rhs import _disk_path
    if os.environ.get("GQIS_DISK_CACHE", "1") == "0":
        return None
    path = _disk_path(key)
    try:
        with open(path, "rb") as f:
            stored_key, mm = pickle.load(f)
    except Exception:
        return None
    return mm if stored_key == key else None


def _disk_store(key, mm):
    import pickle
    from .rhs import _disk_path
    if os.environ.get("GQIS_DISK_CACHE", "1") == "0":
        return
    path = _disk_path(key)
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(f".{os.getpid()}.tmp")
        with open(tmp, "wb") as f:
            pickle.dump((key, mm), f, protocol=pickle.HIGHEST_PROTOCOL)
        os.replace(tmp, path)
    except Exception:
        pass


# ----------------------------------------------------------------------------------------
# module source
# ----------------------------------------------------------------------------------------

def _array(name, ctype, values, per_line=8):
    vals = list(values) or [0]
    fmt = (lambda v: f"{float(v):.17e}") if ctype in ("double", "mreal") else (lambda v: str(int(v)))
    rows = [", ".join(fmt(v) for v in vals[i:i + per_line]) for i in range(0, len(vals), per_line)]
    body = ",\n    ".join(rows)
    return f"__device__ __align__(16) const {ctype} {name}[{len(vals)}] = {{\n    {body}}};"


def _interleave(z):
    z = np.asarray(z, dtype=np.complex128).reshape(-1)
    out = np.empty(2 * z.size)
    out[0::2], out[1::2] = z.real, z.imag
    return out


def tensor_core_jump_lists(mm: MatrixModel, rows_per_thread=8):
    """Jump terms of the tensor-core kernel grouped by thread: thread (column j, row block b)
    owns rows b*8 .. b*8+7 of column j; each term is (row e in the block, source, coef, rate index
    or -1). The source is a population index a >= 0 (rho_aa, shared between threads) or -1 for the
    element (e, j) itself (element-wise terms on coherences, read back by the thread).
    Returns (lists[j][b], has_own_element_terms)."""
    Np = mm.Np
    H = Np // rows_per_thread
    lists = [[[] for _ in range(H)] for _ in range(Np)]
    own = False

    def add(n, j, src_pop, coef, rate):
        nonlocal own
        if src_pop < 0:
            own = True
        lists[j][n // rows_per_thread].append((n % rows_per_thread, src_pop, complex(coef), rate))

    for dst, src, coef, rate in mm.jumps:
        n, j = divmod(dst, Np)
        a, b = divmod(src, Np)
        if dst == src:
            add(n, j, n if n == j else -1, coef, rate)
        elif a == b:
            add(n, j, a, coef, rate)
        else:
            raise ValueError("tensor-core jump lists need population or element-wise sources")
    for n in range(Np):
        for j in range(Np):
            w = complex(mm.wjump[n, j])
            if w != 0:
                add(n, j, n if n == j else -1, w, -1)
    return lists, own


def diag_in_mma(mm: MatrixModel):
    """Whether the tensor-core kernel multiplies the diagonal operator terms on the tensor cores
    (one more MMA term per diagonal operator) or in its epilogue: on the tensor cores wherever the MMA
    is wide enough (2 x rows x terms <= 256 columns). With FP16 operands (K = 16 per MMA) that is the
    faster side at every N: 4096 points x 2000 steps, N = 32 113 ms vs 130 ms with the diagonal terms
    in the epilogue (which reads the stage input back from A), N = 64 1081 vs 1165 ms."""
    rows = mm.Np // (2 if mm.Np >= TC_CLUSTER_FROM else 1)
    return 2 * rows * (1 + mm.num_dense + mm.num_diag) <= 256


# Rows of a column per thread of the tensor-core kernel, by padded dimension (4 or 8). Four rows double
# a CTA's threads and halve each thread's epilogue chain, but measured slower (4096 points x 2000 steps:
# N = 8 10.4 -> 11.0 ms, N = 16 30.1 -> 38.3 ms with 64 registers per thread), so every dimension uses 8.
TC_ROWS_PER_THREAD = {8: 8, 16: 8, 32: 8, 64: 8}


def tensor_core_rows(mm: MatrixModel):
    return TC_ROWS_PER_THREAD.get(mm.Np, 8)


def _tensor_core_tables(mm: MatrixModel):
    E = tensor_core_rows(mm)
    lists, own = tensor_core_jump_lists(mm, rows_per_thread=E)
    Np = mm.Np
    H = Np // E
    jmax = max(1, max(len(lists[j][b]) for j in range(Np) for b in range(H)))
    count, e, a, coef, rate = [], [], [], [], []
    for j in range(Np):
        for b in range(H):
            terms = lists[j][b] + [(0, 0, 0j, -1)] * (jmax - len(lists[j][b]))
            count.append(len(lists[j][b]))
            for (ee, aa, cc, rr) in terms:
                e.append(ee)
                a.append(aa)
                coef.append(cc)
                rate.append(rr)
    arrays = [
        _array("mm_tcj_count", "int", count),
        _array("mm_tcj_e", "int", e),
        _array("mm_tcj_a", "int", a),
        _array("mm_tcj_rate", "int", rate),
        _array("mm_tcj_coef", "mreal", _interleave(coef)),
    ]
    on_diag = all(e + E * b == j for j in range(Np) for b in range(H) for (e, _, _, _) in lists[j][b])
    members = f"""    static constexpr int TCJ_MAX = {jmax};
    static constexpr bool kOwnTerms = {'true' if own else 'false'};
    static constexpr bool kJumpsOnDiagonal = {'true' if on_diag else 'false'};
    static constexpr bool kDiagInMma = {'true' if diag_in_mma(mm) else 'false'};
    static constexpr bool kObsDiagonal = {'true' if not np.any(mm.obs - np.diag(np.diag(mm.obs))) else 'false'};
    static constexpr int TC_CL = {tensor_core_shape(mm)[0]};
    static constexpr int TC_E = {E};
    __device__ __forceinline__ static const int* tcj_count() {{ return mm_tcj_count; }}
    __device__ __forceinline__ static const int* tcj_e() {{ return mm_tcj_e; }}
    __device__ __forceinline__ static const int* tcj_a() {{ return mm_tcj_a; }}
    __device__ __forceinline__ static const int* tcj_rate() {{ return mm_tcj_rate; }}
    __device__ __forceinline__ static const mreal* tcj_coef() {{ return mm_tcj_coef; }}
"""
    return arrays, members


def emit_matrix_model(mm: MatrixModel, form: str, uses_rho0_values: bool, tensor_cores=False):
    """C++ text of the model data and ``struct MM`` for ``csrc/gqis_matrix.cuh``.

    Operator data are printed with 17 significant digits in the form's type (``mreal``);
    the mean operator and rho0 stay FP64. Coefficient functions are FP64 C expressions of
    ``t``, ``ParX``, ``ParY`` and ``Const_arr[k]`` (runtime constants in call order).
    """
    Np = mm.Np
    TR, TC, threads = tile_shape(Np)
    const_names = [(str(s), f"Const_arr[{k}]") for k, s in enumerate(mm.runtime_const_syms)]
    coef_lines = []
    for q, e in enumerate(mm.coef_exprs):
        text = emit.ccode(e, cast=False)
        coef_lines.append(f"c[{q}] = {emit._substitute(text, const_names)};")
    dst = np.array([j[0] for j in mm.jumps], dtype=np.int64)
    order = np.argsort(dst, kind="stable")
    jumps = [mm.jumps[i] for i in order]
    begin = np.zeros(Np * Np + 1, dtype=np.int64)
    for dj, _, _, _ in jumps:
        begin[dj + 1] += 1
    begin = np.cumsum(begin)
    real = "double" if form == "fp64" else "float"
    parts = [
        f"using mreal = {real};",
        _array("mm_heff", "mreal", _interleave(mm.heff0)),
        _array("mm_dense", "mreal", np.concatenate([_interleave(m) for m in mm.dense]) if mm.dense else []),
        _array("mm_diag", "mreal", np.concatenate([_interleave(v) for v in mm.diag]) if mm.diag else []),
        _array("mm_wjump", "mreal", _interleave(mm.wjump)),
        _array("mm_jbegin", "int", begin),
        _array("mm_jsrc", "int", [j[1] for j in jumps]),
        _array("mm_jrate", "int", [j[3] for j in jumps]),
        _array("mm_jcoef", "mreal", _interleave([j[2] for j in jumps]) if jumps else []),
        _array("mm_obs_t", "double", _interleave(mm.obs.T)),
        _array("mm_rho0", "double", _interleave(mm.rho0)),
    ]
    nconst = max(1, len(mm.runtime_const_syms))
    body = "\n".join("        " + ln for ln in coef_lines) or "        /* none */"
    tc_members = ""
    if tensor_cores:
        tc_arrays, tc_members = _tensor_core_tables(mm)
        parts += tc_arrays
    struct = f"""struct MM {{
    using real = mreal;
    static constexpr int N = {Np};
    static constexpr int NO = {mm.N};
    static constexpr int S = {mm.state_size};
    static constexpr int ND = {mm.num_dense};
    static constexpr int NG = {mm.num_diag};
    static constexpr int NCOEF = {len(mm.coef_exprs)};
    static constexpr int NJ = {len(jumps)};
    static constexpr int NCONST = {nconst};
    static constexpr int TR = {TR}, TC = {TC}, THREADS = {threads};
    static constexpr bool kInitFromArray = {'true' if uses_rho0_values else 'false'};

    __device__ __forceinline__ static void coef(double t, double ParX, double ParY,
                                                const double* __restrict__ Const_arr, double* __restrict__ c) {{
        (void)t; (void)ParX; (void)ParY; (void)Const_arr; (void)c;
{body}
    }}
    __device__ __forceinline__ static const mreal* heff() {{ return mm_heff; }}
    __device__ __forceinline__ static const mreal* dense(int q) {{ return mm_dense + 2 * N * N * q; }}
    __device__ __forceinline__ static const mreal* diag(int g) {{ return mm_diag + 2 * N * g; }}
    __device__ __forceinline__ static const mreal* wjump() {{ return mm_wjump; }}
    __device__ __forceinline__ static const int* jbegin() {{ return mm_jbegin; }}
    __device__ __forceinline__ static const int* jsrc() {{ return mm_jsrc; }}
    __device__ __forceinline__ static const int* jrate() {{ return mm_jrate; }}
    __device__ __forceinline__ static const mreal* jcoef() {{ return mm_jcoef; }}
    __device__ __forceinline__ static const double* obs_t() {{ return mm_obs_t; }}
    __device__ __forceinline__ static const double* rho0() {{ return mm_rho0; }}
{tc_members}}};"""
    return "\n".join(parts + [struct])


OUTPUT_IDS = {"mean": 0, "final": 1, "final_rho": 2}
TENSOR_DIMS = (8, 16, 32, 64)
SMEM_LIMIT = 232448  # shared memory of one CTA on sm_100a (bytes)
# Padded dimension from which a tile is split over a cluster of two CTAs. Only N = 64 needs it (one
# SM's registers cannot hold the tile); splitting N = 16 / 32 tiles as well, which would let two CTAs
# share an SM, measured slower (30 -> 44 ms, 146 -> 212 ms for 4096 points x 2000 steps): the exchange
# of every stage costs more than the overlap of one CTA's MMA with the other's epilogue gains.
TC_CLUSTER_FROM = 64


def tensor_core_shape(mm: MatrixModel):
    """(cluster CTAs, rows per CTA, MMA columns, shared-memory bytes) of the tcgen05 kernel for this model,
    the TcShape of csrc/gqis_matrix_tc.cuh (a generated module asserts that the sizes agree)."""
    Np = mm.Np
    cl = 2 if Np >= TC_CLUSTER_FROM else 1
    nh = Np // cl
    P, E = 128 // Np, tensor_core_rows(mm)
    H = nh // E
    terms = 1 + mm.num_dense + (mm.num_diag if diag_in_mma(mm) else 0)
    nmma = 2 * nh * terms
    kdim = 2 * Np
    nc = max(1, len(mm.coef_exprs))
    b = nmma * kdim * 2  # one FP16 part of B
    k = P * nh * (Np + 2) * 8
    x = P * H * E * Np * 8 if cl > 1 else 0
    rd = 2 * P * Np * 4
    cs = 2 * 24 * P * nc * 4  # coefficient table: 2 buffers x 3 stage times x 8 steps
    cg = Np // 32 if Np > 32 else 1
    off_red = -(-(2 * b + k + x + rd + cs) // 8) * 8
    dv = 0 if diag_in_mma(mm) or mm.num_diag == 0 else P * Np * 8  # the epilogue's diagonal coefficients
    needed = off_red + 2 * H * cg * P * 8 + 2 * P * 8 + dv + 128  # + mbarriers, flags, B-term maxima
    return cl, nh, nmma, needed


def tensor_core_blockers(mm: MatrixModel, form: str):
    """Reasons the tensor-core kernel (csrc/gqis_matrix_tc.cuh) cannot run this model; [] if it can."""
    out = []
    if form != "fp32":
        out.append("the tensor-core form is an FP32 form (precision='fp32')")
    if mm.Np not in TENSOR_DIMS:
        out.append(f"padded dimension {mm.Np} is not one of {TENSOR_DIMS}")
    else:
        _, nh, nmma, smem = tensor_core_shape(mm)
        if nmma > 256:
            out.append(f"{mm.num_dense + mm.num_diag} coefficient operator terms exceed one MMA "
                       f"(2 x {nh} rows x (1 + terms) <= 256)")
        elif smem > SMEM_LIMIT:
            out.append(f"{mm.num_dense} dense coefficient operators need {smem} bytes of shared memory per CTA "
                       f"(at most {SMEM_LIMIT})")
    if any(src != dst and src // mm.Np != src % mm.Np for dst, src, _, _ in mm.jumps):
        out.append("a jump term moves a coherence to another element (only populations may feed other elements)")
    elif mm.Np in TENSOR_DIMS:
        lists, _ = tensor_core_jump_lists(mm, rows_per_thread=tensor_core_rows(mm))
        if max(len(x) for col in lists for x in col) > 32:
            out.append("more than 32 jump terms land in one thread's rows")
    return out


def module_source(mm: MatrixModel, form: str, output_mode: str, uses_rho0_values: bool, tensor_cores=False,
                  trace=False):
    """Complete translation unit of one matrix-form module (C ABI of include/gqis_b200.h);
    ``tensor_cores`` selects the tcgen05 kernel of csrc/gqis_matrix_tc.cuh, ``trace`` records the
    observable every trace_stride steps."""
    if output_mode not in OUTPUT_IDS:
        raise ValueError(f"the matrix form supports the outputs {sorted(OUTPUT_IDS)}, not '{output_mode}'")
    if tensor_cores:
        blockers = tensor_core_blockers(mm, form)
        if blockers:
            raise ValueError("the tensor-core matrix form cannot run this model: " + "; ".join(blockers))
    model = emit_matrix_model(mm, form, uses_rho0_values, tensor_cores)
    model_hash = int(hashlib.sha256(model.encode()).hexdigest()[:16], 16)
    form_type = {"fp64": "FormFP64", "fp32": "FormFP32"}[form]
    return "\n".join([
        "// Matrix-form model module generated by gqis (B200 sweep engine). Do not edit.",
        '#include "gqis_common.cuh"',
        '#include "gqis_matrix_tc.cuh"' if tensor_cores else '#include "gqis_matrix.cuh"',
        "namespace gqmodel {",
        model,
        "}  // namespace gqmodel",
        f"#define GQ_MATRIX {2 if tensor_cores else 1}",
        "#define GQ_MODEL gqmodel::MM",
        f"#define GQ_FORM {form_type}",
        "#define GQ_SOLVER_ID 0",
        "#define GQ_ADAPTIVE 0",
        f"#define GQ_OUT {OUTPUT_IDS[output_mode]}",
        f"#define GQ_TRACE {1 if trace else 0}",
        f"#define GQ_MODEL_HASH 0x{model_hash:016x}ULL",
        '#include "gqis_module.cuh"',
    ] + ([f"static_assert(gqmatrix_tc::TcShape<gqmodel::MM>::NEEDED == {tensor_core_shape(mm)[3]}, "
          '"shared-memory size of matrix_form.tensor_core_shape");'] if tensor_cores else []) + [""])


def flops_per_point_step(mm: MatrixModel):
    """Arithmetic of one RK4 step of one point in the matrix kernel (an FMA counts 2 flops).

    Per RHS: H(t) = Heff0 + sum c_k M_k (4 ND per entry), the complex product H(t) rho
    (8 Np^3), the diagonal terms (8 per element plus 4 NG per row), -i (K - K^dag) (2 per
    element) and the jump terms (8 per element-wise and per listed term). Per step: 4 RHS, the
    RK4 stage inputs and combinations (26 per element) and the <O> accumulation (8 per element).
    """
    Np = mm.Np
    nn = Np * Np
    per_rhs = 8 * Np ** 3 + 4 * mm.num_dense * nn + (8 * nn + 4 * mm.num_diag * Np if mm.num_diag else 0)
    per_rhs += 2 * nn + 8 * nn + 8 * len(mm.jumps)
    return 4 * per_rhs + 26 * nn + 8 * nn


def algorithmic_flops_per_point_step(mm: MatrixModel):
    """Flops of one RK4 step of one point as the benchmark's roofline counts them, for any form:
    per RHS the two complex N x N products of -i(H rho - rho H^dag) (16 N^3, 8 real flops per
    complex multiply-add) plus the kernel's element-wise terms (coefficients, diagonal and jump
    terms, -i(K - K^dag)); per step 4 RHS, the RK4 stage arithmetic (26 per element) and <O>
    (8 per element). Uses the model's dimension N, not the padded tile, and counts neither the
    padding nor the extra split-FP16 passes of the tensor-core kernel."""
    N = mm.N
    nn = N * N
    elementwise = 4 * mm.num_dense * nn + (8 * nn + 4 * mm.num_diag * N if mm.num_diag else 0)
    elementwise += 2 * nn + 8 * nn + 8 * len(mm.jumps)
    return 4 * (16 * N ** 3 + elementwise) + 26 * nn + 8 * nn


def tensor_flops_per_point_step(mm: MatrixModel):
    """Tensor-pipe arithmetic of one RK4 step of one point in the tcgen05 kernel: per RHS the
    point's N rows of D (2 N (1 + ND + NG) columns) over K = 2 N, three split-FP16 passes."""
    Np = mm.Np
    terms = 1 + mm.num_dense + (mm.num_diag if diag_in_mma(mm) else 0)
    return 4 * 3 * 2 * Np * (2 * Np * terms) * (2 * Np)


def dense_operators(mm: MatrixModel, X, Y, t, consts=()):
    """Numeric H_eff(t) and the coefficient values at one point, as the module evaluates them
    (coefficients with their printed 10-digit literals); NumPy, used by the tests."""
    syms = {"ParX": X, "ParY": Y, "t": t}
    for s, v in zip(mm.runtime_const_syms, consts):
        syms[str(s)] = v

    def value(e):
        e = _round10(e)
        return complex(e.xreplace({s: sp.Float(syms[str(s)]) for s in e.free_symbols}).evalf())
    cvals = [value(e) for e in mm.coef_exprs]
    H = mm.heff0.copy()
    for q, m in enumerate(mm.dense):
        H = H + cvals[q] * m
    for g, v in enumerate(mm.diag):
        H = H + cvals[mm.num_dense + g] * np.diag(v)
    return H, cvals
