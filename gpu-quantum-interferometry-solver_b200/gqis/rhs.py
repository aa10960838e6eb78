"""Model preparation and device-independent optimisation of the ODE right-hand side.

Pipeline (the reference's L3/L4, ``gqis/solver.py:1374-1589`` and ``:550-625``):

1. ``prepare_model``: rename the sweep symbols to ``ParX``/``ParY``, fold fixed constants
   as Floats, keep runtime constants symbolic (``Const_arr`` order: kept symbols sorted by
   name, then derived constant-only subexpressions), and drop unused runtime constants.
2. derive the real ODE (``lindblad.build_reduced_lindblad_rhs``) or take the user ODE.
3. ``optimize_rhs``: common-subexpression elimination that leaves the state untouched,
   and a level for every state-independent temporary: ``inline`` (constants only),
   ``negate`` (minus a value already bound), ``static`` (sweep parameters and constants:
   once per point) or ``drive`` (time dependent: once per stage time).

The resulting :class:`CompiledRHS` is cached by a structural key; it carries no device
code. ``emit.py`` turns its plan into the model functions the CUDA templates call.
"""

from __future__ import annotations

import hashlib
import os
import pickle
import time
from dataclasses import dataclass, field

import numpy as np
import sympy as sp

from .lindblad import build_reduced_lindblad_rhs, reduced_symbols, rho_matrix_to_independent_exprs

# Process-local caches (names of ``gqis/solver.py:31-34``; tests clear them).
_RHS_CODE_CACHE: dict = {}

PARAM_NAMES = ("ParX", "ParY")


@dataclass(eq=False)
class CompiledRHS:
    """Prepared and optimised right-hand side, independent of any device code.

    Made by ``compile_lindblad_rhs`` or ``compile_ode_rhs``; pass it to ``mesolve_2D`` or
    ``odesolve_2D`` in place of the model to start the call at code emission. Fields follow
    ``gqis/solver.py:1344-1371``.
    """

    kind: str
    state_size: int
    sweep_symbols: tuple
    state_symbols: tuple
    equations: tuple
    mean_re: object
    mean_im: object
    drive_map: object
    rho0_exprs: object
    runtime_const_syms: tuple
    base_runtime_syms: tuple
    derived_const_exprs: tuple
    const_values: dict
    plan: dict
    cache_key: tuple
    timings: dict
    ode: object = None
    emitted: dict = field(default_factory=dict, repr=False)
    model: dict = field(default_factory=dict, repr=False)  # prepared symbolic model (adjoint, matrix form)


# ----------------------------------------------------------------------------------------
# 1. model preparation
# ----------------------------------------------------------------------------------------

def _map_drive(Drive, fn):
    return {k: fn(v) for k, v in Drive.items()} if isinstance(Drive, dict) else fn(Drive)


def _derived_name(expr, idx, taken):
    """Readable unique symbol for a constant-only subexpression (``x__sqrt``, ``x__inv`` ...)."""
    name = None
    if expr.is_Pow and expr.base.is_Symbol:
        name = {sp.Rational(1, 2): f"{expr.base}__sqrt", sp.Rational(-1, 2): f"{expr.base}__rsqrt",
                sp.Integer(-1): f"{expr.base}__inv"}.get(expr.exp)
    elif (expr.func in (sp.sin, sp.cos, sp.tan, sp.exp, sp.log) and len(expr.args) == 1
          and expr.args[0].is_Symbol):
        name = f"{expr.args[0]}__{expr.func.__name__}"
    base = name or f"ConstExpr_{idx}"
    name, n = base, 1
    while name in taken:
        name = f"{base}_{n}"
        n += 1
    taken.add(name)
    return sp.Symbol(name, real=True)


def prepare_model(H, Drive, Col_Ops, mean_operator, *, sweep_symbols, const_values,
                  runtime_consts, keep_symbolic_consts, auto_runtime_consts, rho0, ode_size):
    """Validate a model and substitute sweep symbols and constants (``gqis/solver.py:1374-1521``)."""
    const_values = {} if const_values is None else const_values
    runtime_consts = runtime_consts or {}
    if not isinstance(runtime_consts, dict):
        raise ValueError("runtime_consts must be a dict of {Symbol: value}")
    N = H.shape[0]
    size = N * N - 1 if ode_size is None else ode_size
    rho0_exprs = None
    if rho0 is not None:
        rho0_exprs = (rho_matrix_to_independent_exprs(rho0) if ode_size is None
                      else [sp.sympify(v) for v in rho0])
        if len(rho0_exprs) != size:
            raise ValueError("rho0 does not match Hamiltonian size.")
    for L in Col_Ops:
        if L.shape != (N, N):
            raise ValueError(f"Collapse operator dimension {L.shape} does not match H {N, N}")
    if ode_size is None and mean_operator.shape != (N, N):
        raise ValueError(f"Mean operator dimension {mean_operator.shape} does not match H {N, N}")

    rename = {s: sp.Symbol(name, real=True) for s, name in zip(sweep_symbols, PARAM_NAMES)}
    H = H.subs(rename)
    Drive = _map_drive(Drive, lambda e: sp.sympify(e).subs(rename)) if isinstance(Drive, dict) \
        else sp.sympify(Drive).subs(rename)
    Col_Ops = [L.subs(rename) for L in Col_Ops]
    mean_operator = mean_operator.subs(rename)
    if rho0_exprs is not None:
        rho0_exprs = [e.subs(rename) for e in rho0_exprs]

    if keep_symbolic_consts is None:
        keep = set(const_values) if auto_runtime_consts else set()
    elif keep_symbolic_consts in ("all", "auto", "const_values"):
        keep = set(const_values)
    else:
        keep = set(keep_symbolic_consts)
    keep |= set(runtime_consts)
    if any(not isinstance(s, sp.Symbol) for s in keep):
        raise ValueError("keep_symbolic_consts/runtime_consts keys must be SymPy Symbols")
    runtime = sorted(keep, key=str)

    folded = {k: v for k, v in const_values.items() if k not in set(runtime)}
    if folded:
        as_float = {k: sp.Float(float(v)) for k, v in folded.items()}
        H = H.xreplace(as_float)
        Drive = _map_drive(Drive, lambda e: e.xreplace(as_float))
        Col_Ops = [L.xreplace(as_float) for L in Col_Ops]
        mean_operator = mean_operator.xreplace(as_float)
        if rho0_exprs is not None:
            rho0_exprs = [e.xreplace(as_float) for e in rho0_exprs]

    def all_exprs():
        yield from H
        yield from (Drive.values() if isinstance(Drive, dict) else [Drive])
        for L in Col_Ops:
            yield from L
        yield from mean_operator
        yield from (rho0_exprs or [])

    runtime_set = set(runtime)
    used = set()
    for e in all_exprs():
        used |= e.free_symbols & runtime_set
    runtime = [s for s in runtime if s in used]
    runtime_set = set(runtime)

    derived_exprs = []
    if runtime_set:
        seen = {}
        for e in all_exprs():
            for sub in sp.preorder_traversal(e):
                if sub.is_Number or sub.is_Symbol:
                    continue
                fs = sub.free_symbols
                if fs and fs <= runtime_set:
                    seen[sp.srepr(sub)] = sub
        derived_exprs = [x for x in seen.values() if x.count_ops() > 0]
        derived_exprs.sort(key=lambda x: (x.count_ops(), sp.srepr(x)), reverse=True)
    taken = {str(s) for s in runtime}
    derived_syms = [_derived_name(e, i, taken) for i, e in enumerate(derived_exprs)]
    if derived_exprs:
        table = dict(zip(derived_exprs, derived_syms))
        H = H.xreplace(table)
        Drive = _map_drive(Drive, lambda e: e.xreplace(table))
        Col_Ops = [L.xreplace(table) for L in Col_Ops]
        mean_operator = mean_operator.xreplace(table)
        if rho0_exprs is not None:
            rho0_exprs = [e.xreplace(table) for e in rho0_exprs]

    defaults = {s: v for s, v in {**const_values, **runtime_consts}.items() if s in runtime_set}
    return {"N": N, "state_size": size, "H": H, "Drive": Drive, "Col_Ops": Col_Ops,
            "mean_operator": mean_operator, "rho0_exprs": rho0_exprs,
            "base_runtime_syms": tuple(runtime), "derived_const_exprs": tuple(derived_exprs),
            "runtime_const_syms": tuple(runtime) + tuple(derived_syms),
            "const_values_eff": folded, "defaults": defaults}


# ----------------------------------------------------------------------------------------
# 3. optimisation plan
# ----------------------------------------------------------------------------------------

def cse_plan(exprs, states, *, batch_size=None, do_simplify=True, hoist_rho_independent=False):
    """CSE of the RHS that never factors the state symbols (``gqis/solver.py:749-804``).

    Returns ``(hoisted, blocks)``. ``hoisted`` lists state-independent temporaries
    ``(symbol, expr)`` in dependency order; each block is ``(scoped, temps, outputs)``
    with ``outputs`` as ``(state index, expr)``. With ``batch_size`` every slice of that
    many equations gets its own CSE pass and braces (fewer live temporaries).
    """
    state_set = set(states)

    def one_block(chunk, first, prefix, scoped):
        subs, reduced = sp.cse(chunk, symbols=sp.numbered_symbols(prefix=prefix), ignore=state_set)
        hoisted, kept, dependent = [], [], set()
        for s, e in subs:
            if hoist_rho_independent and not (e.free_symbols & (state_set | dependent)):
                hoisted.append((s, e))
            else:
                kept.append((s, e))
                dependent.add(s)
        fix = sp.simplify if do_simplify else (lambda x: x)
        temps = [(s, fix(e)) for s, e in kept]
        outputs = [(first + k, fix(e)) for k, e in enumerate(reduced)]
        return hoisted, (scoped, temps, outputs)

    if batch_size is None:
        hoisted, block = one_block(list(exprs), 0, "t", False)
        return hoisted, [block]
    size = int(batch_size)
    if size <= 0:
        raise ValueError("batch_size must be a positive integer, or None")
    hoisted_all, blocks = [], []
    for b, start in enumerate(range(0, len(exprs), size)):
        hoisted, block = one_block(list(exprs[start:start + size]), start, f"t{b}_", True)
        hoisted_all += hoisted
        blocks.append(block)
    return hoisted_all, blocks


def drive_plan(drive_map, *, inline_single_use_funcs=True):
    """Drive placeholders, shared function temporaries and expressions (``gqis/solver.py:851-886``).

    A placeholder named ``Drive`` takes slot 0; the others keep their dict order. A function
    call (``cos(w*t)`` ...) used by more than one drive is computed once into a temporary.
    """
    if not drive_map:
        return [], [], []
    syms = list(drive_map)
    for k, s in enumerate(syms):
        if str(s) == "Drive":
            syms.insert(0, syms.pop(k))
            break
    exprs = [sp.factor(sp.expand(drive_map[s])) for s in syms]
    counts = {}
    for e in exprs:
        for f in e.atoms(sp.Function):
            counts[f] = counts.get(f, 0) + 1
    shared = {}
    for k, f in enumerate(sorted(counts, key=str)):
        if inline_single_use_funcs and counts[f] <= 1:
            continue
        shared[sp.Symbol(f"d{k}")] = f
    out = []
    for e in exprs:
        for sym, f in shared.items():
            e = e.subs(f, sym)
        out.append(e)
    return syms, list(shared.items()), out


def optimize_rhs(eqs, mean_re, mean_im, states, Drive_symbol, drive_expr, *, runtime_const_syms=(),
                 cse_batch_size=None, cse_simplify=True, hoist_rho_independent=True,
                 extract_independent=False):
    """Evaluation-level plan of the RHS (``gqis/solver.py:550-625``); see the module docstring."""
    state_names = {str(s) for s in states}
    independent = {}
    if extract_independent and hoist_rho_independent:
        state_set = set(states)

        def lift(e):
            if not e.is_Atom and e.free_symbols and not (e.free_symbols & state_set):
                if e not in independent:
                    independent[e] = sp.Symbol(f"ode_hoist_{len(independent)}", real=True)
                return independent[e]
            return e.func(*(lift(a) for a in e.args)) if e.args else e
        eqs = [lift(e) for e in eqs]
        mean_re, mean_im = lift(mean_re), lift(mean_im)
    hoisted, blocks = cse_plan(eqs, states, batch_size=cse_batch_size, do_simplify=cse_simplify,
                               hoist_rho_independent=hoist_rho_independent)
    hoisted = [(s, e) for e, s in independent.items()] + hoisted
    dmap = {}
    if drive_expr is not None:
        dmap = drive_expr if isinstance(drive_expr, dict) else {Drive_symbol: drive_expr}
    dplan = drive_plan(dmap)

    bound = {str(s) for s in dplan[0]}
    const_like = {str(s) for s in (runtime_const_syms or ())}
    static_names = set()
    hoists = []
    if hoist_rho_independent and hoisted:
        for s, e in hoisted:
            names = {str(x) for x in e.free_symbols}
            coeff, rest = e.as_coeff_Mul()
            if not names or names <= const_like:
                level = "inline"
                const_like.add(str(s))
            elif coeff == -1 and isinstance(rest, sp.Symbol) and str(rest) in bound:
                level = "negate"
            elif names <= const_like | set(PARAM_NAMES) | static_names:
                level = "static"
                static_names.add(str(s))
            else:
                level = "drive"
            hoists.append((s, e, level))
            bound.add(str(s))

    subs, mean_exprs = sp.cse([mean_re, mean_im], symbols=sp.numbered_symbols("mean_tmp"))
    inline_mean = {}
    mean_hoists = []
    for s, e in subs:
        e = e.xreplace(inline_mean)
        names = {str(x) for x in e.free_symbols}
        if names & state_names or not names:
            inline_mean[s] = e
            mean_exprs = [sp.simplify(m.subs(s, e)) for m in mean_exprs]
        elif names <= const_like | set(PARAM_NAMES) | static_names:
            mean_hoists.append((s, e, "static"))
            static_names.add(str(s))
        else:
            mean_hoists.append((s, e, "drive"))
    return {"blocks": blocks, "drive_plan": dplan, "hoists": hoists, "mean_hoists": mean_hoists,
            "mean_exprs": mean_exprs, "runtime_const_syms": tuple(runtime_const_syms or ())}


# ----------------------------------------------------------------------------------------
# 2 + cache: CompiledRHS
# ----------------------------------------------------------------------------------------

def _frozen(x):
    """Hashable, structurally compared form of a call argument (SymPy matrices become immutable)."""
    if x is None or isinstance(x, (bool, int, float, complex, str)):
        return x
    if isinstance(x, sp.MatrixBase):
        return sp.ImmutableMatrix(x)
    if isinstance(x, dict):
        return ("dict",) + tuple(sorted(((_frozen(k), _frozen(v)) for k, v in x.items()), key=lambda kv: str(kv[0])))
    if isinstance(x, (list, tuple)):
        return ("seq",) + tuple(_frozen(v) for v in x)
    if isinstance(x, np.ndarray):
        return ("nd", x.shape, x.dtype.str, x.tobytes())
    return sp.sympify(x)


def compile_rhs(H, Drive, Col_Ops, mean_operator, *, sweep_symbols, const_values=None,
                runtime_consts=None, keep_symbolic_consts=None, auto_runtime_consts=False, rho0=None,
                ode_size=None, pre_expand=True, collect_rho=False, factor_terms=False,
                cse_batch_size=None, cse_simplify=False, hoist_rho_independent=True, reuse=True,
                symbolic_workers="auto", max_symbolic_workers=None):
    """Prepare and optimise the RHS; returns ``(CompiledRHS, "hit" | "miss")``.

    A repeated call with the same arguments is found by a key of the arguments themselves (their
    immutable SymPy forms) before the model is prepared and printed for the structural key; runtime
    constant values are not part of either key (they are launch inputs).
    """
    start = time.time()
    raw_key = None
    if reuse:
        try:
            raw_key = ("b200_rhs_args_v1", _frozen(H), _frozen(Drive), _frozen(list(Col_Ops)),
                       _frozen(mean_operator), _frozen(tuple(sweep_symbols)), _frozen(const_values or {}),
                       tuple(sorted(str(k) for k in (runtime_consts or {}))) if isinstance(runtime_consts, dict)
                       else None, _frozen(keep_symbolic_consts), bool(auto_runtime_consts), _frozen(rho0),
                       ode_size, pre_expand, collect_rho, factor_terms, cse_batch_size, cse_simplify,
                       hoist_rho_independent)
            hit = _RHS_CODE_CACHE.get(raw_key)
        except (TypeError, sp.SympifyError):
            raw_key, hit = None, None
        if hit is not None:
            return hit, "hit"
    model = prepare_model(H, Drive, Col_Ops, mean_operator, sweep_symbols=sweep_symbols,
                          const_values=const_values, runtime_consts=runtime_consts,
                          keep_symbolic_consts=keep_symbolic_consts,
                          auto_runtime_consts=auto_runtime_consts, rho0=rho0, ode_size=ode_size)
    Drive = model["Drive"]
    drive_key = (tuple((str(k), sp.srepr(v)) for k, v in Drive.items()) if isinstance(Drive, dict)
                 else sp.srepr(Drive))
    key = ("b200_rhs_v1", model["N"], ode_size, sp.srepr(model["H"]), drive_key,
           tuple(sp.srepr(L) for L in model["Col_Ops"]), sp.srepr(model["mean_operator"]),
           tuple((str(k), float(v)) for k, v in sorted(model["const_values_eff"].items(), key=lambda kv: str(kv[0]))),
           tuple(str(s) for s in model["runtime_const_syms"]),
           None if model["rho0_exprs"] is None else tuple(sp.srepr(e) for e in model["rho0_exprs"]),
           pre_expand, collect_rho, factor_terms, cse_batch_size, cse_simplify, hoist_rho_independent)
    if reuse and key in _RHS_CODE_CACHE:
        if raw_key is not None:
            _RHS_CODE_CACHE[raw_key] = _RHS_CODE_CACHE[key]
        return _RHS_CODE_CACHE[key], "hit"
    if reuse:
        stored = _disk_get(key)
        if stored is not None:
            _RHS_CODE_CACHE[key] = stored
            if raw_key is not None:
                _RHS_CODE_CACHE[raw_key] = stored
            return stored, "hit"

    size = model["state_size"]
    if ode_size is None:
        eqs, mean_re, mean_im, meta = build_reduced_lindblad_rhs(
            model["N"], model["H"], model["Col_Ops"], model["mean_operator"], pre_expand=pre_expand,
            collect_rho=collect_rho, factor_terms=factor_terms, symbolic_workers=symbolic_workers,
            max_symbolic_workers=max_symbolic_workers)
        states = meta["rho_syms"]
    else:
        states = reduced_symbols(size)
        eqs = list(model["H"])
        if pre_expand:
            eqs = [sp.expand(e) for e in eqs]
        if collect_rho:
            eqs = [sp.collect(e, states) for e in eqs]
        if factor_terms:
            eqs = [sp.factor_terms(e) for e in eqs]
        mean_re, mean_im = sp.re(model["mean_operator"][0]), sp.im(model["mean_operator"][0])
    prepared = time.time()
    plan = optimize_rhs(eqs, mean_re, mean_im, states, sp.Symbol("Drive", real=True), Drive,
                        runtime_const_syms=model["runtime_const_syms"], cse_batch_size=cse_batch_size,
                        cse_simplify=cse_simplify, hoist_rho_independent=hoist_rho_independent,
                        extract_independent=ode_size is not None)
    compiled = CompiledRHS(
        kind="lindblad" if ode_size is None else "ode", state_size=size,
        sweep_symbols=tuple(sweep_symbols), state_symbols=tuple(states), equations=tuple(eqs),
        mean_re=mean_re, mean_im=mean_im, drive_map=Drive,
        rho0_exprs=None if model["rho0_exprs"] is None else tuple(model["rho0_exprs"]),
        runtime_const_syms=model["runtime_const_syms"], base_runtime_syms=model["base_runtime_syms"],
        derived_const_exprs=model["derived_const_exprs"], const_values=model["defaults"], plan=plan,
        cache_key=key, timings={"ode_prepare_s": prepared - start, "ode_optimize_s": time.time() - prepared},
        model=model)
    if reuse:
        _RHS_CODE_CACHE[key] = compiled
        if raw_key is not None:
            _RHS_CODE_CACHE[raw_key] = compiled
        _disk_put(key, compiled)
    return compiled, "miss"


# ----------------------------------------------------------------------------------------
# persistent cache of prepared RHS objects
# ----------------------------------------------------------------------------------------
# The symbolic derivation of larger models takes tens of seconds (N = 8: ~30 s) and, like the
# reference (which recompiles per process), would repeat in every new process. Prepared
# CompiledRHS objects are therefore pickled next to the model modules, keyed by the structural
# cache key. GQIS_DISK_CACHE=0 disables it.

def _disk_path(key):
    from .engine import cache_dir
    digest = hashlib.sha256(repr(key).encode()).hexdigest()[:32]
    return cache_dir().parent / "rhs" / f"{digest}.pkl"


def _disk_get(key):
    if os.environ.get("GQIS_DISK_CACHE", "1") == "0":
        return None
    path = _disk_path(key)
    if not path.exists():
        return None
    try:
        with open(path, "rb") as f:
            stored_key, compiled = pickle.load(f)
    except Exception:
        return None
    if stored_key != key:
        return None
    compiled.emitted = {}
    return compiled


def _disk_put(key, compiled):
    if os.environ.get("GQIS_DISK_CACHE", "1") == "0":
        return
    path = _disk_path(key)
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(f".{os.getpid()}.tmp")
        with open(tmp, "wb") as f:
            pickle.dump((key, compiled), f, protocol=pickle.HIGHEST_PROTOCOL)
        os.replace(tmp, path)
    except Exception:
        pass


def runtime_const_values(compiled, runtime_consts, const_values, use_defaults):
    """Values of the runtime constants for one call, in ``Const_arr`` order (``gqis/solver.py:1695-1709``)."""
    if not compiled.runtime_const_syms:
        return []
    values = dict(compiled.const_values) if use_defaults else {}
    values.update(const_values or {})
    values.update(runtime_consts or {})
    base = {}
    for s in compiled.base_runtime_syms:
        if s not in values:
            raise ValueError(f"Missing value for runtime constant symbol: {s}")
        base[s] = float(values[s])
    out = [base[s] for s in compiled.base_runtime_syms]
    out += [float(e.evalf(subs=base)) for e in compiled.derived_const_exprs]
    return out
