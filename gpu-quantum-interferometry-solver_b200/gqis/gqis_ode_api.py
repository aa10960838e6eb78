"""``odesolve_2D``: real first-order ODE sweeps on the same engine (``gqis/gqis_ode_api.py``).

User symbols are renamed to the engine's internal names - states to ``rho[i]``, time to the
drive ``ode_stage_time`` (evaluated in FP64 once per stage time), other parameters to
``ode_param_i`` - and the model goes through ``solver._solve_symbolic_system`` with
``_ode_size`` set (reference ``gqis/gqis_ode_api.py:115-255``). Without an observable the
outputs are states (``final_rho`` / ``mean_state`` modes); with one, the complex observable.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import sympy as sp

from ._options import OPTION_GROUPS, apply_option_groups

# Unlike Lindblad equations, user expressions are not simplified before CSE, so CSE
# simplification stays on for ODEs (e.g. (x + 1)**2 - x*(x + 2) becomes 1 only with it).
_ODE_CODEGEN_DEFAULTS = {"pre_expand": False, "collect_rho": False, "cse_simplify": True}
_ODE_CODEGEN_OPTIONS = ("pre_expand", "collect_rho", "factor_terms", "cse_batch_size",
                        "cse_simplify", "hoist_rho_independent", "RHSreuse")
_DUMMY_SWEEP = sp.Symbol("ode_dummy", real=True)


def odesolve_2D(rhs, state_symbols=None, y0=None, tlist=None, *, var_arrays=None,
                const_values=None, time_symbol=None, observable=None, output_mode="final",
                y0_values=None, runtime_consts=None, keep_symbolic_consts=None, solver="rk4",
                fp64=False, return_time_trace=False, time_trace_every=None, t_in=0.0,
                return_device=False, calibrate_timesteps=None, consts=None, initial=None, output=None,
                solver_options=None, codegen=None, diagnostics=None, **option_set):
    """Solve real first-order ODEs over zero, one or two parameter-sweep axes.

    ``rhs``: dy/dt expressions in ``state_symbols`` order (or ``Eq(Derivative(s, t), f)``), or a
    ``CompiledRHS`` from ``compile_ode_rhs``. ``y0``: initial values (may depend on sweep
    parameters) or None with ``y0_values`` of shape (nx, ny, n) / (nx, n). ``observable``:
    optional scalar expression; without it the output is the state vector.
    ``output_mode``: ``"final"`` or ``"mean"`` (right-endpoint average for fixed steps).
    Results have shape (nx, ny, n) without an observable, (nx, ny) complex with one; traces
    (nx, ny, nsamples, n) or (nx, ny, nsamples). Unused sweep axes have length one. Other
    ``mesolve_2D`` options (solver, precision, adaptive_options, codegen, diagnostics, ...)
    are forwarded; ``return_device=True`` returns torch CUDA tensors.
    """
    args = dict(locals())
    option_set = args.pop("option_set")
    groups = {name: args.pop(name) for name in OPTION_GROUPS}
    args, option_set = apply_option_groups(odesolve_2D, args, groups, option_set)
    return _solve_ode_system(**args, **option_set)


def compile_ode_rhs(rhs, state_symbols, y0=None, sweep_symbols=(), *, const_values=None,
                    runtime_consts=None, keep_symbolic_consts=None, time_symbol=None,
                    observable=None, **codegen_options):
    """Prepare and optimise an ODE RHS without device code (``gqis/gqis_ode_api.py:70-112``)."""
    unknown = set(codegen_options) - set(_ODE_CODEGEN_OPTIONS)
    if unknown:
        raise TypeError(f"Unknown compile_ode_rhs option(s): {sorted(unknown)}")
    sweep_symbols = tuple(sweep_symbols)
    if len(sweep_symbols) > 2:
        raise ValueError("At most two sweep symbols are supported.")
    model = _prepare_ode_model(rhs, state_symbols, y0, dict.fromkeys(sweep_symbols), const_values,
                               runtime_consts, keep_symbolic_consts, time_symbol, observable)
    from .solver import _compile_rhs
    options = {**_ODE_CODEGEN_DEFAULTS, **codegen_options}
    reuse = options.pop("RHSreuse", True)
    compiled, _ = _compile_rhs(
        model["H"], model["drive"], [], model["mean"], sweep_symbols=tuple(model["sweeps"]),
        const_values=model["constants"], runtime_consts=model["runtime"],
        keep_symbolic_consts=model["keep"], rho0=model["initial"], ode_size=model["size"],
        reuse=reuse, **options)
    return dataclasses.replace(compiled, ode={"symbol_map": model["replacements"],
                                              "sweep_symbols": sweep_symbols,
                                              "has_observable": observable is not None})


def _prepare_ode_model(rhs, state_symbols, y0, var_arrays, const_values, runtime_consts,
                       keep_symbolic_consts, time_symbol, observable):
    """Validate a user ODE and rename its symbols to the engine's internal names."""
    states = tuple(state_symbols)
    if (not states or any(not isinstance(s, sp.Symbol) for s in states)
            or len(set(states)) != len(states)):
        raise ValueError("state_symbols must contain distinct SymPy Symbols.")
    if any(s.is_real is False for s in states):
        raise ValueError("State symbols must represent real variables.")
    exprs = [sp.sympify(e) for e in rhs]
    if len(exprs) != len(states):
        raise ValueError("Provide one RHS expression per state symbol.")
    initial = None if y0 is None else [sp.sympify(e) for e in y0]
    if initial is not None and len(initial) != len(states):
        raise ValueError("y0 must contain one initial value per state symbol.")
    obs = sp.sympify(observable) if observable is not None else sp.Integer(0)
    symbols = set().union(*(e.free_symbols for e in [*exprs, *(initial or []), obs]))
    named_t = [s for s in symbols if s.name == "t" and s not in states]
    if time_symbol is None:
        if len(named_t) > 1:
            raise ValueError("Specify time_symbol when multiple different symbols are named t.")
        time_symbol = named_t[0] if named_t else sp.Symbol("t", real=True)
    if not isinstance(time_symbol, sp.Symbol) or time_symbol in states:
        raise ValueError("time_symbol must be a Symbol distinct from state_symbols.")
    for k, e in enumerate(exprs):
        if isinstance(e, sp.Equality):
            if e.lhs != sp.Derivative(states[k], time_symbol, evaluate=False):
                raise ValueError("Each equation must explicitly define its state derivative.")
            exprs[k] = e.rhs
    if any(e.has(sp.Derivative) for e in exprs):
        raise ValueError("Supply explicit first-order RHS expressions, without derivatives.")

    sweeps = {} if var_arrays is None else dict(var_arrays)
    constants = {} if const_values is None else dict(const_values)
    runtime = {} if runtime_consts is None else dict(runtime_consts)
    params = set(sweeps) | set(constants) | set(runtime)
    if any(not isinstance(s, sp.Symbol) for s in params) or params & (set(states) | {time_symbol}):
        raise ValueError("Parameter keys must be Symbols distinct from the state and time symbols.")
    if set(sweeps) & (set(constants) | set(runtime)):
        raise ValueError("A swept parameter cannot also be a constant.")
    unknown = symbols - set(states) - {time_symbol} - params
    if unknown:
        raise ValueError(f"Unassigned ODE parameters: {sorted(map(str, unknown))}")
    if initial is not None and any(e.free_symbols & (set(states) | {time_symbol}) for e in initial):
        raise ValueError("Initial values may depend on parameters, not on state or time.")
    names = {s: sp.Symbol(f"rho[{k}]", real=True) for k, s in enumerate(states)}
    stage_time = sp.Symbol("ode_stage_time", real=True)
    names[time_symbol] = stage_time
    names.update({s: sp.Symbol(f"ode_param_{k}", real=True)
                  for k, s in enumerate(sorted(params, key=sp.srepr))})
    exprs = [e.xreplace(names) for e in exprs]
    initial = None if initial is None else [e.xreplace(names) for e in initial]
    if any(sp.simplify(sp.im(e)) != 0 for e in [*exprs, *(initial or [])]):
        raise ValueError("ODE states and RHS must be real; split complex states into real/imaginary parts.")
    obs = obs.xreplace(names)

    def rename(mapping):
        return {names[s]: v for s, v in mapping.items()}
    sweeps = rename(sweeps) or {_DUMMY_SWEEP: np.zeros(1)}
    if keep_symbolic_consts is not None and not isinstance(keep_symbolic_consts, str):
        keep_symbolic_consts = [names[s] for s in keep_symbolic_consts]
    drive = {stage_time: sp.Symbol("t", real=True)} if time_symbol in symbols else {}
    return {"H": sp.Matrix(exprs), "drive": drive, "mean": sp.Matrix([obs]), "initial": initial,
            "sweeps": sweeps, "constants": rename(constants), "runtime": rename(runtime),
            "keep": keep_symbolic_consts, "size": len(states), "replacements": names}


def _solve_ode_system(rhs, state_symbols, y0, tlist, *, var_arrays, const_values, time_symbol,
                      observable, output_mode, y0_values, runtime_consts, keep_symbolic_consts,
                      solver, fp64, return_time_trace, time_trace_every, t_in, return_device,
                      calibrate_timesteps, **option_set):
    from .solver import CompiledRHS, _check_sweep_arrays_nonempty, _solve_symbolic_system
    if tlist is None:
        raise TypeError("odesolve_2D needs tlist.")
    _check_sweep_arrays_nonempty(var_arrays)
    if output_mode not in {"mean", "final"}:
        raise ValueError("output_mode must be 'mean' or 'final'.")
    if y0 is not None and y0_values is not None:
        raise ValueError("Use either y0 or y0_values, not both.")
    if y0_values is not None and not hasattr(y0_values, "data_ptr") and np.iscomplexobj(y0_values):
        raise ValueError("y0_values must be real; split complex states into real/imaginary parts.")
    if y0_values is not None and hasattr(y0_values, "is_complex") and y0_values.is_complex():
        raise ValueError("y0_values must be real; split complex states into real/imaginary parts.")
    if any((k.startswith("_") and k not in ("_prebuild_only", "_prepare_only"))
           or k in {"rho0", "rho0_values", "rho0_var_arrays", "compiled_rhs"} for k in option_set):
        raise ValueError("Use y0/y0_values and var_arrays for ODE initial conditions.")

    if isinstance(rhs, CompiledRHS):
        compiled = rhs
        if compiled.kind != "ode" or compiled.ode is None:
            raise ValueError("Pass a CompiledRHS from compile_ode_rhs (compile_lindblad_rhs "
                             "results go to mesolve_2D).")
        if any(v is not None for v in (state_symbols, y0, const_values, keep_symbolic_consts,
                                       time_symbol, observable)):
            raise ValueError("state_symbols, y0, const_values, keep_symbolic_consts, time_symbol "
                             "and observable are fixed when the RHS is compiled.")
        if y0_values is None and compiled.rho0_exprs is None:
            raise ValueError("Provide y0_values: no y0 was given when the RHS was compiled.")
        if tuple(var_arrays or {}) != compiled.ode["sweep_symbols"]:
            raise ValueError(f"var_arrays must sweep {compiled.ode['sweep_symbols']}, in the order "
                             "given when the RHS was compiled.")
        smap = compiled.ode["symbol_map"]

        def remap(mapping, what):
            bad = [s for s in mapping if s not in smap]
            if bad:
                raise ValueError(f"{what} contains symbols unknown to the compiled RHS: {bad}")
            return {smap[s]: v for s, v in mapping.items()}
        sweeps = remap(var_arrays or {}, "var_arrays") or {_DUMMY_SWEEP: np.zeros(1)}
        runtime = remap(runtime_consts or {}, "runtime_consts")
        has_obs = compiled.ode["has_observable"]
        mode = output_mode if has_obs else {"final": "final_rho", "mean": "mean_state"}[output_mode]
        return _solve_symbolic_system(
            None, None, None, None, tlist, var_arrays=sweeps, runtime_consts=runtime,
            rho0_values=y0_values, output_mode=mode, solver=solver, fp64=fp64,
            return_time_trace=return_time_trace, time_trace_every=time_trace_every, t_in=t_in,
            return_device=return_device, calibrate_timesteps=calibrate_timesteps,
            compiled_rhs=compiled, _ode_size=compiled.state_size, _state_trace=not has_obs, **option_set)

    if state_symbols is None:
        raise TypeError("odesolve_2D needs state_symbols (or a CompiledRHS as rhs).")
    if y0 is None and y0_values is None:
        raise ValueError("Provide y0 or y0_values.")
    model = _prepare_ode_model(rhs, state_symbols, y0, var_arrays, const_values, runtime_consts,
                               keep_symbolic_consts, time_symbol, observable)
    for name, value in _ODE_CODEGEN_DEFAULTS.items():
        option_set.setdefault(name, value)
    mode = output_mode if observable is not None else {"final": "final_rho", "mean": "mean_state"}[output_mode]
    return _solve_symbolic_system(
        model["H"], model["drive"], [], model["mean"], tlist, var_arrays=model["sweeps"],
        const_values=model["constants"], runtime_consts=model["runtime"],
        keep_symbolic_consts=model["keep"], rho0=model["initial"], rho0_values=y0_values,
        output_mode=mode, solver=solver, fp64=fp64, return_time_trace=return_time_trace,
        time_trace_every=time_trace_every, t_in=t_in, return_device=return_device,
        calibrate_timesteps=calibrate_timesteps, _ode_size=model["size"],
        _state_trace=observable is None, **option_set)
