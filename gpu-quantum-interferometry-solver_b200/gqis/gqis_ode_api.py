"""``odesolve_2D`` and ``compile_ode_rhs``: real first-order ODE sweeps on the sweep engine.

Interface of the reference's ``gqis/gqis_ode_api.py:17-255``: the signatures, defaults, output
shapes, the internal names a compiled RHS reports (``rho[i]`` for states, ``ParX``/``ParY`` for
sweeps, ``ode_param_i`` for other parameters) and the error messages (the reference's tests match
them).

How it maps onto the engine: an ODE is a "model" whose equations take the place of the reduced
Lindblad equations. :func:`_translate` checks the user's model and renames its symbols -
states to ``rho[i]``, time to the drive symbol ``ode_stage_time`` (the engine evaluates drives in
FP64 once per stage time), parameters to ``ode_param_i`` - giving an :class:`OdeModel`; the
engine call then carries ``_ode_size`` (the state count) instead of a Hilbert-space dimension.
Without an observable the outputs are states (the engine's ``final_rho`` / ``mean_state``
modes); with one, the complex observable.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import sympy as sp

from ._options import OPTION_GROUPS, apply_option_groups

# User ODE expressions, unlike derived Lindblad equations, reach CSE unsimplified, so CSE
# simplification is on for them (e.g. (x + 1)**2 - x*(x + 2) becomes 1 only with it).
_ODE_CODEGEN_DEFAULTS = {"pre_expand": False, "collect_rho": False, "cse_simplify": True}
_ODE_CODEGEN_OPTIONS = ("pre_expand", "collect_rho", "factor_terms", "cse_batch_size",
                        "cse_simplify", "hoist_rho_independent", "RHSreuse")
_DUMMY_SWEEP = sp.Symbol("ode_dummy", real=True)  # the sweep axis of a call that sweeps nothing
_STAGE_TIME = sp.Symbol("ode_stage_time", real=True)
_STATE_OUTPUT = {"final": "final_rho", "mean": "mean_state"}  # engine modes without an observable
_INITIAL_STATE_OPTIONS = {"rho0", "rho0_values", "rho0_var_arrays", "compiled_rhs"}


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
    call = dict(locals())
    forwarded = call.pop("option_set")
    grouped = {group: call.pop(group) for group in OPTION_GROUPS}
    call, forwarded = apply_option_groups(odesolve_2D, call, grouped, forwarded)
    return _solve_ode_system(**call, **forwarded)


def compile_ode_rhs(rhs, state_symbols, y0=None, sweep_symbols=(), *, const_values=None,
                    runtime_consts=None, keep_symbolic_consts=None, time_symbol=None,
                    observable=None, **codegen_options):
    """Check and optimise an ODE RHS without device code (reference ``gqis/gqis_ode_api.py:70-112``);
    ``odesolve_2D(compiled, tlist=..., var_arrays=...)`` then starts from code emission."""
    unknown = set(codegen_options) - set(_ODE_CODEGEN_OPTIONS)
    if unknown:
        raise TypeError(f"Unknown compile_ode_rhs option(s): {sorted(unknown)}")
    sweep_symbols = tuple(sweep_symbols)
    if len(sweep_symbols) > 2:
        raise ValueError("At most two sweep symbols are supported.")
    model = _translate(rhs, state_symbols, y0, dict.fromkeys(sweep_symbols), const_values, runtime_consts,
                       keep_symbolic_consts, time_symbol, observable)
    from .solver import _compile_rhs
    options = dict(_ODE_CODEGEN_DEFAULTS, **codegen_options)
    reuse = options.pop("RHSreuse", True)
    compiled, _ = _compile_rhs(*model.engine_model(), sweep_symbols=tuple(model.sweeps),
                               const_values=model.constants, runtime_consts=model.runtime,
                               keep_symbolic_consts=model.keep, rho0=model.initial, ode_size=model.size,
                               reuse=reuse, **options)
    # the user-to-internal name map belongs to this call: equal internal models can come from other names
    return dataclasses.replace(compiled, ode={"symbol_map": model.names, "sweep_symbols": sweep_symbols,
                                              "has_observable": observable is not None})


# ------------------------------------------------------------------------------ the model

@dataclasses.dataclass
class OdeModel:
    """A checked ODE in the engine's internal names."""
    equations: list
    initial: list | None
    observable: sp.Expr
    uses_time: bool
    sweeps: dict
    constants: dict
    runtime: dict
    keep: object
    names: dict  # user symbol -> internal symbol

    @property
    def size(self):
        return len(self.equations)

    def engine_model(self):
        """(H, Drive, Col_Ops, mean_operator) positional arguments of the engine for this ODE: the
        equations in place of H, time as the one drive, no collapse operators."""
        drive = {_STAGE_TIME: sp.Symbol("t", real=True)} if self.uses_time else {}
        return sp.Matrix(self.equations), drive, [], sp.Matrix([self.observable])


def _states_of(state_symbols):
    states = tuple(state_symbols)
    if not states or not all(isinstance(s, sp.Symbol) for s in states) or len(set(states)) < len(states):
        raise ValueError("state_symbols must contain distinct SymPy Symbols.")
    if any(s.is_real is False for s in states):
        raise ValueError("State symbols must represent real variables.")
    return states


def _time_symbol_of(time_symbol, found, states):
    """The given time symbol, else the one free symbol named ``t`` that is not a state."""
    if time_symbol is None:
        named_t = {s for s in found if s.name == "t"} - set(states)
        if len(named_t) > 1:
            raise ValueError("Specify time_symbol when multiple different symbols are named t.")
        time_symbol = named_t.pop() if named_t else sp.Symbol("t", real=True)
    if not isinstance(time_symbol, sp.Symbol) or time_symbol in states:
        raise ValueError("time_symbol must be a Symbol distinct from state_symbols.")
    return time_symbol


def _explicit_rhs(expressions, states, time_symbol):
    """Right-hand sides, with ``Eq(Derivative(state, t), f)`` forms reduced to ``f``."""
    out = []
    for state, expression in zip(states, expressions):
        if isinstance(expression, sp.Equality):
            if expression.lhs != sp.Derivative(state, time_symbol, evaluate=False):
                raise ValueError("Each equation must explicitly define its state derivative.")
            expression = expression.rhs
        out.append(expression)
    if any(e.has(sp.Derivative) for e in out):
        raise ValueError("Supply explicit first-order RHS expressions, without derivatives.")
    return out


def _translate(rhs, state_symbols, y0, var_arrays, const_values, runtime_consts, keep_symbolic_consts,
               time_symbol, observable):
    """Check a user ODE and rename it into the engine's internal symbols."""
    states = _states_of(state_symbols)
    expressions = [sp.sympify(e) for e in rhs]
    if len(expressions) != len(states):
        raise ValueError("Provide one RHS expression per state symbol.")
    initial = None if y0 is None else [sp.sympify(v) for v in y0]
    if initial is not None and len(initial) != len(states):
        raise ValueError("y0 must contain one initial value per state symbol.")
    observed = sp.Integer(0) if observable is None else sp.sympify(observable)
    found = set().union(*(e.free_symbols for e in (*expressions, *(initial or ()), observed)))
    time_symbol = _time_symbol_of(time_symbol, found, states)
    expressions = _explicit_rhs(expressions, states, time_symbol)

    sweeps, constants, runtime = (dict(m or {}) for m in (var_arrays, const_values, runtime_consts))
    parameters = set(sweeps) | set(constants) | set(runtime)
    reserved = set(states) | {time_symbol}
    if not all(isinstance(p, sp.Symbol) for p in parameters) or parameters & reserved:
        raise ValueError("Parameter keys must be Symbols distinct from the state and time symbols.")
    if set(sweeps) & (set(constants) | set(runtime)):
        raise ValueError("A swept parameter cannot also be a constant.")
    unassigned = found - reserved - parameters
    if unassigned:
        raise ValueError(f"Unassigned ODE parameters: {sorted(map(str, unassigned))}")
    if initial is not None and any(v.free_symbols & reserved for v in initial):
        raise ValueError("Initial values may depend on parameters, not on state or time.")

    # internal names cannot collide with the kernel's locals or CSE temporaries
    names = {state: sp.Symbol(f"rho[{k}]", real=True) for k, state in enumerate(states)}
    names[time_symbol] = _STAGE_TIME
    for k, p in enumerate(sorted(parameters, key=sp.srepr)):
        names[p] = sp.Symbol(f"ode_param_{k}", real=True)
    expressions = [e.xreplace(names) for e in expressions]
    initial = None if initial is None else [v.xreplace(names) for v in initial]
    if any(sp.simplify(sp.im(e)) != 0 for e in (*expressions, *(initial or ()))):
        raise ValueError("ODE states and RHS must be real; split complex states into real/imaginary parts.")
    keep = keep_symbolic_consts
    if keep is not None and not isinstance(keep, str):
        keep = [names[s] for s in keep]

    def internal(mapping):
        return {names[s]: v for s, v in mapping.items()}
    return OdeModel(equations=expressions, initial=initial, observable=observed.xreplace(names),
                    uses_time=time_symbol in found, sweeps=internal(sweeps) or {_DUMMY_SWEEP: np.zeros(1)},
                    constants=internal(constants), runtime=internal(runtime), keep=keep, names=names)


# -------------------------------------------------------------------------------- the call

def _check_call(tlist, var_arrays, output_mode, y0, y0_values, option_set):
    """Checks that apply to compiled and symbolic ODE calls alike."""
    from .solver import _check_sweep_arrays_nonempty
    if tlist is None:
        raise TypeError("odesolve_2D needs tlist.")
    _check_sweep_arrays_nonempty(var_arrays)
    if output_mode not in _STATE_OUTPUT:
        raise ValueError("output_mode must be 'mean' or 'final'.")
    if y0 is not None and y0_values is not None:
        raise ValueError("Use either y0 or y0_values, not both.")
    if y0_values is not None:
        complex_values = (y0_values.is_complex() if hasattr(y0_values, "is_complex")
                          else np.iscomplexobj(y0_values))
        if complex_values:
            raise ValueError("y0_values must be real; split complex states into real/imaginary parts.")
    internal = {"_prebuild_only", "_prepare_only"}  # set by prebuild / prepare_sweep, not by users
    if any(k in _INITIAL_STATE_OPTIONS or (k.startswith("_") and k not in internal) for k in option_set):
        raise ValueError("Use y0/y0_values and var_arrays for ODE initial conditions.")


def _from_compiled(compiled, state_symbols, y0, const_values, keep_symbolic_consts, time_symbol,
                   observable, y0_values, var_arrays, runtime_consts):
    """Engine sweeps and runtime constants of a call on a ``compile_ode_rhs`` result."""
    if compiled.kind != "ode" or compiled.ode is None:
        raise ValueError("Pass a CompiledRHS from compile_ode_rhs (compile_lindblad_rhs "
                         "results go to mesolve_2D).")
    if any(v is not None for v in (state_symbols, y0, const_values, keep_symbolic_consts, time_symbol, observable)):
        raise ValueError("state_symbols, y0, const_values, keep_symbolic_consts, time_symbol "
                         "and observable are fixed when the RHS is compiled.")
    if y0_values is None and compiled.rho0_exprs is None:
        raise ValueError("Provide y0_values: no y0 was given when the RHS was compiled.")
    expected = compiled.ode["sweep_symbols"]
    if tuple(var_arrays or {}) != expected:
        raise ValueError(f"var_arrays must sweep {expected}, in the order given when the RHS was compiled.")
    names = compiled.ode["symbol_map"]

    def internal(mapping, what):
        foreign = [s for s in mapping if s not in names]
        if foreign:
            raise ValueError(f"{what} contains symbols unknown to the compiled RHS: {foreign}")
        return {names[s]: v for s, v in mapping.items()}
    sweeps = internal(var_arrays or {}, "var_arrays") or {_DUMMY_SWEEP: np.zeros(1)}
    return sweeps, internal(runtime_consts or {}, "runtime_consts")


def _solve_ode_system(rhs, state_symbols, y0, tlist, *, var_arrays, const_values, time_symbol,
                      observable, output_mode, y0_values, runtime_consts, keep_symbolic_consts,
                      solver, fp64, return_time_trace, time_trace_every, t_in, return_device,
                      calibrate_timesteps, **option_set):
    from .solver import CompiledRHS, _solve_symbolic_system
    _check_call(tlist, var_arrays, output_mode, y0, y0_values, option_set)
    shared = dict(rho0_values=y0_values, solver=solver, fp64=fp64, return_time_trace=return_time_trace,
                  time_trace_every=time_trace_every, t_in=t_in, return_device=return_device,
                  calibrate_timesteps=calibrate_timesteps)

    if isinstance(rhs, CompiledRHS):
        sweeps, runtime = _from_compiled(rhs, state_symbols, y0, const_values, keep_symbolic_consts, time_symbol,
                                         observable, y0_values, var_arrays, runtime_consts)
        observed = rhs.ode["has_observable"]
        return _solve_symbolic_system(
            None, None, None, None, tlist, var_arrays=sweeps, runtime_consts=runtime,
            output_mode=output_mode if observed else _STATE_OUTPUT[output_mode], compiled_rhs=rhs,
            _ode_size=rhs.state_size, _state_trace=not observed, **shared, **option_set)

    if state_symbols is None:
        raise TypeError("odesolve_2D needs state_symbols (or a CompiledRHS as rhs).")
    if y0 is None and y0_values is None:
        raise ValueError("Provide y0 or y0_values.")
    model = _translate(rhs, state_symbols, y0, var_arrays, const_values, runtime_consts, keep_symbolic_consts,
                       time_symbol, observable)
    options = dict(_ODE_CODEGEN_DEFAULTS, **option_set)
    observed = observable is not None
    return _solve_symbolic_system(
        *model.engine_model(), tlist, var_arrays=model.sweeps, const_values=model.constants,
        runtime_consts=model.runtime, keep_symbolic_consts=model.keep, rho0=model.initial,
        output_mode=output_mode if observed else _STATE_OUTPUT[output_mode], _ode_size=model.size,
        _state_trace=not observed, **shared, **options)
