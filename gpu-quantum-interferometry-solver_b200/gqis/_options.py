"""Grouped keyword options shared by ``mesolve_2D`` and ``odesolve_2D``.

The group table is part of the public interface of the reference package
(``gqis/_options.py:7-18``): callers may pass e.g. ``codegen=dict(cse_batch_size=8)``
instead of the flat keyword, so the group names and members are the reference's, plus this
engine's ``precision`` and ``rhs_form``. The error messages are the reference's too (its tests
match them).
"""

from collections.abc import Mapping
import inspect

OPTION_GROUPS = {
    "consts": ("const_values", "runtime_consts", "keep_symbolic_consts", "auto_runtime_consts"),
    "initial": ("rho0", "rho0_var_arrays", "rho0_values", "y0_values", "t_in"),
    "output": ("warmup_time", "return_time_trace", "time_trace_every", "time_trace_samples_per_period",
               "solver_samples_per_period", "return_device"),
    "solver_options": ("solver", "fp64", "solver_frequency", "adaptive_options", "precision", "rhs_form"),
    "codegen": ("RHSreuse", "kernel_template_file", "unroll", "pre_expand", "collect_rho", "factor_terms",
                "cse_batch_size", "cse_simplify", "hoist_rho_independent", "symbolic_workers",
                "max_symbolic_workers", "nvrtc_options"),
    "diagnostics": ("timings", "return_timing_info", "Actual_Kernel_Save", "beep_on_error",
                    "ignore_non_finite_output"),
}


_PLAIN_DEFAULTS = (bool, int, float, str, tuple)


def _untouched(value, default):
    """A flat option counts as set by the caller unless it is its signature default (the object
    itself, or an equal value of the same plain type)."""
    return value is default or (isinstance(default, _PLAIN_DEFAULTS) and type(value) is type(default)
                                and value == default)


def _grouped(groups):
    """``(group, option, value)`` for every option given inside a group, checked against the table."""
    for group, given in groups.items():
        if given is None:
            continue
        if not isinstance(given, Mapping):
            raise TypeError(f"{group} must be a dict of option names and values.")
        members = OPTION_GROUPS[group]
        for option, value in given.items():
            if option not in members:
                raise ValueError(f"Unknown {group} option '{option}'. Valid options: {', '.join(members)}.")
            yield group, option, value


def apply_option_groups(func, args, groups, extra=None):
    """Move options given inside groups into the flat keyword dict ``args`` of ``func``.

    ``groups`` maps a group name to a dict or None; ``extra`` is the ``**option_set`` dict of a
    function that forwards options it does not name. An option goes to ``args`` when ``func``
    names it, else to ``extra``; one given both flat and in its group, one outside its group, or
    one that ``func`` cannot take raises ``ValueError``. Returns ``(args, extra)``.
    """
    defaults = {name: p.default for name, p in inspect.signature(func).parameters.items()}
    for group, option, value in _grouped(groups):
        if option in defaults:
            target, taken = args, not _untouched(args[option], defaults[option])
        elif extra is not None:
            target, taken = extra, option in extra
        else:
            raise ValueError(f"{func.__name__} does not accept the {group} option '{option}'.")
        if taken:
            raise ValueError(f"'{option}' is given both directly and in {group}; use one.")
        target[option] = value
    return args, extra
