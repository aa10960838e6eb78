"""Grouped keyword options shared by ``mesolve_2D`` and ``odesolve_2D``.

The group table is part of the public interface of the reference package
(``gqis/_options.py:7-18``): callers may pass e.g. ``codegen=dict(cse_batch_size=8)``
instead of the flat keyword. The group names and their members are therefore kept
identical; the merge logic below is this package's own.
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


def _still_default(value, default):
    """True when ``value`` is the untouched signature default of a flat option."""
    if value is default:
        return True
    simple = (bool, int, float, str, tuple)
    return isinstance(default, simple) and type(value) is type(default) and value == default


def apply_option_groups(func, args, groups, extra=None):
    """Fold grouped options into the flat keyword dict ``args`` of ``func``.

    ``groups`` maps a group name to a dict (or None); ``extra`` is the ``**option_set``
    dict of a function that forwards unknown options. Each option may be given either
    flat or inside its group; giving it both ways, naming an option that does not belong
    to the group, or naming one that ``func`` cannot accept raises ``ValueError``
    (behaviour of ``gqis/_options.py:30-57``).
    """
    signature = inspect.signature(func).parameters
    for group_name, members in groups.items():
        if members is None:
            continue
        if not isinstance(members, Mapping):
            raise TypeError(f"{group_name} must be a dict of option names and values.")
        allowed = OPTION_GROUPS[group_name]
        for name, value in members.items():
            if name not in allowed:
                raise ValueError(f"Unknown {group_name} option '{name}'. "
                                 f"Valid options: {', '.join(allowed)}.")
            if name in signature:
                if not _still_default(args[name], signature[name].default):
                    raise ValueError(f"'{name}' is given both directly and in {group_name}; use one.")
                args[name] = value
            elif extra is not None:
                if name in extra:
                    raise ValueError(f"'{name}' is given both directly and in {group_name}; use one.")
                extra[name] = value
            else:
                raise ValueError(f"{func.__name__} does not accept the {group_name} option '{name}'.")
    return args, extra
