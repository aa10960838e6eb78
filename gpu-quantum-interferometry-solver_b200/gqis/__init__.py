"""GQIS on B200: drop-in sweep engine for ``mesolve_2D`` / ``odesolve_2D``.

Same public names as the reference package (``gqis/__init__.py:5-6``). The symbolic front end
imports eagerly (it needs only SymPy and NumPy); the GPU is touched only when a sweep runs.
"""

__version__ = "0.3.0+b200"

__all__ = ["build_independent_rho", "build_reduced_lindblad_rhs", "mesolve_2D", "odesolve_2D",
           "compile_lindblad_rhs", "compile_ode_rhs", "CompiledRHS"]

from .lindblad import build_independent_rho, build_reduced_lindblad_rhs  # noqa: E402
from .rhs import CompiledRHS  # noqa: E402
from .solver import compile_lindblad_rhs, mesolve_2D  # noqa: E402
from .gqis_ode_api import compile_ode_rhs, odesolve_2D  # noqa: E402
