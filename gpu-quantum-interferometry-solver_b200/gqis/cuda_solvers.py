"""Integrator registry: names, aliases, orders, tableaus and per-launch parameters.

The solver names, aliases, orders and RHS counts are the public vocabulary of the reference
(``gqis/cuda_solvers.py:993-1052``) and are kept, so ``solver="RK45"`` or ``"DOP-853"`` mean
the same method. The device code is not generated text here: each solver names one of the
hand-written CUDA templates in ``csrc/`` (``gqis_fixed.cuh``, ``gqis_adaptive.cuh``), and
explicit Runge-Kutta methods pass their Butcher tableau, printed as ``constexpr`` data into
the model module. ``dop853a`` (adaptive DOP853) is new; the reference has only the fixed-step
main formula.

Tableau sources: classical RK4; Dormand & Prince (1980) and DOP853 (Hairer, Norsett & Wanner,
"Solving ODEs I") taken from SciPy's published implementation (``scipy.integrate._ivp``);
Tsitouras (2011) "Runge-Kutta pairs of order 5(4) satisfying only the first column simplifying
assumption"; Alshina, Zaks & Kalitkin (2008) six-stage order-6 scheme; Anastassi & Simos
(2005) frequency-fitted fifth-order method; Carpenter & Kennedy (1994) 2N-storage RK4.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import mpmath as mp

TSIT5A_DEFAULTS = {
    "step_rtol": 1e-5,     # per-step relative tolerance of the local error estimate
    "step_atol": 1e-5,     # per-step absolute tolerance
    "max_substeps": 64,    # accepted + rejected steps allowed per output interval of tlist
    "fp64_time": True,     # accepted for compatibility: time is always FP64 in this engine
    "count_steps": False,  # return accepted/rejected step counts per point (timing info)
}
ADAPTIVE_DEFAULTS = TSIT5A_DEFAULTS


@dataclass(frozen=True)
class Tableau:
    """Explicit RK tableau; ``a1``/``b1`` hold the part proportional to the fitted parameter w."""

    c: tuple
    a: tuple
    b: tuple
    a1: tuple = ()
    b1: tuple = ()
    e: tuple = ()    # Tsit5 error weights b - b_hat (index 6 weights f(y_new))
    e5: tuple = ()   # DOP853 fifth-order error weights
    e3: tuple = ()   # DOP853 third-order error weights

    @property
    def stages(self):
        return len(self.b)


@dataclass(frozen=True)
class SolverSpec:
    """Metadata of one integrator and the CUDA template that runs it."""

    name: str
    label: str
    order: int
    rhs_evaluations: int
    template: str                 # C++ integrator type in csrc/
    solver_id: int                # GQIS_SOLVER_* of include/gqis_b200.h
    adaptive: bool = False
    tableau: Tableau | None = field(default=None, repr=False)
    parameters: tuple = ()        # per-launch values for gqis_sweep_desc.solver_params

    @property
    def source(self):
        """Identifier of the device code (the template type), kept for introspection."""
        return self.template


def _rows(n, entries):
    """Lower-triangular ``a`` rows of an n-stage tableau from {(i, j): value}."""
    return tuple(tuple(float(entries.get((i, j), 0.0)) for j in range(n)) for i in range(n))


def _tsit5():
    c = (0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0)
    a = {(1, 0): 0.161,
         (2, 0): -0.008480655492356989, (2, 1): 0.335480655492357,
         (3, 0): 2.897153057105493, (3, 1): -6.359448489975075, (3, 2): 4.3622954328695815,
         (4, 0): 5.325864828439257, (4, 1): -11.748883564062828, (4, 2): 7.4955393428898365,
         (4, 3): -0.09249506636175525,
         (5, 0): 5.86145544294642, (5, 1): -12.92096931784711, (5, 2): 8.159367898576159,
         (5, 3): -0.071584973281401, (5, 4): -0.028269050394068383}
    b = (0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081,
         2.324710524099774)
    e = (-0.00178001105222577714, -0.0008164344596567469, 0.007880878010261995, -0.1447110071732629,
         0.5823571654525552, -0.45808210592918697, 0.015151515151515152)
    return Tableau(c=c, a=_rows(6, a), b=b, e=e)


def _dp5():
    from scipy.integrate._ivp.rk import RK45
    n = 6
    a = {(i, j): RK45.A[i, j] for i in range(n) for j in range(min(i, RK45.A.shape[1]))}
    return Tableau(c=tuple(float(x) for x in RK45.C), a=_rows(n, a), b=tuple(float(x) for x in RK45.B))


def _dop853():
    from scipy.integrate._ivp import dop853_coefficients as dc
    n = dc.N_STAGES
    a = {(i, j): dc.A[i, j] for i in range(n) for j in range(i)}
    return Tableau(c=tuple(float(x) for x in dc.C[:n]), a=_rows(n, a), b=tuple(float(x) for x in dc.B),
                   e5=tuple(float(x) for x in dc.E5[:n]), e3=tuple(float(x) for x in dc.E3[:n]))


def _alshina6():
    s5 = math.sqrt(5.0)
    c = (0.0, 4 / 7, 5 / 7, 6 / 7, (5 - s5) / 10, (5 + s5) / 10, 1.0)
    a = {(1, 0): 4 / 7,
         (2, 0): 115 / 112, (2, 1): -5 / 16,
         (3, 0): 589 / 630, (3, 1): 5 / 18, (3, 2): -16 / 45,
         (4, 0): 0.18002567144208434, (4, 1): 0.14737940683961614, (4, 2): 0.016070163293314288,
         (4, 3): -0.0670820393249937,
         (5, 0): -0.07979765856603138, (5, 1): 0.025290591998992584, (5, 2): -0.3516326202266813,
         (5, 3): 0.3207294901687516, (5, 4): 0.8090169943749475,
         (6, 0): 0.4988599356197352, (6, 1): -0.8633499941930429, (6, 2): 1.6778122846668349,
         (6, 3): -1.2682372542187894, (6, 4): -0.42705098312484235, (6, 5): 1.381966011250105}
    return Tableau(c=c, a=_rows(7, a), b=(1 / 12, 0.0, 0.0, 0.0, 5 / 12, 5 / 12, 1 / 12))


def _anas5():
    c = (0.0, 0.1, 1 / 3, 2 / 3, 0.9, 1.0)
    a = {(1, 0): 1 / 10,
         (2, 0): -2 / 9, (2, 1): 5 / 9,
         (3, 0): 28 / 9, (3, 1): -40 / 9, (3, 2): 2.0,
         (4, 0): -11277 / 8000, (4, 1): 171 / 80, (4, 2): -459 / 2000, (4, 3): 3213 / 8000,
         (5, 0): -4.0, (5, 1): 5.0}
    a1 = {(5, 0): -0.595, (5, 2): 1.89, (5, 3): -2.295, (5, 4): 1.0}  # times the fitted w
    b = (23 / 216, 0.0, 63 / 136, 9 / 56, 1000 / 3213, -1 / 24)
    return Tableau(c=c, a=_rows(6, a), b=b, a1=_rows(6, a1), b1=(0.0,) * 6)


def _rk4_tableau():
    return Tableau(c=(0.0, 0.5, 0.5, 1.0), a=_rows(4, {(1, 0): 0.5, (2, 1): 0.5, (3, 2): 1.0}),
                   b=(1 / 6, 1 / 3, 1 / 3, 1 / 6))


def _spec(name, label, order, rhs, template, sid, adaptive=False, tableau=None):
    return SolverSpec(name, label, order, rhs, template, sid, adaptive, tableau)


_SOLVERS = {
    "rk4": _spec("rk4", "RK4", 4, 4, "gqfixed::RK4", 0, tableau=_rk4_tableau()),
    "lserk4": _spec("lserk4", "LSRK4", 4, 5, "gqfixed::LowStorageRK4", 1),
    "lserk4f": _spec("lserk4f", "LSRK4F", 4, 5, "gqfixed::LowStorageRK4", 2),
    "dp5": _spec("dp5", "DP5", 5, 6, "gqfixed::ExplicitRK<gqmodel::Tableau>", 3, tableau=_dp5()),
    "ab5": _spec("ab5", "AB5", 5, 1, "gqfixed::AdamsBashforth5", 4),
    "anas5": _spec("anas5", "Anas5", 5, 6, "gqfixed::ExplicitRK<gqmodel::Tableau>", 5, tableau=_anas5()),
    "tsit5": _spec("tsit5", "Tsit5", 5, 6, "gqfixed::ExplicitRK<gqmodel::Tableau>", 6, tableau=_tsit5()),
    "alshina6": _spec("alshina6", "Alshina6", 6, 7, "gqfixed::ExplicitRK<gqmodel::Tableau>", 7,
                      tableau=_alshina6()),
    "dop853": _spec("dop853", "DOP853", 8, 12, "gqfixed::ExplicitRK<gqmodel::Tableau>", 8, tableau=_dop853()),
    "tsit5a": _spec("tsit5a", "Tsit5A", 5, 6, "gqadaptive::Tsit5Pair<gqmodel::Tableau>", 9, True, _tsit5()),
    "dop853a": _spec("dop853a", "DOP853A", 8, 12, "gqadaptive::Dop853Pair<gqmodel::Tableau>", 10, True,
                     _dop853()),
}

_ALIASES = {
    "classical_rk4": "rk4",
    "carpenter_kennedy": "lserk4",
    "carpenter_kennedy_2n54": "lserk4",
    "dormand_prince": "dp5",
    "dormand_prince_5": "dp5",
    "rk45": "dp5",
    "anastassi5": "anas5",
    "anastassi_simos": "anas5",
    "adams_bashforth_5": "ab5",
    "alshina": "alshina6",
    "dormand_prince_853": "dop853",
    "dop_853": "dop853",
    "dop853_adaptive": "dop853a",
    "adaptive_dop853": "dop853a",
}


def available_solvers():
    """Canonical solver names in display order."""
    return tuple(_SOLVERS)


def normalize_solver_name(solver):
    """Canonical lower-case solver name; ``ValueError`` for an unknown one."""
    key = str(solver).strip().lower().replace(" ", "_").replace("-", "_")
    key = _ALIASES.get(key, key)
    if key not in _SOLVERS:
        raise ValueError(f"Unsupported solver '{solver}'. Use one of: {', '.join(_SOLVERS)}")
    return key


def anas5_fitted_parameter(frequency, step_size):
    """Frequency-fitted coefficient w of Anas5 from v = frequency * dt (evaluated in 60 digits).

    Anastassi & Simos (2005): with a43 = 2 the fitted weight is
    w = -(8000/1071) * (-2 v^5 + 6 tan(v) v^4 + 24 v^3 - 72 tan(v) v^2 - 144 v + 144 tan(v))
        / (v^5 (2 tan(v) v + 12 - 20)),
    and w = -800/1071 in the limit v -> 0 (the non-fitted method).
    """
    if not (step_size is not None and mp.isfinite(step_size) and step_size > 0.0):
        raise ValueError("anas5 requires a positive finite step_size")
    frequency = 1.0 if frequency is None else float(frequency)
    if not mp.isfinite(frequency) or frequency < 0.0:
        raise ValueError("solver_frequency must be a finite non-negative angular frequency")
    with mp.workdps(60):
        v = mp.mpf(str(frequency)) * mp.mpf(str(step_size))
        if v == 0:
            return float(mp.mpf(-800) / 1071)
        tv = mp.tan(v)
        num = -2 * v**5 + 6 * tv * v**4 + 24 * v**3 - 72 * tv * v**2 - 144 * v + 144 * tv
        den = v**5 * (2 * tv * v + 12 - 20)
        return float((-mp.mpf(8000) / 1071) * num / den)


def _adaptive_parameters(adaptive_options):
    options = dict(TSIT5A_DEFAULTS)
    unknown = set(adaptive_options or {}) - set(options)
    if unknown:
        raise ValueError(f"Unknown adaptive_options {sorted(unknown)}; use {sorted(options)}.")
    options.update(adaptive_options or {})
    rtol, atol = float(options["step_rtol"]), float(options["step_atol"])
    if not (rtol >= 0.0 and atol >= 0.0 and rtol + atol > 0.0 and math.isfinite(rtol + atol)):
        raise ValueError("step_rtol and step_atol must be finite, non-negative and not both zero.")
    max_substeps = int(options["max_substeps"])
    if max_substeps < 1:
        raise ValueError("max_substeps must be at least 1.")
    return (rtol, atol, float(max_substeps)), bool(options["count_steps"])


def get_solver_spec(solver, *, frequency=None, step_size=None, adaptive_options=None, fp64=False):
    """Spec of ``solver`` with its per-launch parameters (``gqis/cuda_solvers.py:1041-1075``)."""
    spec = _SOLVERS[normalize_solver_name(solver)]
    if spec.adaptive:
        params, _ = _adaptive_parameters(adaptive_options)
        return SolverSpec(spec.name, spec.label, spec.order, spec.rhs_evaluations, spec.template,
                          spec.solver_id, True, spec.tableau, params)
    if adaptive_options:
        raise ValueError("adaptive_options apply only to the adaptive solvers ('tsit5a', 'dop853a').")
    params = ()
    if spec.name == "anas5" and step_size is not None:
        params = (anas5_fitted_parameter(frequency, step_size),)
    return SolverSpec(spec.name, spec.label, spec.order, spec.rhs_evaluations, spec.template,
                      spec.solver_id, False, spec.tableau, params)


def counts_steps(adaptive_options):
    """True when the adaptive options ask for per-point accepted/rejected counts."""
    return _adaptive_parameters(adaptive_options)[1]


def tableau_source(spec):
    """``constexpr`` C++ struct ``Tableau`` of an explicit RK spec (empty for other solvers)."""
    t = spec.tableau
    if t is None or spec.template in ("gqfixed::RK4",):
        return ""
    n = t.stages
    a1 = t.a1 or tuple((0.0,) * n for _ in range(n))
    b1 = t.b1 or (0.0,) * n

    def arr(vals):
        return "{" + ", ".join(repr(float(v)) for v in vals) + "}"

    def mat(rows):
        return "{" + ", ".join(arr(r) for r in rows) + "}"

    def vec_fn(name, vals):
        if not vals:
            return f"    __host__ __device__ static constexpr double {name}(int) {{ return 0.0; }}\n"
        return (f"    __host__ __device__ static constexpr double {name}(int i) {{\n"
                f"        constexpr double v[{len(vals)}] = {arr(vals)};\n        return v[i];\n    }}\n")

    return (
        "struct Tableau {\n"
        f"    static constexpr int NS = {n};\n"
        + vec_fn("c", t.c)
        + f"    __host__ __device__ static constexpr double a(int i, int j, double w = 0.0) {{\n"
        f"        constexpr double v0[{n}][{n}] = {mat(t.a)};\n"
        f"        constexpr double v1[{n}][{n}] = {mat(a1)};\n"
        "        return v0[i][j] + v1[i][j] * w;\n    }\n"
        f"    __host__ __device__ static constexpr bool nonzero_a(int i, int j) {{\n"
        f"        constexpr double v0[{n}][{n}] = {mat(t.a)};\n"
        f"        constexpr double v1[{n}][{n}] = {mat(a1)};\n"
        "        return v0[i][j] != 0.0 || v1[i][j] != 0.0;\n    }\n"
        f"    __host__ __device__ static constexpr double b(int j, double w = 0.0) {{\n"
        f"        constexpr double v0[{n}] = {arr(t.b)};\n"
        f"        constexpr double v1[{n}] = {arr(b1)};\n"
        "        return v0[j] + v1[j] * w;\n    }\n"
        f"    __host__ __device__ static constexpr bool nonzero_b(int j) {{\n"
        f"        constexpr double v0[{n}] = {arr(t.b)};\n"
        f"        constexpr double v1[{n}] = {arr(b1)};\n"
        "        return v0[j] != 0.0 || v1[j] != 0.0;\n    }\n"
        + vec_fn("e", t.e) + vec_fn("e5", t.e5) + vec_fn("e3", t.e3)
        + "};\n")
