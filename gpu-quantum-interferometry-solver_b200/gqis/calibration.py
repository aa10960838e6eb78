"""``calibrate_timesteps``: choose the step (or step tolerance) of a sweep on an undersampled grid.

Reference behaviour (``gqis/solver.py:928-1341``): the coarsest uniform step - for the adaptive
solvers, the loosest step tolerance - whose map on every ``sample_stride``-th point of each sweep
axis meets the requested RMS / max limits, estimated by Richardson extrapolation between two
resolutions; the settings, their defaults and every user-facing message are that interface.

The search is organised around three small objects:

* :class:`Settings` - the validated request (a ``dict``-like view for callers that index it);
* :class:`Ladder`   - the resolution axis: step counts refined by 2, or 1/tolerance refined by 10;
* :class:`TestGrid` - runs candidate resolutions on the undersampled grid and keeps their maps.

``search`` climbs the ladder until a resolution passes against the next finer one, ``narrow`` then
coarsens a passing start and bisects the bracket geometrically against that finer reference, and
``solve_calibrated`` caches the outcome per model and accuracy request and runs the full sweep.

The solver module's names ``_solve_symbolic_system``, ``_calibrate_timestep``,
``_device_run_many`` and ``_TIMESTEP_CALIBRATION_CACHE`` are looked up at call time, so a test that
replaces one of them on ``gqis.solver`` sees every call.
"""

from __future__ import annotations

import dataclasses
import math
import time
import warnings

import numpy as np
import sympy as sp

from .cuda_solvers import TSIT5A_DEFAULTS, get_solver_spec

DEFAULTS = {
    "rms_atol": 1e-3, "rms_rtol": 0.0,
    "max_atol": 1e-2, "max_rtol": 0.0,
    "sample_stride": 8,
    "max_steps": 2**20,
    "min_step_tol": 1e-12,
    "bisection_steps": 2,
    "full_grid_bisection": False,
    "recalibrate_every": None,
    "reset": False,
    "on_fail": "warning",
    "range_warning": True,
    "batch_levels": 1,
}
ODE_DEFAULTS = {"rms_atol": 1e-4, "max_atol": 1e-3}
MAX_COARSENINGS = 6  # a passing start is coarsened at most this many times before bisection


def _solver_module():
    from . import solver
    return solver


# ----------------------------------------------------------------------------------- settings

@dataclasses.dataclass(frozen=True)
class Settings:
    rms_atol: float
    rms_rtol: float
    max_atol: float
    max_rtol: float
    sample_stride: int
    max_steps: int
    min_step_tol: float
    bisection_steps: int
    full_grid_bisection: bool
    recalibrate_every: int | None
    reset: bool
    on_fail: str
    range_warning: bool
    batch_levels: int

    @property
    def check_rms(self):
        return self.rms_atol > 0.0 or self.rms_rtol > 0.0

    @property
    def check_max(self):
        return self.max_atol > 0.0 or self.max_rtol > 0.0

    def __getitem__(self, name):
        return getattr(self, name)

    def get(self, name, default=None):
        return getattr(self, name, default)

    def accuracy_key(self):
        """The settings that change which step is found (part of the cache key)."""
        return (self.rms_atol, self.rms_rtol, self.max_atol, self.max_rtol, self.sample_stride,
                self.max_steps, self.bisection_steps, self.full_grid_bisection)

    @classmethod
    def from_request(cls, request, ode=False):
        """``True`` (defaults) or a dict of overrides; ODE calls default to tighter limits."""
        merged = dict(DEFAULTS, **(ODE_DEFAULTS if ode else {}))
        if request is not True:
            if not isinstance(request, dict):
                raise TypeError("calibrate_timesteps must be True, None or a dict of settings.")
            unknown = sorted(set(request) - set(merged))
            if unknown:
                raise ValueError(f"Unknown calibrate_timesteps setting(s) {unknown}. "
                                 f"Valid settings: {', '.join(merged)}.")
            merged.update(request)
        limits = {name: float(merged[name]) for name in ("rms_atol", "rms_rtol", "max_atol", "max_rtol")}
        negative = [name for name, v in limits.items() if v < 0.0]
        if negative:
            raise ValueError(f"calibrate_timesteps {negative[0]} must be non-negative.")
        if not any(v > 0.0 for v in limits.values()):
            raise ValueError("calibrate_timesteps needs at least one non-zero RMS or max tolerance.")
        stride, max_steps = int(merged["sample_stride"]), int(merged["max_steps"])
        min_tol = float(merged["min_step_tol"])
        if min(stride, max_steps) < 1 or not min_tol > 0.0:
            raise ValueError("calibrate_timesteps sample_stride, max_steps and min_step_tol must be positive.")
        bisections = int(merged["bisection_steps"])
        if bisections < 0:
            raise ValueError("calibrate_timesteps bisection_steps must be zero or a positive integer.")
        every = merged["recalibrate_every"]
        if every is not None:
            every = int(every)
            if every < 1:
                raise ValueError("calibrate_timesteps recalibrate_every must be None or a positive integer.")
        if merged["on_fail"] not in ("warning", "ignore", "error"):
            raise ValueError("calibrate_timesteps on_fail must be 'warning', 'ignore' or 'error'.")
        return cls(**limits, sample_stride=stride, max_steps=max_steps, min_step_tol=min_tol,
                   bisection_steps=bisections, full_grid_bisection=bool(merged["full_grid_bisection"]),
                   recalibrate_every=every, reset=bool(merged["reset"]), on_fail=merged["on_fail"],
                   range_warning=bool(merged["range_warning"]), batch_levels=max(1, int(merged["batch_levels"])))


# ------------------------------------------------------------------ adaptive step tolerances

def step_tolerance(args):
    """The larger of the adaptive step tolerances (rtol, atol) a call asks for."""
    opts = {**TSIT5A_DEFAULTS, **(args["adaptive_options"] or {})}
    return max(float(opts["step_rtol"]), float(opts["step_atol"]))


def adaptive_options_at(args, tol):
    """The call's adaptive options with rtol and atol scaled by one factor, so the larger is ``tol``."""
    given = dict(args["adaptive_options"] or {})
    full = {**TSIT5A_DEFAULTS, **given}
    factor = tol / step_tolerance(args)
    return {**given, "step_rtol": float(full["step_rtol"]) * factor, "step_atol": float(full["step_atol"]) * factor}


# ------------------------------------------------------------------------------- the ladder

@dataclasses.dataclass(frozen=True)
class Ladder:
    """The resolution being searched: step counts (refined x2) or 1/step tolerance (refined x10).

    A resolution x is "finer" when larger; ``user(x)`` is what the report calls it (steps, or the
    tolerance 1/x) and ``order`` the convergence order of the Richardson estimate.
    """
    adaptive: bool
    order: int
    start: float
    top: float

    @property
    def label(self):
        return "step_tol" if self.adaptive else "steps"

    @property
    def ratio(self):
        return 10.0 if self.adaptive else 2

    def finer(self, x):
        return x * self.ratio

    def coarser(self, x):
        return x / 10.0 if self.adaptive else x // 2

    def can_coarsen(self, x):
        return self.adaptive or x >= 2

    def user(self, x):
        return 1.0 / x if self.adaptive else x

    def from_user(self, v):
        return 1.0 / v if self.adaptive else v

    def between(self, lo, hi):
        mid = math.sqrt(lo * hi)
        return mid if self.adaptive else int(round(mid))

    def describe(self, x):
        return f"step tolerance {self.user(x):.2e}" if self.adaptive else f"{x} steps"

    @classmethod
    def for_call(cls, args, settings, base_steps):
        if get_solver_spec(args["solver"]).adaptive:
            return cls(True, 1, 1.0 / step_tolerance(args), 1.0 / settings.min_step_tol)
        averaged = args.get("output_mode") in ("mean", "mean_state") and float(args.get("warmup_time", 0.0)) < 1.0
        # a right-endpoint time average converges at first order whatever the integrator
        order = 1 if averaged else get_solver_spec(args["solver"]).order
        return cls(False, order, base_steps, settings.max_steps)


# ------------------------------------------------------------------------------ test grid

def _every_nth_with_end(n, stride):
    idx = list(range(0, n, stride))
    if idx[-1] != n - 1:
        idx.append(n - 1)
    return idx


def _subset(values, idx):
    return [values[i] for i in idx] if isinstance(values, (list, tuple)) else values[idx]


def test_grid_arguments(args, stride):
    """The call restricted to every ``stride``-th point of each sweep axis, both axis ends kept.

    Returns ``(arguments, covers_full_grid)``; outputs that only the final run needs (traces,
    timing dicts, device results, saved kernels) are switched off and non-finite maps are allowed.
    """
    call = dict(args, calibrate_timesteps=None, return_time_trace=False, return_timing_info=False,
                timings=False, return_device=False, ignore_non_finite_output=True,
                Actual_Kernel_Save=False, beep_on_error=False)
    picked = []
    for field in ("var_arrays", "rho0_var_arrays"):
        if not args[field]:
            continue
        call[field] = {}
        for symbol, values in args[field].items():
            idx = _every_nth_with_end(len(values), stride)
            picked.append((idx, len(values)))
            call[field][symbol] = _subset(values, idx)
    if args["rho0_values"] is not None:
        states = args["rho0_values"]
        states = states if hasattr(states, "ndim") else np.asarray(states)
        if picked:
            states = states[picked[0][0]]
            if states.ndim == 3 and len(picked) > 1:
                states = states[:, picked[1][0]]
        call["rho0_values"] = states
    return call, all(len(idx) == n for idx, n in picked)


class TestGrid:
    """Candidate maps on the undersampled grid, computed once per resolution.

    Fixed-step candidates after the first reuse its prepared launch with only the step count
    changed, so the front end (symbolic model, module lookup, uploads) runs once per search;
    ``batch`` > 1 launches the next few candidates of the ladder together on separate streams.
    """

    def __init__(self, args, settings, ladder, duration):
        self.base, self.covers_full_grid = test_grid_arguments(args, settings.sample_stride)
        self.args, self.ladder, self.duration = args, ladder, duration
        self.batch = settings.batch_levels
        self.maps = {}
        self._prepared = None

    def _call(self, x):
        call = dict(self.base)
        if self.ladder.adaptive:
            call["adaptive_options"] = adaptive_options_at(self.args, 1.0 / x)
        else:
            call["tlist"] = np.linspace(0.0, self.duration, int(x) + 1)
        return call

    def compute(self, resolutions):
        core = _solver_module()
        todo = [x for x in dict.fromkeys(resolutions) if x not in self.maps]
        launches = []
        for x in todo:
            if self._prepared is not None and not self.ladder.adaptive:
                launches.append((x, core._with_steps(self._prepared, x, self.duration,
                                                      self.args.get("warmup_time", 0.0))))
                continue
            holder = {}
            direct = core._solve_symbolic_system(**dict(self._call(x), _prepare_only=holder))
            if "launch" not in holder:  # a stand-in solver that returns the map itself
                self.maps[x] = np.asarray(direct)
                continue
            launches.append((x, holder["launch"]))
            self._prepared = self._prepared or holder["launch"]
        if launches:
            outputs = core._device_run_many([launch for _, launch in launches])
            for (x, launch), out in zip(launches, outputs):
                self.maps[x] = core._calibration_map(launch, out[0])

    def map(self, x):
        self.compute([x])
        return self.maps[x]

    def ladder_from(self, x, count):
        """The next ``count`` finer resolutions after x that the ladder allows."""
        out = []
        for _ in range(count):
            x = self.ladder.finer(x)
            if x > self.ladder.top:
                break
            out.append(x)
        return out


# ------------------------------------------------------------------------ error estimates

@dataclasses.dataclass
class Trial:
    """One comparison of a candidate map against a finer reference map."""
    x: float
    rms: float = np.inf
    max: float = np.inf
    passed: bool = False
    reference: float | None = None

    def record(self, ladder):
        rec = {ladder.label: ladder.user(self.x), "rms": self.rms, "max": self.max}
        if self.reference is not None:
            rec[f"reference_{ladder.label}"] = ladder.user(self.reference)
        return rec


def compare(settings, ladder, x, coarse, x_ref, fine, reference=None):
    """Richardson-scaled change between the maps at resolutions x and x_ref (> x), checked
    against ``atol + rtol * size of the finer map`` for the RMS and max limits that are set."""
    trial = Trial(x, reference=reference)
    if not (np.all(np.isfinite(coarse)) and np.all(np.isfinite(fine))):
        return trial  # a non-finite map never passes
    change = np.abs(fine - coarse) / (1.0 - (x / x_ref) ** ladder.order)
    size = np.abs(fine)
    with np.errstate(over="ignore"):  # squares of a diverging map overflow to inf: it fails
        trial.rms = float(np.sqrt(np.mean(change ** 2)))
        rms_limit = settings.rms_atol + settings.rms_rtol * float(np.sqrt(np.mean(size ** 2)))
    trial.max = float(np.max(change))
    max_limit = settings.max_atol + settings.max_rtol * float(np.max(size))
    trial.passed = ((not settings.check_rms or trial.rms <= rms_limit)
                    and (not settings.check_max or trial.max <= max_limit))
    return trial


# ---------------------------------------------------------------------------------- search

@dataclasses.dataclass
class Outcome:
    status: str
    accepted: float
    trials: list
    reference: float | None = None  # the finer resolution the accepted one passed against


def search(grid, settings, ladder):
    """Climb the ladder from its start until a resolution passes against the next finer one.

    Stops early at the ladder's top (``max_steps`` / ``min_step_tol``), when an adaptive map turns
    non-finite (``max_substeps``), or when refining no longer lowers the RMS change (the precision
    floor of the form: the best resolution seen is kept).
    """
    x = ladder.start
    grid.compute([x] + grid.ladder_from(x, grid.batch - 1))
    trials = []
    while True:
        x_ref = ladder.finer(x)
        if x_ref > ladder.top:
            return Outcome("min_step_tol" if ladder.adaptive else "max_steps", x, trials)
        if x_ref not in grid.maps:
            grid.compute(grid.ladder_from(x, grid.batch))
        coarse, fine = grid.maps[x], grid.maps[x_ref]
        if ladder.adaptive and np.all(np.isfinite(coarse)) and not np.all(np.isfinite(fine)):
            return Outcome("max_substeps", x, trials)
        trial = compare(settings, ladder, x, coarse, x_ref, fine)
        trials.append(trial)
        if trial.passed:
            return Outcome("converged", x, trials, reference=x_ref)
        if len(trials) > 1 and np.isfinite(trial.rms) and trial.rms >= trials[-2].rms:
            best = min(trials, key=lambda t: t.rms)
            return Outcome("precision_floor", best.x, trials)
        x = x_ref


def narrow(grid, settings, ladder, outcome):
    """Coarsest passing resolution of a converged search: a passing start is coarsened until a
    candidate fails, then the [failing, passing] bracket is bisected geometrically
    ``bisection_steps`` times. Every candidate is checked against the search's finer reference map."""
    ref_x = outcome.reference
    ref_map = grid.maps[ref_x]
    accepted = outcome.accepted

    def passes(x):
        trial = compare(settings, ladder, x, grid.map(x), ref_x, ref_map, reference=ref_x)
        outcome.trials.append(trial)
        return trial.passed

    # the search refined past the start: the next coarser resolution has failed already
    failing = ladder.coarser(accepted) if accepted > ladder.start else None
    coarsened = 0
    while failing is None and ladder.can_coarsen(accepted) and coarsened < MAX_COARSENINGS:
        coarsened += 1
        candidate = ladder.coarser(accepted)
        if candidate not in grid.maps and grid.batch > 1:
            ahead, c = [], accepted
            while len(ahead) < min(grid.batch, MAX_COARSENINGS - coarsened + 1) and ladder.can_coarsen(c):
                c = ladder.coarser(c)
                ahead.append(c)
            grid.compute(ahead)
        if passes(candidate):
            accepted = candidate
        else:
            failing = candidate
    if failing is not None:
        for _ in range(settings.bisection_steps):
            candidate = ladder.between(failing, accepted)
            if not failing < candidate < accepted:
                break
            if passes(candidate):
                accepted = candidate
            else:
                failing = candidate
    return accepted


def _failure_message(settings, ladder, outcome, fp64):
    def requested(kind):
        atol, rtol = settings[f"{kind}_atol"], settings[f"{kind}_rtol"]
        text = f"{'RMS' if kind == 'rms' else 'max'} {atol:g}"
        return text + (f" + {rtol:g} relative" if rtol else "")
    limits = ", ".join(requested(k) for k in ("rms", "max") if settings[f"check_{k}"])
    why = {"precision_floor": "does not converge",
           "max_steps": "is not reached within max_steps",
           "min_step_tol": "is not reached above min_step_tol",
           "max_substeps": ("needs more than max_substeps steps per output interval "
                            "(increase adaptive_options max_substeps)")}[outcome.status]
    accepted = outcome.accepted
    if outcome.trials:
        best = next((t for t in outcome.trials if t.x == accepted), outcome.trials[-1])
        seen = f"best achieved RMS {best.rms:.2e}, max {best.max:.2e} with {ladder.describe(accepted)}"
    else:
        seen = f"no refinement beyond {ladder.describe(accepted)} was possible"
    message = f"calibrate_timesteps: requested precision ({limits}) {why}; {seen}."
    if outcome.status == "precision_floor" and not fp64:
        message += " If better precision is required, consider switching to fp64=True."
    return message


def calibrate(args, settings, base_steps, duration):
    """Run the search for one call; returns the report dict of ``timestep_calibration.details``
    (plus ``full_grid_results``: the maps of a test grid that is the whole grid, by resolution)."""
    began = time.time()
    ladder = Ladder.for_call(args, settings, base_steps)
    grid = TestGrid(args, settings, ladder, duration)
    outcome = search(grid, settings, ladder)
    first_pass = outcome.accepted
    if (outcome.status == "converged" and settings.bisection_steps > 0
            and (settings.full_grid_bisection or not grid.covers_full_grid)):
        outcome.accepted = narrow(grid, settings, ladder, outcome)
    full_maps = {ladder.user(x): m for x, m in grid.maps.items()} if grid.covers_full_grid else {}
    report = {"status": outcome.status, "tested": [t.record(ladder) for t in outcome.trials],
              "test_grid": grid.maps[ladder.start].shape[:2], "calibration_s": time.time() - began,
              "full_grid_results": full_maps}
    if ladder.adaptive:
        report.update(step_tol=ladder.user(outcome.accepted), doubling_step_tol=ladder.user(first_pass),
                      start_step_tol=ladder.user(ladder.start))
    else:
        report.update(steps=outcome.accepted, dt=duration / outcome.accepted, doubling_steps=first_pass)
    if outcome.status != "converged" and settings.on_fail != "ignore":
        message = _failure_message(settings, ladder, outcome, args["fp64"])
        if settings.on_fail == "error":
            raise RuntimeError(message)
        warnings.warn(message, RuntimeWarning, stacklevel=4)
    return report


# --------------------------------------------------------------------------------- caching

def _hashable(value):
    """A structural key for SymPy inputs (matrices, dicts, sequences, expressions)."""
    if isinstance(value, sp.MatrixBase):
        return ("matrix", value.shape, tuple(value))
    if isinstance(value, dict):
        return ("dict", frozenset((k, sp.sympify(v)) for k, v in value.items()))
    if isinstance(value, (list, tuple)):
        return ("seq", tuple(sp.sympify(v) for v in value))
    return sp.sympify(value)


def cache_key(args, settings):
    """Model and accuracy request of a call. Code-generation options are not part of it: they
    change how the map is computed, not which step meets the limits."""
    constants = args["const_values"] or {}
    keep = args["keep_symbolic_consts"]
    symbolic = set(args["runtime_consts"] or {})
    if args["auto_runtime_consts"] or keep in ("all", "auto", "const_values"):
        symbolic |= set(constants)
    elif keep is not None:
        symbolic |= set(keep)
    baked = tuple(sorted((str(k), float(v)) for k, v in constants.items() if k not in symbolic))
    if args.get("compiled_rhs") is not None:
        model = ("compiled", args["compiled_rhs"].cache_key)
    else:
        model = ("symbolic", _hashable(args["H"]), _hashable(args["Drive"]),
                 tuple(_hashable(L) for L in args["Col_Ops"]), _hashable(args["mean_operator"]),
                 None if args["rho0"] is None else _hashable(args["rho0"]), baked)
    axes = tuple(str(s) for field in ("var_arrays", "rho0_var_arrays") for s in (args[field] or {}))
    spec = get_solver_spec(args["solver"])
    stepping = ("fixed",)
    if spec.adaptive:
        opts = {**TSIT5A_DEFAULTS, **(args["adaptive_options"] or {})}
        rtol, atol = float(opts["step_rtol"]), float(opts["step_atol"])
        stepping = ("adaptive", atol / rtol if rtol > 0.0 else np.inf, int(opts["max_substeps"]),
                    settings.min_step_tol)
    arithmetic = (bool(args["fp64"]), args.get("precision"))
    output = (args["output_mode"], float(args["warmup_time"]), args["_ode_size"])
    return ("gqis-step-calibration", model, axes, spec.name, stepping, arithmetic, output,
            settings.accuracy_key())


def _axis_spans(args):
    spans = []
    for field in ("var_arrays", "rho0_var_arrays"):
        for values in (args[field] or {}).values():
            values = values if hasattr(values, "min") else np.asarray(values)
            spans.append((float(values.min()), float(values.max())))
    return tuple(spans)


class StoredStep:
    """The cache entry of one key: the step (dt or step tolerance) in use, the sweep ranges it was
    tested on, how many calls used it, and whether the range warning was given."""

    def __init__(self, cache, key, settings, spans):
        self.cache, self.key, self.spans = cache, key, spans
        self.entry = None if settings.reset else cache.get(key)

    def due(self, settings):
        """True when this call must run the search (first call, or every ``recalibrate_every``)."""
        if self.entry is None:
            return True
        every = settings.recalibrate_every
        return every is not None and self.entry["calls"] % every == 0

    def record_search(self, found):
        """A new search result; a recalibration keeps the finer of the old and new steps."""
        old = self.entry
        calls = old["calls"] if old else 0
        if old is None:
            value, spans = found, self.spans
        else:
            value = min(old["value"], found)
            spans = tuple((min(a[0], b[0]), max(a[1], b[1])) for a, b in zip(old["ranges"], self.spans))
        self.entry = {"value": value, "ranges": spans, "range_warned": False, "calls": calls}

    def warn_if_outside(self, settings):
        covered = self.entry["ranges"]
        outside = any(lo < clo or hi > chi for (lo, hi), (clo, chi) in zip(self.spans, covered))
        if outside and settings.range_warning and not self.entry["range_warned"]:
            self.entry["range_warned"] = True
            warnings.warn("calibrate_timesteps: the sweep range extends beyond the range used for calibration; "
                          "the stored step is reused without a new test. Use reset=True or recalibrate_every "
                          "to test the new range.", RuntimeWarning, stacklevel=4)

    def commit(self):
        self.entry["calls"] += 1
        self.cache[self.key] = self.entry

    @property
    def value(self):
        return self.entry["value"]

    @value.setter
    def value(self, v):
        self.entry["value"] = v


# ------------------------------------------------------------------------- the full run

def _fixed_step_run(args, settings, run, stored_dt, base_steps, duration):
    """Step count of the full run for a stored dt, and the trace options that keep the caller's
    sample times when the steps are refined by a power of two."""
    steps = int(np.ceil(duration / stored_dt * (1.0 - 1e-9)))
    keep_times = bool(args["return_time_trace"])
    if settings.bisection_steps == 0 or keep_times:
        steps = max(base_steps, steps)
    refine = 1
    if keep_times:
        while base_steps * refine < steps and base_steps * refine < settings.max_steps:
            refine *= 2
        steps = base_steps * refine
    steps = min(steps, max(base_steps, settings.max_steps))
    if keep_times and refine > 1:
        if args["time_trace_samples_per_period"] is not None:
            every = max(1, int(round(int(args["solver_samples_per_period"])
                                     / int(args["time_trace_samples_per_period"]))))
        else:
            every = int(args["time_trace_every"] or 1)
        run.update(time_trace_every=every * refine, time_trace_samples_per_period=None,
                   solver_samples_per_period=None, _time_trace_offset=refine - 1)
    return steps, keep_times


def solve_calibrated(args):
    """``_solve_symbolic_system`` with ``calibrate_timesteps`` set: find (or reuse) the step, run."""
    core = _solver_module()
    settings = core._timestep_calibration_settings(args["calibrate_timesteps"], ode=args["_ode_size"] is not None)
    tlist = np.asarray(args["tlist"], dtype=np.float64)
    if tlist.ndim != 1 or len(tlist) < 2:
        raise ValueError("tlist must be a one-dimensional array with at least two samples.")
    base_steps, duration = len(tlist) - 1, float(tlist[-1] - tlist[0])
    adaptive = get_solver_spec(args["solver"]).adaptive
    stored = StoredStep(core._TIMESTEP_CALIBRATION_CACHE, cache_key(args, settings), settings, _axis_spans(args))
    report = None
    if stored.due(settings):
        report = core._calibrate_timestep(args, settings, base_steps, duration)
        stored.record_search(report["step_tol"] if adaptive else report["dt"])
    else:
        stored.warn_if_outside(settings)
    stored.commit()

    run = dict(args, calibrate_timesteps=None)
    if adaptive:
        chosen, keep_times = stored.value, False

        def use(tol):
            run["adaptive_options"] = adaptive_options_at(args, tol)

        def text(tol):
            return f"step tolerance {tol:.2e}"
        start_text = text(report["start_step_tol"]) if report else ""
    else:
        chosen, keep_times = _fixed_step_run(args, settings, run, stored.value, base_steps, duration)

        def use(steps):
            run["tlist"] = np.linspace(0.0, duration, steps + 1)

        def text(steps):
            return f"{steps} steps"
        start_text = text(base_steps)
    use(chosen)
    if report is not None and args["timings"]:
        last = report["tested"][-1] if report["tested"] else None
        tail = f"; last RMS/max change {last['rms']:.2e}/{last['max']:.2e}" if last else ""
        print(f"calibrate_timesteps: {text(chosen)} ({report['status']}), tested from {start_text} on "
              f"{report['test_grid'][0]}x{report['test_grid'][1]} points in {report['calibration_s']:.2f}s{tail}")

    # a test grid that was the whole grid already holds the chosen map
    if (report is not None and chosen in report["full_grid_results"] and not args["return_time_trace"]
            and not args["return_timing_info"]):
        result = report["full_grid_results"][chosen]
        if not np.all(np.isfinite(result)) and not args["ignore_non_finite_output"]:
            raise RuntimeError("Non-finite values detected in mesolve_2D output. Try reducing dt "
                               "(increase time samples) or check model parameters/RHS.")
        if args["return_device"]:
            import torch
            return torch.as_tensor(result).cuda()
        return result

    # A bisected step passed on the test points only; if the full grid turns non-finite with it,
    # the search's first passing resolution is used instead.
    safer = None
    if report is not None and report["status"] == "converged" and not keep_times:
        first = report["doubling_step_tol"] if adaptive else report["doubling_steps"]
        if (first < chosen) if adaptive else (first > chosen):
            safer = first
    if safer is not None:
        run["ignore_non_finite_output"] = True
    result = core._solve_symbolic_system(**run)
    if safer is not None:
        values = result[0] if isinstance(result, tuple) else result
        if not core._all_finite(values):
            warnings.warn(f"calibrate_timesteps: {text(chosen)} passed on the test points but gave non-finite "
                          f"values on the full grid; using {text(safer)} instead.", RuntimeWarning, stacklevel=3)
            chosen = safer
            stored.value = chosen if adaptive else duration / chosen
            use(chosen)
            run["ignore_non_finite_output"] = args["ignore_non_finite_output"]
            result = core._solve_symbolic_system(**run)
    if args["return_timing_info"]:
        details = {k: v for k, v in report.items() if k != "full_grid_results"} if report else None
        if adaptive:
            opts = run["adaptive_options"]
            summary = {"step_tol": chosen, "step_rtol": opts["step_rtol"], "step_atol": opts["step_atol"]}
        else:
            summary = {"steps": chosen, "dt": duration / chosen}
        result[-1]["timestep_calibration"] = {**summary, "calibrated_this_call": report is not None,
                                              "details": details}
    return result
