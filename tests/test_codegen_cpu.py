"""Code generation, caching, validation and API behaviour on the CPU (fake device seam).

Modelled on the reference's CPU tests (``tests/test_ode_api.py``, ``tests/test_package.py``):
the generated model-module source is inspected instead of launching it.
"""

import unittest
import warnings
from unittest.mock import patch

import numpy as np
import pytest
import sympy as sp

import gqis.solver as core
from gqis import compile_lindblad_rhs, compile_ode_rhs, mesolve_2D, odesolve_2D
from fake_device import fake_device


class OdeApiTests(unittest.TestCase):
    def setUp(self):
        self.x, self.y, self.t, self.a = sp.symbols("x y t a", real=True)
        cm = fake_device()
        self.dev = cm.__enter__()
        self.addCleanup(cm.__exit__, None, None, None)

    @property
    def codes(self):
        return self.dev.sources

    def solve(self, **kwargs):
        return odesolve_2D([self.y, -self.a * self.x + sp.sin(self.t)], [self.x, self.y], [1, 0],
                           np.linspace(0, 1, 9), var_arrays={self.a: np.array([1., 2.])}, **kwargs)

    def test_shapes_and_time_dependent_rhs(self):
        final, trace, times = self.solve(return_time_trace=True, time_trace_every=3)
        self.assertEqual(final.shape, (2, 1, 2))
        self.assertEqual(trace.shape, (2, 1, 3, 2))
        np.testing.assert_allclose(times, [0.125, 0.5, 0.875])
        code = self.codes[-1]
        self.assertIn("static constexpr int S = 2;", code)
        rhs = code.split("static void rhs(")[1].split("static void observe(")[0]
        self.assertNotIn("sin(", rhs)  # evaluated in the stage-drive function
        self.assertIn("F::sin(", code.split("static void drives(")[1].split("static void rhs(")[0])
        self.assertNotIn("ode_stage_time", code)
        self.assertIn("#define GQ_TRACE 2", code)  # state trace

    def test_mean_and_shared_rhs(self):
        mean = self.solve(output_mode="mean")
        self.assertEqual(mean.shape, (2, 1, 2))
        self.assertIn("#define GQ_OUT 3", self.codes[-1])  # mean_state
        count = len(core._RHS_CODE_CACHE)
        self.solve(solver="tsit5")
        self.assertEqual(len(core._RHS_CODE_CACHE), count)
        self.assertIn("ExplicitRK<gqmodel::Tableau>", self.codes[-1])

    def test_time_offset_reuses_kernel_and_shifts_trace_times(self):
        _, _, times = self.solve(t_in=3.0, return_time_trace=True)
        np.testing.assert_allclose(times, 3 + np.arange(1, 9) / 8)
        self.solve(t_in=5.0, return_time_trace=True)
        self.assertEqual(len(self.codes), 1)
        self.assertEqual(self.dev.launches[-1].t_in, 5.0)
        self.solve(t_in=0.0, return_time_trace=True)  # zero and non-zero offsets share one module
        self.assertEqual(len(self.codes), 1)
        self.assertEqual(self.dev.launches[-1].t_in, 0.0)

    def test_observable_and_fp64(self):
        result, trace, times = self.solve(observable=(self.x + self.y)**2 + sp.I * (self.x + self.y)**3 + self.t,
                                          fp64=True, return_time_trace=True)
        self.assertEqual(result.dtype, np.complex128)
        self.assertEqual(trace.shape, (2, 1, 8))
        self.assertEqual(times.dtype, np.float64)
        drives = self.codes[-1].split("static void drives(")[1].split("static void rhs(")[0]
        self.assertNotIn("rho[", drives)
        self.assertIn("#define GQ_FORM FormFP64", self.codes[-1])

    def test_fp32_form_is_the_default(self):
        result = self.solve()
        self.assertEqual(result.dtype, np.float32)
        self.assertIn("#define GQ_FORM FormFP32", self.codes[-1])

    def test_static_precomputation(self):
        odesolve_2D([sp.exp(self.a) * self.x], [self.x], [1], [0, 0.1], var_arrays={self.a: np.array([1.])})
        static = self.codes[-1].split("static void statics(")[1].split("static void drives(")[0]
        self.assertIn("gq::exp(ParX)", static)

    def test_explicit_initial_states_and_equations(self):
        equation = sp.Eq(sp.Derivative(self.x, self.t, evaluate=False), -self.x)
        result = odesolve_2D([equation], [self.x], None, [0, 0.1], y0_values=np.ones((1, 1)))
        self.assertEqual(result.shape, (1, 1, 1))
        self.assertIn("kInitFromArray = true", self.codes[-1])

    def test_invalid_input(self):
        with self.assertRaisesRegex(ValueError, "Unassigned"):
            odesolve_2D([self.a * self.x], [self.x], [1], [0, 1])
        with self.assertRaisesRegex(ValueError, "real"):
            odesolve_2D([sp.I * self.x], [self.x], [1], [0, 1])

    def test_lindblad_entry_point_still_generates(self):
        result = mesolve_2D(sp.zeros(2), {}, [], sp.diag(1, 0), [0, 0.1], var_arrays={self.a: np.array([0.])})
        self.assertEqual(result.shape, (1, 1))
        self.assertIn("static constexpr int S = 3;", self.codes[-1])

    def test_square_of_a_sum_keeps_its_parentheses(self):
        odesolve_2D([self.y, -(self.x + 1)**2 - self.a * self.y], [self.x, self.y], [1, 0], [0, 0.1],
                    var_arrays={self.a: np.array([1.])}, cse_simplify=False)
        rhs = self.codes[-1].split("static void rhs(")[1].split("static void observe(")[0]
        self.assertIn("((rho[0] + 1)*(rho[0] + 1))", rhs)
        self.assertNotIn("pow(", rhs)

    def test_cubes_print_as_products(self):
        odesolve_2D([self.y, -self.x**3], [self.x, self.y], [1, 0], [0, 0.1], var_arrays={self.a: np.array([1.])})
        self.assertIn("gq::ipow<3>(rho[0])", self.codes[-1])

    def test_exact_constants_print_as_float_literals(self):
        odesolve_2D([self.y, -sp.sqrt(2) * self.x - sp.pi * self.a * self.y + sp.E * sp.cos(2 * sp.pi * self.t)],
                    [self.x, self.y], [1, 0], [0, 0.1], var_arrays={self.a: np.array([1.])})
        self.assertNotRegex(self.codes[-1], r"\bM_\w+")
        self.assertIn("1.414213562e+00", self.codes[-1])

    def test_compiled_ode_rhs_starts_from_code_emission(self):
        compiled = compile_ode_rhs([self.y, -self.a * self.x + sp.sin(self.t)], [self.x, self.y], [1, 0], [self.a])
        self.assertEqual(set(compiled.timings), {"ode_prepare_s", "ode_optimize_s"})
        self.assertEqual(self.codes, [])
        core._RHS_CODE_CACHE.clear()
        with patch.object(core, "_compile_rhs", side_effect=AssertionError("ODE prepared again")):
            via = odesolve_2D(compiled, tlist=np.linspace(0, 1, 9), var_arrays={self.a: np.array([1., 2.])})
        self.assertEqual(via.shape, (2, 1, 2))
        self.solve()
        self.assertEqual(len(self.codes), 1)
        core._KERNEL_CACHE.clear()
        self.solve()
        self.assertEqual(self.codes[0], self.codes[1])
        with self.assertRaisesRegex(ValueError, "var_arrays must sweep"):
            odesolve_2D(compiled, tlist=[0, 1], var_arrays={})
        with self.assertRaisesRegex(ValueError, "fixed when the RHS is compiled"):
            odesolve_2D(compiled, tlist=[0, 1], var_arrays={self.a: np.array([1.])}, observable=self.x)
        with self.assertRaisesRegex(ValueError, "mesolve_2D"):
            odesolve_2D(compile_lindblad_rhs(sp.zeros(2), {}, [], sp.diag(1, 0), [self.a]),
                        tlist=[0, 1], var_arrays={self.a: np.array([0.])})

    def test_compiled_lindblad_rhs_matches_direct_call(self):
        model = (sp.Matrix([[self.a, 1], [1, -self.a]]), {}, [sp.Matrix([[0, 1], [0, 0]])], sp.diag(1, 0))
        compiled = compile_lindblad_rhs(*model, [self.a])
        mesolve_2D(compiled, tlist=[0, 0.1], var_arrays={self.a: np.array([0.])})
        mesolve_2D(*model, [0, 0.1], var_arrays={self.a: np.array([0.])}, RHSreuse=False)
        self.assertEqual(self.codes[0], self.codes[1])
        with self.assertRaisesRegex(ValueError, "order given when the RHS was compiled"):
            mesolve_2D(compiled, tlist=[0, 0.1], var_arrays={self.x: np.array([0.])})
        with self.assertRaisesRegex(ValueError, "do not pass the model"):
            mesolve_2D(compiled, {}, tlist=[0, 0.1], var_arrays={self.a: np.array([0.])})

    def test_grouped_options_match_flat_options(self):
        flat = self.solve(solver="tsit5", fp64=True, return_time_trace=True, time_trace_every=3, cse_batch_size=1)
        grouped = self.solve(solver_options={"solver": "tsit5", "fp64": True}, codegen={"cse_batch_size": 1},
                             output={"return_time_trace": True, "time_trace_every": 3})
        self.assertEqual(len(self.codes), 1)
        for a, b in zip(flat, grouped):
            np.testing.assert_array_equal(a, b)

    def test_grouped_options_reject_conflicts_and_unknown_names(self):
        with self.assertRaisesRegex(ValueError, "both directly"):
            self.solve(fp64=True, solver_options={"fp64": False})
        with self.assertRaisesRegex(ValueError, "Unknown codegen option"):
            self.solve(codegen={"fp64": True})
        with self.assertRaisesRegex(ValueError, "does not accept"):
            mesolve_2D(sp.zeros(2), {}, [], sp.diag(1, 0), [0, 0.1], var_arrays={self.a: np.array([0.])},
                       initial={"y0_values": None})

    def test_adaptive_solvers_pass_tolerances_and_use_work_stealing_kernel(self):
        self.solve(solver="dop853a", adaptive_options={"step_rtol": 1e-8, "step_atol": 1e-10, "max_substeps": 99})
        launch = self.dev.launches[-1]
        self.assertTrue(launch.adaptive)
        self.assertEqual(launch.solver_params, (1e-8, 1e-10, 99.0))
        self.assertIn("Dop853Pair", self.codes[-1])
        self.assertIn("#define GQ_ADAPTIVE 1", self.codes[-1])

    def test_timestep_calibration_reuse_and_recalibration(self):
        with patch.object(core, "_calibrate_timestep", wraps=core._calibrate_timestep) as calibrate:
            settings = dict(rms_atol=1e-4, sample_stride=2)
            self.solve(calibrate_timesteps=settings)
            self.solve(calibrate_timesteps=settings)
            self.assertEqual(calibrate.call_count, 1)
            self.solve(calibrate_timesteps=settings, cse_batch_size=1)
            self.assertEqual(calibrate.call_count, 1)
            self.solve(calibrate_timesteps=dict(settings, rms_atol=1e-5))
            self.assertEqual(calibrate.call_count, 2)
            every = dict(settings, recalibrate_every=2, max_atol=0)
            for _ in range(3):
                self.solve(calibrate_timesteps=every)
            self.assertEqual(calibrate.call_count, 4)
            self.solve(calibrate_timesteps=dict(every, reset=True))
            self.assertEqual(calibrate.call_count, 5)

    def test_timestep_calibration_never_accepts_unstable_runs(self):
        def fake_solve(**kwargs):
            steps = len(kwargs["tlist"]) - 1
            return np.full((2, 2), np.nan) if steps < 4 else np.ones((2, 2))
        args = dict(var_arrays={self.a: np.arange(10.)}, rho0_var_arrays=None, rho0_values=None,
                    solver="rk4", fp64=False)
        settings = core._timestep_calibration_settings(dict(rms_atol=0, max_atol=0, rms_rtol=1e-3))
        with patch.object(core, "_solve_symbolic_system", fake_solve):
            info = core._calibrate_timestep(args, settings, base_steps=1, duration=1.0)
        self.assertEqual(info["steps"], 4)

    def test_timestep_calibration_test_grid_keeps_axis_ends(self):
        args = dict(var_arrays={self.a: np.arange(10.)}, rho0_var_arrays=None, rho0_values=np.zeros((10, 3)),
                    solver="rk4", fp64=False)
        test, full_grid = core._undersampled_arguments(args, 4)
        np.testing.assert_array_equal(test["var_arrays"][self.a], [0, 4, 8, 9])
        self.assertEqual(test["rho0_values"].shape, (4, 3))
        self.assertFalse(full_grid)
        self.assertTrue(core._undersampled_arguments(args, 1)[1])

    def test_timestep_calibration_warns_once_for_wider_sweep_range(self):
        settings = dict(rms_atol=1e-4, sample_stride=2)
        self.solve(calibrate_timesteps=settings)
        wider = dict(var_arrays={self.a: np.array([1., 3.])})
        model = ([self.y, -self.a * self.x + sp.sin(self.t)], [self.x, self.y], [1, 0], np.linspace(0, 1, 9))
        with self.assertWarnsRegex(RuntimeWarning, "beyond the range used for calibration"):
            odesolve_2D(*model, calibrate_timesteps=settings, **wider)
        with warnings.catch_warnings():
            warnings.simplefilter("error")
            odesolve_2D(*model, calibrate_timesteps=settings, **wider)

    def test_timestep_calibration_bisection_finds_coarsest_passing_step(self):
        real = core._solve_symbolic_system

        def fake(**kwargs):
            if kwargs.get("calibrate_timesteps"):
                return real(**kwargs)
            steps = len(kwargs["tlist"]) - 1
            shape = tuple(len(v) for v in kwargs["var_arrays"].values()) + (1,)
            result = np.full(shape[:2], 0.3 + 3e4 / steps**4, dtype=complex)
            return (result, {}) if kwargs.get("return_timing_info") else result

        def steps_for(start, bisection_steps):
            core._TIMESTEP_CALIBRATION_CACHE.clear()
            with patch.object(core, "_solve_symbolic_system", side_effect=fake):
                _, info = real(H=sp.eye(2), Drive=sp.Integer(0), Col_Ops=[], mean_operator=sp.eye(2),
                               tlist=np.linspace(0, 1, start + 1), var_arrays={self.a: np.ones(4)},
                               return_timing_info=True, output_mode="final",
                               calibrate_timesteps=dict(rms_atol=1e-3, max_atol=1e-2,
                                                        bisection_steps=bisection_steps))
            return info["timestep_calibration"]["steps"]

        self.assertEqual(steps_for(16, 0), 128)
        self.assertEqual(steps_for(16, 2), 76)
        self.assertEqual(steps_for(512, 2), 76)
        self.assertEqual(steps_for(512, 0), 512)

    def _calibrated_with(self, value_of, **kwargs):
        """Calibration report of a mesolve_2D call whose uncalibrated runs return ``value_of(call)`` at
        every point (a 4-point sweep, 16 starting steps on [0, 1])."""
        real = core._solve_symbolic_system

        def run(**call):
            if call.get("calibrate_timesteps"):
                return real(**call)
            nx, ny = (len(v) for v in (list(call["var_arrays"].values()) + [[0.0]])[:2])
            out = np.full((nx, ny), value_of(call), dtype=complex)
            return (out, {}) if call.get("return_timing_info") else out

        core._TIMESTEP_CALIBRATION_CACHE.clear()
        with patch.object(core, "_solve_symbolic_system", side_effect=run):
            _, info = real(H=sp.eye(2), Drive=sp.Integer(0), Col_Ops=[], mean_operator=sp.eye(2),
                           tlist=np.linspace(0, 1, 17), var_arrays={self.a: np.ones(4)},
                           return_timing_info=True, **kwargs)
        return info["timestep_calibration"]

    def test_timestep_calibration_mean_uses_first_order_estimate(self):
        """tests/test_ode_api.py:293-300 of the reference: a time average whose error is 1/steps is
        extrapolated as first order (1e-3 needs 1024 steps); the same error read as RK4's fourth
        order would pass at 724."""
        limits = dict(rms_atol=1e-3, max_atol=1e-2)
        def value(call):
            return 0.3 + 1.0 / (len(call["tlist"]) - 1)
        self.assertEqual(self._calibrated_with(value, output_mode="mean", calibrate_timesteps=limits)["steps"], 1024)
        self.assertEqual(self._calibrated_with(value, output_mode="final", calibrate_timesteps=limits)["steps"], 724)

    def test_tsit5a_calibration_scales_both_tolerances(self):
        """tests/test_ode_api.py:302-313: an error of 7 x the step tolerance meets 1e-3 from 1.4e-4 down;
        the search moves by decades from either side and keeps the rtol / atol ratio; output times
        never change."""
        def value(call):
            self.assertEqual(len(call["tlist"]), 17)
            o = call["adaptive_options"]
            return 0.3 + 7.0 * max(o["step_rtol"], o["step_atol"])
        for start in (1e-5, 1e-2):
            r = self._calibrated_with(value, solver="tsit5a", calibrate_timesteps=dict(rms_atol=1e-3, max_atol=1e-2),
                                      adaptive_options=dict(step_rtol=start, step_atol=start / 5))
            self.assertAlmostEqual(r["step_tol"], 1e-4)
            self.assertAlmostEqual(r["step_rtol"], 1e-4)
            self.assertAlmostEqual(r["step_atol"], 2e-5)

    def test_tsit5a_calibration_stops_at_max_substeps(self):
        """tests/test_ode_api.py:315-322: tolerances below 1e-6 exceed max_substeps (NaN points); the
        search stops at 1e-6, warns and reports the status."""
        def value(call):
            tol = call["adaptive_options"]["step_rtol"]
            return np.nan if tol < 0.99e-6 else 0.3 + 1e3 * tol
        with self.assertWarnsRegex(RuntimeWarning, "max_substeps"):
            r = self._calibrated_with(value, solver="tsit5a", calibrate_timesteps=dict(rms_atol=1e-3, max_atol=1e-2))
        self.assertAlmostEqual(r["step_tol"], 1e-6)
        self.assertEqual(r["details"]["status"], "max_substeps")

    def test_timestep_calibration_key_includes_max_steps_and_reuses_full_grid(self):
        """tests/test_ode_api.py:228-247: max_steps is part of the cache key; a full-grid test reuses its
        final run and skips bisection (two launches), unless full_grid_bisection asks for it. Launches
        are counted on the device seam: every candidate here comes from one prepared launch."""
        with patch.object(core, "_calibrate_timestep", wraps=core._calibrate_timestep) as calibrate:
            self.solve(calibrate_timesteps=dict(rms_atol=1e-4, sample_stride=1))
            self.solve(calibrate_timesteps=dict(rms_atol=1e-4, sample_stride=1, max_steps=2**10))
            self.assertEqual(calibrate.call_count, 2)

        def launches(**settings):
            before = len(self.dev.launches)
            self.solve(calibrate_timesteps=dict(rms_atol=1e-4, sample_stride=1, reset=True, **settings))
            return len(self.dev.launches) - before
        self.assertEqual(launches(bisection_steps=0), 2)
        self.assertEqual(launches(bisection_steps=2), 2)
        self.assertEqual(launches(), 2)
        self.assertGreater(launches(full_grid_bisection=True), 2)

    def test_timestep_calibration_defaults_differ_for_lindblad_and_ode(self):
        lindblad = core._timestep_calibration_settings(True)
        ode = core._timestep_calibration_settings(True, ode=True)
        self.assertEqual((lindblad["rms_atol"], lindblad["max_atol"]), (1e-3, 1e-2))
        self.assertEqual((ode["rms_atol"], ode["max_atol"]), (1e-4, 1e-3))

    def test_timestep_calibration_rejects_unknown_settings(self):
        with self.assertRaisesRegex(ValueError, "Unknown calibrate_timesteps"):
            self.solve(calibrate_timesteps=dict(rms_tol=1e-4))
        with self.assertRaisesRegex(ValueError, "at least one"):
            self.solve(calibrate_timesteps=dict(rms_atol=0, max_atol=0))


def _minimal_model():
    sweep = sp.Symbol("sweep", real=True)
    return sp.zeros(2), sp.Integer(0), [], sp.eye(2), {sweep: np.array([0.0])}


def test_nonuniform_time_grid_is_rejected_before_gpu_launch():
    import pytest
    H, D, C, O, sweep = _minimal_model()
    with pytest.raises(ValueError, match="uniformly spaced"):
        mesolve_2D(H, D, C, O, [0.0, 1.0, 2.5], var_arrays=sweep)
    with pytest.raises(ValueError, match="begin at zero"):
        mesolve_2D(H, D, C, O, [1.0, 2.0], var_arrays=sweep)
    with pytest.raises(ValueError, match="Unsupported solver"):
        mesolve_2D(H, D, C, O, [0.0, 1.0], var_arrays=sweep, solver="not_a_solver")
    with pytest.raises(ValueError, match="unroll must be True or False"):
        mesolve_2D(H, D, C, O, [0.0, 1.0], var_arrays=sweep, unroll="False")
    with pytest.raises(ValueError, match="precision must be"):
        mesolve_2D(H, D, C, O, [0.0, 1.0], var_arrays=sweep, precision="bf16")


class TimeFunctionTests(unittest.TestCase):
    """Functions of time alone in the drives become Tf[k] (evaluated once per warp by RK4), and the
    runtime constants they read keep their values through the renumbering of used constants."""

    def setUp(self):
        cm = fake_device()
        self.dev = cm.__enter__()
        self.addCleanup(cm.__exit__, None, None, None)

    def test_time_functions_and_constant_renumbering(self):
        import re
        eps, A, w, g, unused, t, Drive = sp.symbols("eps A w g unused t Drive", real=True)
        sz, sx, sm = sp.Matrix([[1, 0], [0, -1]]), sp.Matrix([[0, 1], [1, 0]]), sp.Matrix([[0, 1], [0, 0]])
        H = eps / 2 * sz + sp.Rational(1, 2) * sx + Drive * sz
        mesolve_2D(H, A * sp.cos(w * t) + eps * sp.sin(2 * t), [sp.sqrt(g) * sm], sp.diag(0, 1),
                   np.linspace(0, 1, 11), var_arrays={eps: np.array([-1., 1.]), A: np.array([0., 1.])},
                   runtime_consts={w: 2.0, g: 0.01, unused: 5.0})
        code, launch = self.dev.sources[-1], self.dev.launches[-1]
        self.assertIn("static constexpr int NTF = 2;", code)
        body = code[code.index("static void time_funcs"):code.index("template <class F>")]
        k = int(re.search(r"cos\(t\*Const_d\[(\d+)\]\)", body).group(1))
        self.assertEqual(launch.consts[k], 2.0)             # w, read only by a drive
        self.assertIn("sin(2*t)", body)
        refs = {int(m) for m in re.findall(r"Const_(?:arr|d)\[(\d+)\]", code)}
        self.assertEqual(refs, set(range(len(launch.consts))))  # every index read has a value, none idle
        self.assertNotIn(5.0, launch.consts)                 # the unused constant is dropped


def test_repeated_call_skips_model_preparation_and_follows_mutated_matrices():
    """A repeated call is found by its arguments before the model is prepared; a matrix changed in
    place between calls is a new model (the key holds an immutable copy of its entries)."""
    from gqis import rhs
    eps, A, t = sp.symbols("eps A t", real=True)
    H = sp.Matrix([[eps / 2, 0.5], [0.5, -eps / 2]])
    ops = [0.1 * sp.Matrix([[0, 1], [0, 0]])]
    call = dict(sweep_symbols=(eps, A), const_values={})
    rhs._RHS_CODE_CACHE.clear()
    with patch.dict("os.environ", {"GQIS_DISK_CACHE": "0"}):
        first, status = rhs.compile_rhs(H, A * sp.cos(t), ops, sp.diag(0, 1), **call)
        assert status == "miss"
        with patch.object(rhs, "prepare_model", side_effect=AssertionError("prepared again")):
            again, status = rhs.compile_rhs(H, A * sp.cos(t), ops, sp.diag(0, 1), **call)
        assert status == "hit" and again is first
        H[0, 1] = H[1, 0] = 0.7  # the same Matrix object, new entries
        changed, status = rhs.compile_rhs(H, A * sp.cos(t), ops, sp.diag(0, 1), **call)
        assert status == "miss" and changed is not first
    rhs._RHS_CODE_CACHE.clear()


def test_non_finite_output_raises_unless_ignored():
    """A non-finite point in the returned map raises RuntimeError (gqis/solver.py:2351-2362 of the
    reference); ignore_non_finite_output returns the map with it. The failure is made on the host."""
    eps, A, t = sp.symbols("eps A t", real=True)
    H = sp.Matrix([[eps / 2, 0.5], [0.5, -eps / 2]])
    call = ((H, A * sp.cos(t), [0.1 * sp.Matrix([[0, 1], [0, 0]])], sp.diag(0, 1), np.linspace(0, 1, 5)),
            dict(var_arrays={eps: np.linspace(-1, 1, 4), A: np.linspace(0, 1, 3)}, fp64=True))

    def values(launch):
        v = np.zeros((len(launch.par_x) * len(launch.par_y), 2))
        v[5, 0] = np.nan
        return v
    with fake_device(values):
        with pytest.raises(RuntimeError, match="Non-finite"):
            mesolve_2D(*call[0], **call[1])
        out = mesolve_2D(*call[0], **call[1], ignore_non_finite_output=True)
    assert out.shape == (4, 3) and int(np.isnan(out.real).sum()) == 1 and np.isnan(out.real[1, 2])


def test_empty_sweep_axis_is_rejected_before_any_compile():
    """A sweep array without values gives a zero-point grid, which the launch rejects; the front end says
    so before deriving or compiling anything (for either axis, and for odesolve_2D)."""
    eps, A, x, k = sp.symbols("eps A x k", real=True)
    H = eps / 2 * sp.Matrix([[1, 0], [0, -1]]) + sp.Symbol("Drive", real=True) / 2 * sp.Matrix([[0, 1], [1, 0]])
    tl = np.linspace(0.0, 1.0, 11)
    with fake_device() as dev:
        for va in ({eps: np.array([]), A: np.linspace(0, 1, 3)}, {eps: np.linspace(0, 1, 3), A: []}):
            with pytest.raises(ValueError, match="is empty"):
                mesolve_2D(H, A, [], sp.diag(0, 1), tl, var_arrays=va, fp64=True)
        with pytest.raises(ValueError, match="sweep array of k is empty"):
            odesolve_2D([-k * x], [x], [1.0], tl, var_arrays={k: np.zeros(0)}, fp64=True)
        assert not dev.sources and not dev.launches


def test_forced_unrolling_is_reported_and_builds_the_same_module():
    """After the reference's tests/test_gpu_solver.py:59-73: ``unroll=True`` is accepted and reported in
    the timing dictionary. The templates already unroll every loop over the state (which keeps it
    in registers), so both settings build one module with the same flags."""
    d = sp.Symbol("dummy", real=True)
    model = (sp.zeros(2), sp.Integer(0), [], sp.eye(2), np.linspace(0.0, 1.0, 5))
    with fake_device() as dev:
        _, timing = mesolve_2D(*model, var_arrays={d: np.array([0.0])}, output_mode="final_rho", unroll=True,
                               return_timing_info=True)
        assert timing["solver"] == "rk4" and timing["unroll"] is True
        flags = [core.prebuild("mesolve_2D", *model, var_arrays={d: np.array([0.0])}, output_mode="final_rho",
                               unroll=u, source_only=True) for u in (False, True)]
        assert flags[0] == flags[1]
        assert len(set(dev.sources)) == 1


def test_calibrated_trace_keeps_the_sample_times_of_the_given_grid():
    """After the reference's tests/test_gpu_solver.py:206-228: when calibration refines the step, the
    trace is still sampled at the times of the supplied grid (stride and offset scaled with it)."""
    eps, A, t = sp.symbols("eps A t", real=True)
    H = eps / 2 * sp.Matrix([[1, 0], [0, -1]]) + sp.Symbol("Drive", real=True) / 2 * sp.Matrix([[0, 1], [1, 0]])
    period = 2 * np.pi
    call = dict(var_arrays={eps: np.linspace(-1, 1, 4), A: np.linspace(0.1, 1, 3)}, output_mode="final",
                return_time_trace=True, time_trace_every=8, fp64=True)
    model = (H, A * sp.cos(t), [], sp.diag(0, 1), np.linspace(0.0, period, 33))
    with fake_device(values=lambda launch: 0.3 + 3e4 / launch.num_steps ** 4) as dev:
        _, plain_trace, plain_times = mesolve_2D(*model, **call)
        _, trace, times, info = mesolve_2D(*model, **call, calibrate_timesteps=dict(rms_atol=1e-3, max_atol=1e-2),
                                           return_timing_info=True)
        final = dev.launches[-1]
    assert info["timestep_calibration"]["steps"] > 32  # the grid was refined
    np.testing.assert_allclose(plain_times, (np.arange(4) * 8 + 1) * period / 32)
    np.testing.assert_allclose(times, plain_times, rtol=1e-12)
    assert trace.shape == plain_trace.shape
    assert final.num_steps % 32 == 0 and final.trace_stride == 8 * final.num_steps // 32


@pytest.mark.parametrize("name", ["rk4", "lserk4", "lserk4f", "dp5", "ab5", "anas5", "tsit5", "alshina6",
                                  "dop853", "tsit5a", "dop853a"])
def test_each_module_selects_only_its_own_integrator(name):
    """After the reference's tests/test_cuda_solvers.py:21-32: the generated module names exactly one
    integrator (its template and solver id), and carries a Butcher tableau only when that template
    reads one, with the method's stage count."""
    from gqis.cuda_solvers import get_solver_spec
    x, t = sp.symbols("x t", real=True)
    kw = {"solver_frequency": 1.0} if name == "anas5" else {}
    with fake_device() as dev:
        odesolve_2D([-x + sp.cos(t)], [x], [1.0], np.linspace(0.0, 1.0, 9), solver=name, fp64=True, **kw)
    src = dev.sources[-1]
    spec = get_solver_spec(name, frequency=1.0, step_size=0.125) if name == "anas5" else get_solver_spec(name)
    solver_lines = [ln for ln in src.splitlines() if ln.startswith("#define GQ_SOLVER ")]
    assert solver_lines == [f"#define GQ_SOLVER {spec.template}"]
    assert f"#define GQ_SOLVER_ID {spec.solver_id}\n" in src
    assert f"#define GQ_ADAPTIVE {1 if spec.adaptive else 0}\n" in src
    if "gqmodel::Tableau" in spec.template:
        assert src.count("struct Tableau {") == 1
        assert f"static constexpr int NS = {len(spec.tableau.b)};" in src
    else:
        assert "struct Tableau" not in src


def test_solver_ids_are_distinct():
    from gqis.cuda_solvers import available_solvers, get_solver_spec
    ids = [get_solver_spec(s, frequency=1.0, step_size=0.1).solver_id if s == "anas5" else get_solver_spec(s).solver_id
           for s in available_solvers()]
    assert len(set(ids)) == len(ids)


def test_fitted_solver_parameter_is_a_runtime_value():
    """After the reference's tests/test_cuda_solvers.py:56-59: anas5's frequency-fitted coefficient is
    passed at launch, so other frequencies reuse the module."""
    x, t = sp.symbols("x t", real=True)
    with fake_device() as dev:
        for f in (1.0, 1.14, 2.5):
            odesolve_2D([-x + sp.cos(t)], [x], [1.0], np.linspace(0.0, 1.0, 9), solver="anas5", solver_frequency=f,
                        fp64=True)
    assert len(dev.sources) == 1
    params = [launch.solver_params for launch in dev.launches]
    assert all(len(p) == 1 for p in params) and len(set(params)) == 3
