"""Model-module variants used by GPU tests beyond the reference cases (prebuilt by build()).

Not a test module itself: ``__graft_entry__.build()`` imports ``calls()`` so that the GPU tests
load these modules instead of compiling them.
"""

import numpy as np
import sympy as sp

import ref_cases
from gqis.cuda_solvers import available_solvers, get_solver_spec

ADAPTIVE_OPTIONS = {"step_rtol": 1e-8, "step_atol": 1e-10, "max_substeps": 4000, "count_steps": True}


def duffing_case(side=8, solver="dop853a", **extra):
    d = ref_cases.workloads().duffing(side=side)
    kwargs = dict(var_arrays=d["var_arrays"], y0_values=d["y0_values"], solver=solver, fp64=True,
                  return_time_trace=True, adaptive_options=dict(ADAPTIVE_OPTIONS))
    kwargs.update(extra)
    return d, (d["rhs"], d["states"], None, d["tlist"]), kwargs


# the serving and fit request models live with the other workloads (the serving bench uses them)
SERVING_SIDES = ref_cases.workloads().SERVING_SIDES
serving_model = ref_cases.workloads().serving_model
qubit_fit_model = ref_cases.workloads().qubit_fit_model


MATRIX_DIMS = (16, 32, 64)
GIVE_UP = ("-DGQ_TC_MAX_POLLS=0",)  # every in-loop MMA wait of the tensor-core kernel gives up at once
TENSOR_DIMS = (8, 16, 32, 64)


def hilbert_model(N, side=(4, 3), steps=100, duration=5.0):
    """(workload, args, kwargs) of the N-level scaling model on a small grid (matrix-form tests)."""
    W = ref_cases.workloads()
    w = W.n_level(N, side=64, steps=steps, duration=duration)
    eps, A = w["symbols"]
    var = {eps: np.linspace(-0.5, 0.5, side[0]), A: np.linspace(0.0, 2.0, side[1])}
    return w, (w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"]), {"var_arrays": var}


def matrix_calls():
    """Matrix-form module variants of the GPU tests and the Hilbert-space scaling benchmark."""
    out = []
    for N in (8,) + MATRIX_DIMS:
        _, args, kwargs = hilbert_model(N)
        for form in ("fp64", "fp32"):
            out.append(("mesolve_2D", args, dict(kwargs, precision=form, rhs_form="matrix")))
    for N in TENSOR_DIMS:
        _, args, kwargs = hilbert_model(N)
        out.append(("mesolve_2D", args, dict(kwargs, precision="fp32", rhs_form="matrix_tc")))
    for N in (16, 64):
        _, args, kwargs = hilbert_model(N)
        out.append(("mesolve_2D", args, dict(kwargs, precision="fp32", rhs_form="matrix_tc", output_mode="final_rho")))
    _, args, kwargs = hilbert_model(40)  # a dimension of 33 .. 48: 48-wide CUDA-core tile, 64 on the tensor cores
    out.append(("mesolve_2D", args, dict(kwargs, fp64=True, rhs_form="matrix")))
    out.append(("mesolve_2D", args, dict(kwargs, precision="fp32")))
    _, args, kwargs = hilbert_model(16)  # the give-up path of the tensor-core kernel's MMA waits
    out.append(("mesolve_2D", args, dict(kwargs, precision="fp32", rhs_form="matrix_tc", nvrtc_options=GIVE_UP)))
    _, args, kwargs = hilbert_model(64)  # the two-CTA tensor-core kernel's trace against the FP64 matrix form
    trace64 = dict(kwargs, return_time_trace=True, time_trace_every=9)
    out.append(("mesolve_2D", args, dict(trace64, fp64=True, rhs_form="matrix")))
    out.append(("mesolve_2D", args, dict(trace64, precision="fp32", rhs_form="matrix_tc")))
    _, args, kwargs = hilbert_model(16)
    out.append(("mesolve_2D", args, dict(kwargs, fp64=True, rhs_form="matrix", output_mode="final_rho")))
    rho0 = np.zeros((4, 3, 16 * 16 - 1))
    out.append(("mesolve_2D", args, dict(kwargs, fp64=True, rhs_form="matrix", output_mode="final_rho",
                                         rho0_values=rho0)))
    out += runtime_rate_calls()
    out += wide_range_calls()
    out += epilogue_diagonal_calls()
    out += offdiagonal_observable_calls()
    args, kwargs = serving_model(8, 6)  # observable traces through the matrix kernels
    args = args[:4] + (np.linspace(0.0, 5.0, 101),)
    trace = dict(kwargs, return_time_trace=True, time_trace_every=7)
    out.append(("mesolve_2D", args, dict(trace, fp64=True, rhs_form="reduced")))
    for form, rf in (("fp64", "matrix"), ("fp32", "matrix"), ("fp32", "matrix_tc")):
        out.append(("mesolve_2D", args, dict(trace, precision=form, rhs_form=rf)))
    return out


def runtime_rate_calls():
    """The fit model with one swept axis and a numeric rho0 through the matrix and reduced forms."""
    import sympy as sp
    args, kwargs, (G1, Gp, D, A) = qubit_fit_model(side=(9, 5), steps=200, duration=10.0)
    rho0 = sp.Matrix([[0.7, 0.2 - 0.1j], [0.2 + 0.1j, 0.3]])
    eps = list(kwargs["var_arrays"])[0]
    one_axis = dict(kwargs, var_arrays={eps: kwargs["var_arrays"][eps]}, rho0=rho0)
    args1 = (args[0], args[1].subs(A, 0.8)) + args[2:]
    out = []
    for mode in ("mean", "final"):
        out.append(("mesolve_2D", args1, dict(one_axis, output_mode=mode, fp64=True, rhs_form="reduced")))
        for form, rf in (("fp64", "matrix"), ("fp32", "matrix"), ("fp32", "matrix_tc")):
            out.append(("mesolve_2D", args1, dict(one_axis, output_mode=mode, precision=form, rhs_form=rf)))
    return out


def calls():
    out = []
    for N in (2, 4, 8):
        args, kwargs = serving_model(N, 64)
        for form in ("fp32", "fp64"):
            out.append(("mesolve_2D", args, dict(kwargs, precision=form)))
    for solver in ("dop853a", "tsit5a"):
        for extra in ({}, {"nvrtc_options": ("-DGQ_STATIC_SCHEDULE=1",)}):
            _, args, kwargs = duffing_case(solver=solver, **extra)
            out.append(("odesolve_2D", args, kwargs))
    _, args, kwargs = duffing_case(side=16, solver="rk4")  # state trace binned by the rasteriser tests
    kwargs.pop("adaptive_options")
    out.append(("odesolve_2D", args, kwargs))
    args, kwargs, params = qubit_fit_model()  # the final-output adjoint's plain FP64 references
    out.append(("mesolve_2D", args, dict(kwargs, fp64=True, output_mode="final")))
    out.append(("mesolve_2D", args, dict(kwargs, keep_symbolic_consts=list(params[:3]), fp64=True,
                                         output_mode="final")))
    return out


def config_calls():
    """Module variants of the full-size configuration tests (tests/test_gpu_configs.py)."""
    d = ref_cases.workloads().duffing(side=8)
    base = dict(var_arrays=d["var_arrays"], y0_values=d["y0_values"], fp64=True,
                adaptive_options={"step_rtol": 1e-8, "step_atol": 1e-10, "max_substeps": 2000})
    args = (d["rhs"], d["states"], None, d["tlist"])
    return [("odesolve_2D", args, dict(base, solver="tsit5a")),
            ("odesolve_2D", args, dict(base, solver="dop853a", return_time_trace=True))]


# driven dissipative qubit of the reference's calibration tests (tests/test_gpu_solver.py:131-227)
CAL_W = 1.14
CAL_PERIOD = 2.0 * np.pi / CAL_W


def calibration_qubit_call(steps_per_period, periods=10, side=16, span=6.0, **options):
    """(args, kwargs) of the driven qubit: H = Delta/2 sx + Drive/2 sz, Drive = eps + A sin(w t),
    w = 1.14, L = sqrt(g1) s-, sqrt(g2) sz (g1 = 0.05 / period, g2 = g1 / 2 + 0.04 / period),
    O = |1><1|; eps in +-span w, A in [0, span w] on a side x side grid."""
    D, eps, Drive, A, t = sp.symbols("Delta eps Drive A t", real=True)
    sz, sm, sx = sp.Matrix([[1, 0], [0, -1]]), sp.Matrix([[0, 1], [0, 0]]), sp.Matrix([[0, 1], [1, 0]])
    g1 = 0.05 / CAL_PERIOD
    g2 = g1 / 2.0 + 0.04 / CAL_PERIOD
    axes = {eps: np.linspace(-span * CAL_W, span * CAL_W, side), A: np.linspace(0.0, span * CAL_W, side)}
    args = (0.5 * D * sx + 0.5 * Drive * sz, eps + A * sp.sin(CAL_W * t), [sp.sqrt(g1) * sm, sp.sqrt(g2) * sz],
            sp.diag(0, 1), np.linspace(0.0, periods * CAL_PERIOD, periods * steps_per_period + 1))
    return args, dict(var_arrays=axes, const_values={D: 1.0}, **options)


def calibration_oscillator_call(steps, **options):
    """(args, kwargs) of the damped driven oscillator x'' = -d x' - x - 0.2 x^3 + a cos(1.3 t) of the
    reference's ODE calibration test (tests/test_gpu_solver.py:234-266), 16 x 16 (d, a) grid."""
    x, v, t, damping, amplitude = sp.symbols("x v t damping amplitude", real=True)
    axes = {damping: np.linspace(0.1, 0.5, 16), amplitude: np.linspace(0.1, 1.0, 16)}
    args = ([v, -damping * v - x - 0.2 * x**3 + amplitude * sp.cos(1.3 * t)], [x, v], [1.0, 0.0],
            np.linspace(0.0, 20.0, steps + 1))
    options = dict(options)
    if options.pop("observable", False):
        options["observable"] = x**2 + v**2
    return args, dict(var_arrays=axes, **options)


def calibration_calls():
    """Module variants of the calibration and Tsit5A known-answer tests."""
    out = []
    for solver in ("rk4", "tsit5a"):
        for mode in ("mean", "final", "final_rho"):
            out.append(("mesolve_2D",) + calibration_qubit_call(8, output_mode=mode, solver=solver))
        out.append(("mesolve_2D",) + calibration_qubit_call(8, output_mode="final", solver=solver,
                                                            return_time_trace=True, time_trace_every=8))
        for extra in ({}, {"output_mode": "mean"}, {"observable": True},
                      {"return_time_trace": True, "time_trace_every": 8}):
            out.append(("odesolve_2D",) + calibration_oscillator_call(64, solver=solver, **extra))
    out.append(("mesolve_2D",) + tsit5a_coarse_output_call())
    out.append(("mesolve_2D",) + tsit5a_average_call())
    return out


def tsit5a_coarse_output_call():
    """H = (1 + (2/5) sin t) sx / 2 from |0>, 4 output intervals on [0, 1.7], Tsit5A at 1e-12
    (tests/test_gpu_solver.py:271-290): rho00(T) = cos^2((T + 0.4 (1 - cos T)) / 2)."""
    dummy, Drive, t = sp.symbols("dummy Drive t", real=True)
    H = (1 + Drive) * sp.Matrix([[0, 1], [1, 0]]) / 2
    kw = dict(var_arrays={dummy: np.array([0.0])}, output_mode="final_rho", solver="tsit5a", fp64=True,
              adaptive_options={"step_rtol": 1e-12, "step_atol": 1e-12, "max_substeps": 10000})
    return (H, {Drive: sp.Rational(2, 5) * sp.sin(t)}, [], sp.eye(2), np.linspace(0.0, 1.7, 5)), kw


def tsit5a_average_call(fp64_time=True):
    """H = sx / 2 from |0>, mean of |0><0| over [2, 10] (warmup 0.2 of 5 intervals of length 2),
    Tsit5A at 1e-10 (tests/test_gpu_solver.py:294-311): 1/2 + (sin 10 - sin 2) / 16."""
    dummy = sp.Symbol("dummy", real=True)
    kw = dict(var_arrays={dummy: np.array([0.0])}, rho0=sp.Matrix([[1, 0], [0, 0]]), output_mode="mean",
              warmup_time=0.2, solver="tsit5a", fp64=True, return_timing_info=True,
              adaptive_options={"step_rtol": 1e-10, "step_atol": 1e-10, "fp64_time": fp64_time,
                                "count_steps": True, "max_substeps": 10000})
    return (sp.Matrix([[0, 1], [1, 0]]) / 2, sp.Integer(0), [], sp.Matrix([[1, 0], [0, 0]]),
            np.linspace(0.0, 10.0, 6)), kw


def adjoint_problems():
    """(args, kwargs) of the adjoint problems the GPU tests and the serving bench build."""
    args, kwargs, params = qubit_fit_model()
    out = [(args, dict(kwargs, params=list(params))), (args, dict(kwargs, params=list(params[:3]))),
           (args, dict(kwargs, params=list(params), output="final"))]
    args, kwargs, params = qubit_fit_model(side=(256, 256), steps=4000, duration=200.0)
    out.append((args, dict(kwargs, params=list(params[:3]))))
    return out


# analytic known-answer cases (tests/test_gpu_known_answers.py)
FIXED = [s for s in available_solvers() if not get_solver_spec(s).adaptive]
ADAPTIVE = [s for s in available_solvers() if get_solver_spec(s).adaptive]
SX = sp.Matrix([[0, 1], [1, 0]])
SZ = sp.Matrix([[1, 0], [0, -1]])


def rabi_call(solver, fp64):
    Om, eps, Drive = sp.symbols("Omega eps Drive", real=True)
    kw = dict(var_arrays={Om: np.linspace(0.5, 2.0, 4), eps: np.array([0.0])}, output_mode="final_rho",
              solver=solver)
    kw.update(dict(fp64=True) if fp64 else dict(precision="fp32"))
    if solver == "anas5":
        kw["solver_frequency"] = 1.0
    return (Drive / 2 * SX + eps / 2 * SZ, Om, [], sp.diag(0, 1), np.linspace(0.0, np.pi, 801)), kw


def commuting_call(solver, output_mode="final_rho"):
    A, eps, Drive, t = sp.symbols("A eps Drive t", real=True)
    kw = dict(var_arrays={A: np.linspace(0.5, 2.0, 4), eps: np.array([0.0])}, output_mode=output_mode,
              solver=solver, fp64=True)
    if solver == "anas5":
        kw["solver_frequency"] = 1.0
    if get_solver_spec(solver).adaptive:
        kw["adaptive_options"] = {"step_rtol": 1e-12, "step_atol": 1e-12, "max_substeps": 4000}
    return (Drive / 2 * SX + eps / 2 * SZ, A * sp.cos(t), [], sp.diag(0, 1), np.linspace(0.0, 5.0, 2001)), kw


def decay_call():
    eps, Drive = sp.symbols("eps Drive", real=True)
    sm = sp.Matrix([[0, 1], [0, 0]])
    kw = dict(var_arrays={eps: np.linspace(-1.0, 1.0, 3)}, output_mode="final_rho", fp64=True,
              rho0=sp.diag(0, 1))
    return (Drive / 2 * SZ, eps, [sp.sqrt(0.3) * sm], sp.diag(0, 1), np.linspace(0.0, 4.0, 801)), kw


def ode_call():
    x, y, t, k = sp.symbols("x y t k", real=True)
    kw = dict(var_arrays={k: np.linspace(0.5, 2.0, 4)}, fp64=True, output_mode="final")
    return ([-k * x, t], [x, y], [1.0, 0.0], np.linspace(0.0, 2.0, 1001)), kw


def known_answer_calls():
    """(api, args, kwargs) of every known-answer launch."""
    out = []
    for s in FIXED:
        for fp64 in (True, False):
            out.append(("mesolve_2D",) + rabi_call(s, fp64))
        out.append(("mesolve_2D",) + commuting_call(s))
    for s in ADAPTIVE:
        out.append(("mesolve_2D",) + commuting_call(s))
    out.append(("mesolve_2D",) + commuting_call("rk4", "mean"))
    out.append(("mesolve_2D",) + decay_call())
    out.append(("odesolve_2D",) + ode_call())
    return out


def wide_range_model(level, decay=True):
    """(args, kwargs) of an 8-level model whose operator terms span many orders of magnitude: level
    energies up to 45.5 with couplings of 2e-3 and decay terms of 5e-5 in Heff0, a drive operator of
    1 beside 3e-4; resonant drive A cos(6.5 t); mean population of `level`; 7 x 6 (eps, A) grid,
    2000 RK4 steps on [0, 20]."""
    eps, A, Drive, t = sp.symbols("eps A Drive t", real=True)
    N = 8
    H0 = sp.zeros(N)
    for k in range(N):
        H0[k, k] = 6.5 * k
    for k in range(N - 1):
        H0[k, k + 1] = H0[k + 1, k] = 2e-3
    X = sp.zeros(N)
    X[0, 1] = X[1, 0] = 1
    for k in range(1, N - 1):
        X[k, k + 1] = X[k + 1, k] = 3e-4
    H = H0 + eps * sp.diag(*range(N)) + Drive * X
    col = []
    for k in range(1, N) if decay else ():
        L = sp.zeros(N)
        L[k - 1, k] = sp.sqrt(1e-4)
        col.append(L)
    O = sp.zeros(N)
    O[level, level] = 1
    var = {eps: np.linspace(-0.05, 0.05, 7), A: np.linspace(0.2, 2.0, 6)}
    return (H, A * sp.cos(6.5 * t), col, O, np.linspace(0.0, 20.0, 2001)), {"var_arrays": var}


def wide_range_calls():
    out = []
    for level, decay in ((1, True), (1, False), (2, True)):
        args, kwargs = wide_range_model(level, decay)
        out.append(("mesolve_2D", args, dict(kwargs, fp64=True, rhs_form="matrix")))
        if decay:
            out.append(("mesolve_2D", args, dict(kwargs, precision="fp32", rhs_form="matrix_tc")))
    return out


def epilogue_diagonal_model():
    """(args, kwargs) of a 20-level model (padded to 32) with three dense drive operators and one
    diagonal term: 2 x 32 rows x 5 terms = 320 MMA columns exceed one MMA, so the tensor-core kernel
    takes the diagonal term in its epilogue. 4 x 3 (eps, A) points, 300 RK4 steps on [0, 15]."""
    eps, A, t = sp.symbols("eps A t", real=True)
    d1, d2, d3 = sp.symbols("Drive1 Drive2 Drive3", real=True)
    N = 20
    rng = np.random.default_rng(7)

    def hermitian(scale):
        G = (rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))) * scale / np.sqrt(2 * N)
        return sp.Matrix(np.round((G + G.conj().T) / 2, 6).tolist())
    H = hermitian(1.0) + eps * sp.diag(*range(N)) + d1 * hermitian(1.0) + d2 * hermitian(0.5) + d3 * hermitian(0.3)
    col = []
    for k in range(1, N):
        L = sp.zeros(N)
        L[k - 1, k] = sp.sqrt(0.01)
        col.append(L)
    O = sp.zeros(N)
    O[N - 1, N - 1] = 1
    drive = {"Drive1": A * sp.cos(t), "Drive2": A * sp.sin(t), "Drive3": A * sp.cos(2 * t)}
    var = {eps: np.linspace(-0.5, 0.5, 4), A: np.linspace(0.0, 2.0, 3)}
    return (H, drive, col, O, np.linspace(0.0, 15.0, 301)), {"var_arrays": var}


def epilogue_diagonal_calls():
    args, kwargs = epilogue_diagonal_model()
    return [("mesolve_2D", args, dict(kwargs, fp64=True, rhs_form="matrix")),
            ("mesolve_2D", args, dict(kwargs, precision="fp32", rhs_form="matrix_tc"))]


def offdiagonal_observable_model(N):
    """(args, kwargs) of the N-level scaling model on its small test grid with a Hermitian observable
    that has off-diagonal entries (a coherence between levels 0 and 1, one between N - 2 and N - 1,
    and a population): the general observable path of the tensor-core kernel."""
    _, args, kwargs = hilbert_model(N)
    O = sp.zeros(N)
    O[0, 1] = O[1, 0] = 1
    O[N - 2, N - 1] = sp.I / 2
    O[N - 1, N - 2] = -sp.I / 2
    O[N - 1, N - 1] = sp.Rational(1, 3)
    return args[:3] + (O,) + args[4:], kwargs


def offdiagonal_observable_calls():
    out = []
    for N in (16, 64):
        args, kwargs = offdiagonal_observable_model(N)
        out.append(("mesolve_2D", args, dict(kwargs, fp64=True, rhs_form="matrix")))
        out.append(("mesolve_2D", args, dict(kwargs, precision="fp32", rhs_form="matrix_tc")))
    return out
