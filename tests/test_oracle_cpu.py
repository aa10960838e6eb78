"""Pin the CPU oracles to the reference's own outputs (golden fixtures), on the CPU.

The golden fixtures are the reference's generated kernels run in FP64 (tests/golden). Before
an oracle checks the GPU path, it must reproduce them: the NumPy density-matrix oracle for the
Lindblad cases, the C oracle for the adaptive Duffing case.
"""

from pathlib import Path

import numpy as np
import pytest

import lindblad_oracle
import ode_oracle
import ref_cases

GOLDEN = Path(__file__).resolve().parent / "golden"
W = ref_cases.workloads()


def test_matrix_oracle_matches_reference_two_level_map_rows():
    w = W.two_level()
    eps, A = w["symbols"]
    g = np.load(GOLDEN / "c1_fp64_mean.npz")["result"]
    rows = [0, 21, 63]  # a few eps rows over the whole A axis keep the CPU time short
    sub = {eps: w["var_arrays"][eps][rows], A: w["var_arrays"][A]}
    model = lindblad_oracle.from_workload(w, sub)
    got = lindblad_oracle.rk4_sweep(model, w["tlist"])
    assert np.max(np.abs(got - g[rows])) < 1e-13


def test_matrix_oracle_matches_reference_four_level_subgrid():
    w = W.four_level(side=32)
    eps, A = w["symbols"]
    g = np.load(GOLDEN / "c2_fp64_mean_sub32.npz")["result"]
    cols = [0, 13, 31]
    sub = {eps: w["var_arrays"][eps], A: w["var_arrays"][A][cols]}
    got = lindblad_oracle.rk4_sweep(lindblad_oracle.from_workload(w, sub), w["tlist"])
    assert np.max(np.abs(got - g[:, cols])) < 1e-13


@pytest.mark.parametrize("name,mode", [("qubit_rk4_final_rho", "final_rho"), ("qubit_rk4_final", "final")])
def test_matrix_oracle_output_modes(name, mode):
    q = ref_cases.small_qubit()
    g = np.load(GOLDEN / f"{name}.npz")["result"]
    got = lindblad_oracle.rk4_sweep(lindblad_oracle.from_workload(q), q["tlist"], output_mode=mode)
    assert np.max(np.abs(got - g)) < 1e-13


def test_matrix_oracle_warmup_and_time_offset():
    q = ref_cases.small_qubit()
    model = lindblad_oracle.from_workload(q)
    g = np.load(GOLDEN / "qubit_rk4_mean_warmup_trace.npz")["result"]
    assert np.max(np.abs(lindblad_oracle.rk4_sweep(model, q["tlist"], warmup_time=0.3) - g)) < 1e-13
    g = np.load(GOLDEN / "qubit_rk4_t_in.npz")["result"]
    assert np.max(np.abs(lindblad_oracle.rk4_sweep(model, q["tlist"], t_in=3.25) - g)) < 1e-13


def test_c_oracle_matches_reference_adaptive_tsit5_duffing():
    d = W.duffing(side=12)
    F, Wv = d["var_arrays"].values()
    g = np.load(GOLDEN / "duffing_tsit5a_trace.npz")
    final, trace, _ = ode_oracle.sweep("tsit5a", F, Wv, d["y0_values"], d["tlist"])
    assert np.max(np.abs(final - g["result"])) < 1e-10
    assert np.max(np.abs(trace[:, :, ::int(g["trace_stride"])] - g["trace"])) < 1e-10


def test_c_oracle_rk4_matches_reference_duffing_observable_trace():
    d = W.duffing(side=12)
    F, Wv = d["var_arrays"].values()
    g = np.load(GOLDEN / "duffing_rk4_observable_trace.npz")
    tl = np.linspace(0.0, 50.0, 5001)
    final, trace, _ = ode_oracle.sweep("rk4", F, Wv, d["y0_values"], tl)
    x, v = trace[..., 0], trace[..., 1]
    obs = x**2 + 1j * v
    stride = 10 * int(g["trace_stride"])
    assert np.max(np.abs(obs[:, :, ::stride] - g["trace"])) < 1e-12  # samples after steps 0, 10, ..


def test_c_oracle_adaptive_dop853_agrees_with_scipy():
    """Adaptive DOP853 has no reference implementation: pin it to SciPy's DOP853 instead."""
    from scipy.integrate import solve_ivp
    d = W.duffing(side=3)
    F, Wv = d["var_arrays"].values()
    final, _, counts = ode_oracle.sweep("dop853a", F, Wv, d["y0_values"], d["tlist"], want_trace=False)
    for i in range(3):
        for j in range(3):
            sol = solve_ivp(lambda t, y: [y[1], -0.1 * y[1] - y[0] - y[0]**3 + F[i] * np.cos(Wv[j] * t)],
                            (0.0, 500.0), d["y0_values"][i, j], method="DOP853", rtol=1e-12, atol=1e-13)
            assert np.max(np.abs(sol.y[:, -1] - final[i, j])) < 5e-6
    assert counts[..., 0].min() > 100


@pytest.mark.parametrize("case", ["rabi", "commuting", "mean", "decay"])
def test_matrix_oracle_known_answers(case):
    """The density-matrix oracle reproduces the analytic answers the GPU known-answer tests use."""
    import test_support_calls as ka
    args, kw = {"rabi": lambda: ka.rabi_call("rk4", True), "commuting": lambda: ka.commuting_call("rk4"),
                "mean": lambda: ka.commuting_call("rk4", "mean"), "decay": ka.decay_call}[case]()
    H, Drive, Col_Ops, O, tlist = args
    rho0 = np.array(kw["rho0"].tolist(), dtype=complex) if "rho0" in kw else None
    model = lindblad_oracle.MatrixModel(H, Drive, Col_Ops, O, kw["var_arrays"])
    out = lindblad_oracle.rk4_sweep(model, tlist, output_mode=kw["output_mode"], rho0=rho0)
    x = np.linspace(0.5, 2.0, 4)
    if case == "rabi":
        got, exact = out[:, 0, 0], np.cos(x * np.pi / 2) ** 2
    elif case == "commuting":
        got, exact = out[:, 0, 0], np.cos(x * np.sin(5.0) / 2) ** 2
    elif case == "mean":
        got = out.real[:, 0]
        exact = np.mean(np.sin(x[:, None] * np.sin(tlist[1:]) / 2) ** 2, axis=1)
    else:
        got, exact = out[..., 0], 1 - np.exp(-0.3 * 4.0)
    assert np.max(np.abs(got - exact)) <= 1e-9
