"""Known analytic answers on the GPU (the reference's test_gpu_solver / test_ode_api known answers,
written here from the physics):

* Rabi rotation H = (Omega / 2) sigma_x from the ground state: rho00(T) = cos^2(Omega T / 2), every
  fixed-step integrator, FP64 and the FP32 form;
* a commuting time-dependent drive H = (A cos t / 2) sigma_x: rho00(T) = cos^2(A sin T / 2), every
  fixed-step integrator and the adaptive ones, and the right-endpoint time average of rho11;
* pure decay sqrt(gamma) sigma_- from the excited state: rho11(T) = exp(-gamma T);
* the ODE front end on x' = -k x, y' = t: x(T) = exp(-k T), y(T) = T^2 / 2.
"""

import numpy as np
import pytest

from gqis.cuda_solvers import get_solver_spec
from test_support_calls import ADAPTIVE, FIXED, commuting_call, decay_call, ode_call, rabi_call


@pytest.mark.gpu
@pytest.mark.parametrize("solver", FIXED)
@pytest.mark.parametrize("fp64", [True, False])
def test_rabi_rotation(solver, fp64):
    import gqis
    args, kw = rabi_call(solver, fp64)
    rho = np.asarray(gqis.mesolve_2D(*args, **kw))
    Om = np.linspace(0.5, 2.0, 4)
    exact = np.cos(Om * np.pi / 2) ** 2
    err = float(np.max(np.abs(rho[:, 0, 0] - exact)))
    assert err <= (1e-9 if fp64 else 2e-6), (solver, err)


@pytest.mark.gpu
@pytest.mark.parametrize("solver", FIXED + ADAPTIVE)
def test_commuting_drive(solver):
    import gqis
    args, kw = commuting_call(solver)
    rho = np.asarray(gqis.mesolve_2D(*args, **kw))
    A = np.linspace(0.5, 2.0, 4)
    exact = np.cos(A * np.sin(5.0) / 2) ** 2
    err = float(np.max(np.abs(rho[:, 0, 0] - exact)))
    assert err <= (1e-8 if get_solver_spec(solver).adaptive else 1e-9), (solver, err)


@pytest.mark.gpu
def test_time_average_is_the_right_endpoint_mean():
    import gqis
    args, kw = commuting_call("rk4", "mean")
    mean = np.asarray(gqis.mesolve_2D(*args, **kw)).real[:, 0]
    A = np.linspace(0.5, 2.0, 4)[:, None]
    t = np.linspace(0.0, 5.0, 2001)[1:]
    exact = np.mean(np.sin(A * np.sin(t) / 2) ** 2, axis=1)
    assert float(np.max(np.abs(mean - exact))) <= 1e-9


@pytest.mark.gpu
def test_pure_decay():
    import gqis
    args, kw = decay_call()
    rho = np.asarray(gqis.mesolve_2D(*args, **kw))
    assert float(np.max(np.abs(rho[..., 0] - (1 - np.exp(-0.3 * 4.0))))) <= 1e-10


@pytest.mark.gpu
def test_ode_front_end_known_answers():
    import gqis
    args, kw = ode_call()
    out = np.asarray(gqis.odesolve_2D(*args, **kw)).reshape(4, 2)
    k = np.linspace(0.5, 2.0, 4)
    assert float(np.max(np.abs(out[:, 0] - np.exp(-2.0 * k)))) <= 1e-10
    assert float(np.max(np.abs(out[:, 1] - 2.0))) <= 1e-10


@pytest.mark.gpu
def test_tsit5a_matches_time_dependent_solution_between_coarse_output_points():
    """Four output intervals on [0, 1.7]: the adaptive steps inside each interval follow the drive
    (1 + 0.4 sin t) sx / 2, and rho00(T) = cos^2((T + 0.4 (1 - cos T)) / 2)
    (the reference's tests/test_gpu_solver.py:271-290)."""
    import gqis
    from test_support_calls import tsit5a_coarse_output_call
    args, kw = tsit5a_coarse_output_call()
    rho = np.asarray(gqis.mesolve_2D(*args, **kw))
    T = 1.7
    expected = np.cos(0.5 * (T + 0.4 * (1.0 - np.cos(T)))) ** 2
    assert abs(float(rho[0, 0, 0]) - expected) < 2.0e-7


@pytest.mark.gpu
@pytest.mark.parametrize("fp64_time", (True, False))
def test_tsit5a_time_average_integrates_over_adaptive_steps(fp64_time):
    """The time average of rho00 = cos^2(t/2) over [2, 10] is 1/2 + (sin 10 - sin 2) / 16; Tsit5A
    integrates it with the trapezoid rule over its own steps (second order, about
    h^2/12 |f'(10) - f'(2)| / 8), not over the 5 output points (the reference's
    tests/test_gpu_solver.py:294-311)."""
    import gqis
    from test_support_calls import tsit5a_average_call
    args, kw = tsit5a_average_call(fp64_time)
    value, info = gqis.mesolve_2D(*args, **kw)
    expected = 0.5 + (np.sin(10.0) - np.sin(2.0)) / (2.0 * 8.0)
    assert abs(float(np.real(value[0, 0])) - expected) < 5.0e-5
    assert info["adaptive_steps"]["accepted"][0, 0] > 5
