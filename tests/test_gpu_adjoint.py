"""Gradients on the GPU: the checkpointed RK4 adjoint against forward sensitivities and central
finite differences (FP64, h = 1e-6), and through torch.autograd."""

import numpy as np
import pytest

from test_support_calls import qubit_fit_model


def _scaled(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.gpu
def test_adjoint_mean_equals_plain_fp64_sweep():
    import gqis
    from gqis import adjoint
    args, kwargs, params = qubit_fit_model()
    mean, grad = adjoint.mean_gradient(*args, **kwargs, params=list(params))
    plain = gqis.mesolve_2D(*args, **kwargs, keep_symbolic_consts=list(params[:3]), fp64=True)
    assert _scaled(mean, plain.real) < 1e-13
    assert grad.shape == (8, 6, 4)


@pytest.mark.gpu
def test_adjoint_matches_forward_sensitivities():
    from gqis import adjoint
    args, kwargs, params = qubit_fit_model()
    mean, grad = adjoint.mean_gradient(*args, **kwargs, params=list(params))
    fmean, fgrad = adjoint.forward_sensitivity(*args, **kwargs, params=list(params))
    assert _scaled(mean, fmean) < 1e-12
    for m in range(4):
        assert _scaled(grad[..., m], fgrad[..., m]) < 1e-9, m


@pytest.mark.gpu
def test_adjoint_matches_central_differences():
    import gqis
    from gqis import adjoint
    args, kwargs, params = qubit_fit_model()
    G1, Gp, D, A = params
    _, grad = adjoint.mean_gradient(*args, **kwargs, params=[G1, Gp, D])
    h = 1e-6
    base = kwargs["runtime_consts"]
    for m, p in enumerate((G1, Gp, D)):
        up, dn = dict(base), dict(base)
        up[p] = base[p] + h
        dn[p] = base[p] - h
        fp = gqis.mesolve_2D(*args, **dict(kwargs, runtime_consts=up), fp64=True).real
        fm = gqis.mesolve_2D(*args, **dict(kwargs, runtime_consts=dn), fp64=True).real
        fd = (fp - fm) / (2 * h)
        assert _scaled(grad[..., m], fd) < 1e-6, (p, _scaled(grad[..., m], fd))


@pytest.mark.gpu
def test_autograd_backward_contracts_the_gradient():
    import torch
    from gqis import adjoint
    args, kwargs, params = qubit_fit_model()
    prob = adjoint.Problem(*args, **kwargs, params=list(params[:3]))
    theta = torch.tensor([0.01, 0.02, 1.0], dtype=torch.float64, requires_grad=True)
    out = adjoint.MeanMap.apply(theta, prob)
    weights = torch.linspace(0.5, 1.5, out.numel(), dtype=torch.float64, device=out.device).reshape(out.shape)
    loss = (weights * out).sum()
    loss.backward()
    _, grad = prob.run({"Gamma1": 0.01, "Gammaphi": 0.02, "Delta": 1.0})
    expect = (weights.unsqueeze(-1) * grad).sum(dim=(0, 1)).cpu()
    assert torch.allclose(theta.grad, expect, rtol=1e-12, atol=0)
    assert torch.isfinite(theta.grad).all()


@pytest.mark.gpu
def test_adjoint_of_the_final_observable():
    """output="final": the final <O> map equals the plain FP64 sweep's final output, and its gradient
    in the fit parameters (Gamma1, Gamma_phi, Delta) and the swept drive amplitude A equals central
    differences of that sweep (h = 1e-6)."""
    import gqis
    from gqis import adjoint
    args, kwargs, params = qubit_fit_model()
    final, grad = adjoint.mean_gradient(*args, **kwargs, params=list(params), output="final")
    plain = gqis.mesolve_2D(*args, **kwargs, keep_symbolic_consts=list(params[:3]), fp64=True, output_mode="final")
    assert _scaled(final, plain.real) < 1e-13
    h = 1e-6
    base = kwargs["runtime_consts"]
    for m, p in enumerate(params[:3]):
        up, dn = dict(base), dict(base)
        up[p] = base[p] + h
        dn[p] = base[p] - h
        fp = gqis.mesolve_2D(*args, **dict(kwargs, runtime_consts=up), fp64=True, output_mode="final").real
        fm = gqis.mesolve_2D(*args, **dict(kwargs, runtime_consts=dn), fp64=True, output_mode="final").real
        assert _scaled(grad[..., m], (fp - fm) / (2 * h)) < 1e-6, p
    eps, A = list(kwargs["var_arrays"])
    up, dn = dict(kwargs["var_arrays"]), dict(kwargs["var_arrays"])
    up[A] = up[A] + h
    dn[A] = dn[A] - h
    fp = gqis.mesolve_2D(*args, **dict(kwargs, var_arrays=up), fp64=True, output_mode="final").real
    fm = gqis.mesolve_2D(*args, **dict(kwargs, var_arrays=dn), fp64=True, output_mode="final").real
    assert _scaled(grad[..., 3], (fp - fm) / (2 * h)) < 1e-6
