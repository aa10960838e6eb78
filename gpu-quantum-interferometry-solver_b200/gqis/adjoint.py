"""Gradients of the time-averaged (or final) observable: checkpointed discrete adjoint of RK4 (FP64).

``mean_gradient(model..., params=[...])`` returns the ``mesolve_2D`` mean map (FP64, bit-identical
to the plain sweep) and d<O>_avg/dtheta for every point; with ``output="final"`` the final map
(``output_mode="final"``) and d<O>_final/dtheta. theta are runtime constants of the
model (e.g. Gamma1, Gamma_phi, Delta) and/or the swept parameters. ``MeanMap`` wraps it as a
``torch.autograd.Function`` for interferogram fitting: its backward contracts the per-point
derivatives with the incoming map gradient.

The device side is ``csrc/gqis_adjoint.cuh``; this module emits the adjoint struct it calls:
J(u, t)^T kb (the transposed Jacobian of the reduced RHS), (dF/dtheta)(u, t)^T kb including the
drives' parameter dependence, the drives and their parameter derivatives, and dO/dy - all derived
by SymPy from the same equations the sweep uses. ``forward_sensitivity`` is the independent
check: RK4 applied to the model augmented with its variational equations (run through
``odesolve_2D``), which equals the derivative of the discrete RK4 map.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import sympy as sp

from . import emit


# ----------------------------------------------------------------------------------------
# symbolic part
# ----------------------------------------------------------------------------------------

def _drive_items(compiled):
    dm = compiled.drive_map
    if isinstance(dm, dict):
        return list(dm.items())
    if dm is None:
        return []
    return [(sp.Symbol("Drive", real=True), sp.sympify(dm))]


def _param_symbols(compiled, params):
    """Map user parameter symbols (runtime constants or sweep symbols) to the internal symbols."""
    by_name = {str(s): s for s in compiled.base_runtime_syms}
    sweep = {str(s): name for s, name in zip(compiled.sweep_symbols, ("ParX", "ParY"))}
    out = []
    for p in params:
        name = str(p)
        if name in by_name:
            out.append(by_name[name])
        elif name in sweep:
            out.append(sp.Symbol(sweep[name], real=True))
        elif name in ("ParX", "ParY"):
            out.append(sp.Symbol(name, real=True))
        else:
            raise ValueError(f"parameter {p} is neither a runtime constant of the model nor a sweep symbol; "
                             "keep it symbolic with runtime_consts or keep_symbolic_consts")
    return out


def adjoint_equations(compiled, params):
    """SymPy pieces of the adjoint: (eqs, drives, states, params, g_obs)."""
    derived = dict(zip(compiled.runtime_const_syms[len(compiled.base_runtime_syms):], compiled.derived_const_exprs))
    eqs = [sp.sympify(e).xreplace(derived) for e in compiled.equations]
    drives = [(d, sp.sympify(e).xreplace(derived)) for d, e in _drive_items(compiled)]
    states = list(compiled.state_symbols)
    theta = _param_symbols(compiled, params)
    mean_re = sp.sympify(compiled.mean_re).xreplace(derived)
    return eqs, drives, states, theta, mean_re


def _lines(assigns, prefix):
    """CSE a list of (lhs, expr) and print as double-precision C++ lines."""
    if not assigns:
        return []
    subs, reduced = sp.cse([e for _, e in assigns], symbols=sp.numbered_symbols(prefix))
    out = [f"const double {s} = {emit.ccode(e, cast=False)};" for s, e in subs]
    out += [f"{lhs} {emit.ccode(e, cast=False)};" for (lhs, _), e in zip(assigns, reduced)]
    return out


def emit_adjoint(compiled, params):
    """C++ ``struct Adjoint`` for ``csrc/gqis_adjoint.cuh``; returns (source, meta)."""
    eqs, drives, states, theta, mean_re = adjoint_equations(compiled, params)
    S, P, ND = len(states), len(theta), len(drives)
    dsyms = [d for d, _ in drives]
    kb = [sp.Symbol(f"kb[{j}]", real=True) for j in range(S)]
    dD = [[sp.Symbol(f"dD[{k * P + m}]", real=True) for m in range(P)] for k in range(ND)]
    jt = []
    for i, yi in enumerate(states):
        jt.append((f"ub[{i}] =", sp.Add(*[kb[j] * sp.diff(eqs[j], yi) for j in range(S)])))
    fp = []
    for m, th in enumerate(theta):
        total = sp.Integer(0)
        for j in range(S):
            term = sp.diff(eqs[j], th)
            for k, dk in enumerate(dsyms):
                term += sp.diff(eqs[j], dk) * dD[k][m]
            total += kb[j] * term
        fp.append((f"tb[{m}] +=", total))
    # Functions of time alone (cos(w t), with runtime constants at most) in the drives and their
    # parameter derivatives are the same for every point: Tf[k], which the kernel evaluates once per
    # warp for the stage times of a block of steps (time_funcs).
    uniform = {str(s) for s in compiled.runtime_const_syms} | {"t"}
    time_funcs = {}

    def factor_time(e):
        found = {}
        walk = sp.preorder_traversal(sp.sympify(e))
        for sub in walk:
            names_in = {str(x) for x in sub.free_symbols} if isinstance(sub, sp.Function) else set()
            if names_in and names_in <= uniform and "t" in names_in:
                k = time_funcs.setdefault(sub, len(time_funcs))
                found[sub] = sp.Symbol(f"Tf[{k}]", real=True)
                walk.skip()
        return sp.sympify(e).xreplace(found) if found else e

    dr = [(f"D[{k}] =", factor_time(e)) for k, (_, e) in enumerate(drives)]
    ddr = [(f"dD[{k * P + m}] =", factor_time(sp.diff(e, th)))
           for k, (_, e) in enumerate(drives) for m, th in enumerate(theta)]
    tf = [(f"Tf[{k}] =", f) for k, f in enumerate(sorted(time_funcs, key=time_funcs.get))]
    dob = [(f"g[{i}] =", sp.diff(mean_re, yi)) for i, yi in enumerate(states)]

    names = {str(d): f"D[{k}]" for k, d in enumerate(dsyms)}
    names.update({str(s): f"C[{k}]" for k, s in enumerate(compiled.runtime_const_syms)})

    def fix(lines):
        out = []
        for ln in lines:
            ln = ln.replace("rho[", "u[")
            for name, repl in names.items():
                ln = emit._word(name).sub(lambda _m, r=repl: r, ln)
            out.append(ln)
        return out

    def body(lines):
        return "\n".join("        " + ln for ln in lines) if lines else "        /* none */"

    src = f"""struct Adjoint {{
    static constexpr int P = {P};
    static constexpr int ND = {ND};
    static constexpr int NTF = {len(time_funcs)};
    __device__ __forceinline__ static void time_funcs(double t, const double* C, double* Tf) {{
        (void)t; (void)C; (void)Tf;
{body(fix(_lines(tf, "at")))}
    }}
    __device__ __forceinline__ static void drives(double t, const double* Tf, double ParX, double ParY,
                                                  const double* C, double* D) {{
        (void)t; (void)Tf; (void)ParX; (void)ParY; (void)C; (void)D;
{body(fix(_lines(dr, "ad")))}
    }}
    __device__ __forceinline__ static void ddrives(double t, const double* Tf, double ParX, double ParY,
                                                   const double* C, double* dD) {{
        (void)t; (void)Tf; (void)ParX; (void)ParY; (void)C; (void)dD;
{body(fix(_lines(ddr, "add")))}
    }}
    __device__ __forceinline__ static void jt(const double* u, const double* kb, const double* D, double ParX,
                                              double ParY, const double* C, double* ub) {{
        (void)u; (void)kb; (void)D; (void)ParX; (void)ParY; (void)C;
{body(fix(_lines(jt, "aj")))}
    }}
    __device__ __forceinline__ static void fparam(const double* u, const double* kb, const double* D,
                                                  const double* dD, double ParX, double ParY, const double* C,
                                                  double* tb) {{
        (void)u; (void)kb; (void)D; (void)dD; (void)ParX; (void)ParY; (void)C; (void)tb;
{body(fix(_lines(fp, "af")))}
    }}
    __device__ __forceinline__ static void dobs(const double* u, const double* D, double ParX, double ParY,
                                                const double* C, double* g) {{
        (void)u; (void)D; (void)ParX; (void)ParY; (void)C;
{body(fix(_lines(dob, "ao")))}
    }}
}};
"""
    return src, {"P": P, "params": [str(t) for t in theta], "S": S}


# ----------------------------------------------------------------------------------------
# device call
# ----------------------------------------------------------------------------------------

def module_source(H, Drive, Col_Ops, mean_operator, tlist, *, var_arrays, params, const_values=None,
                  runtime_consts=None, warmup_time=0.0, t_in=0.0, rho0=None, rho0_values=None, output="mean",
                  **codegen):
    """Front end of an adjoint problem without a GPU: returns (module source, SweepLaunch, meta).
    ``output``: "mean" (d<O>_avg/dtheta) or "final" (d<O>/dtheta at the last step)."""
    from . import engine, solver
    if output not in ("mean", "final"):
        raise ValueError("the adjoint differentiates output 'mean' or 'final'")
    const_values = dict(const_values or {})
    runtime_consts = dict(runtime_consts or {})
    keep = [p for p in params if p in const_values or p in runtime_consts]
    holder = {}
    solver.mesolve_2D(H, Drive, Col_Ops, mean_operator, tlist, var_arrays=var_arrays,
                      const_values=const_values, runtime_consts=runtime_consts,
                      keep_symbolic_consts=keep or None, fp64=True, output_mode=output,
                      warmup_time=warmup_time, t_in=t_in, rho0=rho0, rho0_values=rho0_values,
                      _prepare_only=holder, **codegen)
    launch = holder["launch"]
    adj_src, meta = emit_adjoint(launch.entry["compiled"], params)
    source = engine.module_source(launch.entry["frag"], launch.entry["spec"], "fp64", output, None,
                                  extra_code=adj_src,
                                  defines={"GQ_WITH_ADJOINT": 1, "GQ_ADJOINT_FINAL": int(output == "final")})
    meta["defaults"] = {**const_values, **runtime_consts}
    return source, launch, meta


def const_values(compiled, defaults, values=None):
    """Full runtime-constant array (kept symbols, then derived expressions) for given values."""
    vals = {str(k): v for k, v in (defaults or {}).items()}
    vals.update({str(k): v for k, v in (values or {}).items()})
    base = {s: float(vals[str(s)]) for s in compiled.base_runtime_syms}
    return [base[s] for s in compiled.base_runtime_syms] + [float(e.evalf(subs=base))
                                                            for e in compiled.derived_const_exprs]


class Problem:
    """A mean-map + gradient problem prepared once (module built, inputs uploaded)."""

    def __init__(self, H, Drive, Col_Ops, mean_operator, tlist, *, var_arrays, params, const_values=None,
                 runtime_consts=None, warmup_time=0.0, t_in=0.0, rho0=None, rho0_values=None,
                 checkpoint_every=None, output="mean", **codegen):
        from . import abi, engine, solver
        import torch
        const_values = dict(const_values or {})
        runtime_consts = dict(runtime_consts or {})
        source, launch, meta = module_source(H, Drive, Col_Ops, mean_operator, tlist, var_arrays=var_arrays,
                                             params=params, const_values=const_values,
                                             runtime_consts=runtime_consts, warmup_time=warmup_time, t_in=t_in,
                                             rho0=rho0, rho0_values=rho0_values, output=output, **codegen)
        self.output = output
        self.compiled = launch.entry["compiled"]
        self.params = meta["params"]
        self.P = meta["P"]
        self.module = engine.load_module(source)
        self.launch_spec = launch
        self.torch = torch
        self.desc_sweep, self.buf = solver._device_buffers(launch)
        npts = int(self.desc_sweep.point_count)
        N = int(launch.num_steps)
        self.checkpoint_every = int(checkpoint_every or max(1, math.ceil(math.sqrt(N))))
        nbytes = ctypes.c_int64()
        rc = self.module.lib.gqis_adjoint_scratch_bytes(npts, N, self.checkpoint_every, ctypes.byref(nbytes))
        abi.check(rc, self.module.lib)
        dev = self.buf["results"].device
        self.scratch = torch.empty(max(1, nbytes.value // 8), dtype=torch.float64, device=dev)
        self.grad = torch.empty((npts, max(1, self.P)), dtype=torch.float64, device=dev)
        self.const_syms = list(self.compiled.runtime_const_syms)
        self.base_syms = list(self.compiled.base_runtime_syms)
        self.defaults = {**{k: v for k, v in const_values.items()}, **runtime_consts}
        self.shape = (len(launch.par_x), len(launch.par_y))
        self.scratch_bytes = nbytes.value

    def const_array(self, values=None):
        """Full runtime-constant array (kept symbols, then derived expressions) for given values."""
        return const_values(self.compiled, self.defaults, values)

    def run(self, values=None, stream=None):
        """Launch; returns device tensors (mean map (nx, ny), grad (nx, ny, P))."""
        from . import abi
        torch = self.torch
        consts_full = self.const_array(values)
        # The forward module reads only the constants its emitted code uses, in that order.
        used = self.launch_spec.entry["frag"]["used_const_indices"]
        fwd = [consts_full[i] for i in used] if used else []
        dev = self.buf["results"].device
        self._cf = torch.tensor(fwd or [0.0], dtype=torch.float64, device=dev)
        self._ca = torch.tensor(consts_full or [0.0], dtype=torch.float64, device=dev)
        d = abi.AdjointDesc()
        d.sweep = self.desc_sweep
        d.sweep.consts = self._cf.data_ptr() if fwd else None
        d.num_params = self.P
        d.checkpoint_every = self.checkpoint_every
        d.adjoint_consts = self._ca.data_ptr()
        d.grad = self.grad.data_ptr()
        d.scratch = self.scratch.data_ptr()
        d.scratch_bytes = self.scratch_bytes
        st = stream or torch.cuda.current_stream()
        rc = self.module.lib.gqis_adjoint_launch(ctypes.byref(d), ctypes.c_void_p(st.cuda_stream))
        abi.check(rc, self.module.lib)
        nx, ny = self.shape
        return self.buf["results"][:, 0].reshape(nx, ny), self.grad[:, :self.P].reshape(nx, ny, self.P)


def mean_gradient(H, Drive, Col_Ops, mean_operator, tlist, *, var_arrays, params, values=None, **kwargs):
    """Mean map and d<O>_avg/dtheta per point (NumPy, FP64); see :class:`Problem`."""
    prob = Problem(H, Drive, Col_Ops, mean_operator, tlist, var_arrays=var_arrays, params=params, **kwargs)
    mean, grad = prob.run(values)
    return mean.cpu().numpy(), grad.cpu().numpy()


def _autograd_function():
    import torch

    class MeanMap(torch.autograd.Function):
        """<O>_avg map as a differentiable function of the parameter vector theta.

        ``MeanMap.apply(theta, problem)``: theta is a 1-D tensor of the problem's runtime-constant
        parameters in ``problem.params`` order; returns the (nx, ny) mean map; backward returns
        sum over points of grad_out * d<O>/dtheta.
        """

        @staticmethod
        def forward(ctx, theta, problem):
            names = problem.params
            values = {name: float(v) for name, v in zip(names, theta.detach().cpu().tolist())}
            mean, grad = problem.run(values)
            ctx.save_for_backward(grad.clone())
            ctx.theta_device = theta.device
            return mean.clone().to(theta.dtype)

        @staticmethod
        def backward(ctx, grad_out):
            (grad,) = ctx.saved_tensors
            g = (grad_out.to(grad.device, grad.dtype).unsqueeze(-1) * grad).sum(dim=(0, 1))
            return g.to(ctx.theta_device), None

    return MeanMap


def __getattr__(name):
    if name == "MeanMap":
        return _autograd_function()
    raise AttributeError(name)


# ----------------------------------------------------------------------------------------
# forward-mode reference: RK4 on the model augmented with its variational equations
# ----------------------------------------------------------------------------------------

def forward_sensitivity(H, Drive, Col_Ops, mean_operator, tlist, *, var_arrays, params, const_values=None,
                        runtime_consts=None, warmup_time=0.0, t_in=0.0):
    """d<O>_avg/dtheta by forward sensitivities (FP64), through ``odesolve_2D``.

    The reduced Lindblad equations y' = F(y, t) are augmented with s_m' = J s_m + dF/dtheta_m for
    each parameter, the drives written out as functions of t; RK4 of the augmented system is the
    tangent of the RK4 map, so the result equals the discrete adjoint up to rounding.
    Returns (mean (nx, ny), grad (nx, ny, P)).
    """
    from . import rhs as rhs_mod
    from .gqis_ode_api import odesolve_2D
    const_values = dict(const_values or {})
    runtime_consts = dict(runtime_consts or {})
    keep = [p for p in params if p in const_values or p in runtime_consts]
    compiled, _ = rhs_mod.compile_rhs(H, Drive, Col_Ops, mean_operator, sweep_symbols=tuple(var_arrays),
                                      const_values=const_values, runtime_consts=runtime_consts,
                                      keep_symbolic_consts=keep or None, reuse=False)
    eqs, drives, states, theta, mean_re = adjoint_equations(compiled, params)
    t = sp.Symbol("t", real=True)
    dmap = {d: e.subs({s: t for s in e.free_symbols if s.name == "t"}) for d, e in drives}
    F = [e.xreplace(dmap) for e in eqs]
    S, P = len(states), len(theta)
    sens = [[sp.Symbol(f"s_{m}_{i}", real=True) for i in range(S)] for m in range(P)]
    ys = [sp.Symbol(f"y_{i}", real=True) for i in range(S)]
    ren = dict(zip(states, ys))
    aug = [f.xreplace(ren) for f in F]
    for m, th in enumerate(theta):
        for j in range(S):
            expr = sp.diff(F[j], th) + sp.Add(*[sp.diff(F[j], yi) * sens[m][i] for i, yi in enumerate(states)])
            aug.append(expr.xreplace(ren))
    all_states = ys + [s for row in sens for s in row]
    y0 = [1] + [0] * (S - 1) + [0] * (S * P)
    # runtime constants become ODE parameters with their values
    param_vals = {}
    pmap = {}
    for s in compiled.base_runtime_syms:
        v = runtime_consts.get(s, const_values.get(s))
        sym = sp.Symbol(str(s), real=True)
        pmap[s] = sym
        param_vals[sym] = v
    sweep_ren = {sp.Symbol(n, real=True): s for n, s in zip(("ParX", "ParY"), var_arrays)}
    aug = [e.xreplace(pmap).xreplace(sweep_ren) for e in aug]
    mean_state = odesolve_2D(aug, all_states, y0, tlist, var_arrays=var_arrays, const_values=param_vals,
                             output_mode="mean", fp64=True, warmup_time=warmup_time, t_in=t_in)
    g = np.array([float(sp.diff(mean_re, yi)) for yi in states])
    c0 = float(mean_re.xreplace({yi: 0 for yi in states}))
    mean = mean_state[..., :S] @ g + c0
    grad = np.stack([mean_state[..., S * (1 + m):S * (2 + m)] @ g for m in range(P)], axis=-1)
    return mean, grad
