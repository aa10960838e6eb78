"""CPU oracle: density-matrix form of the Lindblad sweep, batched over points in NumPy (FP64).

Oracle infrastructure only (tests/, ``__graft_entry__.smoke()`` and bench.py's CPU baseline
leg). It restates the algorithm of the reference sweep without any of the product's code:

* the master equation in full matrix form, d rho/dt = -i[H(t), rho] + sum_L (L rho L^dag
  - 1/2 {L^dag L, rho}) (reference ``gqis/solver.py:452-457``), with H = H_static + sum_d
  Drive_d(t) H_d evaluated per point;
* the reference RK4 step (``gqis/cuda_solvers.py:470-517``): stage times t + dt/2 and
  (t + dt/2) + dt/2 computed from the step index;
* the outputs of ``gqis/solver.py:2126-2196``: the right-endpoint mean of <O> over the steps
  after warmup, the final <O>, or the final reduced state (``gqis/solver.py:202-250`` layout).

Floats of H, the drives and O are rounded to ten significant digits, as the reference code
printer does (``gqis/solver.py:166-170``), so the oracle integrates the same numbers as the
reference kernel. Collapse operators enter quadratically and are left unrounded.
"""

from __future__ import annotations

import numpy as np
import sympy as sp


def round_literals(expr):
    """Evaluate exact irrationals and round every Float to 10 significant digits."""
    expr = sp.sympify(expr)
    found = {}
    walk = sp.preorder_traversal(expr)
    for sub in walk:
        if sub.is_number and not (sub.is_Rational or sub.is_Float) and sub.is_real:
            found[sub] = sub.evalf()
            walk.skip()
    expr = expr.xreplace(found)
    return expr.xreplace({f: sp.Float(float(f"{float(f):.9e}")) for f in expr.atoms(sp.Float)})


class MatrixModel:
    """Numeric form of a (H, Drive, Col_Ops, O) model on a 1-D / 2-D sweep."""

    def __init__(self, H, Drive, Col_Ops, mean_operator, var_arrays, const_values=None, t_symbol="t"):
        const_values = dict(const_values or {})
        syms = list(var_arrays)
        self.N = H.shape[0]
        H = H.xreplace({k: sp.Float(float(v)) for k, v in const_values.items()})
        drive_map = Drive if isinstance(Drive, dict) else {sp.Symbol("Drive", real=True): Drive}
        placeholders = [s for s in drive_map]
        t = sp.Symbol(t_symbol, real=True)
        for k, v in const_values.items():
            drive_map = {d: sp.sympify(e).xreplace({k: sp.Float(float(v))}) for d, e in drive_map.items()}
        H = H.applyfunc(round_literals)
        self.H_parts = []
        static = H.xreplace({d: 0 for d in placeholders})
        self.static_fn = sp.lambdify(syms, static, "numpy")
        for d in placeholders:
            self.H_parts.append(np.array(H.diff(d).tolist(), dtype=complex))
        self.drive_fns = [sp.lambdify([t] + syms, round_literals(drive_map[d]), "numpy") for d in placeholders]
        self.L = [np.array(L.xreplace({k: sp.Float(float(v)) for k, v in const_values.items()}).evalf().tolist(),
                           dtype=complex) for L in Col_Ops]
        self.O = np.array(mean_operator.applyfunc(round_literals).tolist(), dtype=complex)
        axes = [np.asarray(v, dtype=np.float64) for v in var_arrays.values()]
        if len(axes) == 1:
            axes.append(np.zeros(1))
        self.shape = (len(axes[0]), len(axes[1]))
        X, Y = np.meshgrid(axes[0], axes[1], indexing="ij")
        self.params = [X.ravel(), Y.ravel()][:len(syms)]
        P = X.size
        Hs = np.empty((P, self.N, self.N), dtype=complex)
        for p in range(P):
            Hs[p] = np.array(self.static_fn(*[a[p] for a in self.params]), dtype=complex)
        self.H_static = Hs
        self.LdL = sum((L.conj().T @ L for L in self.L), np.zeros((self.N, self.N), dtype=complex))
        # L rho L^dag of sparse collapse operators as one sparse map on row-major vec(rho):
        # (L rho L^dag)_ij = sum_ab L_ia rho_ab conj(L_jb); dense operators stay as products.
        import scipy.sparse as sps
        rows, cols, vals, self.L_dense = [], [], [], []
        for L in self.L:
            nz = list(zip(*np.nonzero(L)))
            if len(nz) ** 2 > 4 * self.N * self.N:
                self.L_dense.append(L)
                continue
            for (i, a) in nz:
                for (j, b) in nz:
                    rows.append(i * self.N + j)
                    cols.append(a * self.N + b)
                    vals.append(L[i, a] * np.conj(L[j, b]))
        self.jump_T = sps.csr_matrix((np.array(vals, dtype=complex), (cols, rows)), shape=(self.N**2,) * 2)
        # Row-major vectorisation, vec(A rho B) = (A kron B^T) vec(rho): for small N the RHS is a
        # per-point superoperator applied to vec(rho) (same equation, far fewer NumPy calls).
        self.superop = self.N <= 8
        if self.superop:
            I = np.eye(self.N)
            diss = sum((np.kron(L, L.conj()) for L in self.L), np.zeros((self.N**2,) * 2, dtype=complex))
            diss = diss - 0.5 * (np.kron(self.LdL, I) + np.kron(I, self.LdL.T))
            self.M_static = np.stack([-1j * (np.kron(h, I) - np.kron(I, h.T)) + diss for h in Hs])
            self.M_drive = [-1j * (np.kron(h, I) - np.kron(I, h.T)) for h in self.H_parts]

    def drives(self, t):
        P = self.H_static.shape[0]
        return [np.broadcast_to(np.asarray(fn(t, *self.params), dtype=np.float64), (P,)) for fn in self.drive_fns]

    def hamiltonian(self, t):
        if self.superop:
            return self.drives(t)
        H = self.H_static.copy()
        for Hd, fn in zip(self.H_parts, self.drive_fns):
            d = np.broadcast_to(np.asarray(fn(t, *self.params), dtype=np.float64), (H.shape[0],))
            H += d[:, None, None] * Hd
        return H

    def rhs(self, H, rho):
        if self.superop:  # H holds the drive values; rho is (P, N, N)
            v = rho.reshape(rho.shape[0], -1)
            out = np.matmul(self.M_static, v[..., None])[..., 0]
            for d, Md in zip(H, self.M_drive):
                out += d[:, None] * (v @ Md.T)
            return out.reshape(rho.shape)
        # -i[H, rho] - 1/2 {LdL, rho} = -i (Heff rho - rho Heff^dag), Heff = H - i/2 LdL
        Heff = H - 0.5j * self.LdL
        out = -1j * (Heff @ rho - rho @ np.conj(np.swapaxes(Heff, -1, -2)))
        for L in self.L_dense:
            out += L @ rho @ L.conj().T
        P = rho.shape[0]
        out += (rho.reshape(P, -1) @ self.jump_T).reshape(rho.shape)
        return out

    def observe(self, rho):
        return np.einsum("ij,pji->p", self.O, rho)

    def initial(self, rho0=None):
        P = self.H_static.shape[0]
        rho = np.zeros((P, self.N, self.N), dtype=complex)
        if rho0 is None:
            rho[:, 0, 0] = 1.0
        else:
            rho[:] = rho0
        return rho


def reduced_state(rho):
    """(P, N, N) density matrices -> (P, N*N-1) reduced real vectors (reference layout)."""
    P, N, _ = rho.shape
    cols = [rho[:, i, i].real for i in range(N - 1)]
    for i in range(N):
        for j in range(i + 1, N):
            cols.append(rho[:, i, j].real)
            cols.append(rho[:, i, j].imag)
    return np.stack(cols, axis=1)


def rk4_sweep(model, tlist, *, output_mode="mean", warmup_time=0.0, t_in=0.0, rho0=None):
    """Reference-order RK4 over the whole grid; returns the map in the API's shape."""
    tlist = np.asarray(tlist, dtype=np.float64)
    steps = len(tlist) - 1
    dt = float((tlist[-1] - tlist[0]) / steps)
    warm = steps if warmup_time >= 1.0 else int(np.floor(warmup_time * steps))
    rho = model.initial(rho0)
    acc = np.zeros(rho.shape[0], dtype=complex)
    half = dt * 0.5
    for step in range(steps):
        t_mid = (step + 0.5) * dt
        H_mid = model.hamiltonian(t_in + t_mid)
        H_end = model.hamiltonian(t_in + (t_mid + half))
        H0 = model.hamiltonian(t_in + step * dt) if step == 0 else H_prev_end
        k1 = model.rhs(H0, rho)
        k2 = model.rhs(H_mid, rho + half * k1)
        k3 = model.rhs(H_mid, rho + half * k2)
        k4 = model.rhs(H_end, rho + dt * k3)
        rho = rho + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
        H_prev_end = H_end
        if output_mode == "mean" and step >= warm:
            acc += model.observe(rho)
    nx, ny = model.shape
    if output_mode == "mean" and warm < steps:
        return (acc / (steps - warm)).reshape(nx, ny)
    if output_mode in ("mean", "final"):
        return model.observe(rho).reshape(nx, ny)
    if output_mode == "final_rho":
        return reduced_state(rho).reshape(nx, ny, -1)
    raise ValueError(output_mode)


def from_workload(w, side_arrays=None):
    """MatrixModel of a ``gqis.workloads`` dict."""
    return MatrixModel(w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], side_arrays or w["var_arrays"],
                       w.get("const_values"))
