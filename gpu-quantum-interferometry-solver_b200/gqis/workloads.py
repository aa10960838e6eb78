"""Synthetic sweep workloads: the benchmark and parity models, defined once.

Pure SymPy/NumPy with no package-relative imports, so the oracle recipes can load this file on
its own (importlib by path) next to another ``gqis`` package. Every constant that reaches
generated code is a short decimal (couplings are rounded to six digits after drawing them), so
the ten-significant-digit literals of the code printer represent the model exactly and CPU
oracles can use the same numbers.

* ``two_level``   - driven qubit: H = eps/2 sz + Delta/2 sx + A cos(w t) sz, Delta = 1,
                    w = 2 pi 0.5; L = sqrt(G1) s-, sqrt(Gphi/2) sz (G1 = 0.01, Gphi = 0.02);
                    rho0 = ground; O = excited projector; tlist = linspace(0, 200, 4001);
                    eps in linspace(-5, 5, 64) x A in linspace(0, 5, 64).
* ``four_level``  - interferogram: H = diag(0, eps, 2 eps + 1.3, 3 eps + 0.7) + nearest-
                    neighbour couplings g_k ~ U(0.1, 1) (seed 0, six digits) + A cos(2 pi 0.3 t)
                    diag(0, 1, 2, 3); L = sqrt(0.005)|k-1><k| (k = 1..3), sqrt(0.01)|k><k|
                    (k = 0..3); O = |3><3|; RK4, 8000 steps on [0, 400]; 2048 x 2048 grid of
                    eps in [-5, 5] x A in [0, 5].
* ``duffing``     - x'' + 0.1 x' + x + x^3 = F cos(W t) as a first-order system; F in [0, 2],
                    W in [0.5, 2]; (x, x') ~ U(-1, 1)^2 (seed 0); t in [0, 500], 512 intervals.
* ``n_level``     - N-level scaling model (N in 8..64) with seeded GUE-like H0, swept
                    eps diag(0..N-1), drive A cos(t) X, N-1 lowering and N dephasing operators.
"""

from __future__ import annotations

import numpy as np
import sympy as sp


def _axis(lo, hi, full, side):
    """``side`` evenly strided samples of ``linspace(lo, hi, full)`` (the full axis when equal)."""
    values = np.linspace(lo, hi, full)
    if side is None or side >= full:
        return values
    idx = np.round(np.linspace(0, full - 1, side)).astype(int)
    return values[idx]


def two_level(side=None, full=64, steps=4000, duration=200.0):
    """The driven-qubit model of the module docstring on a ``full``-point axis pair (``side``: a
    strided subgrid of it)."""
    eps, A, Delta, Drive, t = sp.symbols("eps A Delta Drive t", real=True)
    sz = sp.Matrix([[1, 0], [0, -1]])
    sx = sp.Matrix([[0, 1], [1, 0]])
    sm = sp.Matrix([[0, 1], [0, 0]])
    H = eps / 2 * sz + Delta / 2 * sx + Drive * sz
    drive = A * sp.cos(2 * sp.pi * 0.5 * t)
    col = [sp.sqrt(0.01) * sm, sp.sqrt(0.02 / 2) * sz]
    return {"name": "two_level", "H": H, "Drive": drive, "Col_Ops": col, "mean_operator": sp.diag(0, 1),
            "tlist": np.linspace(0.0, duration, steps + 1),
            "var_arrays": {eps: _axis(-5.0, 5.0, full, side), A: _axis(0.0, 5.0, full, side)},
            "const_values": {Delta: 1.0}, "symbols": (eps, A), "N": 2,
            "omega": 2 * np.pi * 0.5}


def four_level_couplings(seed=0):
    """The three nearest-neighbour couplings of the four-level model, U(0.1, 1), six digits."""
    rng = np.random.default_rng(seed)
    return [round(float(g), 6) for g in rng.uniform(0.1, 1.0, 3)]


def four_level(side=None, steps=8000, duration=400.0, full=2048):
    """The four-level interferogram model of the module docstring (``side``: a strided subgrid
    of the ``full`` x ``full`` grid)."""
    eps, A, Drive, t = sp.symbols("eps A Drive t", real=True)
    g = four_level_couplings(0)
    H = sp.diag(0, eps, 2 * eps + sp.Float(1.3), 3 * eps + sp.Float(0.7)) + Drive * sp.diag(0, 1, 2, 3)
    for k, gk in enumerate(g):
        H[k, k + 1] = H[k, k + 1] + sp.Float(gk)
        H[k + 1, k] = H[k + 1, k] + sp.Float(gk)
    col = []
    for k in range(1, 4):
        L = sp.zeros(4)
        L[k - 1, k] = sp.sqrt(0.005)
        col.append(L)
    for k in range(4):
        L = sp.zeros(4)
        L[k, k] = sp.sqrt(0.01)
        col.append(L)
    O = sp.zeros(4)
    O[3, 3] = 1
    return {"name": "four_level", "H": H, "Drive": A * sp.cos(2 * sp.pi * 0.3 * t), "Col_Ops": col,
            "mean_operator": O, "tlist": np.linspace(0.0, duration, steps + 1),
            "var_arrays": {eps: _axis(-5.0, 5.0, full, side), A: _axis(0.0, 5.0, full, side)},
            "const_values": {}, "symbols": (eps, A), "N": 4, "couplings": g,
            "omega": 2 * np.pi * 0.3}


def duffing(side=None, full=1024, duration=500.0, intervals=512, seed=0):
    """The driven Duffing oscillator of the module docstring as an ``odesolve_2D`` workload."""
    x, v, t, F, W = sp.symbols("x v t F W", real=True)
    rhs = [v, -0.1 * v - x - x**3 + F * sp.cos(W * t)]
    Fs = _axis(0.0, 2.0, full, side)
    Ws = _axis(0.5, 2.0, full, side)
    rng = np.random.default_rng(seed)
    y0_full = rng.uniform(-1.0, 1.0, size=(full, full, 2))
    if side is not None and side < full:
        idx = np.round(np.linspace(0, full - 1, side)).astype(int)
        y0 = y0_full[np.ix_(idx, idx)]
    else:
        y0 = y0_full
    return {"name": "duffing", "rhs": rhs, "states": [x, v], "tlist": np.linspace(0.0, duration, intervals + 1),
            "var_arrays": {F: Fs, W: Ws}, "y0_values": y0, "symbols": (F, W), "gamma": 0.1, "beta": 1.0}


def n_level(N, side=64, steps=2000, duration=100.0, seed=0):
    """N-level scaling model; matrices are numeric (seeded) and returned with the SymPy model.

    eps spans [-0.5, 0.5]: the level spread eps (N-1) then stays below 32 at N = 64, so that
    the largest transition frequency times dt = 0.05 (about 2) lies inside RK4's stability
    interval on the imaginary axis (|omega dt| < 2.83); with eps in [-1, 1] RK4 diverges at N = 64.
    """
    eps, A, Drive, t = sp.symbols("eps A Drive t", real=True)
    rng = np.random.default_rng(seed + N)
    G = (rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))) / np.sqrt(2 * N)
    H0 = np.round((G + G.conj().T) / 2, 6)
    Xr = (rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))) / np.sqrt(2 * N)
    X = np.round((Xr + Xr.conj().T) / 2, 6)
    D = np.diag(np.arange(N, dtype=float))
    H = (sp.Matrix(H0.tolist()) + eps * sp.Matrix(D.tolist()) + Drive * sp.Matrix(X.tolist()))
    col = []
    for k in range(1, N):
        L = sp.zeros(N)
        L[k - 1, k] = sp.sqrt(0.01)
        col.append(L)
    for k in range(N):
        L = sp.zeros(N)
        L[k, k] = sp.sqrt(0.005)
        col.append(L)
    O = sp.zeros(N)
    O[N - 1, N - 1] = 1
    return {"name": f"n_level_{N}", "H": H, "Drive": A * sp.cos(t), "Col_Ops": col, "mean_operator": O,
            "tlist": np.linspace(0.0, duration, steps + 1),
            "var_arrays": {eps: np.linspace(-0.5, 0.5, side), A: np.linspace(0.0, 2.0, side)},
            "const_values": {}, "symbols": (eps, A), "N": N, "H0": H0, "X": X, "D": D,
            "lowering_rate": 0.01, "dephasing_rate": 0.005, "omega": 1.0}


# ---------------------------------------------------------------- serving and fit requests

SERVING_SIDES = (64, 128, 256, 512, 1024)  # grid sides of the mixed serving stream (64^2 .. 1024^2)


def serving_model(N, side):
    """(args, kwargs) of one ``mesolve_2D`` serving request: the Lindblad model of dimension N
    (two-level, four-level, or the N-level scaling model) on a side x side (eps, A) grid."""
    if N == 2:
        w = two_level()
    elif N == 4:
        w = four_level(full=side)
    else:
        w = n_level(N, side=side)
    eps, A = w["symbols"]
    var = {eps: np.linspace(float(np.min(w["var_arrays"][eps])), float(np.max(w["var_arrays"][eps])), side),
           A: np.linspace(float(np.min(w["var_arrays"][A])), float(np.max(w["var_arrays"][A])), side)}
    return ((w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"]),
            {"var_arrays": var, "const_values": w["const_values"]})


def qubit_fit_model(side=(8, 6), steps=400, duration=20.0):
    """Fit-request model: the two-level qubit with Gamma1, Gamma_phi and Delta kept as runtime
    constants (the parameters an interferogram fit adjusts; defaults 0.01, 0.02, 1.0) and drive
    A cos(pi t). Returns (args, kwargs, (Gamma1, Gamma_phi, Delta, A))."""
    eps, A, D, Drive, t, G1, Gp = sp.symbols("eps A Delta Drive t Gamma1 Gammaphi", real=True)
    sz, sx, sm = sp.Matrix([[1, 0], [0, -1]]), sp.Matrix([[0, 1], [1, 0]]), sp.Matrix([[0, 1], [0, 0]])
    H = eps / 2 * sz + D / 2 * sx + Drive * sz
    args = (H, A * sp.cos(sp.pi * t), [sp.sqrt(G1) * sm, sp.sqrt(Gp / 2) * sz], sp.diag(0, 1),
            np.linspace(0.0, duration, steps + 1))
    kwargs = {"var_arrays": {eps: np.linspace(-3.0, 3.0, side[0]), A: np.linspace(0.0, 2.0, side[1])},
              "runtime_consts": {G1: 0.01, Gp: 0.02, D: 1.0}}
    return args, kwargs, (G1, Gp, D, A)
