"""Python side of the C ODE oracle (``ode_oracle.c``): Duffing sweeps on the CPU in FP64.

Oracle infrastructure only. The Tsit5 tableau is Tsitouras (2011); the DOP853 tableau and
error weights come from SciPy's published implementation (an independent source of the same
table). ``sweep(method, F, W, y0, tlist, ...)`` returns ``(final, trace, counts)`` with the
shapes of ``odesolve_2D``: final (nF, nW, 2), trace (nF, nW, n_intervals, 2).
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libode_oracle.so"

TSIT5_C = [0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0]
TSIT5_A = [[0.161],
           [-0.008480655492356989, 0.335480655492357],
           [2.897153057105493, -6.359448489975075, 4.3622954328695815],
           [5.325864828439257, -11.748883564062828, 7.4955393428898365, -0.09249506636175525],
           [5.86145544294642, -12.92096931784711, 8.159367898576159, -0.071584973281401, -0.028269050394068383]]
TSIT5_B = [0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081,
           2.324710524099774]
TSIT5_E = [-0.00178001105222577714, -0.0008164344596567469, 0.007880878010261995, -0.1447110071732629,
           0.5823571654525552, -0.45808210592918697, 0.015151515151515152]

METHODS = {"rk4": 0, "tsit5a": 1, "dop853a": 2}
MODELS = {"duffing": 0, "decay_ramp": 1}


def build():
    LIB.parent.mkdir(exist_ok=True)
    subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-ffp-contract=off", "-o", str(LIB),
                    str(HERE / "ode_oracle.c"), "-lm"], check=True)


def _lib():
    if not LIB.exists():
        build()
    lib = ctypes.CDLL(str(LIB))
    dp = ctypes.POINTER(ctypes.c_double)
    lib.oracle_sweep.argtypes = [ctypes.c_int] * 5 + [dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                      ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                                      dp, dp, dp, dp, dp, dp, dp, ctypes.POINTER(ctypes.c_int)]
    lib.oracle_sweep.restype = ctypes.c_int
    return lib


def _tableau(method):
    if method == "tsit5a":
        ns = 6
        a = np.zeros((ns, ns))
        for i, row in enumerate(TSIT5_A, start=1):
            a[i, :len(row)] = row
        return ns, np.array(TSIT5_C), a, np.array(TSIT5_B), np.array(TSIT5_E), np.zeros(ns)
    if method == "dop853a":
        from scipy.integrate._ivp import dop853_coefficients as dc
        ns = dc.N_STAGES
        return ns, dc.C[:ns].copy(), dc.A[:ns, :ns].copy(), dc.B.copy(), dc.E5[:ns].copy(), dc.E3[:ns].copy()
    z = np.zeros(1)
    return 1, z, z, z, z, z


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def sweep(method, F, W, y0, tlist, *, model="duffing", gamma=0.1, beta=1.0, t_in=0.0, rtol=1e-8, atol=1e-10,
          max_substeps=4000, want_trace=True):
    F, W = np.asarray(F, float), np.asarray(W, float)
    nF, nW = len(F), len(W)
    FF, WW = np.meshgrid(F, W, indexing="ij")
    params = np.ascontiguousarray(np.stack([np.full(FF.size, gamma), np.full(FF.size, beta), FF.ravel(),
                                            WW.ravel()], axis=1))
    y0 = np.ascontiguousarray(np.asarray(y0, float).reshape(nF * nW, 2))
    tlist = np.asarray(tlist, float)
    nsteps = len(tlist) - 1
    dt = float((tlist[-1] - tlist[0]) / nsteps)
    ns, c, a, b, e, e3 = (np.ascontiguousarray(x, dtype=float) if isinstance(x, np.ndarray) else x
                          for x in _tableau(method))
    final = np.zeros((nF * nW, 2))
    trace = np.zeros((nF * nW, nsteps, 2)) if want_trace else None
    counts = np.zeros((nF * nW, 2), dtype=np.int32)
    rc = _lib().oracle_sweep(METHODS[method], MODELS[model], 2, 4, nF * nW, _ptr(params), _ptr(y0), float(t_in), dt,
                             nsteps, float(rtol), float(atol), int(max_substeps), int(ns), _ptr(c), _ptr(a.ravel()),
                             _ptr(b), _ptr(e), _ptr(e3), _ptr(final),
                             _ptr(trace) if trace is not None else None,
                             counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != 0:
        raise RuntimeError("oracle_sweep rejected its arguments")
    return (final.reshape(nF, nW, 2), None if trace is None else trace.reshape(nF, nW, nsteps, 2),
            counts.reshape(nF, nW, 2))
