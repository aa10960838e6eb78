"""CPU tests of the symbolic front end (no GPU): layout, Lindblad equations, emission, options."""

import numpy as np
import pytest
import sympy as sp

from gqis import build_independent_rho, build_reduced_lindblad_rhs, compile_lindblad_rhs
from gqis import emit, rhs as rhs_mod
from gqis._options import OPTION_GROUPS, apply_option_groups


def test_independent_density_matrix_layout():
    rho, meta = build_independent_rho(3)
    assert rho.shape == (3, 3)
    assert len(meta["rho_syms"]) == 8
    assert meta["num_coherences"] == 3
    assert sp.simplify(sp.trace(rho) - 1) == 0
    # Hermitian by construction
    assert sp.simplify(rho - rho.H) == sp.zeros(3)


def test_reduced_lindblad_rhs_matches_two_level_bloch_equations():
    delta, drive, g1, g2 = sp.symbols("delta drive gamma1 gamma2", real=True, nonnegative=True)
    sx, sz, sm = sp.Matrix([[0, 1], [1, 0]]), sp.Matrix([[1, 0], [0, -1]]), sp.Matrix([[0, 1], [0, 0]])
    eqs, mean_re, mean_im, meta = build_reduced_lindblad_rhs(
        2, delta * sx / 2 + drive * sz / 2, [sp.sqrt(g1) * sm, sp.sqrt(g2) * sz], sp.diag(0, 1))
    r00, r01re, r01im = meta["rho_syms"]
    decay = g1 / 2 + 2 * g2
    expected = [g1 * (1 - r00) - delta * r01im,
                drive * r01im - decay * r01re,
                delta * (r00 - sp.Rational(1, 2)) - drive * r01re - decay * r01im]
    assert all(sp.simplify(a - b) == 0 for a, b in zip(eqs, expected))
    assert sp.simplify(mean_re - (1 - r00)) == 0 and mean_im == 0


def test_emitted_literals_use_ten_significant_digits():
    eps, A, t, Drive = sp.symbols("eps A t Drive", real=True)
    c = compile_lindblad_rhs(eps / 2 * sp.Matrix([[1, 0], [0, -1]]) + Drive * sp.Matrix([[0, 1], [1, 0]]),
                             A * sp.cos(sp.pi * t), [sp.sqrt(0.01) * sp.Matrix([[0, 1], [0, 0]])],
                             sp.diag(0, 1), [eps, A], RHSreuse=False)
    frag = emit.emit_model(c, False)
    # cos(pi t) depends on time alone: it is a time function Tf[0], printed for the per-point drives
    # (phase-reduced, F::cos) and for the per-warp table (FP64)
    assert frag["n_time_funcs"] == 1 and any("Tf[0]" in ln for ln in frag["drive_lines"])
    assert any("3.141592654e+00" in ln and "F::cos(" in ln for ln in frag["time_lines_inline"])
    assert any("3.141592654e+00" in ln and "gq::cos(" in ln for ln in frag["time_lines_exact"])
    lines = frag["drive_lines"] + frag["rhs_lines"] + frag["time_lines_inline"] + frag["time_lines_exact"]
    assert all("M_PI" not in ln for ln in lines)
    assert frag["state_size"] == 3


def test_option_groups_merge_and_reject_conflicts():
    def f(a=1, fp64=False, solver="rk4"):
        return a
    args = {"a": 1, "fp64": False, "solver": "rk4"}
    merged, _ = apply_option_groups(f, dict(args), {"solver_options": {"fp64": True}})
    assert merged["fp64"] is True
    with pytest.raises(ValueError, match="both directly"):
        apply_option_groups(f, dict(args, fp64=True), {"solver_options": {"fp64": False}})
    with pytest.raises(ValueError, match="Unknown codegen option"):
        apply_option_groups(f, dict(args), {"codegen": {"fp64": True}})
    assert "precision" in OPTION_GROUPS["solver_options"]


def test_api_reference_documents_every_parameter():
    """After the reference's tests/test_package.py:42-46: the API reference names every parameter of
    both entry points."""
    import inspect
    from pathlib import Path

    from gqis import mesolve_2D, odesolve_2D
    doc = (Path(__file__).resolve().parents[1] / "API.md").read_text(encoding="utf-8")
    for func in (mesolve_2D, odesolve_2D):
        missing = [name for name in inspect.signature(func).parameters if f"`{name}`" not in doc]
        assert missing == [], (func.__name__, missing)


def test_package_import_needs_no_cupy_or_triton():
    """After the reference's tests/test_package.py:15-39 (import without CuPy): the package and every
    submodule import in a fresh process without a GPU, and load neither CuPy nor Triton."""
    import subprocess
    import sys
    from pathlib import Path

    pkg = Path(__file__).resolve().parents[1] / "gpu-quantum-interferometry-solver_b200"
    code = ("import sys; sys.path.insert(0, %r)\n"
            "import gqis, gqis.solver, gqis.serving, gqis.adjoint, gqis.render, gqis.shard, gqis.matrix_form\n"
            "bad = sorted(m for m in sys.modules if m.split('.')[0] in ('cupy', 'triton'))\n"
            "assert not bad, bad\n") % str(pkg)
    proc = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr[-2000:]


def test_rabi_rhs_at_the_ground_state():
    """After the reference's environment check (gqis/check_environment.py:284-293): for
    H = (A/2) sigma_x at rho = |0><0|, d rho/dt = -i[H, rho] has Im(rho_01)' = A/2 and the rest 0."""
    from gqis import compile_lindblad_rhs
    A, dummy, Drive = sp.symbols("A dummy Drive", real=True)
    rhs = compile_lindblad_rhs(Drive / 2 * sp.Matrix([[0, 1], [1, 0]]), A, [], sp.diag(0, 1), [A, dummy])
    assert rhs.state_size == 3 and len(rhs.equations) == 3
    at_ground = dict(zip(rhs.state_symbols, (1, 0, 0)))
    drive = rhs.drive_map[Drive] if isinstance(rhs.drive_map, dict) else rhs.drive_map
    values = [float(sp.sympify(e).subs(Drive, drive).subs({**at_ground, sp.Symbol("ParX", real=True): 2.0}))
              for e in rhs.equations]
    np.testing.assert_allclose(values, [0.0, 0.0, 1.0], atol=1e-12)
