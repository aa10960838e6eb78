"""Print an optimised RHS plan as the C++ model struct consumed by the CUDA templates.

The struct exposes five device functions that ``csrc/gqis_sweep.cuh`` calls:

* ``statics``  once per parameter point, in FP64;
* ``drives``   once per stage time; FP64 time and phase, results stored in the form's type;
* ``rhs``      the reduced ODE, in the form's arithmetic type ``R``;
* ``observe``  the observable (real, imaginary), in ``R``;
* ``init``     symbolic initial state, in FP64.

Floating literals are printed with ten significant digits (``%.9e``), the convention of the
reference printer (``gqis/solver.py:158-199``): the plain FP64 form then evaluates exactly the
same numbers as the reference kernel, which the <=1e-10 parity target needs. Exact irrational
constants are evaluated before printing, squares print as products.
"""

from __future__ import annotations

import hashlib
import re

import sympy as sp
from sympy.printing.c import C99CodePrinter
from sympy.printing.precedence import PRECEDENCE

_MATH = ("sqrt", "cbrt", "sin", "cos", "tan", "asin", "acos", "atan", "atan2", "sinh", "cosh",
         "tanh", "asinh", "acosh", "atanh", "exp", "expm1", "log", "log1p", "log10", "log2",
         "pow", "fabs", "floor", "ceil", "fmax", "fmin", "erf", "erfc", "tgamma", "lgamma", "hypot")
_PHASED = ("sin", "cos", "tan")  # periodic functions evaluated through the form's phase reduction
_MATH_CALL = re.compile(r"(?<![\w:.])(" + "|".join(_MATH) + r")\(")


PHASE_OPEN, PHASE_CLOSE = "\x01", "\x02"  # marks the FP64 argument of a periodic drive function


class _ModelPrinter(C99CodePrinter):
    """C99 printer with ten-digit literals; ``cast=True`` wraps literals as ``R(...)``.

    With ``phased=True`` the argument of ``sin``/``cos``/``tan`` is printed in FP64 (plain
    literals) between the phase markers; ``_phase_names`` later points the symbols inside the
    markers to their FP64 copies.
    """

    def __init__(self, cast, phased=False):
        super().__init__()
        self._cast = cast
        self._phased = phased

    def _print_Function(self, expr):
        name = expr.func.__name__
        if self._phased and name in _PHASED and len(expr.args) == 1:
            inner = _ModelPrinter(cast=False).doprint(expr.args[0])
            return f"{name}({PHASE_OPEN}{inner}{PHASE_CLOSE})"
        return super()._print_Function(expr)

    def _print_sin(self, expr):
        return self._print_Function(expr)

    def _print_cos(self, expr):
        return self._print_Function(expr)

    def _print_tan(self, expr):
        return self._print_Function(expr)

    def _lit(self, text):
        return f"R({text})" if self._cast else text

    def _print_Float(self, expr):
        return self._lit(f"{float(expr):.9e}")

    def _print_Rational(self, expr):
        return self._lit(f"{int(expr.p)}.0/{int(expr.q)}.0")

    def _print_Pow(self, expr):
        base, exp = expr.base, expr.exp
        if exp == 2:
            b = self.parenthesize(base, PRECEDENCE["Mul"])
            return f"({b}*{b})"
        if exp.is_Integer and 3 <= int(exp) <= 8:
            return f"gq::ipow<{int(exp)}>({self._print(base)})"
        if exp == -1:
            return f"{self._lit('1.0')}/{self.parenthesize(base, PRECEDENCE['Mul'])}"
        if exp == sp.Rational(1, 2):
            return f"sqrt({self._print(base)})"
        if exp == sp.Rational(-1, 2):
            return f"{self._lit('1.0')}/sqrt({self._print(base)})"
        return f"pow({self._print(base)}, {self._print(exp)})"


def _evaluate_constants(expr):
    """Replace exact irrational numbers (pi, E, sqrt(2) ...) by Floats before printing."""
    if not isinstance(expr, sp.Basic):
        return expr
    found = {}
    walk = sp.preorder_traversal(expr)
    for sub in walk:
        if sub.is_number and not (sub.is_Rational or sub.is_Float) and sub.is_real:
            found[sub] = sub.evalf()
            walk.skip()
    return expr.xreplace(found) if found else expr


def ccode(expr, *, cast=True, phased=False):
    """Print one expression for the model struct.

    ``cast``: literals become ``R(...)`` (arithmetic in the form's type); otherwise they stay
    FP64. ``phased``: ``sin/cos/tan`` go through ``F::`` (the form's phase-reduced versions) and
    their arguments are FP64 (see ``_phase_names``).
    """
    text = _ModelPrinter(cast, phased).doprint(_evaluate_constants(sp.sympify(expr)))

    def repl(m):
        name = m.group(1)
        return f"F::{name}(" if phased and name in _PHASED else f"gq::{name}("
    return _MATH_CALL.sub(repl, text)


def _fp64_names(line):
    """A drive line evaluated entirely in FP64: FP64 copies of every input, results in ``Dd``.

    Rounding a sweep parameter to FP32 before it enters a drive (``eps + A cos(w t)``) shifts
    the model by a fixed amount at every step, a systematic error that reached 1.5e-6 at sharp
    resonances of the four-level map; evaluated in FP64 and rounded once per stage time, the
    drive's rounding varies in time and averages out (5e-8 there).
    """
    line = line.replace(PHASE_OPEN, "").replace(PHASE_CLOSE, "")
    line = re.sub(r"(?<![\w])ParX(?![\w])", "ParXd", line)
    line = re.sub(r"(?<![\w])ParY(?![\w])", "ParYd", line)
    line = line.replace("Static_arr[", "Static_d[").replace("Const_arr[", "Const_d[")
    return line.replace("Drive_arr[", "Dd[")


def _word(name):
    return re.compile(r"(?<![0-9A-Za-z_])" + re.escape(name) + r"(?![0-9A-Za-z_])")


def _substitute(text, table):
    for name, repl in table:
        if repl is not None:
            text = _word(name).sub(lambda _m, r=repl: r, text)
    return text


def emit_model(compiled, uses_rho0_values):
    """Model fragments of a :class:`~gqis.rhs.CompiledRHS`.

    Returns a dict with the C++ bodies of the five model functions, the array sizes and the
    ``Const_arr`` indices the code reads (unused runtime constants are removed and the rest
    renumbered, as ``gqis/solver.py:1649-1692`` does).
    """
    plan = compiled.plan
    drive_syms, func_temps, drive_exprs = plan["drive_plan"]
    names = {str(s): f"Drive_arr[{k}]" for k, s in enumerate(drive_syms)}
    static_lines, drive_lines = [], []
    n_static = 0
    n_drive = len(drive_syms)

    # Functions of time alone (cos(w t), with runtime constants at most) are the same for every
    # point: they become Tf[k], which the RK4 kernel evaluates once per warp for a block of steps.
    uniform = {str(x) for x in plan.get("runtime_const_syms", ())} | {"t"}
    time_funcs = {}

    def factor_time(e):
        found = {}
        walk = sp.preorder_traversal(sp.sympify(e))
        for sub in walk:
            if isinstance(sub, sp.Function) and sub.free_symbols \
                    and {str(x) for x in sub.free_symbols} <= uniform and "t" in {str(x) for x in sub.free_symbols}:
                k = time_funcs.setdefault(sub, len(time_funcs))
                found[sub] = sp.Symbol(f"GQTF{k}")
                walk.skip()
        return sp.sympify(e).xreplace(found) if found else e

    drive_lines += [f"const double {s} = {ccode(factor_time(f), cast=False, phased=True)};" for s, f in func_temps]
    drive_lines += [f"Drive_arr[{k}] = {ccode(factor_time(e), cast=False, phased=True)};"
                    for k, e in enumerate(drive_exprs)]

    def bind(s, e, level):
        nonlocal n_static, n_drive
        if level == "static":
            line = f"Static_arr[{n_static}] = {ccode(e, cast=False)};"
            static_lines.append(_substitute(line, list(names.items())))
            names[str(s)] = f"Static_arr[{n_static}]"
            n_static += 1
        else:
            line = f"Drive_arr[{n_drive}] = {ccode(factor_time(e), cast=False, phased=True)};"
            drive_lines.append(_substitute(line, list(names.items())))
            names[str(s)] = f"Drive_arr[{n_drive}]"
            n_drive += 1

    inline_consts = {}
    for s, e, level in plan["hoists"]:
        if level == "negate":
            target = names[str(e.as_coeff_Mul()[1])]
            names[str(s)] = target[1:] if target.startswith("-") else "-" + target
        elif level == "inline":
            inline_consts[str(s)] = e
            names[str(s)] = None  # printed per use in the precision of the using line
        else:
            bind(s, e, level)
    for s, e, level in plan["mean_hoists"]:
        bind(s, e, level)

    rhs_lines = []
    for scoped, temps, outputs in plan["blocks"]:
        if scoped:
            rhs_lines.append("{")
        rhs_lines += [f"const R {s} = {ccode(e)};" for s, e in temps]
        rhs_lines += [f"d_rho[{k}] = {ccode(e)};" for k, e in outputs]
        if scoped:
            rhs_lines.append("}")
    obs_re = ccode(plan["mean_exprs"][0])
    obs_im = ccode(plan["mean_exprs"][1])

    size = compiled.state_size
    if uses_rho0_values:
        init_lines = []  # the template reads Rho0_arr
    elif compiled.rho0_exprs is None:
        init_lines = [f"rho[{k}] = {1.0 if k == 0 else 0.0};" for k in range(size)]
    else:
        init_lines = [f"rho[{k}] = {ccode(e, cast=False)};" for k, e in enumerate(compiled.rho0_exprs)]

    const_names = [(str(sym), f"Const_arr[{k}]") for k, sym in enumerate(plan["runtime_const_syms"])]

    def finish(lines, cast):
        out = []
        for line in lines:
            for name, e in reversed(list(inline_consts.items())):  # later ones may use earlier ones
                line = _word(name).sub(lambda _m, e=e: f"({ccode(e, cast=cast)})", line)
            line = _substitute(line, [(k, v) for k, v in names.items() if v is not None])
            out.append(_substitute(line, const_names))
        return out

    static_lines = finish(static_lines, False)
    drive_lines = [_fp64_names(ln) for ln in finish(drive_lines, False)]
    tf_names = [(f"GQTF{k}", f"Tf[{k}]") for k in range(len(time_funcs))]
    drive_lines = [_substitute(ln, tf_names) for ln in drive_lines]
    funcs = sorted(time_funcs, key=time_funcs.get)
    time_inline = [_fp64_names(ln) for ln in finish([f"Tf[{k}] = {ccode(f, cast=False, phased=True)};"
                                                     for k, f in enumerate(funcs)], False)]
    time_exact = [_fp64_names(ln) for ln in finish(
        [f"Tf[{k}] = {ccode(f, cast=False)};" for k, f in enumerate(funcs)], False)]
    rhs_lines = finish(rhs_lines, True)
    init_lines = finish(init_lines, False)
    obs_re, obs_im = finish([obs_re, obs_im], True)

    # drive and time lines read the FP64 copies (Const_d), the others Const_arr: both count and both
    # are renumbered
    used = sorted({int(m) for part in (static_lines, drive_lines, rhs_lines, init_lines, [obs_re, obs_im],
                                       time_inline, time_exact)
                   for line in part for m in re.findall(r"Const_(?:arr|d)\[(\d+)\]", line)})
    if used and used != list(range(len(plan["runtime_const_syms"]))):
        remap = {old: new for new, old in enumerate(used)}

        def renumber(line):
            return re.sub(r"Const_(arr|d)\[(\d+)\]",
                          lambda m: f"Const_{m.group(1)}[{remap[int(m.group(2))]}]", line)
        static_lines, drive_lines, rhs_lines, init_lines, time_inline, time_exact = (
            [renumber(x) for x in part]
            for part in (static_lines, drive_lines, rhs_lines, init_lines, time_inline, time_exact))
        obs_re, obs_im = renumber(obs_re), renumber(obs_im)

    return {"state_size": size, "n_static": max(1, n_static), "n_drive": max(1, n_drive),
            "n_drive_used": n_drive,
            "n_const": max(1, len(used)), "used_const_indices": tuple(used),
            "static_lines": tuple(static_lines), "drive_lines": tuple(drive_lines),
            "rhs_lines": tuple(rhs_lines), "obs_re": obs_re, "obs_im": obs_im,
            "init_lines": tuple(init_lines), "uses_rho0_values": bool(uses_rho0_values),
            "n_time_funcs": len(time_funcs), "time_lines_inline": tuple(time_inline),
            "time_lines_exact": tuple(time_exact),
            "has_time": any(re.search(r"(?<![\w])t(?![\w])", ln) for ln in drive_lines)}


def model_source(frag, struct_name="Model"):
    """C++ text of the model struct for the fragments of :func:`emit_model`."""
    def body(lines, indent="        "):
        return "\n".join(indent + ln for ln in lines) if lines else indent + "/* none */"

    return f"""struct {struct_name} {{
    static constexpr int S = {frag['state_size']};
    static constexpr int NSTAT = {frag['n_static']};
    static constexpr int NDRV = {frag['n_drive']};
    static constexpr int NCONST = {frag['n_const']};
    static constexpr int NTF = {frag.get('n_time_funcs', 0)};
    static constexpr bool kInitFromArray = {'true' if frag['uses_rho0_values'] else 'false'};

    __device__ __forceinline__ static void statics(double ParX, double ParY, double* __restrict__ Static_arr,
                                                   const double* __restrict__ Const_arr) {{
        (void)ParX; (void)ParY; (void)Static_arr; (void)Const_arr;
{body(frag['static_lines'])}
    }}

    // the functions of time alone at time t, in FP64 (one evaluation serves every point)
    __device__ __forceinline__ static void time_funcs(double t, const double* __restrict__ Const_d,
                                                      double* __restrict__ Tf) {{
        (void)t; (void)Const_d; (void)Tf;
{body(frag.get('time_lines_exact', ()))}
    }}

    template <class F>
    __device__ __forceinline__ static void drives(double ParXd, double ParYd, double t,
                                                  typename F::real ParX, typename F::real ParY,
                                                  typename F::real* __restrict__ Drive_arr,
                                                  const double* __restrict__ Static_d,
                                                  const typename F::real* __restrict__ Static_arr,
                                                  const double* __restrict__ Const_d,
                                                  const typename F::real* __restrict__ Const_arr) {{
        double Tf[NTF > 0 ? NTF : 1];
        (void)Tf;
{body(frag.get('time_lines_inline', ()))}
        drives_tf<F>(ParXd, ParYd, t, ParX, ParY, Drive_arr, Static_d, Static_arr, Const_d, Const_arr, Tf);
    }}

    // drives with the functions of time given (Tf, from time_funcs)
    template <class F>
    __device__ __forceinline__ static void drives_tf(double ParXd, double ParYd, double t,
                                                     typename F::real ParX, typename F::real ParY,
                                                     typename F::real* __restrict__ Drive_arr,
                                                     const double* __restrict__ Static_d,
                                                     const typename F::real* __restrict__ Static_arr,
                                                     const double* __restrict__ Const_d,
                                                     const typename F::real* __restrict__ Const_arr,
                                                     const double* __restrict__ Tf) {{
        using R = typename F::real;
        (void)ParXd; (void)ParYd; (void)ParX; (void)ParY; (void)t; (void)Drive_arr;
        (void)Static_d; (void)Static_arr; (void)Const_d; (void)Const_arr; (void)Tf;
        double Dd[NDRV];
        (void)Dd;
{body(frag['drive_lines'])}
#pragma unroll
        for (int k = 0; k < {frag['n_drive_used']}; ++k) Drive_arr[k] = (R)Dd[k];
    }}

    template <class R>
    __device__ __forceinline__ static void rhs(const R* __restrict__ rho, R ParX, R ParY,
                                               const R* __restrict__ Drive_arr,
                                               const R* __restrict__ Static_arr, R* __restrict__ d_rho,
                                               const R* __restrict__ Const_arr) {{
        (void)ParX; (void)ParY; (void)Drive_arr; (void)Static_arr; (void)Const_arr;
{body(frag['rhs_lines'])}
    }}

    template <class R>
    __device__ __forceinline__ static void observe(const R* __restrict__ rho, R ParX, R ParY,
                                                   const R* __restrict__ Drive_arr,
                                                   const R* __restrict__ Static_arr,
                                                   const R* __restrict__ Const_arr, R& re, R& im) {{
        (void)rho; (void)ParX; (void)ParY; (void)Drive_arr; (void)Static_arr; (void)Const_arr;
        re = {frag['obs_re']};
        im = {frag['obs_im']};
    }}

    __device__ __forceinline__ static void init(double* __restrict__ rho, double ParX, double ParY,
                                                const double* __restrict__ Const_arr) {{
        (void)rho; (void)ParX; (void)ParY; (void)Const_arr;
{body(frag['init_lines'])}
    }}
}};
"""


def fragments_digest(frag):
    """Stable hash of the emitted model text (part of the module cache key)."""
    return hashlib.sha256(model_source(frag).encode()).hexdigest()[:16]


def _count_ops(lines):
    n = 0
    for line in lines:
        if "=" not in line:
            continue
        expr = line.split("=", 1)[1]
        expr = re.sub(r"\[[0-9]+\]", "", expr)
        expr = re.sub(r"R\(([^()]*)\)", "c", expr)
        expr = re.sub(r"\d+\.\d*e[+-]\d+", "c", expr)
        expr = re.sub(r"(^|[=(,*/+-])\s*-", r"\1", expr)
        n += len(re.findall(r"[+\-*/]", expr))
    return n


def count_drive_flops(frag):
    """Arithmetic operators of one ``drives`` call (sin/cos calls not included)."""
    return _count_ops(frag["drive_lines"])


def count_rhs_flops(frag):
    """Floating-point operations of one ``rhs`` call, counted from the emitted lines.

    Every binary ``+ - *`` and ``/`` counts one, an ``FMA``-contractible pair counts two as
    well (so the count equals the number of arithmetic operators); unary minus on a literal or
    an array element and integer indexing are not counted. Used for the roofline.
    """
    n = 0
    for line in frag["rhs_lines"]:
        if "=" not in line:
            continue
        expr = line.split("=", 1)[1]
        expr = re.sub(r"\[[0-9]+\]", "", expr)            # array indices
        expr = re.sub(r"R\(([^()]*)\)", "c", expr)        # literals
        expr = re.sub(r"\d+\.\d*e[+-]\d+", "c", expr)
        expr = re.sub(r"(^|[=(,*/+-])\s*-", r"\1", expr)  # unary minus
        n += len(re.findall(r"[+\-*/]", expr))
    return n
