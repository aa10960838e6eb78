"""The C ABI on the CPU: header parsing, module build, exported symbols (no compute calls)."""

import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest
import sympy as sp

from gqis import abi, engine, solver
from gqis.cuda_solvers import available_solvers, get_solver_spec, normalize_solver_name

HEADER = Path(engine.INCLUDE_DIR) / "gqis_b200.h"


def _module_path():
    t, a, Drive = sp.symbols("t a Drive", real=True)
    return solver.prebuild("mesolve_2D", sp.Matrix([[a, Drive], [Drive, -a]]) / 2, sp.cos(t),
                           [sp.Matrix([[0, 0.1], [0, 0]])], sp.diag(0, 1), np.linspace(0, 1, 11),
                           var_arrays={a: np.linspace(-1, 1, 3)})


def test_header_declares_the_module_entry_points():
    declared = set(abi.header_symbols(HEADER.read_text()))
    assert set(abi.MODULE_SYMBOLS) <= declared


def test_model_module_builds_loads_and_exports_every_declared_symbol():
    path = _module_path()
    lib = ctypes.CDLL(str(path))  # loading needs no GPU; no entry point is called here
    for name in abi.header_symbols(HEADER.read_text()):
        if name in abi.MODULE_SYMBOLS:
            assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(abi.MODULE_SYMBOLS) <= exported
    assert not any(s.startswith("_ZN") and "gqfixed" in s for s in exported)  # templates stay hidden


def test_model_module_rejects_invalid_descriptors_before_any_cuda_call():
    """The descriptor check of ``gqis_sweep_launch`` runs before any CUDA call, and a zero-point launch
    returns before one too, so both are testable without a GPU."""
    lib = ctypes.CDLL(str(_module_path()))
    lib.gqis_last_error.restype = ctypes.c_char_p
    launch = lib.gqis_sweep_launch
    launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p]

    def desc(**kw):
        d = abi.SweepDesc(abi_version=abi.ABI_VERSION, num_x=3, num_y=1, num_steps=10, warmup_steps=0,
                          point_begin=0, point_count=0, dt=0.1, t_in=0.0)
        for k, v in kw.items():
            setattr(d, k, v)
        return d

    def rejects(d, text):
        assert launch(ctypes.byref(d), None) == 1
        assert text in lib.gqis_last_error(), lib.gqis_last_error()

    assert launch(None, None) == 1 and b"descriptor is NULL" in lib.gqis_last_error()
    assert lib.gqis_model_info_get(None) == 1
    rejects(desc(abi_version=abi.ABI_VERSION + 1), b"ABI version")
    rejects(desc(num_x=0), b"sweep axes must be non-empty")
    rejects(desc(point_begin=2, point_count=2), b"outside the 3-point grid")
    rejects(desc(num_steps=0), b"num_steps must be at least 1")
    rejects(desc(warmup_steps=11), b"warmup_steps must lie in")
    rejects(desc(warmup_steps=10), b"needs at least one step after warmup")
    rejects(desc(dt=0.0), b"dt must be positive")
    rejects(desc(dt=float("inf")), b"dt must be positive")
    rejects(desc(point_count=3), b"par_x, par_y and results are required")
    assert launch(ctypes.byref(desc()), None) == 0  # no points: nothing to launch


def test_adaptive_launch_rejects_more_points_than_its_work_counter_can_count():
    """The adaptive kernels hand out points from a 32-bit counter, so one launch takes at most
    2^31 - 1 points (a wrapped counter would never mark the grid exhausted). Both launches check
    this before any CUDA call, so it is testable without a GPU."""
    t, a, Drive = sp.symbols("t a Drive", real=True)
    path = solver.prebuild("mesolve_2D", sp.Matrix([[a, Drive], [Drive, -a]]) / 2, sp.cos(t),
                           [sp.Matrix([[0, 0.1], [0, 0]])], sp.diag(0, 1), np.linspace(0, 1, 11),
                           var_arrays={a: np.linspace(-1, 1, 3)}, solver="tsit5a", fp64=True)
    lib = ctypes.CDLL(str(path))
    abi.bind_module(lib)
    fake = 0x10000  # never dereferenced: the launch is refused first
    d = abi.SweepDesc(abi_version=abi.ABI_VERSION, num_x=65536, num_y=65536, num_steps=10, warmup_steps=0,
                      point_begin=0, point_count=1 << 32, dt=0.1, t_in=0.0, par_x=fake, par_y=fake,
                      results=fake, work_counter=fake)
    d.solver_params[0], d.solver_params[1], d.solver_params[2] = 1e-6, 1e-8, 64.0
    for launch in (lib.gqis_sweep_launch, lib.gqis_sweep_launch_noalloc):
        assert launch(ctypes.byref(d), None) == abi.ERR_TOO_LARGE
        assert b"exceed the maximum" in lib.gqis_last_error()
    d.point_count = (1 << 31) - 1  # at the limit the main launch passes the check and needs CUDA;
    d.num_x = 0                    # an invalid axis makes it stop at the descriptor check instead
    assert lib.gqis_sweep_launch(ctypes.byref(d), None) == abi.ERR_INVALID


def test_adjoint_scratch_size_and_modules_without_an_adjoint():
    """``gqis_adjoint_scratch_bytes`` is host arithmetic: (checkpoints + one interval of recomputed
    states) x S x points x 8 bytes; a module built without an adjoint answers GQIS_ERR_UNSUPPORTED."""
    lib = ctypes.CDLL(str(_module_path()))  # S = 3, no adjoint
    lib.gqis_last_error.restype = ctypes.c_char_p
    nbytes = ctypes.c_int64()
    assert lib.gqis_adjoint_scratch_bytes(ctypes.c_int64(1000), 4000, 64, ctypes.byref(nbytes)) == 0
    assert nbytes.value == (63 + 64) * 3 * 1000 * 8  # ceil(4000 / 64) = 63 checkpoints
    assert lib.gqis_adjoint_scratch_bytes(ctypes.c_int64(1000), 4000, 0, ctypes.byref(nbytes)) == 1
    assert lib.gqis_adjoint_scratch_bytes(ctypes.c_int64(-1), 4000, 64, ctypes.byref(nbytes)) == 1
    assert lib.gqis_adjoint_scratch_bytes(ctypes.c_int64(1), 4000, 64, None) == 1
    P, S = ctypes.c_int32(), ctypes.c_int32()
    assert lib.gqis_adjoint_info(ctypes.byref(P), ctypes.byref(S)) == 3
    assert lib.gqis_adjoint_launch(None, None) == 3 and b"without an adjoint" in lib.gqis_last_error()


def _struct_fields(text, name):
    import re
    body = text[text.index(f"typedef struct {name}"):text.index(f"}} {name};")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S).split("{", 1)[1]
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        decl = re.sub(r"\[\d+\]", "", decl)
        head, *rest = decl.split(",")
        fields.append(head.replace("*", " ").split()[-1])
        fields += [r.strip().lstrip("*") for r in rest]
    return fields


def test_descriptor_layout_matches_header_order():
    text = HEADER.read_text()
    assert _struct_fields(text, "gqis_sweep_desc") == [f for f, _ in abi.SweepDesc._fields_]
    assert _struct_fields(text, "gqis_model_info") == [f for f, _ in abi.ModelInfo._fields_]
    # The C compiler's layout (sizes and every offset) equals the ctypes mirror.
    prog = ['#include <stdio.h>', '#include <stddef.h>', '#include "gqis_b200.h"', "int main(void) {"]
    for struct, mirror in (("gqis_sweep_desc", abi.SweepDesc), ("gqis_model_info", abi.ModelInfo)):
        prog.append(f'printf("%zu\\n", sizeof({struct}));')
        prog += [f'printf("%zu\\n", offsetof({struct}, {f}));' for f, _ in mirror._fields_]
    prog.append("return 0; }")
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        src, exe = Path(tmp) / "layout.c", Path(tmp) / "layout"
        src.write_text("\n".join(prog))
        subprocess.run(["gcc", f"-I{HEADER.parent}", str(src), "-o", str(exe)], check=True)
        got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    want = []
    for mirror in (abi.SweepDesc, abi.ModelInfo):
        want.append(ctypes.sizeof(mirror))
        want += [getattr(mirror, f).offset for f, _ in mirror._fields_]
    assert got == want


def test_solver_names_and_aliases():
    assert available_solvers() == ("rk4", "lserk4", "lserk4f", "dp5", "ab5", "anas5", "tsit5", "alshina6",
                                   "dop853", "tsit5a", "dop853a")
    assert normalize_solver_name("RK45") == "dp5"
    assert normalize_solver_name("Anastassi-Simos") == "anas5"
    assert normalize_solver_name("DOP-853") == "dop853"
    assert normalize_solver_name("adaptive_dop853") == "dop853a"
    with pytest.raises(ValueError, match="Unsupported solver"):
        normalize_solver_name("not_a_solver")


def test_solver_orders_rhs_counts_and_tableaus():
    # steady-state RHS evaluations per step, FSAL reuse included (tests/test_cuda_solvers.py:35-42)
    assert get_solver_spec("rk4").rhs_evaluations == 4
    assert get_solver_spec("lserk4").rhs_evaluations == 5
    for name in ("dp5", "anas5", "tsit5"):
        assert get_solver_spec(name, step_size=0.1).rhs_evaluations == 6
    assert get_solver_spec("alshina6").rhs_evaluations == 7
    assert get_solver_spec("dop853").rhs_evaluations == 12
    assert get_solver_spec("ab5").rhs_evaluations == 1
    for name in ("dp5", "tsit5", "alshina6", "dop853"):
        t = get_solver_spec(name).tableau
        assert abs(sum(t.b) - 1.0) < 1e-12, name                     # consistency
        for i, row in enumerate(t.a):
            assert abs(sum(row) - t.c[i]) < 1e-10, (name, i)         # row sums = nodes
    anas = get_solver_spec("anas5", frequency=1.14, step_size=0.01)
    assert len(anas.parameters) == 1
    spec = get_solver_spec("tsit5a", step_size=0.1, adaptive_options={"step_rtol": 1e-6})
    assert spec.parameters[:3] == (1e-6, 1e-5, 64.0)
    with pytest.raises(ValueError, match="only to the adaptive solvers"):
        get_solver_spec("tsit5", step_size=0.1, adaptive_options={"step_rtol": 1e-6})
    with pytest.raises(ValueError, match="Unknown adaptive_options"):
        get_solver_spec("tsit5a", adaptive_options={"rtol": 1e-6})


@pytest.mark.parametrize("rhs_form,precision", [("matrix", "fp64"), ("matrix_tc", "fp32")])
def test_density_matrix_modules_export_the_module_entry_points(rhs_form, precision):
    """The density-matrix modules (CUDA-core and tcgen05) are model modules with the same C ABI."""
    from gqis import workloads
    w = workloads.n_level(16, side=2, steps=10, duration=1.0)
    path = solver.prebuild("mesolve_2D", w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"],
                           var_arrays=w["var_arrays"], precision=precision, rhs_form=rhs_form)
    lib = ctypes.CDLL(str(path))
    for name in ("gqis_model_info_get", "gqis_sweep_launch", "gqis_last_error", "gqis_sweep_launch_noalloc"):
        assert hasattr(lib, name), name
    src = Path(str(path).replace(".so", ".cu")).read_text()
    assert ("#define GQ_MATRIX 2" in src) == (rhs_form == "matrix_tc")


def test_module_cache_key_follows_the_callers_template_headers(tmp_path):
    """A module built with a caller's template directory (kernel_template_file) is rebuilt when a
    header there changes, and found again when it is restored."""
    from gqis import engine
    (tmp_path / "extra.cuh").write_text("#define GQIS_TEST_VALUE 1\n")
    src = '#include "extra.cuh"\nextern "C" int gqis_test_value(void) { return GQIS_TEST_VALUE; }\n'
    flags = (f"-I{tmp_path}",)
    first = engine.build_module(src, extra_flags=flags)
    (tmp_path / "extra.cuh").write_text("#define GQIS_TEST_VALUE 2\n")
    second = engine.build_module(src, extra_flags=flags)
    assert first != second
    (tmp_path / "extra.cuh").write_text("#define GQIS_TEST_VALUE 1\n")
    assert engine.build_module(src, extra_flags=flags) == first


def test_callers_template_directory_is_searched_before_the_packaged_headers(tmp_path):
    """kernel_template_file names a directory searched before the packaged CUDA templates: a header
    there with a packaged header's name replaces it in the build."""
    import ctypes
    from gqis import engine
    (tmp_path / "gqis_b200.h").write_text("#define GQIS_TEMPLATE_OVERRIDE 7\n")
    src = ('#include "gqis_b200.h"\n#ifndef GQIS_TEMPLATE_OVERRIDE\n#define GQIS_TEMPLATE_OVERRIDE 0\n#endif\n'
           'extern "C" __attribute__((visibility("default"))) int gqis_test_override(void) '
           '{ return GQIS_TEMPLATE_OVERRIDE; }\n')
    lib = ctypes.CDLL(str(engine.build_module(src, extra_flags=(f"-I{tmp_path}",))))
    assert lib.gqis_test_override() == 7
    lib = ctypes.CDLL(str(engine.build_module(src)))
    assert lib.gqis_test_override() == 0


def test_batch_launch_checks_its_arguments_before_any_cuda_call():
    """``gqis_sweep_launch_batch`` validates the batch size and every descriptor on the host; a
    density-matrix module answers GQIS_ERR_UNSUPPORTED."""
    lib = ctypes.CDLL(str(_module_path()))
    abi.bind_module(lib)
    d = abi.SweepDesc(abi_version=abi.ABI_VERSION, num_x=3, num_y=1, num_steps=10, warmup_steps=0,
                      point_begin=0, point_count=0, dt=0.1, t_in=0.0)
    descs = (abi.SweepDesc * (abi.BATCH_MAX + 1))(*([d] * (abi.BATCH_MAX + 1)))
    assert lib.gqis_sweep_launch_batch(descs, abi.BATCH_MAX + 1, None, None) == abi.ERR_TOO_LARGE
    assert lib.gqis_sweep_launch_batch(descs, 0, None, None) == abi.ERR_INVALID
    assert lib.gqis_sweep_launch_batch(None, 1, None, None) == abi.ERR_INVALID
    descs[2].num_x = 0
    assert lib.gqis_sweep_launch_batch(descs, 3, None, None) == abi.ERR_INVALID
    assert b"batch item 2: sweep axes must be non-empty" in lib.gqis_last_error()
    assert lib.gqis_sweep_launch_batch(descs, 2, None, None) == abi.OK  # no points: nothing to launch
    from gqis import workloads
    w = workloads.n_level(16, side=2, steps=10, duration=1.0)
    path = solver.prebuild("mesolve_2D", w["H"], w["Drive"], w["Col_Ops"], w["mean_operator"], w["tlist"],
                           var_arrays=w["var_arrays"], precision="fp64", rhs_form="matrix")
    mlib = ctypes.CDLL(str(path))
    abi.bind_module(mlib)
    assert mlib.gqis_sweep_launch_batch(descs, 1, None, None) == abi.ERR_UNSUPPORTED


def test_probe_library_exports_the_fma_and_tensor_core_probes():
    """The roofline denominators: FMA-pipe probes and the tcgen05 kind::tf32 / kind::f16 MMA probes
    (loading needs no GPU; nothing is called)."""
    from gqis import native
    lib = ctypes.CDLL(str(native.build("gqis_probe")))
    for name in ("gqis_probe_fma", "gqis_probe_tc_tf32", "gqis_probe_tc_f16"):
        assert hasattr(lib, name), name
