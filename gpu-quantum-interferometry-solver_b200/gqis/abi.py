"""ctypes mirror of ``include/gqis_b200.h`` (structures, constants and error handling)."""

from __future__ import annotations

import ctypes

ABI_VERSION = 1
OK, ERR_INVALID, ERR_CUDA, ERR_UNSUPPORTED, ERR_TOO_LARGE, ERR_CANCELLED, ERR_TIMEOUT, ERR_BUSY = range(8)


class GqisError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code, message):
        super().__init__(f"gqis status {code}: {message}")
        self.code = code


class ModelInfo(ctypes.Structure):
    _fields_ = [("abi_version", ctypes.c_int32), ("state_size", ctypes.c_int32),
                ("num_consts", ctypes.c_int32), ("form", ctypes.c_int32), ("solver", ctypes.c_int32),
                ("output_mode", ctypes.c_int32), ("trace_mode", ctypes.c_int32),
                ("init_from_array", ctypes.c_int32), ("block_threads", ctypes.c_int32),
                ("registers_per_thread", ctypes.c_int32), ("sm_count", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("model_hash", ctypes.c_uint64)]


class SweepDesc(ctypes.Structure):
    _fields_ = [("abi_version", ctypes.c_int32), ("num_x", ctypes.c_int32), ("num_y", ctypes.c_int32),
                ("num_steps", ctypes.c_int32), ("warmup_steps", ctypes.c_int32),
                ("trace_stride", ctypes.c_int32), ("trace_offset", ctypes.c_int32),
                ("num_trace", ctypes.c_int32), ("point_begin", ctypes.c_int64),
                ("point_count", ctypes.c_int64), ("dt", ctypes.c_double), ("t_in", ctypes.c_double),
                ("par_x", ctypes.c_void_p), ("par_y", ctypes.c_void_p), ("consts", ctypes.c_void_p),
                ("rho0", ctypes.c_void_p), ("results", ctypes.c_void_p), ("trace", ctypes.c_void_p),
                ("step_counts", ctypes.c_void_p), ("work_counter", ctypes.c_void_p),
                ("solver_params", ctypes.c_double * 8)]


class AdjointDesc(ctypes.Structure):
    _fields_ = [("sweep", SweepDesc), ("num_params", ctypes.c_int32), ("checkpoint_every", ctypes.c_int32),
                ("adjoint_consts", ctypes.c_void_p), ("grad", ctypes.c_void_p), ("scratch", ctypes.c_void_p),
                ("scratch_bytes", ctypes.c_int64)]


BATCH_MAX = 64  # GQIS_BATCH_MAX

MODULE_SYMBOLS = ("gqis_model_info_get", "gqis_sweep_launch", "gqis_last_error", "gqis_sweep_launch_noalloc",
                  "gqis_sweep_launch_batch",
                  "gqis_adjoint_info", "gqis_adjoint_scratch_bytes", "gqis_adjoint_launch")


def bind_module(lib):
    """Declare argument and return types of a model module's entry points."""
    lib.gqis_model_info_get.argtypes = [ctypes.POINTER(ModelInfo)]
    lib.gqis_model_info_get.restype = ctypes.c_int
    lib.gqis_sweep_launch.argtypes = [ctypes.POINTER(SweepDesc), ctypes.c_void_p]
    lib.gqis_sweep_launch.restype = ctypes.c_int
    lib.gqis_sweep_launch_noalloc.argtypes = [ctypes.POINTER(SweepDesc), ctypes.c_void_p]
    lib.gqis_sweep_launch_noalloc.restype = ctypes.c_int
    lib.gqis_sweep_launch_batch.argtypes = [ctypes.POINTER(SweepDesc), ctypes.c_int32, ctypes.c_void_p,
                                            ctypes.c_void_p]
    lib.gqis_sweep_launch_batch.restype = ctypes.c_int
    lib.gqis_adjoint_info.argtypes = [ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    lib.gqis_adjoint_info.restype = ctypes.c_int
    lib.gqis_adjoint_scratch_bytes.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                               ctypes.POINTER(ctypes.c_int64)]
    lib.gqis_adjoint_scratch_bytes.restype = ctypes.c_int
    lib.gqis_adjoint_launch.argtypes = [ctypes.POINTER(AdjointDesc), ctypes.c_void_p]
    lib.gqis_adjoint_launch.restype = ctypes.c_int
    lib.gqis_last_error.argtypes = []
    lib.gqis_last_error.restype = ctypes.c_char_p


def check(rc, lib):
    if rc != OK:
        msg = lib.gqis_last_error()
        raise GqisError(rc, msg.decode(errors="replace") if msg else "")


def header_symbols(header_text):
    """Function names declared in a C header (``type name(args);`` lines)."""
    import re
    body = re.sub(r"/\*.*?\*/", "", header_text, flags=re.S)
    return re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(gqis_\w+)\s*\(", body, flags=re.M)
