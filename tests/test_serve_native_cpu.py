"""The native sweep server's C ABI on the CPU: the library builds, loads and exports every function
include/gqis_serve.h declares, and rejects invalid arguments (the only calls made: a running server
needs a GPU)."""

import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_serve_library_exports_the_header_symbols():
    from gqis import native
    lib = ctypes.CDLL(str(native.build("gqis_serve")))  # nvcc builds it here; loading needs no GPU
    header = (ROOT / "include" / "gqis_serve.h").read_text()
    names = re.findall(r"^(?:int|const char\*)\s+(gqis_serve_\w+)\(", header, re.M)
    assert len(names) == 8
    for n in names:
        assert hasattr(lib, n), n


def test_serve_rejects_invalid_arguments_before_any_cuda_call():
    """Argument checks run before the server touches a device, so they are testable without a GPU:
    every entry point returns GQIS_ERR_INVALID (1) with a message for NULL or out-of-range input."""
    from gqis import native
    lib = ctypes.CDLL(str(native.build("gqis_serve")))
    lib.gqis_serve_last_error.restype = ctypes.c_char_p
    out = ctypes.c_void_p(1)
    assert lib.gqis_serve_open(0, 2, 4, ctypes.c_int64(1024), ctypes.c_int64(0), None) == 1
    assert b"out is NULL" in lib.gqis_serve_last_error()
    assert lib.gqis_serve_open(0, 0, 4, ctypes.c_int64(1024), ctypes.c_int64(0), ctypes.byref(out)) == 1
    assert out.value is None  # cleared on failure
    assert b"invalid server sizes" in lib.gqis_serve_last_error()
    assert lib.gqis_serve_open(0, 2, 4, ctypes.c_int64(0), ctypes.c_int64(0), ctypes.byref(out)) == 1
    assert lib.gqis_serve_open(0, 2, 4, ctypes.c_int64(64), ctypes.c_int64(-1), ctypes.byref(out)) == 1
    state, rid, buf = ctypes.c_int32(), ctypes.c_int64(), ctypes.create_string_buffer(16)
    assert lib.gqis_serve_submit(None, b"x.so", None, ctypes.c_int64(0), ctypes.byref(rid)) == 1
    assert lib.gqis_serve_poll(None, ctypes.c_int64(0), ctypes.byref(state)) == 1
    assert lib.gqis_serve_wait(None, ctypes.c_int64(0), ctypes.c_double(1.0), ctypes.byref(state)) == 1
    assert lib.gqis_serve_cancel(None, ctypes.c_int64(0)) == 1
    assert lib.gqis_serve_request_error(None, ctypes.c_int64(0), buf, ctypes.c_int64(16)) == 1
    assert lib.gqis_serve_close(None) == 1
    assert b"NULL server" in lib.gqis_serve_last_error()
