"""The native sweep server's C ABI on the CPU: the library builds, loads and exports every function
include/gqis_serve.h declares (no call is made: the server needs a GPU)."""

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
