"""Recording stand-in for CuPy, used only by oracle/ref_capture.py.

The reference package imports CuPy for device arrays and NVRTC. This module gives it NumPy
arrays instead and records, rather than runs, every ``RawKernel``: the generated CUDA source
and the positional launch arguments. The oracle recipe then compiles that source itself.
"""
import numpy as np

float32, float64 = np.float32, np.float64
complex64, complex128 = np.complex64, np.complex128
int32 = np.int32
ndarray = np.ndarray
asarray, asnumpy, zeros, all, isfinite = np.asarray, np.asarray, np.zeros, np.all, np.isfinite

RECORDS = []


class RawKernel:
    def __init__(self, code, name, options=()):
        self.code, self.name, self.options = code, name, tuple(options)

    def compile(self):
        return None

    def __call__(self, grid, block, args):
        RECORDS.append({"code": self.code, "name": self.name, "grid": tuple(grid), "block": tuple(block),
                        "args": list(args)})


class _Event:
    def record(self, *a):
        return None

    def synchronize(self):
        return None


class cuda:  # noqa: N801 - mirrors the module layout the reference touches
    Event = _Event

    @staticmethod
    def get_elapsed_time(a, b):
        return 0.0
