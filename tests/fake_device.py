"""CPU stand-in for the device seam of ``gqis.solver`` (for tests that need no GPU).

``_load_kernel`` records the generated module source instead of running nvcc, and
``_device_run`` returns zero-filled outputs of the right shapes, so code generation, caching,
validation and calibration logic run on the CPU - the role the reference's NumPy CuPy stand-in
plays in its tests (``tests/test_ode_api.py:14-33``).
"""

from contextlib import contextmanager
from unittest.mock import patch

import numpy as np

import gqis.solver as core
from gqis.rhs import _RHS_CODE_CACHE


class FakeDevice:
    def __init__(self, values=None):
        self.sources = []
        self.launches = []
        self.values = values  # optional callable(launch) -> value written into every result

    def load_kernel(self, entry):
        if entry.get("module") is None:
            entry["module"] = "fake"
            self.sources.append(entry["source"])
        return entry["module"]

    def device_run(self, launch):
        self.launches.append(launch)
        nx = len(launch.par_x)
        ny = len(launch.par_y)
        width = 2 if launch.output_mode in ("mean", "final") else launch.state_size
        dtype = np.float64 if launch.form == "fp64" else np.float32
        res = np.zeros((nx * ny, width), dtype=dtype)
        if self.values is not None:
            res[:] = self.values(launch)
        trace = None
        if launch.trace_mode is not None:
            tw = 2 if launch.trace_mode == "observable" else launch.state_size
            trace = np.zeros((nx * ny, launch.num_trace, tw), dtype=dtype)
        counts = np.zeros((nx * ny, 2), dtype=np.int32) if launch.count_steps else None
        return res, trace, counts, 0.0


    def device_run_many(self, launches):
        return [self.device_run(launch) for launch in launches]


def clear_caches():
    for cache in (_RHS_CODE_CACHE, core._KERNEL_CACHE, core._TIMESTEP_CALIBRATION_CACHE):
        cache.clear()


@contextmanager
def fake_device(values=None):
    dev = FakeDevice(values)
    clear_caches()
    with patch.dict("os.environ", {"GQIS_DISK_CACHE": "0"}), \
            patch.object(core, "_load_kernel", dev.load_kernel), patch.object(core, "_device_run", dev.device_run), \
            patch.object(core, "_device_run_many", dev.device_run_many):
        try:
            yield dev
        finally:
            clear_caches()
