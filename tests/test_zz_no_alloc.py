"""The allocation-free launch, ``gqis_sweep_launch_noalloc``, on the GPU.

Some callers cannot call cudaMalloc: a host whose caching allocator owns the device memory, a
real-time loop where an allocation would synchronize the device, a plugin handed only its input
and output buffers. For them the module exports a launch whose scratch (the adaptive kernels'
work-stealing counter) lives in a fixed device array inside the library. This file calls it
through the C ABI twice in a row and checks both results against the ordinary launch, which
takes its scratch from the caller. It is named to run last, after every other test.
"""

import ctypes

import numpy as np
import pytest

import ref_cases


def _scaled_err(got, ref):
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.gpu
def test_noalloc_launch_matches_the_allocating_launch_on_two_calls_in_a_row():
    import torch
    from gqis import abi, solver
    torch.cuda.set_device(0)
    case = ref_cases.cases()["qubit_tsit5a_mean"]  # adaptive work-stealing kernel: uses scratch
    sweep = solver.prepare_sweep(case["api"], *case["args"], **case["kwargs"])
    stream = torch.cuda.current_stream()
    sweep.launch(stream)
    torch.cuda.synchronize()
    expected = sweep.results.double().cpu().numpy()
    expected_counts = sweep.tensors["step_counts"].cpu().numpy()

    lib = sweep.module.lib
    desc = abi.SweepDesc.from_buffer_copy(sweep.desc)
    desc.work_counter = None  # ignored by the no-alloc launch: its scratch lives in the library
    for call in range(2):
        sweep.results.fill_(float("nan"))
        sweep.tensors["step_counts"].fill_(-1)
        rc = lib.gqis_sweep_launch_noalloc(ctypes.byref(desc), ctypes.c_void_p(stream.cuda_stream))
        assert rc == abi.OK, lib.gqis_last_error().decode()
        torch.cuda.synchronize()
        got = sweep.results.double().cpu().numpy()
        err = _scaled_err(got, expected)
        assert err <= 1e-10, f"call {call}: scaled max error {err:.3e}"
        np.testing.assert_array_equal(sweep.tensors["step_counts"].cpu().numpy(), expected_counts)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["qubit_rk4_final", "c2_fp64_mean_sub32"])
def test_noalloc_launch_of_a_fixed_step_module_is_the_ordinary_launch(name):
    """Fixed-step kernels use no scratch: the no-alloc entry point runs the ordinary launch and
    ignores a NULL work counter (for the FP32 four-level case, the packed two-point kernel)."""
    import torch
    from gqis import abi, solver
    torch.cuda.set_device(0)
    case = ref_cases.cases()[name]
    sweep = solver.prepare_sweep(case["api"], *case["args"], **dict(case["kwargs"], fp64=False))
    stream = torch.cuda.current_stream()
    sweep.launch(stream)
    torch.cuda.synchronize()
    expected = sweep.results.clone()
    desc = abi.SweepDesc.from_buffer_copy(sweep.desc)
    desc.work_counter = None
    lib = sweep.module.lib
    for call in range(2):
        sweep.results.fill_(float("nan"))
        rc = lib.gqis_sweep_launch_noalloc(ctypes.byref(desc), ctypes.c_void_p(stream.cuda_stream))
        assert rc == abi.OK, lib.gqis_last_error().decode()
        torch.cuda.synchronize()
        assert torch.equal(sweep.results, expected), f"call {call}"


@pytest.mark.gpu
def test_noalloc_launch_rejects_more_points_than_its_scratch_can_count():
    import torch
    from gqis import abi, solver
    torch.cuda.set_device(0)
    case = ref_cases.cases()["qubit_tsit5a_mean"]
    sweep = solver.prepare_sweep(case["api"], *case["args"], **case["kwargs"])
    desc = abi.SweepDesc.from_buffer_copy(sweep.desc)
    desc.num_x, desc.num_y = 65536, 65536
    desc.point_begin, desc.point_count = 0, 1 << 32  # checked before anything touches the GPU
    lib = sweep.module.lib
    rc = lib.gqis_sweep_launch_noalloc(ctypes.byref(desc), ctypes.c_void_p(0))
    assert rc == abi.ERR_TOO_LARGE
    assert b"exceed the maximum" in lib.gqis_last_error()
