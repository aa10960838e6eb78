"""Batch launches (``gqis_sweep_launch_batch``) on the GPU: several sweeps of one module in one grid.

Each sweep's points must come out exactly as in a launch of their own - bit for bit - whatever the
other sweeps of the batch are: different grids and point ranges (odd counts, offsets), step counts
and dt, for the plain FP64 kernel, the packed two-point FP32 kernel and the persistent adaptive
kernels, whose lanes take points of every sweep from one shared counter.
"""

import ctypes

import numpy as np
import pytest

import ref_cases


def _sweeps(case, variants, **override):
    """Prepared sweeps of one module: ``variants`` lists (point_begin, point_count, steps)."""
    from gqis import solver
    kwargs = dict(case["kwargs"], **override)
    out = []
    for begin, count, steps in variants:
        args = list(case["args"])
        if steps is not None:
            tl = np.asarray(args[4] if case["api"] == "mesolve_2D" else args[3])
            new = np.linspace(0.0, float(tl[-1]) * steps / (len(tl) - 1), steps + 1)
            args[4 if case["api"] == "mesolve_2D" else 3] = new
        out.append(solver.prepare_sweep(case["api"], *args, **kwargs, point_begin=begin, point_count=count))
    return out


def _check_batch(sweeps):
    import torch
    from gqis import abi
    stream = torch.cuda.current_stream()
    alone = []
    for sw in sweeps:
        sw.launch(stream)
        torch.cuda.synchronize()
        alone.append({k: v.clone() for k, v in sw.tensors.items() if k in ("results", "trace", "step_counts")
                      and v is not None})
        for k in alone[-1]:
            sw.tensors[k].fill_(-7)
    paths = {str(sw.module.path) for sw in sweeps}
    assert len(paths) == 1, "a batch runs one module"
    lib = sweeps[0].module.lib
    descs = (abi.SweepDesc * len(sweeps))(*[sw.desc for sw in sweeps])
    counter = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.gqis_sweep_launch_batch(descs, len(sweeps), counter.data_ptr(), stream.cuda_stream)
    assert rc == abi.OK, lib.gqis_last_error().decode()
    torch.cuda.synchronize()
    for sw, ref in zip(sweeps, alone):
        for k, v in ref.items():
            assert torch.equal(sw.tensors[k], v), k


@pytest.mark.gpu
@pytest.mark.parametrize("name,fp64", [("c2_fp64_mean_sub32", True), ("c2_fp64_mean_sub32", False),
                                       ("qubit_rk4_mean_warmup_trace", True), ("qubit_rk4_mean_warmup_trace", False)])
def test_fixed_step_batch_equals_separate_launches(name, fp64):
    """FP64 one point per thread, and the packed FP32 kernel (two points per thread): sweeps with
    odd point counts, offsets and different step counts in one grid."""
    import torch
    torch.cuda.set_device(0)
    case = ref_cases.cases()[name]
    n = int(np.prod([len(v) for v in case["kwargs"]["var_arrays"].values()]))
    variants = [(0, n, None), (3, n - 10, None), (1, 33, 37), (n - 5, 5, 60), (7, 1, None)]
    _check_batch(_sweeps(case, variants, fp64=fp64))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["qubit_tsit5a_mean", "duffing_tsit5a_trace"])
def test_adaptive_batch_shares_one_grid_and_equals_separate_launches(name):
    """The adaptive kernels' lanes take points of every sweep of the batch from one counter; each
    point's result, trace and step counts equal those of its own launch."""
    import torch
    torch.cuda.set_device(0)
    case = ref_cases.cases()[name]
    kwargs = dict(case["kwargs"])
    kwargs["adaptive_options"] = dict(kwargs["adaptive_options"], count_steps=True)
    case = dict(case, kwargs=kwargs)
    n = int(np.prod([len(v) for v in case["kwargs"]["var_arrays"].values()]))
    variants = [(0, n, None), (2, n - 3, None), (5, 11, None)]
    _check_batch(_sweeps(case, variants))


@pytest.mark.gpu
def test_batch_rejects_an_invalid_item_before_launching():
    import torch
    from gqis import abi
    torch.cuda.set_device(0)
    case = ref_cases.cases()["qubit_rk4_final"]
    sweeps = _sweeps(case, [(0, 4, None), (0, 4, None)])
    descs = (abi.SweepDesc * 2)(*[sw.desc for sw in sweeps])
    descs[1].num_steps = 0
    lib = sweeps[0].module.lib
    rc = lib.gqis_sweep_launch_batch(descs, 2, None, ctypes.c_void_p(0))
    assert rc == abi.ERR_INVALID and b"batch item 1" in lib.gqis_last_error()
