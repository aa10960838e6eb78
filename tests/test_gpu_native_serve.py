"""The native sweep server (include/gqis_serve.h) on the GPU: requests of three kernel kinds (two adaptive
requests of one module, whose chunks go out as shared batch grids) submitted
together through the C ABI, cut into 97-point chunks on three streams, give the results of their
direct launches bit for bit; a request its module rejects fails alone with the module's message."""

import ctypes

import numpy as np
import pytest

import ref_cases


def _lib():
    from gqis import native
    lib = ctypes.CDLL(str(native.build("gqis_serve")))
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    lib.gqis_serve_open.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, i64, i64, ctypes.POINTER(vp)]
    lib.gqis_serve_submit.argtypes = [vp, ctypes.c_char_p, vp, i64, ctypes.POINTER(i64)]
    lib.gqis_serve_wait.argtypes = [vp, i64, ctypes.c_double, ctypes.POINTER(ctypes.c_int32)]
    lib.gqis_serve_request_error.argtypes = [vp, i64, ctypes.c_char_p, i64]
    lib.gqis_serve_close.argtypes = [vp]
    lib.gqis_serve_last_error.restype = ctypes.c_char_p
    return lib


def _sweeps():
    from gqis import solver
    from test_support_calls import hilbert_model
    cases = ref_cases.cases()
    out = {}
    for name in ("c2_fp64_mean_sub32", "duffing_tsit5a_trace"):  # fixed-step; adaptive with a trace
        c = cases[name]
        out[name] = solver.prepare_sweep(c["api"], *c["args"], **c["kwargs"])
    # a second request of the same adaptive module: its chunks share batch grids with the first's
    c = cases["duffing_tsit5a_trace"]
    out["duffing_part"] = solver.prepare_sweep(c["api"], *c["args"], **c["kwargs"], point_begin=5, point_count=101)
    _, args, kwargs = hilbert_model(16, side=(12, 9))  # tensor cores: 8-point tiles split by the chunks
    out["tc16"] = solver.prepare_sweep("mesolve_2D", *args, **dict(kwargs, precision="fp32", rhs_form="matrix_tc"))
    return out


@pytest.mark.gpu
def test_native_server_gives_each_request_its_direct_results():
    import torch
    torch.cuda.set_device(0)
    lib = _lib()
    sweeps = _sweeps()
    direct = {}
    for k, sw in sweeps.items():
        sw.launch()
        torch.cuda.synchronize()
        direct[k] = {n: t.clone() for n, t in sw.tensors.items() if t is not None and n in ("results", "trace")}
        for n in direct[k]:
            sw.tensors[n].zero_()
    torch.cuda.synchronize()
    server = ctypes.c_void_p()
    assert lib.gqis_serve_open(0, 3, 8, 97, 0, ctypes.byref(server)) == 0, lib.gqis_serve_last_error()
    try:
        ids = {}
        for k, sw in sweeps.items():
            rid = ctypes.c_int64()
            rc = lib.gqis_serve_submit(server, str(sw.module.path).encode(), ctypes.addressof(sw.desc), 0,
                                       ctypes.byref(rid))
            assert rc == 0, lib.gqis_serve_last_error()
            ids[k] = rid.value
        bad = sweeps["c2_fp64_mean_sub32"]
        desc = type(bad.desc).from_buffer_copy(bad.desc)
        desc.num_steps = 0  # the module rejects it at launch
        bad_id = ctypes.c_int64()
        assert lib.gqis_serve_submit(server, str(bad.module.path).encode(), ctypes.addressof(desc), 0,
                                     ctypes.byref(bad_id)) == 0
        for k, rid in ids.items():
            state = ctypes.c_int32()
            assert lib.gqis_serve_wait(server, rid, 300.0, ctypes.byref(state)) == 0, k
            assert state.value == 2, (k, state.value)  # GQIS_REQ_DONE
        state = ctypes.c_int32()
        assert lib.gqis_serve_wait(server, bad_id.value, 60.0, ctypes.byref(state)) == 0
        assert state.value == 3  # GQIS_REQ_FAILED
        msg = ctypes.create_string_buffer(512)
        assert lib.gqis_serve_request_error(server, bad_id.value, msg, 512) == 0
        assert b"num_steps" in msg.value
    finally:
        assert lib.gqis_serve_close(server) == 0
    torch.cuda.synchronize()
    for k, sw in sweeps.items():
        for n, ref in direct[k].items():
            assert torch.equal(sw.tensors[n], ref), (k, n)


@pytest.mark.gpu
def test_native_server_cancels_a_queued_request():
    """With one slot, a request queued behind a long adaptive sweep (1024^2 Duffing points) is
    cancelled before it starts; the running one completes."""
    import torch
    from gqis import solver
    torch.cuda.set_device(0)
    lib = _lib()
    lib.gqis_serve_cancel.argtypes = [ctypes.c_void_p, ctypes.c_int64]
    cases = ref_cases.cases()
    sweeps = [solver.prepare_sweep(c["api"], *c["args"], **c["kwargs"])
              for c in (cases["duffing_tsit5a_full_final"], cases["c2_fp64_mean_sub32"])]
    server = ctypes.c_void_p()
    assert lib.gqis_serve_open(0, 2, 1, 1 << 16, 0, ctypes.byref(server)) == 0
    try:
        ids = []
        for sw in sweeps:
            rid = ctypes.c_int64()
            assert lib.gqis_serve_submit(server, str(sw.module.path).encode(), ctypes.addressof(sw.desc), 0,
                                         ctypes.byref(rid)) == 0
            ids.append(rid.value)
        assert lib.gqis_serve_cancel(server, ids[1]) == 0
        states = []
        for rid in ids:
            state = ctypes.c_int32()
            assert lib.gqis_serve_wait(server, rid, 300.0, ctypes.byref(state)) == 0
            states.append(state.value)
        assert states == [2, 4]  # DONE, CANCELLED
    finally:
        assert lib.gqis_serve_close(server) == 0
