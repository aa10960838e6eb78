"""The continuous-batching server on the GPU: every result is the same alone and in the mix."""

import numpy as np
import pytest

import ref_cases


def _direct(case):
    import gqis
    return getattr(gqis, case["api"])(*case["args"], **case["kwargs"])


@pytest.mark.gpu
def test_each_request_is_the_same_alone_and_in_the_mix():
    from gqis.serving import SweepServer
    cases = ref_cases.cases()
    names = ["c1_fp64_mean", "c2_fp64_mean_sub32", "qubit_dop853_final_rho", "qubit_rk4_mean_warmup_trace",
             "qubit_tsit5a_mean", "duffing_tsit5a_trace", "duffing_rk4_observable_trace", "qubit_ab5_final_rho"]
    alone = {n: _direct(cases[n]) for n in names}
    # Small chunks and several streams: the requests' chunks interleave and overlap on the device.
    with SweepServer(streams=3, chunk_points=256, max_inflight=8) as srv:
        futs = {n: srv.submit(cases[n]["api"], *cases[n]["args"], **cases[n]["kwargs"]) for n in names}
        outs = {n: f.result(300) for n, f in futs.items()}
        stats = dict(srv.stats)
    assert stats["completed"] == len(names)
    assert stats["max_concurrent"] >= 2
    for n in names:
        ref = alone[n]
        ref_result = ref[0] if isinstance(ref, tuple) else ref
        np.testing.assert_array_equal(outs[n]["result"], ref_result, err_msg=n)
        if isinstance(ref, tuple):
            np.testing.assert_array_equal(outs[n]["trace"], ref[1], err_msg=n)


@pytest.mark.gpu
def test_adaptive_requests_share_batched_grids_and_match_their_direct_calls():
    """Adaptive requests of one module (here three Duffing sweeps of different grids and tolerances)
    are served by batch launches whose lanes take points of every request from one counter; each
    request's final states, traces and step counts equal its direct call bit for bit."""
    import gqis
    from gqis.serving import SweepServer
    from test_support_calls import duffing_case
    calls = []
    for side, rtol in ((8, 1e-8), (12, 1e-7), (5, 1e-9)):
        _, args, kwargs = duffing_case(side=side, solver="tsit5a")
        kwargs["adaptive_options"] = dict(kwargs["adaptive_options"], step_rtol=rtol)
        calls.append((args, kwargs))
    alone = [gqis.odesolve_2D(*a, **kw, return_timing_info=True) for a, kw in calls]
    with SweepServer(streams=2, chunk_points=40, max_inflight=8) as srv:
        futs = [srv.submit("odesolve_2D", *a, **kw) for a, kw in calls]
        outs = [f.result(300) for f in futs]
        stats = dict(srv.stats)
    assert stats["batched_launches"] >= 1 and stats["completed"] == len(calls)
    for (final, trace, _, info), out in zip(alone, outs):
        np.testing.assert_array_equal(out["result"], final)
        np.testing.assert_array_equal(out["trace"], trace)
        counts = np.stack([info["adaptive_steps"]["accepted"], info["adaptive_steps"]["rejected"]], -1)
        np.testing.assert_array_equal(out["step_counts"].reshape(counts.shape), counts)


@pytest.mark.gpu
def test_server_isolates_a_request_the_c_abi_rejects():
    """A launch the module rejects (status != 0) fails its own request; the others complete."""
    import dataclasses
    import gqis
    from gqis import solver
    from gqis.serving import FAILED, SweepServer
    good = ref_cases.cases()["qubit_rk4_final"]
    holder = {}
    gqis.mesolve_2D(*good["args"], **good["kwargs"], _prepare_only=holder)
    solver._load_kernel(holder["launch"].entry)
    bad = dataclasses.replace(holder["launch"], num_steps=0)  # "num_steps must be at least 1"
    with SweepServer(streams=2, chunk_points=16) as srv:
        f1 = srv.submit(good["api"], *good["args"], **good["kwargs"])
        f2 = srv.submit_launch(bad)
        f3 = srv.submit(good["api"], *good["args"], **good["kwargs"])
        r1, r3 = f1.result(120), f3.result(120)
        f2._event.wait(120)
    np.testing.assert_array_equal(r1["result"], r3["result"])
    assert f2.state == FAILED and "num_steps" in f2.error


@pytest.mark.gpu
def test_fit_requests_in_the_server_match_the_adjoint_alone():
    from gqis import adjoint
    from gqis.serving import SweepServer
    from test_support_calls import qubit_fit_model
    args, kwargs, params = qubit_fit_model()
    mean, grad = adjoint.mean_gradient(*args, **kwargs, params=list(params[:3]))
    sweep_case = ref_cases.cases()["c1_fp64_mean"]
    with SweepServer(streams=2, chunk_points=16) as srv:
        f_fit = srv.submit_fit(*args, **kwargs, params=list(params[:3]))
        f_sweep = srv.submit(sweep_case["api"], *sweep_case["args"], **sweep_case["kwargs"])
        out = f_fit.result(300)
        f_sweep.result(300)
    np.testing.assert_array_equal(out["result"], mean)
    np.testing.assert_array_equal(out["grad"], grad)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [16, 64])
def test_tensor_core_request_is_the_same_in_chunks_that_split_tiles(N):
    """The tensor-core kernel packs 128 / N points per MMA tile (at N = 64 a tile spans a cluster of
    two CTAs); a chunk size that is not a multiple of the tile moves every point to another row of
    another tile, and the result must not change."""
    import gqis
    from gqis.serving import SweepServer
    from test_support_calls import hilbert_model
    _, args, kwargs = hilbert_model(N, side=(12, 9) if N == 16 else (5, 3))
    alone = gqis.mesolve_2D(*args, **kwargs, precision="fp32", rhs_form="matrix_tc")
    with SweepServer(streams=3, chunk_points=13, max_inflight=4) as srv:
        out = srv.submit("mesolve_2D", *args, **kwargs, precision="fp32", rhs_form="matrix_tc").result(300)
    np.testing.assert_array_equal(out["result"], alone)


@pytest.mark.gpu
def test_tensor_core_requests_of_every_tile_shape_share_the_device():
    """Tensor-core requests of N = 8, 16 and 64 (one CTA per tile, and a two-CTA cluster per tile that
    allocates all of its SMs' tensor memory) and a reduced-form request run concurrently on four
    streams; each result equals the request run alone."""
    import gqis
    from gqis.serving import SweepServer
    from test_support_calls import hilbert_model
    reqs = {}
    for N, side in ((64, (5, 3)), (16, (12, 9)), (8, (4, 3))):
        _, args, kwargs = hilbert_model(N, side=side)
        reqs[f"tc{N}"] = (args, dict(kwargs, precision="fp32", rhs_form="matrix_tc"))
    case = ref_cases.cases()["c2_fp64_mean_sub32"]
    reqs["reduced"] = (tuple(case["args"]), dict(case["kwargs"]))
    alone = {k: gqis.mesolve_2D(*a, **kw) for k, (a, kw) in reqs.items()}
    with SweepServer(streams=4, chunk_points=7, max_inflight=8) as srv:
        futs = {k: srv.submit("mesolve_2D", *a, **kw) for k, (a, kw) in reqs.items()}
        outs = {k: f.result(300) for k, f in futs.items()}
        stats = dict(srv.stats)
    assert stats["completed"] == len(reqs) and stats["max_concurrent"] >= 2
    for k in reqs:
        np.testing.assert_array_equal(outs[k]["result"], alone[k], err_msg=k)
