"""Scheduling logic of the sweep server on the CPU, with a fake device backend.

Failures are made on the host (an allocation that raises, a launch that raises, a cancelled
request); no GPU is involved.
"""

import time

import numpy as np
import pytest

from gqis.serving import CANCELLED, DONE, FAILED, SweepServer
from gqis.solver import SweepLaunch


class FakeEvent:
    def __init__(self, polls):
        self.remaining = polls


class FakeBackend:
    streams = [None, None]

    def __init__(self, polls=3):
        self.polls = polls
        self.launches = []
        self.fail_admit = set()
        self.fail_launch = set()

    def free_bytes(self):
        return 1 << 30

    def admit(self, req, chunk_points):
        if req.launch.extra.get("tag") in self.fail_admit:
            raise MemoryError("injected allocation failure")
        return [(b, min(chunk_points, req.points - b)) for b in range(0, req.points, chunk_points)]

    def launch(self, req, chunk, s):
        tag = req.launch.extra.get("tag")
        if tag in self.fail_launch:
            raise RuntimeError("injected launch failure")
        self.launches.append((tag, chunk[0], s))
        return FakeEvent(self.polls)

    def query(self, ev):
        ev.remaining -= 1
        return ev.remaining <= 0

    def copy_out(self, req, events):
        return FakeEvent(1)

    def results(self, req):
        return {"results": np.full((req.points, 2), float(req.launch.extra["tag"]))}

    def release(self, req):
        pass


def _launch(tag, nx=8, ny=8, steps=10):
    return SweepLaunch(entry={}, form="fp64", output_mode="mean", trace_mode=None, state_size=3,
                       par_x=np.zeros(nx), par_y=np.zeros(ny), consts=[], rho0=None, num_steps=steps,
                       warmup_steps=0, dt=0.1, t_in=0.0, extra={"tag": tag})


def test_requests_complete_with_their_own_results():
    be = FakeBackend()
    with SweepServer(backend=be, memory_budget=1 << 20, chunk_points=16) as srv:
        futs = [srv.submit_launch(_launch(k)) for k in range(5)]
        outs = [f.result(5) for f in futs]
    for k, out in enumerate(outs):
        assert out["result"].shape == (8, 8)
        assert np.all(out["result"] == k + 1j * k)
    assert srv.stats["completed"] == 5


def test_chunks_of_concurrent_requests_interleave():
    be = FakeBackend(polls=5)
    with SweepServer(backend=be, memory_budget=1 << 20, chunk_points=16) as srv:
        futs = [srv.submit_launch(_launch(k)) for k in range(3)]
        [f.result(5) for f in futs]
    first = [tag for tag, _, _ in be.launches[:6]]
    assert len(set(first)) > 1  # not one request's four chunks back to back
    assert srv.stats["max_concurrent"] >= 2


def test_admission_waits_for_memory_budget():
    be = FakeBackend(polls=4)
    with SweepServer(backend=be, memory_budget=1000, chunk_points=16) as srv:
        futs = [srv.submit_launch(_launch(k), nbytes=600) for k in range(3)]
        [f.result(5) for f in futs]
    assert srv.stats["max_concurrent"] == 1
    assert futs[1].admitted_at >= futs[0].finished_at - 1e-3


def test_request_larger_than_budget_fails_at_submission():
    with SweepServer(backend=FakeBackend(), memory_budget=100) as srv:
        fut = srv.submit_launch(_launch(0), nbytes=1000)
        with pytest.raises(RuntimeError, match="budget"):
            fut.result(1)


def test_failures_are_isolated_to_their_request():
    be = FakeBackend()
    be.fail_admit.add(1)
    be.fail_launch.add(2)
    with SweepServer(backend=be, memory_budget=1 << 20, chunk_points=16) as srv:
        futs = [srv.submit_launch(_launch(k)) for k in range(4)]
        for f in futs:
            f._event.wait(5)
    assert [f.state for f in futs] == [DONE, FAILED, FAILED, DONE]
    assert "injected" in futs[1].error and "injected" in futs[2].error


def test_cancel_queued_and_running_requests():
    be = FakeBackend(polls=20000)
    with SweepServer(backend=be, memory_budget=1000, chunk_points=8) as srv:
        a = srv.submit_launch(_launch(0), nbytes=600)
        b = srv.submit_launch(_launch(1), nbytes=600)  # queued behind a (budget)
        deadline = time.time() + 5
        while a.state != "running" and time.time() < deadline:
            time.sleep(1e-4)
        assert srv.cancel(b)
        assert srv.cancel(a)
        for f in (a, b):
            f._event.wait(5)
        be.polls = 3
        c = srv.submit_launch(_launch(2), nbytes=600)
        assert c.result(5)["result"].shape == (8, 8)
    assert a.state == CANCELLED and b.state == CANCELLED
    launched_a = [x for x in be.launches if x[0] == 0]
    assert len(launched_a) < 8  # dispatch stopped before all 8 chunks of a


def test_small_requests_go_before_large_ones_but_waiting_counts():
    """Admission takes the queued request with the least estimated work (point-steps x flops), aged by
    its waiting time; here the slot limit admits one at a time, so the order of admission shows it."""
    be = FakeBackend(polls=2)
    # estimates: 64^2 x 1e7 point-steps (0.2 s at the nominal rate) against 4^2 x 1e7 (0.8 ms)
    big, small = _launch(0, nx=64, ny=64, steps=10**7), _launch(1, nx=4, ny=4, steps=10**7)
    with SweepServer(backend=be, memory_budget=1 << 20, chunk_points=4096, max_inflight=1) as srv:
        first = srv.submit_launch(_launch(2, nx=32, ny=32))   # admitted at once (the server is idle)
        fb, fs = srv.submit_launch(big), srv.submit_launch(small)
        [f.result(5) for f in (first, fb, fs)]
    assert fs.admitted_at < fb.admitted_at  # the small request passed the big one queued before it


def test_close_drains_queued_and_running_requests():
    """close() returns once every request submitted before it has finished; none is dropped."""
    be = FakeBackend(polls=4)
    srv = SweepServer(backend=be, memory_budget=1 << 20, chunk_points=16)
    futs = [srv.submit_launch(_launch(k)) for k in range(4)]
    srv.close(timeout=10)
    assert not srv._thread.is_alive()
    assert all(f.done() and f.state == DONE for f in futs)
    for k, f in enumerate(futs):
        assert np.all(f.result(0)["result"] == k + 1j * k)
    assert srv.stats["completed"] == 4
