"""Continuous-batching sweep server.

Requests - any ``mesolve_2D`` / ``odesolve_2D`` call, of any model, size, integrator or form - are
admitted while device memory and slots allow, split into point chunks, and their chunks are
interleaved across several CUDA streams, so work of requests that arrive while others run overlaps
on the device. Inputs and outputs stay resident in device memory from admission to completion.
The server loop is one host thread; every launch goes through the model module's C ABI
(``gqis_sweep_launch``), a chunk being the descriptor's ``[point_begin, point_begin + point_count)``
slice with per-point pointers offset to that slice.

Adaptive requests steal work across requests: each dispatch pass gathers the next chunk of every
admitted adaptive request of the same module into one ``gqis_sweep_launch_batch`` grid, whose
persistent lanes take points of all those chunks from one counter. Points whose step counts differ
no longer leave a request's launch idle behind its slowest point: other requests' points fill the
lanes that finish early.

Each point's result depends only on its own inputs, so a request returns the same values alone and
in the mix (the GPU tests check that bit for bit).

The device layer is a small backend object so that the scheduling logic (admission by memory
budget and slots, priority dispatch, cancellation, failure isolation) is tested on the CPU with
a fake backend.
"""

from __future__ import annotations

import itertools
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

QUEUED, RUNNING, DONE, FAILED, CANCELLED = "queued", "running", "done", "failed", "cancelled"
BATCH_MAX = 64  # sweeps per gqis_sweep_launch_batch grid (GQIS_BATCH_MAX)


class SweepFuture:
    """Handle of one submitted request."""

    def __init__(self, rid, arrival):
        self.id = rid
        self.arrival = arrival
        self.admitted_at = None
        self.finished_at = None
        self.state = QUEUED
        self.error = None
        self._result = None
        self._event = threading.Event()

    def done(self):
        """True once the request has ended (done, failed or cancelled)."""
        return self._event.is_set()

    def result(self, timeout=None):
        """Wait for the request and return its results; raises if it failed, was cancelled or did
        not end within ``timeout`` seconds."""
        if not self._event.wait(timeout):
            raise TimeoutError(f"request {self.id} not finished within {timeout} s")
        if self.state == FAILED:
            raise RuntimeError(f"request {self.id} failed: {self.error}")
        if self.state == CANCELLED:
            raise RuntimeError(f"request {self.id} was cancelled")
        return self._result

    @property
    def latency(self):
        """Seconds from submission to completion (None while the request runs)."""
        return None if self.finished_at is None else self.finished_at - self.arrival

    def _finish(self, state, result=None, error=None):
        self.state, self._result, self.error = state, result, error
        self.finished_at = time.perf_counter()
        self._event.set()


@dataclass
class FitLaunch:
    """A gradient ("fit") request: the adjoint module and the sweep it differentiates."""

    sweep: object          # solver.SweepLaunch of the mean map
    module: object         # adjoint module (engine.ModelModule)
    P: int
    params: list
    checkpoint_every: int
    forward_consts: list
    adjoint_consts: list

    # the attributes the server reads for budgeting and output shapes
    def __getattr__(self, name):
        return getattr(self.sweep, name)


@dataclass
class _Request:
    future: SweepFuture
    launch: object                 # solver.SweepLaunch (or a backend-specific description)
    shape: tuple                   # output post-processing information
    nbytes: int
    points: int
    point_steps: int
    chunks: deque = field(default_factory=deque)
    inflight: list = field(default_factory=list)
    handle: object = None          # backend state (device buffers)
    cancel: bool = False
    copying: object = None
    kind: str = "sweep"
    work_s: float = 0.0            # estimated device time of the whole request (scheduling priority)
    total_chunks: int = 1


class TorchBackend:
    """Device layer on torch tensors and CUDA streams; launches through the model modules' C ABI."""

    def __init__(self, device=0, streams=4):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device)
        with torch.cuda.device(self.device):
            self.admit_stream = torch.cuda.Stream(self.device)
            self.streams = [torch.cuda.Stream(self.device) for _ in range(streams)]

    def free_bytes(self):
        free, _total = self.torch.cuda.mem_get_info(self.device)
        return free

    def admit(self, req, chunk_points):
        """Allocate and upload on the admission stream; returns the chunk list."""
        if req.kind == "adjoint":
            return self._admit_adjoint(req, chunk_points)
        from . import abi, solver
        torch = self.torch
        with torch.cuda.device(self.device), torch.cuda.stream(self.admit_stream):
            module = solver._load_kernel(req.launch.entry)
            desc, buf = solver._device_buffers(req.launch)
            n = int(desc.point_count)
            starts = list(range(0, n, chunk_points))
            counters = (torch.zeros(len(starts), dtype=torch.int32, device=self.device)
                        if req.launch.adaptive else None)
            ready = torch.cuda.Event()
            ready.record(self.admit_stream)
        real = buf["results"].element_size()
        width = buf["results"].shape[1]
        chunks = []
        for k, b in enumerate(starts):
            c = abi.SweepDesc.from_buffer_copy(desc)
            c.point_begin, c.point_count = b, min(chunk_points, n - b)
            c.results = desc.results + b * width * real
            if desc.rho0:
                c.rho0 = desc.rho0 + b * buf["rho0"].shape[1] * real
            if desc.trace:
                tr = buf["trace"]
                c.trace = desc.trace + b * tr.shape[1] * tr.shape[2] * real
            if desc.step_counts:
                c.step_counts = desc.step_counts + b * 2 * 4
            if counters is not None:
                c.work_counter = counters.data_ptr() + 4 * k
            chunks.append(c)
        req.handle = {"module": module, "buf": buf, "desc": desc, "ready": ready, "counters": counters}
        return chunks

    def _admit_adjoint(self, req, chunk_points):
        import ctypes
        from . import abi, solver
        torch = self.torch
        fit = req.launch  # FitLaunch
        with torch.cuda.device(self.device), torch.cuda.stream(self.admit_stream):
            desc, buf = solver._device_buffers(fit.sweep)
            n = int(desc.point_count)
            N = int(fit.sweep.num_steps)
            region = ctypes.c_int64()
            rc = fit.module.lib.gqis_adjoint_scratch_bytes(min(chunk_points, n), N, fit.checkpoint_every,
                                                           ctypes.byref(region))
            abi.check(rc, fit.module.lib)
            starts = list(range(0, n, chunk_points))
            words = (region.value + 7) // 8
            scratch = torch.empty(max(1, words * len(starts)), dtype=torch.float64, device=self.device)
            grad = torch.empty((n, max(1, fit.P)), dtype=torch.float64, device=self.device)
            cf = torch.tensor(fit.forward_consts or [0.0], dtype=torch.float64, device=self.device)
            ca = torch.tensor(fit.adjoint_consts or [0.0], dtype=torch.float64, device=self.device)
            ready = torch.cuda.Event()
            ready.record(self.admit_stream)
        buf["grad"] = grad
        chunks = []
        for k, b in enumerate(starts):
            a = abi.AdjointDesc()
            a.sweep = abi.SweepDesc.from_buffer_copy(desc)
            a.sweep.point_begin, a.sweep.point_count = b, min(chunk_points, n - b)
            a.sweep.results = desc.results + b * 2 * 8
            a.sweep.consts = cf.data_ptr() if fit.forward_consts else None
            a.num_params = fit.P
            a.checkpoint_every = fit.checkpoint_every
            a.adjoint_consts = ca.data_ptr()
            a.grad = grad.data_ptr() + b * max(1, fit.P) * 8
            a.scratch = scratch.data_ptr() + k * words * 8
            a.scratch_bytes = words * 8
            chunks.append(a)
        req.handle = {"module": fit.module, "buf": buf, "desc": desc, "ready": ready,
                      "keep": (scratch, cf, ca)}
        return chunks

    def launch(self, req, chunk, stream_index):
        torch = self.torch
        st = self.streams[stream_index]
        st.wait_event(req.handle["ready"])
        if req.kind == "adjoint":
            import ctypes
            from . import abi
            lib = req.handle["module"].lib
            rc = lib.gqis_adjoint_launch(ctypes.byref(chunk), ctypes.c_void_p(st.cuda_stream))
            abi.check(rc, lib)
        else:
            req.handle["module"].launch(chunk, st.cuda_stream)
        ev = torch.cuda.Event()
        ev.record(st)
        return ev

    def launch_batch(self, items, stream_index):
        """One grid for chunks of several adaptive requests of one module (``items``: (request, chunk)
        pairs); their lanes share one fresh work counter. Returns the event and the counter, which
        must stay alive until the event completes."""
        from . import abi
        torch = self.torch
        st = self.streams[stream_index]
        for req, _ in items:
            st.wait_event(req.handle["ready"])
        with torch.cuda.device(self.device), torch.cuda.stream(st):
            counter = torch.zeros(1, dtype=torch.int32, device=self.device)
        descs = (abi.SweepDesc * len(items))(*[chunk for _, chunk in items])
        lib = items[0][0].handle["module"].lib
        rc = lib.gqis_sweep_launch_batch(descs, len(items), counter.data_ptr(), st.cuda_stream)
        abi.check(rc, lib)
        ev = torch.cuda.Event()
        ev.record(st)
        return ev, counter

    @staticmethod
    def query(event):
        return event.query()

    def copy_out(self, req, events):
        """D2H of the results after the given chunk events; returns an event."""
        torch = self.torch
        with torch.cuda.device(self.device), torch.cuda.stream(self.admit_stream):
            for ev in events:
                self.admit_stream.wait_event(ev)
            host = {}
            for name in ("results", "trace", "step_counts", "grad"):
                t = req.handle["buf"].get(name)
                if t is not None:
                    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
                    h.copy_(t, non_blocking=True)
                    host[name] = h
            ev = torch.cuda.Event()
            ev.record(self.admit_stream)
        req.handle["host"] = host
        return ev

    def results(self, req):
        return {k: v.numpy() for k, v in req.handle["host"].items()}

    def release(self, req):
        req.handle = None


class SweepServer:
    """Continuous-batching server (see the module docstring).

    ``memory_budget`` caps the device bytes of admitted requests (default: half the free memory at
    start); ``max_inflight`` caps admitted requests; ``chunk_points`` is the launch granularity.
    """

    def __init__(self, device=0, streams=4, memory_budget=None, max_inflight=16, chunk_points=1 << 16,
                 backend=None, poll_s=50e-6):
        self.backend = backend or TorchBackend(device, streams)
        self.nstreams = len(getattr(self.backend, "streams", [None] * streams))
        self.budget = int(memory_budget if memory_budget is not None else self.backend.free_bytes() // 2)
        self.max_inflight = int(max_inflight)
        self.chunk_points = int(chunk_points)
        self.poll_s = poll_s
        self._ids = itertools.count()
        self._lock = threading.Lock()
        self._queue = deque()
        self._active = []
        self._used = 0
        self._stop = False
        self._stream_load = [0] * self.nstreams
        self._batches = hasattr(self.backend, "launch_batch")  # cross-request batches of adaptive chunks
        self.stats = {"submitted": 0, "completed": 0, "failed": 0, "cancelled": 0, "point_steps": 0,
                      "max_concurrent": 0, "batched_launches": 0}
        self._thread = threading.Thread(target=self._loop, name="gqis-serve", daemon=True)
        self._thread.start()

    # ------------------------------------------------------------------ public API
    def submit(self, api, *args, **kwargs):
        """Queue one ``mesolve_2D`` / ``odesolve_2D`` call; returns a :class:`SweepFuture`.

        The symbolic preparation and the module build run here, in the caller's thread (both are
        cached), so the server thread only moves data and launches kernels.
        """
        from . import solver
        holder = {}
        kwargs = dict(kwargs, _prepare_only=holder)
        if api in ("odesolve_2D", "odesolve"):
            from .gqis_ode_api import odesolve_2D
            odesolve_2D(*args, **kwargs)
        else:
            solver.mesolve_2D(*args, **kwargs)
        launch = holder["launch"]
        solver._load_kernel(launch.entry)
        return self.submit_launch(launch)

    def submit_fit(self, *args, params, values=None, checkpoint_every=None, **kwargs):
        """Queue a gradient request: the ``mesolve_2D`` mean map and d<O>_avg/dtheta per point for the
        runtime-constant parameters ``params`` (checkpointed RK4 adjoint, FP64)."""
        import math
        from . import adjoint, engine
        source, launch, meta = adjoint.module_source(*args, params=params, **kwargs)
        module = engine.load_module(source)
        prob_consts = adjoint.const_values(launch.entry["compiled"], meta["defaults"], values)
        used = launch.entry["frag"]["used_const_indices"]
        fit = FitLaunch(sweep=launch, module=module, P=meta["P"], params=meta["params"],
                        checkpoint_every=int(checkpoint_every or max(1, math.ceil(math.sqrt(launch.num_steps)))),
                        forward_consts=[prob_consts[i] for i in used] if used else [],
                        adjoint_consts=prob_consts)
        points = len(launch.par_x) * len(launch.par_y)
        ck = fit.checkpoint_every
        scratch = (math.ceil(launch.num_steps / ck) + ck) * launch.state_size * min(points, self.chunk_points) * 8
        nchunks = math.ceil(points / self.chunk_points)
        nbytes = points * (2 + fit.P) * 8 + scratch * nchunks
        return self.submit_launch(fit, nbytes=nbytes, kind="adjoint")

    def submit_launch(self, launch, nbytes=None, kind="sweep"):
        """Queue a prepared launch; ``nbytes`` is its device memory for admission (estimated from the
        launch when None). A request larger than the whole budget fails at once."""
        rid = next(self._ids)
        fut = SweepFuture(rid, time.perf_counter())
        nx = len(launch.par_x)
        ny = len(launch.par_y)
        points = nx * ny
        if nbytes is None:
            real = 8 if launch.form == "fp64" else 4
            width = 2 if launch.output_mode in ("mean", "final") else launch.state_size
            nbytes = points * width * real + 8 * (nx + ny + len(launch.consts) + 1)
            if launch.rho0 is not None:
                nbytes += points * launch.state_size * real
            if launch.trace_mode is not None:
                tw = 2 if launch.trace_mode == "observable" else launch.state_size
                nbytes += points * launch.num_trace * tw * real
        req = _Request(fut, launch, (nx, ny), int(nbytes), points, points * int(launch.num_steps), kind=kind)
        req.work_s = _work_estimate(launch, kind, req.point_steps)
        if req.nbytes > self.budget:
            fut._finish(FAILED, error=f"request needs {req.nbytes} bytes, more than the budget {self.budget}")
            return fut
        with self._lock:
            self._queue.append(req)
            self.stats["submitted"] += 1
        return fut

    def cancel(self, fut):
        """Cancel a request: a queued one ends at once, a running one after its chunks in flight.
        Returns False if the request has already ended."""
        with self._lock:
            for req in list(self._queue):
                if req.future is fut:
                    self._queue.remove(req)
                    fut._finish(CANCELLED)
                    self.stats["cancelled"] += 1
                    return True
            for req in self._active:
                if req.future is fut:
                    req.cancel = True
                    return True
        return False

    def close(self, timeout=60.0):
        """Stop accepting work once the queue is drained: the scheduler thread finishes every queued and
        running request, then exits; waits up to ``timeout`` seconds for it."""
        self._stop = True
        self._thread.join(timeout)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ server loop
    def _priority(self, req, now):
        """Shortest estimated remaining work first, aged by the time since arrival (seconds): a request
        that has waited longer than its own estimated work goes before any newer one."""
        left = 1.0 if req.future.state == QUEUED else len(req.chunks) / max(1, req.total_chunks)
        return (req.work_s * left - (now - req.future.arrival), req.future.id)

    def _admit(self):
        while True:
            with self._lock:
                if not self._queue or len(self._active) >= self.max_inflight:
                    return
                now = time.perf_counter()
                req = min(self._queue, key=lambda r: self._priority(r, now))
                if self._used + req.nbytes > self.budget:
                    return  # the first in line waits for memory; nothing passes it
                self._queue.remove(req)
            try:
                req.chunks = deque(self.backend.admit(req, self.chunk_points))
                req.total_chunks = max(1, len(req.chunks))
            except Exception as exc:  # allocation or upload failure: this request only
                req.future._finish(FAILED, error=repr(exc))
                self.stats["failed"] += 1
                continue
            req.future.state = RUNNING
            req.future.admitted_at = time.perf_counter()
            self._used += req.nbytes
            with self._lock:
                self._active.append(req)
                self.stats["max_concurrent"] = max(self.stats["max_concurrent"], len(self._active))

    def _dispatch(self):
        # One chunk of each admitted request per pass, onto the least-loaded stream, at most two chunks
        # queued per stream: first the oldest admitted request (so large requests keep progressing
        # beside small ones), then the others in priority order (least estimated work left first, aged).
        progressed = False
        now = time.perf_counter()
        order = sorted(self._active, key=lambda r: self._priority(r, now))
        if order:
            oldest = min(self._active, key=lambda r: r.future.id)
            order.remove(oldest)
            order.insert(0, oldest)
        batched = {}  # adaptive requests by module: their next chunks go out as one grid
        for req in order:
            if req.cancel or not req.chunks or req.copying is not None:
                continue
            if self._batches and req.kind == "sweep" and getattr(req.launch, "adaptive", False):
                batched.setdefault(str(req.handle["module"].path), []).append(req)
                continue
            s = min(range(self.nstreams), key=lambda i: self._stream_load[i])
            if self._stream_load[s] >= 2:
                break
            chunk = req.chunks.popleft()
            try:
                ev = self.backend.launch(req, chunk, s)
            except Exception as exc:
                req.cancel = True
                req.future.error = repr(exc)
                continue
            self._stream_load[s] += 1
            req.inflight.append((ev, s, {}))
            progressed = True
        for reqs in batched.values():
            s = min(range(self.nstreams), key=lambda i: self._stream_load[i])
            if self._stream_load[s] >= 2:
                break
            reqs = reqs[:BATCH_MAX]
            items = [(req, req.chunks.popleft()) for req in reqs]
            try:
                ev, keep = self.backend.launch_batch(items, s)
            except Exception as exc:  # a rejected batch fails its requests only
                for req in reqs:
                    req.cancel = True
                    req.future.error = repr(exc)
                continue
            self._stream_load[s] += 1
            token = {"keep": keep}  # one launch: the stream load is released once
            for req in reqs:
                req.inflight.append((ev, s, token))
            self.stats["batched_launches"] += 1
            progressed = True
        return progressed

    def _complete(self):
        progressed = False
        for req in list(self._active):
            still = []
            for ev, s, token in req.inflight:
                if self.backend.query(ev):
                    if not token.get("done"):
                        token["done"] = True
                        token.pop("keep", None)
                        self._stream_load[s] -= 1
                    progressed = True
                else:
                    still.append((ev, s, token))
            req.inflight = still
            if req.inflight:
                continue
            if req.cancel:
                state = FAILED if req.future.error else CANCELLED
                self._retire(req, state, error=req.future.error)
                progressed = True
            elif not req.chunks:
                if req.copying is None:
                    req.copying = self.backend.copy_out(req, [])
                elif self.backend.query(req.copying):
                    out = self.backend.results(req)
                    self._retire(req, DONE, result=out)
                    progressed = True
        return progressed

    def _retire(self, req, state, result=None, error=None):
        self.backend.release(req)
        self._used -= req.nbytes
        with self._lock:
            self._active.remove(req)
        if state == DONE:
            self.stats["completed"] += 1
            self.stats["point_steps"] += req.point_steps
            result = _shape_outputs(req, result)
        elif state == FAILED:
            self.stats["failed"] += 1
        else:
            self.stats["cancelled"] += 1
        req.future._finish(state, result=result, error=error)

    def _loop(self):
        while True:
            self._admit()
            busy = self._dispatch()
            busy = self._complete() or busy
            with self._lock:
                idle = not self._active and not self._queue
            if self._stop and idle:
                return
            if not busy:
                time.sleep(self.poll_s)


_NOMINAL_FLOPS = 2e13  # flop/s that turn the algorithmic work of a request into seconds (priority only)


def _work_estimate(launch, kind, point_steps):
    """Estimated device seconds of a request: point-steps x the algorithmic flops of one point-step
    (the reduced RHS count, or the density-matrix formula), x 6 for an adjoint (fit) request."""
    try:
        frag = launch.entry["frag"]
        if frag.get("matrix"):
            per = float(frag["flops_per_point_step"])
        else:
            from . import emit
            per = 4.0 * emit.count_rhs_flops(frag) + 13.0 * frag["state_size"] + 2.0 * emit.count_drive_flops(frag)
    except Exception:  # launches without emitted code (test doubles, adjoint problems): point-steps alone
        per = 100.0
    return point_steps * per * (6.0 if kind == "adjoint" else 1.0) / _NOMINAL_FLOPS


def _shape_outputs(req, out):
    """Server outputs -> the shapes ``mesolve_2D`` returns (complex maps, state arrays, traces)."""
    launch = req.launch
    nx, ny = req.shape
    res = np.asarray(out["results"])
    if launch.output_mode in ("mean", "final"):
        r = res.reshape(nx, ny, 2)
        result = r[..., 0] + 1j * r[..., 1]
    else:
        result = res.reshape(nx, ny, launch.state_size)
    payload = {"result": result}
    if out.get("trace") is not None:
        tr = np.asarray(out["trace"])
        if launch.trace_mode == "observable":
            tr = tr.reshape(nx, ny, launch.num_trace, 2)
            payload["trace"] = tr[..., 0] + 1j * tr[..., 1]
        else:
            payload["trace"] = tr.reshape(nx, ny, launch.num_trace, launch.state_size)
    if out.get("step_counts") is not None:
        payload["step_counts"] = np.asarray(out["step_counts"]).reshape(nx, ny, 2)
    if out.get("grad") is not None:
        P = launch.P
        payload["result"] = payload["result"].real
        payload["grad"] = np.asarray(out["grad"])[:, :P].reshape(nx, ny, P)
        payload["params"] = launch.params
    return payload
