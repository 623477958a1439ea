"""Continuous-batching request loop for neighbour-graph jobs.

Requests (an embedding plus n_neighbors / metric / method) arrive at any time.  A scheduler
thread admits them, in arrival order, as soon as an execution slot is free and their device memory
fits the HBM budget; each slot's worker thread enqueues and completes its request.  Admitted requests run on their own CUDA streams, so the work of requests that arrive
while others are on the GPU overlaps on the device: small graphs share the SMs, and a large one
yields slots as its neighbours finish.  Embeddings are uploaded once and results stay in HBM as
device CSR tensors, ready for GPU consumers; a host copy is optional.

Every request's result is the exact graph, so it does not depend on what else was running
(``tests/test_gpu_serve.py`` checks alone-vs-mixed equality).  ``run_trace`` replays a Poisson
arrival trace and reports p50/p99 latency (arrival → result complete on the device and handed to
the caller; with ``to_host``, after the host copy) and cells/s;
``run_offline`` pushes the same requests back to back at full concurrency, the batched-offline
throughput that the served throughput is compared against.
"""

from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import CancelledError
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .neighbors import _torch, _ids, DEFAULT_PRECISION


@dataclass(eq=False)                   # requests compare by identity
class Request:
    X: object                      # host numpy (n, d) float32, or a CUDA tensor
    n_neighbors: int = 15
    metric: str = "euclidean"
    method: str = "umap"
    precision: str = DEFAULT_PRECISION
    to_host: bool = False
    arrival: float = 0.0           # seconds on the server clock (set by submit)
    rid: int = -1
    # filled in by the server
    admitted: float = 0.0
    done: float = 0.0
    result: dict = field(default_factory=dict)
    error: BaseException | None = None
    event: threading.Event = field(default_factory=threading.Event)
    # a CUDA embedding is read only after the work queued on its producer stream at submit time
    ready: object = None

    @property
    def n(self) -> int:
        return int(self.X.shape[0])

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def request_bytes(lib, n, d, k, metric, method, precision) -> int:
    """Device bytes one request holds while in flight: workspace + input + outputs."""
    mid, meth, pid = _ids(metric, method, precision)
    ws = lib.msc_neighbors_workspace_bytes(n, d, k, mid, meth, pid, 0)
    if ws == 0:
        return -1
    m = max(k - 1, 0)
    outs = n * k * 8 + 2 * (n + 1) * 8 + n * m * 8 + 2 * n * m * 8 + 64
    return int(ws + n * d * 4 + outs)


# pinned staging buffers of closed servers, handed to the next server of this process
# (page-locking host memory costs milliseconds per call; a new server would otherwise pay it
# again for every slot); a buffer belongs to one slot of one server at a time
_PINNED_POOL: list = []
_PINNED_LOCK = threading.Lock()


class GraphServer:
    """Admission by HBM budget and free slots; one CUDA stream and one worker thread per slot.

    The scheduler thread admits pending requests in arrival order and hands each to a free slot's
    worker.  The worker enqueues the graph on its slot's stream (the library call releases the
    GIL, so the host work of several slots runs on several cores), waits for it, checks it and
    completes the request, then frees the slot and the bytes."""

    def __init__(self, hbm_budget: int, slots: int = 8, device=None, poll_s: float = 2e-4,
                 pinned_bytes: int = 0, keep_results: bool = True):
        torch = _torch()
        self.torch = torch
        self.lib = _lib.load()
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.budget = int(hbm_budget)
        self.poll_s = poll_s
        # False: a completed request keeps only its checked stats (result["host_stats"])
        self.keep_results = keep_results
        self.slots = [torch.cuda.Stream(device=self.device) for _ in range(slots)]
        self.free_slots = collections.deque(range(slots))
        self.pending: collections.deque[Request] = collections.deque()
        self.inflight: dict[int, tuple[Request, int]] = {}
        self.in_use = 0
        self.lock = threading.Lock()
        self.cv = threading.Condition(self.lock)       # pending work, freed slots, stop
        self.t0 = time.perf_counter()
        self.completed: list[Request] = []
        self._next_id = 0
        self._stop = False
        self.peak_in_use = 0
        self.peak_inflight = 0
        with _PINNED_LOCK:                            # buffers of earlier servers, largest first
            _PINNED_POOL.sort(key=lambda b: b.numel())
            self._pinned = [_PINNED_POOL.pop() if _PINNED_POOL else None for _ in range(slots)]
        if pinned_bytes > 0 and hasattr(torch, "empty"):
            # staging for host embeddings up to pinned_bytes, page-locked now rather than while
            # requests wait
            size = 1 << max(20, (int(pinned_bytes) - 1).bit_length())
            for i, b in enumerate(self._pinned):
                if b is None or b.numel() < size:
                    self._pinned[i] = torch.empty(size, dtype=torch.uint8).pin_memory()
        # a scratch workspace per slot, kept across requests (a fresh one per request made the
        # caching allocator take new device segments for many request sizes on every slot stream)
        from .neighbors import Workspace
        self._ws = [Workspace(self.device, pow2=True) for _ in range(slots)]
        self._work = [collections.deque() for _ in range(slots)]
        self._work_cv = [threading.Condition(threading.Lock()) for _ in range(slots)]
        self._workers = [threading.Thread(target=self._worker, args=(i,), daemon=True)
                         for i in range(slots)]
        for t in self._workers:
            t.start()
        self._thread = threading.Thread(target=self._loop, daemon=True)
        self._thread.start()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def submit(self, req: Request) -> Request:
        """Queue ``req``.  A CUDA embedding may still be in the making on the caller's current
        stream: an event recorded there now is waited on by the request's own stream before it
        reads the tensor, and the tensor is kept alive for that stream until the graph is done."""
        torch = self.torch
        if isinstance(req.X, torch.Tensor) and req.X.is_cuda:
            req.ready = torch.cuda.Event()
            req.ready.record(torch.cuda.current_stream(req.X.device))
        with self.cv:
            req.arrival = self.now()
            req.rid = self._next_id
            self._next_id += 1
            self.pending.append(req)
            self.cv.notify_all()
        return req

    def cancel(self, req: Request) -> bool:
        """Withdraw a request that has not been admitted yet: it completes at once with a
        ``CancelledError`` and never reaches the GPU.  False if it was already admitted or done."""
        with self.cv:
            for i, r in enumerate(self.pending):
                if r is req:
                    del self.pending[i]
                    break
            else:
                return False
            req.error = CancelledError(f"request {req.rid} cancelled before admission")
            req.done = self.now()
            self.completed.append(req)
        req.event.set()
        return True

    def close(self):
        with self.cv:
            self._stop = True
            self.cv.notify_all()
        self._thread.join()
        for i, cv in enumerate(self._work_cv):
            with cv:
                self._work[i].append(None)             # the worker's sentinel
                cv.notify()
        for t in self._workers:
            t.join()
        with _PINNED_LOCK:                            # hand the staging buffers on
            _PINNED_POOL.extend(b for b in self._pinned if b is not None)
            self._pinned = [None] * len(self._pinned)

    # -- workers ------------------------------------------------------------------------------

    def _start(self, req: Request, slot: int):
        torch = self.torch
        st = self.slots[slot]
        from .neighbors import neighbors_device
        with torch.cuda.stream(st):
            X = req.X
            if not isinstance(X, torch.Tensor):
                X = torch.from_numpy(np.ascontiguousarray(X, np.float32))
            if X.is_cuda:
                if req.ready is not None:
                    st.wait_event(req.ready)          # the producer's writes come first
                X.record_stream(st)                   # its memory stays live for this stream
                Xd = X if X.device == self.device else X.to(self.device)
            else:
                Xd = self._upload(X, slot)
            res = neighbors_device(Xd, req.n_neighbors, metric=req.metric, method=req.method,
                                   precision=req.precision, workspace=self._ws[slot])
            res["X"] = Xd
            if req.to_host:
                res["host_stats"] = res["stats"].to("cpu", non_blocking=True)
            # a blocking-sync event: the slot's worker sleeps while it waits instead of spinning
            # on a host core (with a spin per slot the workers starve the threads enqueuing work)
            ev = torch.cuda.Event(blocking=True)
            ev.record(st)
        req.result = res
        return ev

    def _upload(self, X, slot: int):
        """Host embedding -> device on the slot's stream through the slot's pinned buffer (grown
        on demand, reused: the slot's previous request finished before this one started), so the
        copy is asynchronous instead of a blocking copy from pageable memory."""
        torch = self.torch
        if not hasattr(torch, "empty") or not hasattr(X, "numel"):
            return X.to(self.device, non_blocking=True)          # stand-ins in host-only tests
        buf = self._pinned[slot]
        nbytes = X.numel() * 4
        if buf is None or buf.numel() < nbytes:
            # grown to a power of two, so that a slot re-pins only a few times as sizes vary
            size = 1 << max(20, (nbytes - 1).bit_length())
            buf = torch.empty(size, dtype=torch.uint8).pin_memory()
            self._pinned[slot] = buf
        staged = buf[:nbytes].view(torch.float32).view(X.shape)
        staged.copy_(X)
        return staged.to(self.device, non_blocking=True)

    def _wait(self, ev):
        if hasattr(ev, "synchronize"):
            ev.synchronize()                          # blocks without holding the GIL
            return
        while not ev.query():
            time.sleep(self.poll_s)

    def _release(self, req: Request, slot: int, need: int):
        with self.cv:
            self.inflight.pop(slot, None)
            self.in_use -= need
            self.free_slots.append(slot)
            self.completed.append(req)
            self.cv.notify_all()
        req.event.set()

    def _worker(self, slot: int):
        torch = self.torch
        torch.cuda.set_device(self.device)
        q, cv = self._work[slot], self._work_cv[slot]
        while True:
            with cv:
                while not q:
                    cv.wait()
                item = q.popleft()
            if item is None:
                return
            req, need = item
            try:
                ev = self._start(req, slot)
            except BaseException as e:               # e.g. an allocation failure at start
                req.error = e
                req.done = self.now()
                self._release(req, slot, need)
                continue
            self._wait(ev)
            req.done = self.now()
            stats = None
            try:
                stats = req.result["stats"].cpu().numpy()
                _lib.check_stats(stats)
                if req.to_host:
                    from .neighbors import graph_to_host
                    req.result["host"] = graph_to_host(req.result, req.n, req.n_neighbors)
                    req.done = self.now()
            except BaseException as e:                # report per request, keep serving
                req.error = e
            if not self.keep_results:
                # a consumer that only needs the outcome: the device buffers go back to the
                # allocator now instead of piling up until the caller drops the request
                req.result = {"host_stats": stats}
            self._release(req, slot, need)

    # -- scheduler ------------------------------------------------------------------------------

    def _loop(self):
        while True:
            with self.cv:
                while True:
                    if self._stop and not self.pending and not self.inflight:
                        return
                    if self.pending and self.free_slots:
                        break
                    self.cv.wait(0.05)
                req = self.pending[0]
            need = request_bytes(self.lib, req.n, int(req.X.shape[1]), req.n_neighbors,
                                 req.metric, req.method, req.precision)
            with self.cv:
                if not self.pending or self.pending[0] is not req:
                    continue                           # cancelled meanwhile
                if need < 0 or need > self.budget:
                    self.pending.popleft()
                    req.error = ValueError(f"request needs {need} bytes > budget {self.budget}")
                    req.done = self.now()
                    self.completed.append(req)
                    req.event.set()
                    continue
                while self.in_use + need > self.budget or not self.free_slots:
                    self.cv.wait(0.05)                 # FIFO: the head waits for memory
                    if not self.pending or self.pending[0] is not req:
                        break
                if not self.pending or self.pending[0] is not req:
                    continue
                self.pending.popleft()
                slot = self.free_slots.popleft()
                self.in_use += need
                self.peak_in_use = max(self.peak_in_use, self.in_use)
                self.inflight[slot] = (req, need)
                self.peak_inflight = max(self.peak_inflight, len(self.inflight))
                req.admitted = self.now()
            cv = self._work_cv[slot]
            with cv:
                self._work[slot].append((req, need))
                cv.notify()


def _percentile(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else float("nan")


def run_trace(reqs: list[Request], arrivals: list[float], hbm_budget: int, slots: int = 8,
              device=None, pinned_bytes: int = 0, keep_results: bool = True) -> dict:
    """Submit ``reqs`` at ``arrivals`` (seconds from start); wait for all; report latency and
    throughput.  ``pinned_bytes``: page-lock each slot's staging buffer for host embeddings of up
    to that size before the first arrival.  ``keep_results=False``: release every request's
    device results as soon as it completes (a consumer that takes each result and lets it go)."""
    srv = GraphServer(hbm_budget, slots, device, pinned_bytes=pinned_bytes,
                      keep_results=keep_results)
    t_start = srv.now()
    for r, a in zip(reqs, arrivals):
        delay = a - (srv.now() - t_start)
        if delay > 0:
            time.sleep(delay)
        srv.submit(r)
    for r in reqs:
        r.event.wait()
    srv.close()
    ok = [r for r in reqs if r.error is None]
    errors = [f"request {r.rid}: {type(r.error).__name__}: {str(r.error)[:300]}"
              for r in reqs if r.error is not None][:5]
    lat = [r.latency * 1e3 for r in ok]
    queue = [(r.admitted - r.arrival) * 1e3 for r in ok]        # waiting for a slot / memory
    service = [(r.done - r.admitted) * 1e3 for r in ok]         # admitted -> handed back
    makespan = max(r.done for r in reqs) - t_start
    cells = sum(r.n for r in ok)
    # the five slowest requests: what they were and where their time went
    slowest = [{"rid": r.rid, "n": r.n, "d": int(r.X.shape[1]), "k": r.n_neighbors,
                "arrival_s": round(r.arrival - t_start, 4),
                "queue_ms": round((r.admitted - r.arrival) * 1e3, 2),
                "service_ms": round((r.done - r.admitted) * 1e3, 2)}
               for r in sorted(ok, key=lambda r: -r.latency)[:5]]
    return {"requests": len(reqs), "failed": len(reqs) - len(ok),
            "p50_ms": _percentile(lat, 50), "p99_ms": _percentile(lat, 99),
            "mean_ms": float(np.mean(lat)) if lat else float("nan"),
            "queue_p50_ms": _percentile(queue, 50), "queue_p99_ms": _percentile(queue, 99),
            "service_p50_ms": _percentile(service, 50), "service_p99_ms": _percentile(service, 99),
            "cells_per_s": cells / makespan, "makespan_s": makespan,
            "peak_inflight": srv.peak_inflight, "peak_hbm_bytes": srv.peak_in_use,
            "errors": errors, "slowest": slowest}


def run_offline(reqs: list[Request], hbm_budget: int, slots: int = 8, device=None,
                pinned_bytes: int = 0, keep_results: bool = True) -> dict:
    """All requests available at t=0: the batched-offline throughput."""
    return run_trace(reqs, [0.0] * len(reqs), hbm_budget, slots, device, pinned_bytes,
                     keep_results)
