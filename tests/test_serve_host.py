"""Host logic of the serving loop (``msc_b200.serve.GraphServer``) with the GPU replaced by a
fake: streams, events and the graph computation are stand-ins, so the scheduler's admission by
HBM budget and free slots, its FIFO order, and its handling of host-side faults (an oversize
request, an allocation failure when a request starts, a request cancelled before admission) run
on the CPU.  The GPU lane checks the real thing (tests/test_gpu_serve.py)."""
import contextlib
import time
from concurrent.futures import CancelledError

import numpy as np
import pytest

from msc_b200 import serve, neighbors as nbm


class _Tensor:
    def __init__(self, a, cuda=False):
        self.a = np.asarray(a)
        self.is_cuda = cuda
        self.shape = self.a.shape

    def to(self, *args, **kw):
        return _Tensor(self.a, cuda=True)

    def cpu(self):
        return _Tensor(self.a)

    def numpy(self):
        return self.a


class _Event:
    """Completes a fixed time after it is recorded (the fake request's device time)."""
    work_s = 0.02

    def __init__(self, **flags):
        self.t = None

    def record(self, stream):
        self.t = time.perf_counter()

    def query(self):
        return time.perf_counter() - self.t >= self.work_s


class _Cuda:
    Event = _Event

    @staticmethod
    def Stream(device=None):
        return object()

    @staticmethod
    @contextlib.contextmanager
    def stream(st):
        yield

    @staticmethod
    def set_device(d):
        pass

    @staticmethod
    def current_device():
        return 0


class _Torch:
    Tensor = _Tensor
    cuda = _Cuda

    @staticmethod
    def device(*a):
        return ("cuda", 0)

    @staticmethod
    def from_numpy(a):
        return _Tensor(a)


@pytest.fixture
def fake_gpu(monkeypatch):
    """Fake device; each request's footprint is its cell count in bytes; compute calls logged.
    A request whose n is 13 fails to start (an allocation failure)."""
    calls = []

    def fake_neighbors_device(X, n_neighbors, **kw):
        calls.append(int(X.shape[0]))
        if X.shape[0] == 13:
            raise MemoryError("out of device memory (injected)")
        return {"stats": _Tensor(np.zeros(8, np.int64), cuda=True)}

    monkeypatch.setattr(serve, "_torch", lambda: _Torch)
    monkeypatch.setattr(nbm, "neighbors_device", fake_neighbors_device)
    monkeypatch.setattr(serve, "request_bytes",
                        lambda lib, n, d, k, metric, method, precision: n)
    return calls


def _req(n):
    return serve.Request(X=np.zeros((n, 4), np.float32), n_neighbors=3)


def _wait(reqs, timeout=10.0):
    for r in reqs:
        assert r.event.wait(timeout), "request never completed"


def test_budget_and_slots_bound_the_work_in_flight(fake_gpu):
    srv = serve.GraphServer(hbm_budget=100, slots=3)
    reqs = [srv.submit(_req(40)) for _ in range(6)]
    _wait(reqs)
    srv.close()
    assert all(r.error is None for r in reqs)
    assert srv.peak_in_use <= 100 and srv.peak_inflight <= 2      # 2 x 40 fit, 3 do not
    assert srv.in_use == 0 and len(srv.free_slots) == 3
    # FIFO: admitted in submission order
    assert [r.rid for r in sorted(reqs, key=lambda r: r.admitted)] == [r.rid for r in reqs]
    assert fake_gpu == [40] * 6


def test_oversize_request_is_refused_and_the_rest_run(fake_gpu):
    srv = serve.GraphServer(hbm_budget=100, slots=2)
    reqs = [srv.submit(_req(n)) for n in (30, 500, 30)]
    _wait(reqs)
    srv.close()
    assert isinstance(reqs[1].error, ValueError) and "budget" in str(reqs[1].error)
    assert reqs[0].error is None and reqs[2].error is None
    assert fake_gpu == [30, 30]                                   # never started


def test_allocation_failure_releases_its_slot_and_budget(fake_gpu):
    srv = serve.GraphServer(hbm_budget=100, slots=1)
    reqs = [srv.submit(_req(n)) for n in (20, 13, 20, 20)]
    _wait(reqs)
    srv.close()
    assert isinstance(reqs[1].error, MemoryError)
    assert all(r.error is None for i, r in enumerate(reqs) if i != 1)
    assert srv.in_use == 0 and list(srv.free_slots) == [0]


def test_cancel_before_admission(fake_gpu):
    _Event.work_s = 0.2
    try:
        srv = serve.GraphServer(hbm_budget=50, slots=1)
        first = srv.submit(_req(50))                 # occupies the only slot for 0.2 s
        time.sleep(0.05)
        queued = [srv.submit(_req(n)) for n in (41, 42, 43)]
        assert srv.cancel(queued[1]) is True
        assert srv.cancel(queued[1]) is False        # already withdrawn
        _wait([first] + queued)
        assert srv.cancel(first) is False            # already done
        srv.close()
    finally:
        _Event.work_s = 0.02
    assert isinstance(queued[1].error, CancelledError)
    assert first.error is None and queued[0].error is None and queued[2].error is None
    assert fake_gpu == [50, 41, 43]                  # the cancelled request never started


def test_results_released_when_not_kept(fake_gpu):
    srv = serve.GraphServer(hbm_budget=100, slots=2, keep_results=False)
    reqs = [srv.submit(_req(n)) for n in (20, 30)]
    _wait(reqs)
    srv.close()
    assert all(r.error is None for r in reqs)
    for r in reqs:
        assert set(r.result) == {"host_stats"}
        assert np.array_equal(r.result["host_stats"], np.zeros(8, np.int64))
