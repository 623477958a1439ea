"""Serving loop: continuous batching with HBM admission; every result must be the same alone and
in the mix (and equal to the oracle)."""
import numpy as np
import pytest

import oracle
from msc_b200 import serve, synth, neighbors as nbm

pytestmark = pytest.mark.gpu


def make_requests(seed=0, count=24):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        n = int(rng.choice([600, 1500, 4000, 9000, 20000]))
        d = int(rng.choice([30, 50, 100]))
        k = int(rng.choice([10, 15, 30]))
        metric = str(rng.choice(["euclidean", "cosine"]))
        X = synth.gaussian_mixture(n, d, int(rng.integers(3, 12)), seed=seed * 1000 + i,
                                   normalize=metric == "cosine")
        reqs.append(serve.Request(X=X, n_neighbors=k, metric=metric))
    return reqs


def host_result(r):
    import torch
    torch.cuda.synchronize()
    return (r.result["knn_idx"].cpu().numpy(), r.result["knn_dist"].cpu().numpy(),
            *nbm.graph_to_host(r.result, r.n, r.n_neighbors))


def test_mixed_equals_alone_and_oracle():
    reqs = make_requests(3, 16)
    budget = 8 << 30
    # in the mix: Poisson arrivals, 6 slots
    arrivals = np.cumsum(np.random.default_rng(1).exponential(0.002, len(reqs))).tolist()
    rep = serve.run_trace(reqs, arrivals, budget, slots=6)
    assert rep["failed"] == 0 and rep["peak_inflight"] >= 2
    mixed = [host_result(r) for r in reqs]
    # alone: one request at a time
    alone_reqs = [serve.Request(X=r.X, n_neighbors=r.n_neighbors, metric=r.metric)
                  for r in reqs]
    serve.run_trace(alone_reqs, [0.0] * len(alone_reqs), budget, slots=1)
    for a, m in zip((host_result(r) for r in alone_reqs), mixed):
        assert np.array_equal(a[0], m[0]) and np.array_equal(a[1], m[1])
        for ca, cm in ((a[2], m[2]), (a[3], m[3])):
            assert np.array_equal(ca.indptr, cm.indptr)
            assert np.array_equal(ca.indices, cm.indices)
            assert np.array_equal(ca.data, cm.data)
    # and against the oracle for two of them
    for r, res in list(zip(reqs, mixed))[:2]:
        ref = oracle.neighbors_graph(r.X, r.n_neighbors, metric=r.metric)
        assert np.array_equal(res[0], ref["idx"].astype(np.int32))
        assert np.array_equal(res[3].data, ref["connectivities"].data)


def test_admission_respects_budget():
    reqs = make_requests(5, 10)
    lib_bytes = [serve.request_bytes(__import__("msc_b200")._lib.load(), r.n, r.X.shape[1],
                                     r.n_neighbors, r.metric, r.method, r.precision) for r in reqs]
    budget = int(max(lib_bytes) * 1.5)            # at most ~one large request at a time
    rep = serve.run_trace(reqs, [0.0] * len(reqs), budget, slots=8)
    assert rep["failed"] == 0
    assert rep["peak_hbm_bytes"] <= budget
    too_big = serve.Request(X=synth.gaussian_mixture(30000, 50, 5, seed=9), n_neighbors=15)
    rep2 = serve.run_trace([too_big], [0.0], 1 << 20, slots=2)
    assert rep2["failed"] == 1 and isinstance(too_big.error, ValueError)


def test_concurrent_launches_of_different_widths():
    """Host threads on their own streams launch graphs of different widths d (hence different
    shared-memory sizes of the same kernels) at once.  A kernel's shared-memory cap is one
    process-wide attribute: a thread lowering it between another thread's set and launch made
    that launch fail.  Every call must succeed and match its single-thread result."""
    import threading
    import torch
    shapes = [(700, 30, 10), (900, 50, 15), (800, 100, 30), (600, 50, 10)]
    Xs = [torch.from_numpy(synth.gaussian_mixture(n, d, 4, seed=40 + i)).cuda()
          for i, (n, d, _) in enumerate(shapes)]
    alone = []
    for X, (_, _, k) in zip(Xs, shapes):
        r = nbm.neighbors_device(X, k)
        torch.cuda.synchronize()
        alone.append((r["knn_idx"].cpu(), r["knn_dist"].cpu()))
    errors, mismatches = [], []

    def worker(t):
        st = torch.cuda.Stream()
        ws = nbm.Workspace(torch.device("cuda", 0))
        try:
            for it in range(24):
                j = (t + it) % len(shapes)
                with torch.cuda.stream(st):
                    r = nbm.neighbors_device(Xs[j], shapes[j][2], workspace=ws)
                st.synchronize()
                if not (torch.equal(r["knn_idx"].cpu(), alone[j][0])
                        and torch.equal(r["knn_dist"].cpu(), alone[j][1])):
                    mismatches.append((t, it, j))
        except Exception as e:                      # noqa: BLE001 (reported below)
            errors.append(f"thread {t}: {type(e).__name__}: {e}")

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(8)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors[:3]
    assert not mismatches, mismatches[:5]
