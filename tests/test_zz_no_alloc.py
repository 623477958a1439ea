"""msc_fuzzy_union_noalloc: the fuzzy union for callers that cannot give the library device
memory (code under a memory manager that owns the whole GPU, or a hot loop that must not call
cudaMalloc/cudaFree, which can synchronise the device).  It uses a fixed array in the library's
own device memory instead of a workspace.

Checked through the C ABI against msc_fuzzy_union (the workspace entry point) on two calls in a
row with different graphs, to the bit — the tolerance of every parity test in this suite.  This file
is collected last so a failure here cannot stop the rest of a `-x` run; it also passes alone in a
fresh process, where its first call is the one that looks up the array's device address.
"""
import numpy as np
import pytest

from msc_b200 import _lib

pytestmark = pytest.mark.gpu


def _graph(n, k, seed):
    """kNN indices and UMAP memberships of a seeded mixture, computed on the GPU."""
    import torch
    from msc_b200 import synth, neighbors as nbm
    lib = _lib.load()
    X = synth.gaussian_mixture(n, 20, 8, seed=seed)
    idx, dist, _ = nbm.knn_device(torch.from_numpy(X).cuda(), k)
    sigma = torch.empty(n, dtype=torch.float32, device="cuda")
    rho = torch.empty_like(sigma)
    ws = torch.empty(1025 * 8, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.msc_smooth_knn_dist(dist.data_ptr(), n, k, 1.0, sigma.data_ptr(),
                                       rho.data_ptr(), ws.data_ptr(), ws.numel(), st))
    w = torch.empty((n, k), dtype=torch.float32, device="cuda")
    _lib.check(lib.msc_membership(idx.data_ptr(), dist.data_ptr(), sigma.data_ptr(),
                                  rho.data_ptr(), n, k, w.data_ptr(), st))
    return idx, w


def _outputs(n, k):
    import torch
    cap = max(2 * n * (k - 1), 1)
    return (torch.empty(n + 1, dtype=torch.int64, device="cuda"),
            torch.empty(cap, dtype=torch.int32, device="cuda"),
            torch.empty(cap, dtype=torch.float32, device="cuda"),
            torch.empty(1, dtype=torch.int64, device="cuda"))


def _host(indptr, indices, data, nnz):
    import torch
    torch.cuda.synchronize()
    m = int(nnz.item())
    assert m == int(indptr[-1].item())
    return indptr.cpu().numpy(), indices[:m].cpu().numpy(), data[:m].cpu().numpy()


def _with_workspace(idx, w, n, k):
    import torch
    lib = _lib.load()
    nbytes = lib.msc_fuzzy_union_workspace_bytes(n, k)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    out = _outputs(n, k)
    _lib.check(lib.msc_fuzzy_union(idx.data_ptr(), w.data_ptr(), n, k, *[t.data_ptr() for t in out],
                                   ws.data_ptr(), nbytes, torch.cuda.current_stream().cuda_stream))
    return _host(*out)


def _no_alloc(idx, w, n, k):
    import torch
    lib = _lib.load()
    out = _outputs(n, k)
    _lib.check(lib.msc_fuzzy_union_noalloc(idx.data_ptr(), w.data_ptr(), n, k,
                                           *[t.data_ptr() for t in out],
                                           torch.cuda.current_stream().cuda_stream))
    return _host(*out)


def test_no_alloc_union_matches_workspace_entry_point_twice():
    # two calls in a row on different graphs: the shared array keeps the first call's contents,
    # which must not leak into the second result
    for n, k, seed in ((20_000, 15, 1), (7_000, 30, 2)):
        idx, w = _graph(n, k, seed)
        ref = _with_workspace(idx, w, n, k)
        got = _no_alloc(idx, w, n, k)
        for a, b, what in zip(got, ref, ("indptr", "indices", "data")):
            assert np.array_equal(a, b), f"n={n} k={k}: {what} differs"


def test_no_alloc_union_rejects_sizes_beyond_its_scratch():
    lib = _lib.load()
    n = 70_000                                     # > MSC_NOALLOC_MAX_CELLS
    rc = lib.msc_fuzzy_union_noalloc(1, 1, n, 15, 1, 1, 1, 1, None)
    assert rc == _lib.MSC_ERR_INVALID_ARG
    assert "scratch" in _lib.last_error()
    rc = lib.msc_fuzzy_union_noalloc(1, 1, 60_000, 20, 1, 1, 1, 1, None)   # n*k > 2^20
    assert rc == _lib.MSC_ERR_INVALID_ARG


def test_no_alloc_union_at_its_largest_documented_sizes():
    # the two corners of the accepted region: every cell at the cell limit, and the widest lists
    # at the entry limit; both must be accepted and equal the workspace entry point
    for n, k, seed in ((_lib.NOALLOC_MAX_CELLS, 16, 3),
                       (_lib.NOALLOC_MAX_ENTRIES // _lib.MAX_K, _lib.MAX_K, 4)):
        assert n * k <= _lib.NOALLOC_MAX_ENTRIES
        idx, w = _graph(n, k, seed)
        ref = _with_workspace(idx, w, n, k)
        got = _no_alloc(idx, w, n, k)
        for a, b, what in zip(got, ref, ("indptr", "indices", "data")):
            assert np.array_equal(a, b), f"n={n} k={k}: {what} differs"
