"""The default path at the headline size (1,300,000 cells × 50 PCs, k=15: the scale workload),
checked through properties that hold at any size and against the oracle on a seeded sample of
rows (the oracle scans all 1.3M cells for each sampled row).

* every row certified or re-scanned, no device wait gave up, no non-finite input;
* kNN lists: self first at distance 0, then k-1 distinct other cells at ascending distance —
  and bit-identical to the oracle, ties included, on 192 seeded rows;
* distances CSR: row i holds exactly knn row i's columns 1..k-1, column-sorted (the oracle's
  ``distances_csr`` of those rows);
* connectivities: symmetric, no diagonal, values in (0, 1], n(k-1) <= nnz <= 2n(k-1);
* the whole graph: the oracle's ρ/σ, memberships, fuzzy union and distances CSR, run on the host
  over all 1.3M of the GPU's kNN lists (which the sampled rows pin to the oracle's exact kNN),
  equal the GPU's connectivities and distances CSR bit for bit — every row, not a sample.
"""
import numpy as np
import pytest

import oracle
from msc_b200 import neighbors as nbm, synth, _lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scale_graph():
    import torch
    X, p = synth.scale_1m3()
    Xd = torch.from_numpy(X).cuda()
    res = nbm.neighbors_device(Xd, p["n_neighbors"], metric=p["metric"], method=p["method"])
    torch.cuda.synchronize()
    host = {k: v.cpu().numpy() for k, v in res.items()}
    del Xd, res
    torch.cuda.empty_cache()
    return X, p["n_neighbors"], host


def test_full_size_stats(scale_graph):
    X, k, g = scale_graph
    n = X.shape[0]
    st = g["stats"]
    assert int(st[_lib.STAT_TIMEOUT]) == 0 and int(st[_lib.STAT_NONFINITE]) == 0
    assert int(st[_lib.STAT_CERTIFIED]) + int(st[_lib.STAT_RESCANNED]) >= n
    assert int(st[_lib.STAT_PRECISION]) == _lib.PRECISION[nbm.DEFAULT_PRECISION]


def test_full_size_lists(scale_graph):
    X, k, g = scale_graph
    n = X.shape[0]
    idx, dist = g["knn_idx"], g["knn_dist"]
    assert idx.shape == (n, k) and dist.shape == (n, k)
    assert (idx[:, 0] == np.arange(n)).all() and (dist[:, 0] == 0).all()
    assert idx.min() >= 0 and idx.max() < n
    # ascending float32 distances (the order is by the FP64 squared distance, then the index, so
    # equal float32 values may come in either index order; the sampled rows check ties exactly)
    assert (np.diff(dist, axis=1) >= 0).all()
    s = np.sort(idx, axis=1)
    assert (np.diff(s, axis=1) > 0).all()                  # no cell twice in a row


def test_full_size_rows_match_oracle(scale_graph):
    X, k, g = scale_graph
    n = X.shape[0]
    rows = np.sort(np.random.default_rng(20261203).choice(n, 192, replace=False))
    ridx, _, rdist = oracle.knn_exact(X, k, rows=rows)
    np.testing.assert_array_equal(g["knn_idx"][rows], ridx.astype(np.int32))
    np.testing.assert_array_equal(g["knn_dist"][rows], rdist)
    # distances CSR rows of the sampled cells: the oracle's construction of those rows
    ptr, ind, dat = g["dist_indptr"], g["dist_indices"], g["dist_data"]
    assert ptr[n] == n * (k - 1)
    for r, i in enumerate(rows):
        a, b = int(ptr[i]), int(ptr[i + 1])
        o = np.argsort(ridx[r, 1:])
        np.testing.assert_array_equal(ind[a:b], ridx[r, 1:][o].astype(np.int32))
        np.testing.assert_array_equal(dat[a:b], rdist[r, 1:][o])


def test_full_size_connectivities(scale_graph):
    import scipy.sparse as sp
    X, k, g = scale_graph
    n = X.shape[0]
    ptr = g["conn_indptr"]
    nnz = int(ptr[n])
    assert n * (k - 1) <= nnz <= 2 * n * (k - 1)
    C = sp.csr_matrix((g["conn_data"][:nnz], g["conn_indices"][:nnz], ptr), shape=(n, n))
    assert C.has_sorted_indices
    assert (C.data > 0).all() and (C.data <= 1).all()
    assert C.diagonal().sum() == 0
    D = (C - C.T).tocsr()
    D.eliminate_zeros()
    assert D.nnz == 0                                     # symmetric, values bit-equal


def test_full_size_whole_graph_matches_oracle(scale_graph):
    import scipy.sparse as sp
    X, k, g = scale_graph
    n = X.shape[0]
    idx, dist = g["knn_idx"], g["knn_dist"]
    sigma, rho = oracle.smooth_knn_dist(dist, k)
    w = oracle.membership_strengths(idx, dist, sigma, rho)
    ref_conn = oracle.fuzzy_union(idx, w, n)
    ref_dist = oracle.distances_csr(idx, dist, n)
    for what, (ptr, ind, dat), ref in (
            ("connectivities", (g["conn_indptr"], g["conn_indices"], g["conn_data"]), ref_conn),
            ("distances", (g["dist_indptr"], g["dist_indices"], g["dist_data"]), ref_dist)):
        nnz = int(ptr[n])
        assert nnz == ref.nnz, what
        np.testing.assert_array_equal(ptr.astype(np.int64), ref.indptr.astype(np.int64), what)
        np.testing.assert_array_equal(ind[:nnz], ref.indices.astype(np.int32), what)
        np.testing.assert_array_equal(dat[:nnz], ref.data, what)
