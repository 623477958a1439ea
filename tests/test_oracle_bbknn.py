"""The batch-balanced kNN oracle (oracle/bbknn.py) against the reference's own test and against
independent statements of the same graph.

* tests/test_postfix_fixes.py:186-193 — 60×10 N(0,1), batches of 40 / 2 / 18 cells, three
  neighbours per batch: a batch smaller than that must not fail, and the graph is 60×60, non-empty;
* neighbors.py:516-539 — every cell gets min(k, |b|) cells of every batch b, exact here;
* with one batch the untrimmed graph is the ``pp.neighbors`` graph of the same k (same lists, same
  fuzzy set), which the kNN and fuzzy-set pins already cover;
* neighbors.py:554-557 — distances without the diagonal and without zero entries;
* neighbors.py:465-488 — trimming keeps a symmetric graph symmetric (bit-exact against the
  reference's function in test_golden.py).
"""
import numpy as np

import oracle
from oracle import bbknn as obb


def test_reference_tiny_batch_case():
    X = np.random.default_rng(0).standard_normal((60, 10)).astype(np.float32)
    batch = np.array(["a"] * 40 + ["b"] * 2 + ["c"] * 18)
    dist_m, conn, K, inter = obb.bbknn(X, batch, neighbors_within_batch=3)
    assert K == 3 + 2 + 3 and inter["kk"].tolist() == [3, 2, 3]
    assert conn.shape == (60, 60) and conn.nnz > 0 and np.isfinite(conn.data).all()
    assert conn.data.dtype == np.float32 and conn.diagonal().sum() == 0
    idx, dist = inter["idx"], inter["dist"]
    # self first at distance 0, rows ascending, kk cells of every batch in every row
    assert (idx[:, 0] == np.arange(60)).all() and (dist[:, 0] == 0).all()
    assert (np.diff(dist, axis=1) >= 0).all()
    codes = np.searchsorted(np.array(["a", "b", "c"]), batch)
    for i in range(60):
        assert np.bincount(codes[idx[i]], minlength=3).tolist() == [3, 2, 3]
    # the 2-cell batch: both cells are in every row
    assert all({40, 41} <= set(idx[i].tolist()) for i in range(60))
    assert dist_m.diagonal().sum() == 0 and (dist_m.data > 0).all()
    assert dist_m.has_canonical_format and dist_m.nnz == 60 * K - 60


def test_knn_cross_is_brute_force():
    rng = np.random.default_rng(3)
    Q = rng.standard_normal((70, 9)).astype(np.float32)
    B = rng.standard_normal((45, 9)).astype(np.float32)
    B[7] = B[30]                                      # a tie: the lower index first
    idx, d2, dist = obb.knn_cross(Q, B, 6)
    D = ((Q.astype(np.float64)[:, None, :] - B.astype(np.float64)[None]) ** 2).sum(-1)
    for i in range(70):
        o = np.lexsort((np.arange(45), D[i]))[:6]
        assert idx[i].tolist() == o.tolist()
        np.testing.assert_allclose(d2[i], D[i, o], rtol=1e-14)
        if 30 in o:
            assert 7 in o and o.tolist().index(7) < o.tolist().index(30)
    assert dist.dtype == np.float32
    np.testing.assert_array_equal(dist, np.sqrt(d2).astype(np.float32))


def test_single_batch_is_the_neighbors_graph():
    X = np.random.default_rng(5).standard_normal((300, 8)).astype(np.float32)
    k = 12
    dist_m, conn, K, inter = obb.bbknn(X, np.zeros(300, np.int64), neighbors_within_batch=k,
                                       trim=0)
    g = oracle.neighbors_graph(X, k)
    assert K == k
    np.testing.assert_array_equal(inter["idx"], g["idx"])
    np.testing.assert_array_equal(inter["dist"], g["dist"])
    for a, b in ((conn, g["connectivities"]), (dist_m, g["distances"])):
        a, b = a.tocsr(), b.tocsr()
        a.sort_indices(); b.sort_indices()
        np.testing.assert_array_equal(a.indptr, b.indptr)
        np.testing.assert_array_equal(a.indices, b.indices)
        np.testing.assert_array_equal(a.data, b.data)


def test_coincident_cells_across_batches():
    X = np.random.default_rng(8).standard_normal((90, 6)).astype(np.float32)
    X[60:70] = X[0:10]                                # copies of batch-0 cells in batch 2
    batch = np.repeat([0, 1, 2], 30)
    dist_m, conn, K, inter = obb.bbknn(X, batch, neighbors_within_batch=4)
    assert K == 12
    # a copy is at distance 0: in the lists, not in the distances matrix
    assert inter["dist"][0, :2].tolist() == [0.0, 0.0]
    assert set(inter["idx"][0, :2].tolist()) == {0, 60}
    assert dist_m[0, 60] == 0 and (dist_m.data > 0).all()
    assert np.isfinite(conn.data).all() and (conn != conn.T).nnz == 0


def test_trim_keeps_symmetry_and_respects_thresholds():
    X = np.random.default_rng(11).standard_normal((400, 10)).astype(np.float32)
    batch = np.random.default_rng(12).integers(0, 4, 400)
    _, _, K, inter = obb.bbknn(X, batch, neighbors_within_batch=4)
    A = inter["untrimmed"].tocsr()
    assert (A != A.T).nnz == 0
    for t in (5, 9, 16):
        T = obb.trim_graph(A, t)
        assert (T != T.T).nnz == 0
        assert T.nnz < A.nnz
        # every row that had more than t edges keeps at most its t strongest values' ties
        cnt = np.diff(A.indptr)
        for i in np.flatnonzero(cnt > t)[:50]:
            row = np.sort(A.data[A.indptr[i]:A.indptr[i + 1]])
            kept = T.data[T.indptr[i]:T.indptr[i + 1]]
            assert (kept >= row[-t]).all()
    # no trim, or a trim above every row's count: unchanged
    for t in (None, 0, 10 * K):
        T = obb.trim_graph(A, t)
        assert (T != A).nnz == 0


def test_edge_batches():
    rng = np.random.default_rng(21)
    X = rng.standard_normal((200, 5)).astype(np.float32)
    # a one-cell batch: every row holds that cell; its own row holds only itself from its batch
    batch = np.array([0] * 199 + [1])
    _, conn, K, inter = obb.bbknn(X, batch, neighbors_within_batch=4)
    assert K == 4 + 1 and inter["kk"].tolist() == [4, 1]
    assert all(199 in inter["idx"][i].tolist() for i in range(200))
    assert conn.nnz > 0 and np.isfinite(conn.data).all()
    # neighbors_within_batch = 1: a cell of batch b gets itself from b
    batch = rng.integers(0, 3, 200)
    _, _, K, inter = obb.bbknn(X, batch, neighbors_within_batch=1)
    assert K == 3 and (inter["idx"][:, 0] == np.arange(200)).all()
    # 40 batches of 5 cells, 3 each: K = 120 (within the 128-entry limit of the GPU path)
    batch = np.repeat(np.arange(40), 5)
    _, conn, K, inter = obb.bbknn(X, batch, neighbors_within_batch=3)
    assert K == 120 and inter["idx"].shape == (200, 120)
    assert (np.diff(inter["dist"], axis=1) >= 0).all()
    # labels of any sortable type give the same graph as their codes
    labels = np.array([f"s{b:02d}" for b in batch])
    _, conn2, _, _ = obb.bbknn(X, labels, neighbors_within_batch=3)
    assert (conn != conn2).nnz == 0
