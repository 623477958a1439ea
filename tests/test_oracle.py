"""The CPU oracle against the reference's own known answers and against independent restatements.

Pins (the reference's own tests and code for this path):
* tests/test_postfix_fixes.py:108-121 — 500×20 N(0,1), default_rng(0), k ∈ {15, 33, 50}: recall
  ≥ 0.99 against NumPy brute force (`np.argsort(D)[:, :k]`); the oracle must be exact (1.0);
* tests/test_postfix_fixes.py:197-207 — 60×10 + 5 exact duplicates, k=10: finite connectivities;
* neighbors.py:457-461 — ties ordered by (distance, index); neighbors.py:129-131 — self first;
* neighbors.py:755-759 — distances CSR in SciPy canonical form with explicit zeros kept.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle


def brute(X):
    X64 = X.astype(np.float64)
    D = ((X64[:, None, :] - X64[None, :, :]) ** 2).sum(-1)
    return D


@pytest.mark.parametrize("k", [15, 33, 50])
def test_reference_recall_case_is_exact(k):
    rng = np.random.default_rng(0)
    X = rng.standard_normal((500, 20)).astype(np.float32)
    idx, d2, dist = oracle.knn_exact(X, k)
    D = np.sqrt(((X[:, None, :] - X[None, :, :]) ** 2).sum(-1))      # the reference test's own
    ref = np.argsort(D, axis=1)[:, :k]
    recall = np.mean([len(set(idx[i]) & set(ref[i])) / k for i in range(500)])
    assert idx.shape == (500, k) and recall == 1.0
    assert (idx[:, 0] == np.arange(500)).all()
    # independent FP64 brute force, (distance, index) order
    B = brute(X)
    np.fill_diagonal(B, np.inf)
    for i in range(0, 500, 37):
        o = np.lexsort((np.arange(500), B[i]))[: k - 1]
        assert np.array_equal(idx[i, 1:], o)
        np.testing.assert_allclose(dist[i, 1:], np.sqrt(B[i, o]).astype(np.float32), rtol=0)


def test_ties_by_index_and_self_first():
    X = np.zeros((6, 3), np.float32)
    X[3] = [1, 0, 0]
    idx, d2, dist = oracle.knn_exact(X, 4)
    # rows 0,1,2,4,5 coincide: self first, then the lowest other indices
    assert idx[0].tolist() == [0, 1, 2, 4]
    assert idx[4].tolist() == [4, 0, 1, 2]
    assert idx[3].tolist() == [3, 0, 1, 2]
    assert dist[0].tolist() == [0, 0, 0, 0]


def test_coincident_points_connectivities_finite():
    rng = np.random.default_rng(0)
    X = rng.standard_normal((60, 10)).astype(np.float32)
    Xd = np.vstack([X, X[:5]]).astype(np.float32)
    g = oracle.neighbors_graph(Xd, 10)
    conn = g["connectivities"]
    assert conn.shape == (65, 65) and np.isfinite(conn.data).all() and conn.nnz > 0
    assert (conn != conn.T).nnz == 0                      # symmetric
    assert conn.diagonal().sum() == 0


def test_distances_csr_canonical_with_explicit_zeros():
    X = np.zeros((5, 2), np.float32)
    X[4] = [3, 4]
    g = oracle.neighbors_graph(X, 3)
    Dm = g["distances"]
    assert Dm.has_canonical_format and Dm.nnz == 5 * 2
    assert (Dm.data == 0).sum() == 8                      # coincident cells kept as explicit 0
    assert Dm.indices.dtype == np.int32 and Dm.indptr.dtype == np.int32
    assert Dm.data.dtype == np.float32


def test_fuzzy_union_matches_dense_restatement():
    """P = A + Aᵀ − A∘Aᵀ against an element-by-element float32 restatement."""
    rng = np.random.default_rng(5)
    X = rng.standard_normal((300, 8)).astype(np.float32)
    g = oracle.neighbors_graph(X, 12)
    n, k = 300, 12
    A = np.zeros((n, n), np.float32)
    A[np.repeat(np.arange(n), k), g["idx"].ravel()] = g["w"].ravel()
    P = g["connectivities"].toarray()
    for i in range(0, n, 7):
        for j in range(n):
            a, b = A[i, j], A[j, i]
            exp = np.float32(np.float32(a + b) - np.float32(a * b)) if a and b else (a or b)
            assert P[i, j] == np.float32(exp)


def test_smooth_knn_dist_properties():
    rng = np.random.default_rng(2)
    X = rng.standard_normal((400, 12)).astype(np.float32)
    idx, d2, dist = oracle.knn_exact(X, 15)
    sigma, rho = oracle.smooth_knn_dist(dist, 15.0)
    assert np.array_equal(rho, dist[:, 1])                # first non-zero distance
    # the bisection target: Σ_{j≥1} exp(-(d-ρ)/σ) = log2(k) within the tolerance
    s = np.exp(-np.maximum(dist[:, 1:] - rho[:, None], 0) / sigma[:, None]).sum(1)
    assert np.abs(s - np.log2(15)).max() < 2e-4
    w = oracle.membership_strengths(idx, dist, sigma, rho)
    assert (w[:, 0] == 0).all() and (w[:, 1] == 1).all()


def test_local_connectivity_interpolation():
    D = np.array([[0.0, 0.0, 1.0, 2.0, 4.0]], np.float32)
    s1, r1 = oracle.smooth_knn_dist(D, 5.0, local_connectivity=1.0)
    s2, r2 = oracle.smooth_knn_dist(D, 5.0, local_connectivity=1.5)
    assert r1[0] == 1.0 and r2[0] == np.float32(1.5)
    s0, r0 = oracle.smooth_knn_dist(np.zeros((1, 5), np.float32), 5.0)
    assert r0[0] == 0.0


def test_gauss_symmetric_and_in_range():
    X = np.random.default_rng(4).standard_normal((400, 6)).astype(np.float32)
    g = oracle.neighbors_graph(X, 10, method="gauss")
    W = g["connectivities"]
    assert (W != W.T).nnz == 0
    assert (W.data >= 0).all() and (W.data <= 1).all()
    # structure = kNN edges ∪ reverse edges, self excluded
    n = 400
    E = sp.csr_matrix((np.ones(n * 9), (np.repeat(np.arange(n), 9), g["idx"][:, 1:].ravel())),
                      shape=(n, n))
    S = ((E + E.T) > 0).astype(np.int8)
    assert np.array_equal(S.indices, W.indices) and np.array_equal(S.indptr, W.indptr)


def test_cosine_definition():
    X = np.random.default_rng(9).standard_normal((200, 7)).astype(np.float32)
    idx, d2, dist = oracle.knn_exact(X, 5, metric="cosine")
    Xn = X / np.linalg.norm(X, axis=1, keepdims=True)
    cos = 1.0 - (Xn[0] @ Xn[idx[0, 1:]].T)
    np.testing.assert_allclose(dist[0, 1:], cos, rtol=1e-5, atol=1e-6)
