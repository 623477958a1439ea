"""Batch-balanced kNN oracle.  TEST INFRASTRUCTURE ONLY — see ``oracle/__init__.py``.

Restates metalsinglecell ``neighbors.bbknn`` (neighbors.py:491-559) and its ``_trim_graph``
(neighbors.py:465-488), called by ``pp.bbknn`` (pp.py:809-833):

1. the representation is sliced to its first ``n_pcs`` columns (neighbors.py:506-507);
2. for every batch b (the sorted unique labels, neighbors.py:510,516), every cell — of any
   batch — gets its ``kk = min(neighbors_within_batch, |b|)`` nearest cells of b
   (neighbors.py:516-539).
   A cell of b finds itself at distance 0.  Exact here, like ``knn.knn_exact``: FP64 squared
   distance of the float32 inputs, ties to the lower cell index, distance = float32 of the FP64
   square root.  (The reference ranks and reports the FP32 Gram form |x|²+|y|²−2x·y; that form's
   rounding is the only difference, and it can give a cell a small non-zero distance to itself.)
3. the per-batch lists are concatenated and every row sorted by distance (neighbors.py:541-545).
   The reference's ``np.argsort`` leaves the order of equal distances unspecified; nothing
   downstream depends on it (equal distances give equal terms and memberships), and this oracle
   orders them by cell index;
4. connectivities: the umap fuzzy simplicial set with n_neighbors = K = Σ_b kk, the width of the
   combined lists (neighbors.py:547-553) — ``graph.smooth_knn_dist`` /
   ``graph.membership_strengths`` / ``graph.fuzzy_union``;
5. distances: the combined lists as a CSR matrix with the diagonal set to 0 and every zero
   eliminated (neighbors.py:554-557) — unlike ``pp.neighbors``, zero distances to coincident
   cells are dropped too;
6. connectivities trimmed to each cell's ``trim`` strongest edges, ``trim = 10·K`` by default
   (neighbors.py:558, :465-488): θ_i = the trim-th largest value of row i when the row holds more
   than ``trim`` entries (else 0); an edge (i, j) stays when its value is ≥ θ_i and ≥ θ_j (the
   reference applies the row thresholds to the rows, transposes, applies them again and
   transposes back).

Pinning: ``trim_graph`` is checked bit for bit against the reference's own ``_trim_graph`` run on
this machine (``tests/golden/make_golden.py`` → ``reference_trim.npz``).  The kNN lists follow
the exact semantics pinned for ``knn.knn_exact``.  The connectivity values go through the
umap-learn restatement, which no reference test pins (**parity unpinned**, as for
``pp.neighbors``).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .graph import smooth_knn_dist, membership_strengths, fuzzy_union
from .knn import sq_dist_f64


def _cross_full(Q32, B32, rows, kk):
    """Full FP64 scan of B for a few query rows, ordered by (d², B index)."""
    cols = np.arange(B32.shape[0])
    oi = np.empty((rows.size, kk), np.int64)
    od = np.empty((rows.size, kk), np.float64)
    for r, i in enumerate(rows):
        D = sq_dist_f64(Q32[i:i + 1], B32)[0]
        o = np.lexsort((cols, D))[:kk]
        oi[r] = o
        od[r] = D[o]
    return oi, od


def knn_cross(Q: np.ndarray, B: np.ndarray, kk: int, chunk_elems: int = 1 << 25):
    """Exact kk nearest rows of ``B`` for every row of ``Q``: ``(idx int64 (m,kk) into B,
    d2 float64 (m,kk), dist float32 (m,kk))``, ordered by (FP64 squared distance, B index).

    An FP64 Gram form |q|² + |b|² − 2q·b pre-selects kk+8 candidates per row; their distances are
    recomputed as FP64 sums of squared differences in dimension order, and a row whose kk-th
    recomputed value does not clear the pre-selection threshold by the Gram form's error bound
    is scanned in full."""
    Q32 = np.ascontiguousarray(Q, np.float32)
    B32 = np.ascontiguousarray(B, np.float32)
    m, nb = Q32.shape[0], B32.shape[0]
    d = Q32.shape[1]
    if not 0 <= kk <= nb:
        raise ValueError(f"kk={kk} must be in [0, {nb}]")
    idx = np.empty((m, kk), np.int64)
    d2 = np.empty((m, kk), np.float64)
    if kk == 0 or m == 0:
        return idx, d2, np.sqrt(d2).astype(np.float32)
    Q64, B64 = Q32.astype(np.float64), B32.astype(np.float64)
    sq_q = np.einsum("ij,ij->i", Q64, Q64)
    sq_b = np.einsum("ij,ij->i", B64, B64)
    sbmax = float(sq_b.max())
    eps64 = 64.0 * (d + 8) * 2.0 ** -53
    m_extra = min(nb, kk + 8)
    chunk = int(max(8, min(2048, chunk_elems // max(nb, 1))))
    for s in range(0, m, chunk):
        e = min(s + chunk, m)
        V = sq_q[s:e, None] + sq_b[None, :] - 2.0 * (Q64[s:e] @ B64.T)
        if m_extra < nb:
            cand = np.argpartition(V, m_extra - 1, axis=1)[:, :m_extra]
            thr = np.take_along_axis(V, cand, axis=1).max(axis=1)
        else:
            cand = np.broadcast_to(np.arange(nb), (e - s, nb))
            thr = np.full(e - s, np.inf)
        D = sq_dist_f64(Q32[s:e], B32[cand])
        o = np.lexsort((cand, D), axis=1)
        ci = np.take_along_axis(cand, o, axis=1)[:, :kk]
        cd = np.take_along_axis(D, o, axis=1)[:, :kk]
        err = eps64 * (sq_q[s:e] + sbmax)
        bad = np.flatnonzero(~(cd[:, kk - 1] < thr - 2.0 * err))
        if bad.size:
            bi, bd = _cross_full(Q32, B32, s + bad, kk)
            ci[bad] = bi
            cd[bad] = bd
        idx[s:e] = ci
        d2[s:e] = cd
    return idx, d2, np.sqrt(d2).astype(np.float32)


def trim_graph(conn: sp.spmatrix, trim: int | None) -> sp.csr_matrix:
    """Keep the non-zero entries (i, j) with value ≥ θ_i and ≥ θ_j; θ_i = the trim-th largest
    value of row i (its stored entries, explicit zeros included) if it stores more than ``trim``
    entries, else 0.  ``trim`` None or ≤ 0: unchanged.  (The reference zeroes the entries below
    the thresholds and eliminates zeros, which also drops stored zeros.)"""
    A = sp.csr_matrix(conn, copy=True)
    if trim is None or trim <= 0:
        return A
    n = A.shape[0]
    cnt = np.diff(A.indptr)
    theta = np.zeros(n, np.float64)
    for i in np.flatnonzero(cnt > trim):
        row = A.data[A.indptr[i]:A.indptr[i + 1]]
        theta[i] = np.partition(row, row.size - trim)[row.size - trim]
    rows = np.repeat(np.arange(n), cnt)
    keep = (A.data >= theta[rows]) & (A.data >= theta[A.indices]) & (A.data != 0)
    out = sp.csr_matrix((A.data[keep], (rows[keep], A.indices[keep])), shape=A.shape,
                        dtype=A.dtype)
    out.sort_indices()
    return out


def batch_codes(batch) -> tuple[np.ndarray, np.ndarray]:
    """(sorted unique labels, code of every cell) — the batch order of neighbors.py:510."""
    cats, codes = np.unique(np.asarray(batch), return_inverse=True)
    return cats, codes.astype(np.int64)


def bbknn_lists(X: np.ndarray, batch, neighbors_within_batch: int = 3,
                n_pcs: int | None = 50):
    """Steps 1-3: the combined, sorted kNN lists ``(idx int64 (n,K), dist float32 (n,K),
    kk per batch)``."""
    X32 = np.ascontiguousarray(X, np.float32)
    if n_pcs is not None:
        X32 = np.ascontiguousarray(X32[:, :n_pcs])
    n = X32.shape[0]
    cats, codes = batch_codes(batch)
    idx_parts, d_parts, kks = [], [], []
    for b in range(cats.size):
        members = np.flatnonzero(codes == b)
        kk = min(int(neighbors_within_batch), members.size)
        loc, _, dist = knn_cross(X32, X32[members], kk)
        idx_parts.append(members[loc])
        d_parts.append(dist)
        kks.append(kk)
    idx = np.concatenate(idx_parts, axis=1) if idx_parts else np.empty((n, 0), np.int64)
    dist = np.concatenate(d_parts, axis=1) if d_parts else np.empty((n, 0), np.float32)
    o = np.lexsort((idx, dist), axis=1)
    return (np.take_along_axis(idx, o, axis=1), np.take_along_axis(dist, o, axis=1),
            np.asarray(kks, np.int64))


def bbknn_distances(idx: np.ndarray, dist: np.ndarray, n: int) -> sp.csr_matrix:
    """Step 5: the lists as CSR, diagonal and zero distances removed."""
    K = idx.shape[1]
    rows = np.repeat(np.arange(n), K)
    cols = np.asarray(idx).ravel()
    vals = np.asarray(dist, np.float32).ravel()
    keep = (cols != rows) & (vals != 0)
    return sp.csr_matrix((vals[keep], (rows[keep], cols[keep])), shape=(n, n), dtype=np.float32)


def bbknn(X: np.ndarray, batch, neighbors_within_batch: int = 3, n_pcs: int | None = 50,
          trim: int | None = None):
    """The whole batch-balanced graph: ``(distances CSR, connectivities CSR, K)`` plus the
    intermediates in a dict."""
    n = X.shape[0]
    idx, dist, kks = bbknn_lists(X, batch, neighbors_within_batch, n_pcs)
    K = idx.shape[1]
    sigma, rho = smooth_knn_dist(dist, float(K))
    w = membership_strengths(idx, dist, sigma, rho)
    conn = fuzzy_union(idx, w, n)
    distances = bbknn_distances(idx, dist, n)
    trimmed = trim_graph(conn, 10 * K if trim is None else trim)
    return distances, trimmed, K, dict(idx=idx, dist=dist, kk=kks, sigma=sigma, rho=rho, w=w,
                                       untrimmed=conn)
