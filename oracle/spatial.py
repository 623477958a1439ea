"""Spatial (2-D / 3-D) neighbour oracle.  TEST INFRASTRUCTURE ONLY — see ``oracle/__init__.py``.

Restates what metalsinglecell's uniform-grid index computes for spatial coordinates:

* ``grid_knn`` — ``neighbors._knn_grid`` (neighbors.py:333-417): exact self-inclusive k nearest
  neighbours, shape (n, k), self first.  The reference's grid kernel ranks on the float32
  squared distance of float32 differences (neighbors.py:180-183) and reports
  ``sqrt(max(d², 0))`` in float32 (neighbors.py:404-406); rows its completeness test rejects are
  redone by ``_exact_knn_rows`` (neighbors.py:420-462), which orders by (distance, index).
  Here every row follows ONE rule, the grid kernel's arithmetic with that tie order:
  d² = fl(fl(dx²) + fl(dy²)) [+ fl(dz²)] with dx = fl(x_p − x_q), no fused multiply-add;
  distance s = the correctly rounded float32 square root of d²; self first, then the k − 1
  other points in (s, index) order — the order ``gr._knn_edges`` (gr.py:186-195) imposes on
  the grid's lists.
* ``grid_radius`` — ``neighbors._radius_grid`` (neighbors.py:255-330): every other point with
  r_lo² ≤ d² ≤ r_hi² (float32 d² as above; r² = float32 of the float64 square,
  neighbors.py:301-302 and :238), self excluded (:232), as an (n, n) CSR with int64 indptr,
  int32 columns and float32 distances sqrt(d²).  The reference writes a row's columns in its
  cell-walk order; here they are ascending (the same matrix in SciPy's canonical layout).
* ``knn_edges`` — ``gr._knn_edges`` (gr.py:186-195): the directed n_neighs-NN edge list,
  self excluded.

Pinning: the reference's own known-answer criteria, run here.  ``grid_radius`` must give exactly
sklearn's ``radius_neighbors_graph`` pattern on the three seeded inputs of the reference's
``tests/test_spatial_neighbors.py:363-375``; distances of the large-coordinate regression
(:378-387) stay within 1e-3 of 273; ``grid_knn`` agrees with sklearn's exact kNN except where
two candidates are exactly equidistant (the reference's tie-aware comparison, :33-47).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def sq_dist_f32(Q: np.ndarray, P: np.ndarray) -> np.ndarray:
    """(m, n) float32 squared distances, summed axis by axis in order, no fused multiply-add."""
    Q = np.asarray(Q, np.float32)
    P = np.asarray(P, np.float32)
    acc = None
    for a in range(Q.shape[1]):
        diff = P[None, :, a] - Q[:, None, a]
        t = diff * diff
        acc = t if acc is None else acc + t
    return acc


def _row_blocks(n: int, m: int, budget: int = 32_000_000):
    step = max(1, budget // max(m, 1))
    for s in range(0, n, step):
        yield s, min(n, s + step)


def grid_knn(coords: np.ndarray, k: int, rows=None):
    """(idx int64 (m, k), dist float32 (m, k)) for the query ``rows`` (all points by default):
    self first, then (float32 distance, index)."""
    X = np.ascontiguousarray(coords, np.float32)
    n = X.shape[0]
    if not 1 <= k <= n:
        raise ValueError(f"k={k} must be in [1, n={n}]")
    q = np.arange(n) if rows is None else np.asarray(rows, np.int64)
    m = q.size
    idx = np.empty((m, k), np.int64)
    dist = np.empty((m, k), np.float32)
    cols = np.arange(n)
    for s, e in _row_blocks(m, n):
        d2 = sq_dist_f32(X[q[s:e]], X)
        sd = np.sqrt(d2)
        sd[np.arange(e - s), q[s:e]] = -1.0            # self ranks first
        if k < n:
            part = np.argpartition(sd, k - 1, axis=1)[:, :k]
            kth = np.take_along_axis(sd, part, axis=1).max(1)
        else:
            kth = sd.max(1)
        for r in range(e - s):
            c = cols[sd[r] <= kth[r]]                  # every candidate tied at the k-th value
            o = np.lexsort((c, sd[r, c]))[:k]
            idx[s + r] = c[o]
            dist[s + r] = np.maximum(sd[r, c[o]], 0.0)
    return idx, dist


def grid_radius(coords: np.ndarray, radius: float, min_radius: float = 0.0):
    """(indptr int64, cols int32, dist float32) of the (n, n) radius graph, self excluded."""
    X = np.ascontiguousarray(coords, np.float32)
    n = X.shape[0]
    r2hi = np.float32(float(radius) ** 2)
    r2lo = np.float32(float(min_radius) ** 2)
    counts = np.zeros(n, np.int64)
    cols, vals = [], []
    for s, e in _row_blocks(n, n):
        d2 = sq_dist_f32(X[s:e], X)
        keep = (d2 <= r2hi) & (d2 >= r2lo)
        rows = np.arange(s, e)
        keep[rows - s, rows] = False
        r, c = np.nonzero(keep)                        # row-major: columns ascending per row
        counts[s:e] = np.bincount(r, minlength=e - s)
        cols.append(c.astype(np.int32))
        vals.append(np.sqrt(d2[r, c]))
    indptr = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=indptr[1:])
    col = np.concatenate(cols) if cols else np.zeros(0, np.int32)
    val = np.concatenate(vals).astype(np.float32) if vals else np.zeros(0, np.float32)
    return indptr, col, val


def radius_csr(coords: np.ndarray, radius: float, min_radius: float = 0.0) -> sp.csr_matrix:
    n = np.asarray(coords).shape[0]
    indptr, col, val = grid_radius(coords, radius, min_radius)
    return sp.csr_matrix((val, col, indptr), shape=(n, n))


def knn_edges(coords: np.ndarray, n_neighs: int):
    """(rows int64, cols int64, dist float32) of the directed n_neighs-NN graph, self excluded:
    each point's n_neighs nearest other points in (float32 distance, index) order."""
    X = np.asarray(coords, np.float32)
    n = X.shape[0]
    if not 0 < n_neighs < n:
        raise ValueError(f"n_neighs={n_neighs} must be in [1, n - 1 = {n - 1}]")
    idx, dist = grid_knn(X, n_neighs + 1)
    rows = np.repeat(np.arange(n, dtype=np.int64), n_neighs)
    return rows, idx[:, 1:].ravel().astype(np.int64), dist[:, 1:].ravel()


# ---------------------------------------------------------------------------------------------
# The spatial graph builders around the search: gr.spatial_neighbors_knn / _radius
# (gr.py:198-255), their shared tail (gr.py:81-104) and per-library assembly (gr.py:107-147).

def edge_lengths_f64(coords64: np.ndarray, rows: np.ndarray, cols: np.ndarray) -> np.ndarray:
    """gr.py:32-34: Euclidean edge lengths from the float64 coordinates, squares summed axis by
    axis in order, float64 result."""
    X = np.asarray(coords64, np.float64)
    acc = None
    for a in range(X.shape[1]):
        t = X[rows, a] - X[cols, a]
        t = t * t
        acc = t if acc is None else acc + t
    return np.sqrt(acc) if acc is not None else np.zeros(0)


def _masked(M: sp.csr_matrix, keep: np.ndarray) -> sp.csr_matrix:
    """Entries where ``keep`` holds and the value is non-zero (gr.py:88-98)."""
    ok = keep & (M.data != 0)
    rows = np.repeat(np.arange(M.shape[0]), np.diff(M.indptr))[ok]
    indptr = np.zeros(M.shape[0] + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=M.shape[0]), out=indptr[1:])
    return sp.csr_matrix((M.data[ok], M.indices[ok], indptr), shape=M.shape)


def finish_graph(adj, dst, transform=None, set_diag=False, percentile=None):
    """gr.py:81-104, in order: drop every edge whose distance is above the ``percentile``-th
    percentile of the distances (NumPy's default linear interpolation), with the zero
    distances; 1.0 on the adjacency's diagonal (the element-wise maximum with I); the
    distances' diagonal and zeros removed; then the adjacency transform."""
    adj, dst = sp.csr_matrix(adj), sp.csr_matrix(dst)
    if percentile is not None and dst.nnz:
        keep = dst.data <= np.percentile(dst.data, percentile)
        adj, dst = _masked(adj, keep), _masked(dst, keep)
    if set_diag:
        adj = adj.maximum(sp.identity(adj.shape[0], format="csr", dtype=adj.dtype)).tocsr()
    r = np.repeat(np.arange(dst.shape[0]), np.diff(dst.indptr))
    dst = _masked(dst, dst.indices != r)
    return transform_adjacency(adj, transform), dst


def transform_adjacency(adj, transform):
    """gr.py:37-57: None; 'spectral' = D^-1/2 A D^-1/2 with D the COLUMN degrees (in-degree), a
    zero degree giving a zero scale; 'cosine' = sklearn's cosine similarity of the rows."""
    if transform in (None, "none"):
        return adj
    if transform == "spectral":
        deg = np.asarray(adj.sum(axis=0)).ravel()
        inv = np.zeros_like(deg)
        np.divide(1.0, np.sqrt(deg), out=inv, where=deg > 0)
        D = sp.diags(inv)
        return (D @ adj @ D).tocsr()
    if transform == "cosine":
        from sklearn.metrics.pairwise import cosine_similarity
        return sp.csr_matrix(cosine_similarity(adj, dense_output=False))
    raise NotImplementedError(f"transform={transform!r}")


def _per_library(coords64, library, build, transform, set_diag, percentile):
    """gr.py:123-147: one graph per library code (codes in category order, empty ones skipped),
    each finished on its own, combined block-diagonally and put back in observation order."""
    coords64 = np.asarray(coords64, np.float64)
    if library is None:
        return finish_graph(*build(coords64.astype(np.float32), coords64),
                            transform, set_diag, percentile)
    library = np.asarray(library)
    groups = [np.flatnonzero(library == c) for c in range(int(library.max()) + 1)]
    groups = [g for g in groups if g.size]
    parts = [finish_graph(*build(np.ascontiguousarray(coords64[g], np.float32),
                                 np.ascontiguousarray(coords64[g])),
                          transform, set_diag, percentile) for g in groups]
    adj = sp.block_diag([p[0] for p in parts], format="csr")
    dst = sp.block_diag([p[1] for p in parts], format="csr")
    order = np.concatenate(groups)
    if np.any(np.diff(order) < 0):
        back = np.argsort(order)
        adj, dst = adj[back][:, back], dst[back][:, back]
    return adj.tocsr(), dst.tocsr()


def spatial_neighbors_knn(coords64, n_neighs=6, library=None, percentile=None, transform=None,
                          set_diag=False):
    """(connectivities, distances) of gr.spatial_neighbors_knn (gr.py:198-225): the directed
    n_neighs-NN graph, binary float32 adjacency, float64 edge lengths.  ``library`` holds one
    integer category code per observation (or None)."""
    def build(xy, exact):
        n = xy.shape[0]
        rows, cols, _ = knn_edges(xy, n_neighs)
        dist = edge_lengths_f64(exact, rows, cols)
        indptr = np.arange(n + 1, dtype=np.int64) * n_neighs
        return (sp.csr_matrix((np.ones(dist.size, np.float32), cols, indptr), shape=(n, n)),
                sp.csr_matrix((dist, cols, indptr), shape=(n, n)))
    return _per_library(coords64, library, build, transform, set_diag, percentile)


def spatial_neighbors_radius(coords64, radius, library=None, percentile=None, transform=None,
                             set_diag=False):
    """(connectivities, distances) of gr.spatial_neighbors_radius (gr.py:228-255): every pair
    within ``radius`` (a maximum, or a (min, max) interval), binary float32 adjacency, float64
    edge lengths."""
    if np.isscalar(radius):
        lo, hi = 0.0, float(radius)
    else:
        lo, hi = float(min(radius)), float(max(radius))

    def build(xy, exact):
        n = xy.shape[0]
        indptr, cols, _ = grid_radius(xy, hi, lo)
        rows = np.repeat(np.arange(n), np.diff(indptr))
        dist = edge_lengths_f64(exact, rows, cols)
        return (sp.csr_matrix((np.ones(dist.size, np.float32), cols, indptr), shape=(n, n)),
                sp.csr_matrix((dist, cols, indptr), shape=(n, n)))
    return _per_library(coords64, library, build, transform, set_diag, percentile)
