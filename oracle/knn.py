"""Exact kNN oracle (FP64).  TEST INFRASTRUCTURE ONLY — see ``oracle/__init__.py``.

Semantics restated from the reference:

* the kNN list of cell i holds i itself in column 0 (``neighbors.py:129-131`` sorts self first by
  its zero distance; ``neighbors.py:691-692`` prepends it explicitly), then the k-1 nearest other
  cells;
* ties are broken by index: order by (distance, index), as ``neighbors.py:457-461`` does with
  ``np.lexsort((loc, exact))`` "so exact ties resolve the same way as a CPU reference that breaks
  ties by index";
* returned distances are float32 of the square root (``neighbors.py:131``).  Here the squared
  distance is the FP64 sum, in dimension order, of squared FP64 differences of the float32 inputs,
  and the distance is that value's FP64 square root rounded to float32.
* ``metric='cosine'`` (the reference raises, ``pp.py:768-769``): rows are L2-normalised in FP64 and
  rounded to float32, neighbours are ranked by squared euclidean distance between the unit rows,
  and the reported distance is ``1 - cos = |x̂-ŷ|²/2``.
"""

from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np


def l2_normalize_rows(X: np.ndarray) -> np.ndarray:
    """x̂ = float32(x · (1/sqrt(Σ x_t²))) with the sum in FP64 in dimension order; zero rows stay 0."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    X64 = X.astype(np.float64)
    s = np.zeros(X.shape[0], np.float64)
    for t in range(X.shape[1]):
        s += X64[:, t] * X64[:, t]
    with np.errstate(divide="ignore"):
        r = np.where(s > 0, 1.0 / np.sqrt(s), 0.0)
    return np.ascontiguousarray((X64 * r[:, None]).astype(np.float32))


def sq_dist_f64(Q: np.ndarray, Y: np.ndarray) -> np.ndarray:
    """FP64 squared distances, summed in dimension order.

    ``Q`` is (m, d) float32, ``Y`` is (m, c, d) or (c, d) float32; the result is (m, c)."""
    Q64 = Q.astype(np.float64)
    Y64 = Y.astype(np.float64)
    if Y64.ndim == 2:
        Y64 = Y64[None, :, :]
    acc = np.zeros((Q64.shape[0], Y64.shape[1]), np.float64)
    for t in range(Q64.shape[1]):
        diff = Q64[:, None, t] - Y64[:, :, t]
        acc += diff * diff
    return acc


def _rows_exact(X32: np.ndarray, rows: np.ndarray, kk: int):
    """Full-scan exact neighbours for a few rows (used where the FP64 Gram pre-selection cannot
    certify its boundary, e.g. large groups of coincident cells)."""
    n = X32.shape[0]
    oi = np.empty((rows.size, kk), np.int64)
    od = np.empty((rows.size, kk), np.float64)
    cols = np.arange(n)
    for r, i in enumerate(rows):
        D = sq_dist_f64(X32[i:i + 1], X32)[0]
        D[i] = np.inf
        o = np.lexsort((cols, D))[:kk]
        oi[r] = o
        od[r] = D[o]
    return oi, od


def knn_exact(X: np.ndarray, k: int, metric: str = "euclidean", rows=None,
              threads: int | None = None, chunk_elems: int = 1 << 25):
    """Exact kNN.  Returns ``(idx int64 (m,k), d2 float64 (m,k), dist float32 (m,k))`` for the
    query ``rows`` (all cells by default); column 0 is the cell itself.

    For ``metric='cosine'`` ``dist`` is the cosine distance ``d2/2`` on the normalised rows.
    """
    X32 = np.ascontiguousarray(X, dtype=np.float32)
    if metric == "cosine":
        X32 = l2_normalize_rows(X32)
    elif metric != "euclidean":
        raise ValueError(f"unknown metric {metric!r}")
    n, d = X32.shape
    if not 1 <= k <= n:
        raise ValueError(f"n_neighbors={k} must be in [1, n={n}]")
    rows = np.arange(n) if rows is None else np.asarray(rows, np.int64)
    m = rows.size
    kk = k - 1
    idx = np.empty((m, k), np.int64)
    d2 = np.zeros((m, k), np.float64)
    idx[:, 0] = rows
    if kk > 0:
        X64 = X32.astype(np.float64)
        sq = np.einsum("ij,ij->i", X64, X64)
        sqmax = float(sq.max())
        # |V - exact| for V = |x|² + |y|² - 2x·y in FP64 is far below this bound
        eps64 = 64.0 * (d + 8) * 2.0 ** -53
        m_extra = min(n - 1, kk + 8)
        chunk = int(max(8, min(2048, chunk_elems // max(n, 1))))

        def work(s):
            e = min(s + chunk, m)
            r = rows[s:e]
            V = sq[r, None] + sq[None, :] - 2.0 * (X64[r] @ X64.T)
            V[np.arange(e - s), r] = np.inf
            cand = np.argpartition(V, m_extra - 1, axis=1)[:, :m_extra]
            thr = np.take_along_axis(V, cand, axis=1).max(axis=1)
            D = sq_dist_f64(X32[r], X32[cand])
            o = np.lexsort((cand, D), axis=1)
            ci = np.take_along_axis(cand, o, axis=1)[:, :kk]
            cd = np.take_along_axis(D, o, axis=1)[:, :kk]
            err = eps64 * (sq[r] + sqmax)
            ok = (cd[:, kk - 1] < thr - 2.0 * err) | (m_extra == n - 1)
            bad = np.flatnonzero(~ok)
            if bad.size:
                bi, bd = _rows_exact(X32, r[bad], kk)
                ci[bad] = bi
                cd[bad] = bd
            idx[s:e, 1:] = ci
            d2[s:e, 1:] = cd

        starts = range(0, m, chunk)
        nthreads = threads or os.cpu_count() or 1
        try:
            from threadpoolctl import threadpool_limits
            limiter = threadpool_limits(1) if nthreads > 1 else None
        except Exception:           # threadpoolctl missing: BLAS keeps its own threads
            limiter = None
        try:
            if nthreads > 1 and len(starts) > 1:
                with ThreadPoolExecutor(nthreads) as ex:
                    list(ex.map(work, starts))
            else:
                for s in starts:
                    work(s)
        finally:
            if limiter is not None:
                limiter.restore_original_limits()
    dist = np.sqrt(d2).astype(np.float32)
    if metric == "cosine":
        dist = (d2 * 0.5).astype(np.float32)
    return idx, d2, dist
