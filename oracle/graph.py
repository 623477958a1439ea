"""UMAP fuzzy simplicial set, distances CSR and gauss kernel.  TEST INFRASTRUCTURE ONLY.

The reference builds connectivities with umap-learn's ``fuzzy_simplicial_set``
(``neighbors.py:742-753``: X = coo (n,1) dummy, knn given, ``set_op_mix_ratio=1``,
``local_connectivity=1``).  umap-learn 0.5.12 (``CODE_AVAILABILITY.md:24``) is not installed here,
so its published algorithm is restated:

``smooth_knn_dist`` (umap-learn ``umap_.smooth_knn_dist``)
    ρ_i = the ``local_connectivity``-th non-zero distance of row i (linear interpolation for a
    fractional value; the largest non-zero distance if there are fewer; 0 if none).
    σ_i by bisection so that Σ_{j≥1} exp(-max(0, d_ij-ρ_i)/σ_i) = log2(k)·bandwidth, at most 64
    steps, stop when |sum - target| < 1e-5; start lo=0, hi=∞, mid=1; double mid while hi=∞.
    Floor: σ_i ≥ 1e-3·mean(row i) when ρ_i>0, else ≥ 1e-3·mean(all distances).
    umap-learn keeps psum/lo/hi/mid in float32 (numba ``locals``).  This restatement fixes the
    arithmetic exactly so the CUDA kernel can be checked bit-for-bit: float32 state, the sum in
    column order, IEEE float32 division, and exp evaluated in FP64 then rounded to float32
    (``exp_f32``).  umap-learn compiles the loop with numba ``fastmath`` (which may reorder the sum
    and use an approximate float32 exp); against umap-learn itself agreement is therefore within
    the stated 1e-5 relative, not bitwise.  Row means: float32 sum in column order divided by k in
    FP64; the global mean is the FP64 sum divided by n·k.

``compute_membership_strengths``
    w_ij = 0 for the cell itself; 1 if d_ij-ρ_i ≤ 0 or σ_i = 0; else exp(-(d_ij-ρ_i)/σ_i), all in
    float32.

fuzzy union (``set_op_mix_ratio = 1``)
    A = coo(w) with zeros eliminated; P = 1·(A + Aᵀ − A∘Aᵀ) + 0·(A∘Aᵀ), zeros eliminated, CSR —
    performed here with exactly those SciPy operations in float32, so
    P_ij = fl(fl(a+b) − fl(a·b)) with a = A_ij, b = A_ji.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .knn import knn_exact

SMOOTH_K_TOLERANCE = 1e-5
MIN_K_DIST_SCALE = 1e-3


def exp_f32(z: np.ndarray) -> np.ndarray:
    """exp of float32 arguments evaluated in FP64 and rounded to float32."""
    return np.exp(np.asarray(z, np.float32).astype(np.float64)).astype(np.float32)


def _row_sum_f32(a: np.ndarray) -> np.ndarray:
    acc = np.zeros(a.shape[0], np.float32)
    for j in range(a.shape[1]):
        acc = (acc + a[:, j]).astype(np.float32)
    return acc


def smooth_knn_dist(distances: np.ndarray, k: float, n_iter: int = 64,
                    local_connectivity: float = 1.0, bandwidth: float = 1.0):
    """(sigma float32 (n,), rho float32 (n,)) — see the module docstring."""
    D = np.ascontiguousarray(distances, np.float32)
    n, kc = D.shape
    target = np.log2(float(k)) * bandwidth
    rho = np.zeros(n, np.float32)
    # ρ: the local_connectivity-th non-zero distance, in row (ascending) order
    nz = D > 0.0
    nnz = nz.sum(1)
    index = int(np.floor(local_connectivity))
    interpolation = np.float64(local_connectivity - index)
    # position of the r-th non-zero in each row
    csum = np.cumsum(nz, axis=1)
    def nth_nonzero(r):            # value of the r-th (1-based) non-zero entry
        pos = np.argmax(csum >= r, axis=1)
        return D[np.arange(n), pos]
    enough = nnz >= local_connectivity
    # umap-learn adds `interpolation` (a Python float) to float32 values: numba evaluates that in
    # FP64 and stores float32
    if index > 0:
        v = nth_nonzero(index)
        if interpolation > SMOOTH_K_TOLERANCE:
            v_next = nth_nonzero(index + 1)
            gap = (v_next - v).astype(np.float32).astype(np.float64)
            v = (v.astype(np.float64) + interpolation * gap).astype(np.float32)
        rho = np.where(enough, v, rho).astype(np.float32)
    else:
        first = nth_nonzero(1)
        rho = np.where(enough, (interpolation * first.astype(np.float64)).astype(np.float32), rho)
    few = (~enough) & (nnz > 0)
    rho = np.where(few, np.where(nz, D, 0.0).max(1).astype(np.float32), rho).astype(np.float32)

    lo = np.zeros(n, np.float32)
    hi = np.full(n, np.inf, np.float32)
    mid = np.ones(n, np.float32)
    active = np.ones(n, bool)
    for _ in range(n_iter):
        a = np.flatnonzero(active)
        if a.size == 0:
            break
        psum = np.zeros(a.size, np.float32)
        ra, ma = rho[a], mid[a]
        for j in range(1, kc):
            d = (D[a, j] - ra).astype(np.float32)
            with np.errstate(over="ignore", under="ignore", invalid="ignore"):
                q = (d / ma).astype(np.float32)
                term = np.where(d > 0, exp_f32(-q), np.float32(1.0)).astype(np.float32)
            psum = (psum + term).astype(np.float32)
        p64 = psum.astype(np.float64)
        conv = np.abs(p64 - target) < SMOOTH_K_TOLERANCE
        active[a[conv]] = False
        upd = a[~conv]
        gt = p64[~conv] > target
        g, l_ = upd[gt], upd[~gt]
        hi[g] = mid[g]
        mid[g] = ((lo[g] + hi[g]).astype(np.float32) * np.float32(0.5)).astype(np.float32)
        lo[l_] = mid[l_]
        inf_hi = np.isinf(hi[l_])
        li, lf = l_[inf_hi], l_[~inf_hi]
        mid[li] = (mid[li] * np.float32(2.0)).astype(np.float32)
        mid[lf] = ((lo[lf] + hi[lf]).astype(np.float32) * np.float32(0.5)).astype(np.float32)
    result = mid.copy()
    row_mean = _row_sum_f32(D).astype(np.float64) / kc
    all_mean = D.astype(np.float64).sum() / D.size if D.size else 0.0
    floor_row = MIN_K_DIST_SCALE * row_mean
    floor_all = MIN_K_DIST_SCALE * all_mean
    pos = rho > 0
    lift_r = pos & (result.astype(np.float64) < floor_row)
    lift_a = (~pos) & (result.astype(np.float64) < floor_all)
    result[lift_r] = floor_row[lift_r].astype(np.float32)
    result[lift_a] = np.float32(floor_all)
    return result, rho


def membership_strengths(knn_idx: np.ndarray, knn_dist: np.ndarray, sigma: np.ndarray,
                         rho: np.ndarray) -> np.ndarray:
    """float32 (n, k) memberships w_ij (self → 0)."""
    n, k = knn_idx.shape
    D = np.asarray(knn_dist, np.float32)
    d = (D - rho[:, None]).astype(np.float32)
    with np.errstate(over="ignore", under="ignore", invalid="ignore", divide="ignore"):
        q = (d / sigma[:, None]).astype(np.float32)
        val = exp_f32(-q)
    one = (d <= 0) | (sigma[:, None] == 0)
    val = np.where(one, np.float32(1.0), val).astype(np.float32)
    val[knn_idx == np.arange(n)[:, None]] = 0.0
    return val


def fuzzy_union(knn_idx: np.ndarray, w: np.ndarray, n: int) -> sp.csr_matrix:
    """P = A + Aᵀ − A∘Aᵀ with SciPy float32 arithmetic, as umap-learn performs it."""
    k = knn_idx.shape[1]
    rows = np.repeat(np.arange(n, dtype=np.int32), k)
    cols = np.asarray(knn_idx, np.int32).ravel()
    A = sp.coo_matrix((np.asarray(w, np.float32).ravel(), (rows, cols)), shape=(n, n))
    A.eliminate_zeros()
    T = A.transpose()
    prod = A.multiply(T)
    R = 1.0 * (A + T - prod) + (1.0 - 1.0) * prod
    R.eliminate_zeros()
    R = R.tocsr()
    assert R.dtype == np.float32
    return R


def distances_csr(knn_idx: np.ndarray, knn_dist: np.ndarray, n: int) -> sp.csr_matrix:
    """``neighbors.py:755-759``: columns 1..k-1 of every row; SciPy canonical form, explicit
    zeros (coincident cells) kept."""
    k = knn_idx.shape[1]
    rows = np.repeat(np.arange(n), k - 1)
    cols = np.asarray(knn_idx)[:, 1:].ravel()
    vals = np.asarray(knn_dist, np.float32)[:, 1:].ravel()
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def gauss_connectivities(knn_idx: np.ndarray, knn_dist: np.ndarray, n: int) -> sp.csr_matrix:
    """``method='gauss'``: the locally scaled Gaussian kernel of Haghverdi et al. (2016) on the
    kNN graph, as scanpy applies it to a kNN distance graph.

    σ_i² = median of the squared distances to the k-1 nearest other cells (FP64; the mean of the
    two middle values for an even count).  For every pair in the symmetrised kNN structure
    (i→j or j→i): W_ij = sqrt(2σ_iσ_j/(σ_i²+σ_j²))·exp(-d_ij²/(σ_i²+σ_j²)), in FP64, rounded to
    float32.  The kernel is symmetric, so W is.  The reference has no ``method`` parameter
    (``pp.py:780`` always records 'umap'), so this is an addition: parity unpinned.

    Two deliberate departures from scanpy's implementation: an edge to a coincident cell
    (distance 0) is kept, where scanpy's ``eliminate_zeros()`` on the distance matrix drops it
    (and takes that row's median over fewer entries); and the medians and the kernel are FP64,
    rounded once, where scanpy computes in float32.
    """
    k = knn_idx.shape[1]
    D = np.asarray(knn_dist, np.float32)[:, 1:].astype(np.float64)
    Dsq = D * D
    sig2 = np.median(Dsq, axis=1) if k > 1 else np.zeros(n)
    sig = np.sqrt(sig2)
    rows = np.repeat(np.arange(n), k - 1)
    cols = np.asarray(knn_idx)[:, 1:].ravel()
    dsq = Dsq.ravel()
    # union structure; the distance of an edge is the same from either end
    r2 = np.concatenate([rows, cols])
    c2 = np.concatenate([cols, rows])
    d2 = np.concatenate([dsq, dsq])
    key = r2.astype(np.int64) * n + c2
    uk, first = np.unique(key, return_index=True)
    r2, c2, d2 = r2[first], c2[first], d2[first]
    num = 2.0 * sig[r2] * sig[c2]
    den = sig2[r2] + sig2[c2]
    with np.errstate(divide="ignore", invalid="ignore"):
        W = np.sqrt(num / den) * np.exp(-d2 / den)
    W = np.where(den > 0, W, 0.0)     # σ_i = σ_j = 0: coincident neighbourhoods
    return sp.csr_matrix((W.astype(np.float32), (r2, c2)), shape=(n, n))


def neighbors_graph(X: np.ndarray, n_neighbors: int = 15, metric: str = "euclidean",
                    method: str = "umap", threads=None):
    """The whole path on the CPU: kNN → (distances CSR, connectivities CSR) + intermediates."""
    n = X.shape[0]
    idx, d2, dist = knn_exact(X, n_neighbors, metric=metric, threads=threads)
    if method == "umap":
        sigma, rho = smooth_knn_dist(dist, float(n_neighbors))
        w = membership_strengths(idx, dist, sigma, rho)
        conn = fuzzy_union(idx, w, n)
    elif method == "gauss":
        sigma = rho = w = None
        conn = gauss_connectivities(idx, dist, n)
    else:
        raise ValueError(f"unknown method {method!r}")
    distances = distances_csr(idx, dist, n)
    return dict(idx=idx, d2=d2, dist=dist, sigma=sigma, rho=rho, w=w,
                distances=distances, connectivities=conn)
