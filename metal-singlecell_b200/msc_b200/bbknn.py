"""Batch-balanced kNN graph — the compute layer under ``pp.bbknn``.

Mirrors metalsinglecell ``neighbors.bbknn(X_pca, batch, neighbors_within_batch, n_pcs, trim,
random_state)`` (neighbors.py:491-559) → ``(distances, connectivities, n_neighbors)``: every cell
gets its ``min(neighbors_within_batch, n_b)`` nearest cells of every batch b, the combined lists
(K = Σ_b min(neighbors_within_batch, n_b) entries per cell, sorted by distance) go through the
umap fuzzy simplicial set with n_neighbors = K, the distances graph drops the diagonal and zero
distances, and the connectivities are trimmed to each cell's ``trim`` strongest edges
(``10·K`` by default, neighbors.py:465-488).

The reference scans every batch by brute force in FP32; here the lists are exact (tensor-core
candidates, exact re-rank and certificate, FP64 scan of the uncertified cells), so they are the
same lists a CPU scan in exact arithmetic gives.  Every stage runs on the GPU through the C ABI of
``libmsc_b200.so``; PyTorch only provides buffers and the current stream.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .neighbors import DEFAULT_PRECISION, Workspace, _stream, _torch


def batch_codes(batch) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(sorted unique labels, int32 code of every cell, int64 cells per batch) — the batch order
    of neighbors.py:510 (``np.unique``)."""
    cats, codes = np.unique(np.asarray(batch), return_inverse=True)
    counts = np.bincount(codes, minlength=cats.size).astype(np.int64)
    return cats, codes.astype(np.int32), counts


def bbknn_device(X, codes, counts: np.ndarray, neighbors_within_batch: int = 3,
                 trim: int | None = None, *, precision: str = DEFAULT_PRECISION,
                 workspace: Workspace | None = None) -> dict:
    """The batch-balanced graph on device tensors, enqueued on the current stream.

    ``X``: CUDA float32 (n, d); ``codes``: CUDA int32 (n,) batch codes 0..B-1; ``counts``: host
    int64 (B,) cells per batch (the histogram of ``codes``).  Returns a dict of CUDA tensors:
    ``knn_idx`` / ``knn_dist`` (n, K), ``sigma`` / ``rho`` (n,), ``w`` (n, K), the distances
    CSR ``dist_indptr/indices/data`` (valid length ``dist_indptr[n]``), the untrimmed
    connectivities ``union_indptr/indices/data`` and the trimmed ones
    ``conn_indptr/indices/data`` (valid length ``conn_indptr[n]``), ``stats`` (int64[8]) and
    ``K`` / ``trim`` (ints).
    """
    torch = _torch()
    lib = _lib.load()
    if X.dtype != torch.float32 or not X.is_cuda or X.dim() != 2:
        raise ValueError("X must be a 2-D float32 CUDA tensor")
    if codes.dtype != torch.int32 or not codes.is_cuda or codes.numel() != X.shape[0]:
        raise ValueError("codes must be an int32 CUDA tensor with one entry per cell")
    if precision not in _lib.PRECISION:
        raise ValueError(f"precision={precision!r} must be one of {sorted(_lib.PRECISION)}")
    X = X.contiguous()
    codes = codes.contiguous()
    counts = np.ascontiguousarray(counts, dtype=np.int64)
    n, d = X.shape
    nb = int(counts.size)
    kwb = int(neighbors_within_batch)
    pid = _lib.PRECISION[precision]
    cptr = counts.ctypes.data
    nbytes = lib.msc_bbknn_workspace_bytes(n, d, cptr, nb, kwb, pid)
    if nbytes == 0:
        _lib.check(lib.msc_bbknn_knn(0, n, d, 0, cptr, nb, kwb, pid, 0, 0, 0, 0, 0, 0),
                   "msc_bbknn_knn")
        raise ValueError("msc_bbknn_knn: invalid arguments")
    K = int(lib.msc_bbknn_width(cptr, nb, kwb))
    t = 10 * K if trim is None else int(trim)
    dev = X.device
    st = _stream(torch, dev)
    # one scratch buffer for every stage (they run one after the other on the stream)
    ws_bytes = max(nbytes, lib.msc_fuzzy_union_workspace_bytes(n, K),
                   lib.msc_bbknn_distances_workspace_bytes(n),
                   lib.msc_trim_graph_workspace_bytes(n), 256)
    ws = (workspace or Workspace(dev)).get(ws_bytes)
    o = {"K": K, "trim": t}
    e = lambda shape, dt: torch.empty(shape, dtype=dt, device=dev)
    o["knn_idx"] = e((n, K), torch.int32)
    o["knn_dist"] = e((n, K), torch.float32)
    o["stats"] = torch.zeros(_lib.STATS_LEN, dtype=torch.int64, device=dev)
    _lib.check(lib.msc_bbknn_knn(X.data_ptr(), n, d, codes.data_ptr(), cptr, nb, kwb, pid,
                                 o["knn_idx"].data_ptr(), o["knn_dist"].data_ptr(),
                                 o["stats"].data_ptr(), ws.data_ptr(), ws.numel(), st),
               "msc_bbknn_knn")
    # the fuzzy simplicial set of the combined lists, n_neighbors = K (neighbors.py:547-553)
    o["sigma"] = e((n,), torch.float32)
    o["rho"] = e((n,), torch.float32)
    _lib.check(lib.msc_smooth_knn_dist(o["knn_dist"].data_ptr(), n, K, 1.0, o["sigma"].data_ptr(),
                                       o["rho"].data_ptr(), ws.data_ptr(), ws.numel(), st),
               "msc_smooth_knn_dist")
    o["w"] = e((n, K), torch.float32)
    _lib.check(lib.msc_membership(o["knn_idx"].data_ptr(), o["knn_dist"].data_ptr(),
                                  o["sigma"].data_ptr(), o["rho"].data_ptr(), n, K,
                                  o["w"].data_ptr(), st), "msc_membership")
    cap = max(2 * n * K, 1)
    o["union_indptr"] = e((n + 1,), torch.int64)
    o["union_indices"] = e((cap,), torch.int32)
    o["union_data"] = e((cap,), torch.float32)
    nnz_dev = e((1,), torch.int64)
    _lib.check(lib.msc_fuzzy_union(o["knn_idx"].data_ptr(), o["w"].data_ptr(), n, K,
                                   o["union_indptr"].data_ptr(), o["union_indices"].data_ptr(),
                                   o["union_data"].data_ptr(), nnz_dev.data_ptr(), ws.data_ptr(),
                                   ws.numel(), st), "msc_fuzzy_union")
    # distances graph (neighbors.py:554-557)
    o["dist_indptr"] = e((n + 1,), torch.int64)
    o["dist_indices"] = e((max(n * K, 1),), torch.int32)
    o["dist_data"] = e((max(n * K, 1),), torch.float32)
    _lib.check(lib.msc_bbknn_distances_csr(o["knn_idx"].data_ptr(), o["knn_dist"].data_ptr(), n,
                                           K, o["dist_indptr"].data_ptr(),
                                           o["dist_indices"].data_ptr(),
                                           o["dist_data"].data_ptr(), ws.data_ptr(), ws.numel(),
                                           st), "msc_bbknn_distances_csr")
    # trimming (neighbors.py:558, 465-488); trim <= 0 keeps the union as it is
    if t > 0:
        o["conn_indptr"] = e((n + 1,), torch.int64)
        o["conn_indices"] = e((cap,), torch.int32)
        o["conn_data"] = e((cap,), torch.float32)
        _lib.check(lib.msc_trim_graph(o["union_indptr"].data_ptr(), o["union_indices"].data_ptr(),
                                      o["union_data"].data_ptr(), n, t,
                                      o["conn_indptr"].data_ptr(), o["conn_indices"].data_ptr(),
                                      o["conn_data"].data_ptr(), ws.data_ptr(), ws.numel(), st),
                   "msc_trim_graph")
    else:
        o["conn_indptr"] = o["union_indptr"]
        o["conn_indices"] = o["union_indices"]
        o["conn_data"] = o["union_data"]
    return o


def _csr_to_host(indptr, indices, data, n):
    import scipy.sparse as sp
    ptr = indptr.cpu().numpy()
    nnz = int(ptr[n])
    return sp.csr_matrix((data[:nnz].cpu().numpy(), indices[:nnz].cpu().numpy(),
                          ptr.astype(np.int32)), shape=(n, n))


def graph_to_host(res: dict, n: int):
    """Device result of ``bbknn_device`` → (distances CSR, connectivities CSR) on the host, with
    int32 index arrays and sorted columns (SciPy's canonical form, as the reference returns)."""
    stats = res["stats"].cpu().numpy()
    _lib.check_stats(stats)
    dist = _csr_to_host(res["dist_indptr"], res["dist_indices"], res["dist_data"], n)
    conn = _csr_to_host(res["conn_indptr"], res["conn_indices"], res["conn_data"], n)
    return dist, conn


def trim_graph(conn, trim: int | None, *, device=None):
    """``_trim_graph`` (neighbors.py:465-488) of a SciPy CSR matrix on the GPU: the entries with
    value v != 0, v >= θ_i and v >= θ_j, θ_i = the trim-th largest stored value of row i when it
    stores more than ``trim`` entries.  ``trim`` None or <= 0: an unchanged copy."""
    import scipy.sparse as sp
    torch = _torch()
    lib = _lib.load()
    A = sp.csr_matrix(conn, copy=True)
    if trim is None or trim <= 0:
        return A
    A.sort_indices()
    n = A.shape[0]
    dev = torch.device(device) if device is not None else torch.device("cuda",
                                                                       torch.cuda.current_device())
    ptr = torch.from_numpy(A.indptr.astype(np.int64)).to(dev)
    ind = torch.from_numpy(A.indices.astype(np.int32)).to(dev)
    dat = torch.from_numpy(A.data.astype(np.float32)).to(dev)
    cap = max(A.nnz, 1)
    optr = torch.empty(n + 1, dtype=torch.int64, device=dev)
    oind = torch.empty(cap, dtype=torch.int32, device=dev)
    odat = torch.empty(cap, dtype=torch.float32, device=dev)
    ws = Workspace(dev).get(lib.msc_trim_graph_workspace_bytes(n))
    _lib.check(lib.msc_trim_graph(ptr.data_ptr(), ind.data_ptr(), dat.data_ptr(), n, int(trim),
                                  optr.data_ptr(), oind.data_ptr(), odat.data_ptr(),
                                  ws.data_ptr(), ws.numel(), _stream(torch, dev)),
               "msc_trim_graph")
    torch.cuda.current_stream(dev).synchronize()
    return _csr_to_host(optr, oind, odat, n)


def bbknn(X_pca: np.ndarray, batch, neighbors_within_batch: int = 3, n_pcs: int | None = 50,
          trim: int | None = None, random_state: int = 0, *,
          precision: str = DEFAULT_PRECISION, device=None):
    """``(distances, connectivities, n_neighbors)`` as metalsinglecell ``neighbors.bbknn``
    returns them (neighbors.py:491-559); ``n_neighbors`` = K, the width of the combined lists.
    ``random_state`` is accepted for compatibility; the graph is exact and deterministic."""
    torch = _torch()
    X = np.ascontiguousarray(X_pca, dtype=np.float32)
    if X.ndim != 2:
        raise ValueError("X_pca must be 2-D")
    if n_pcs is not None:                       # neighbors.py:506-507
        X = np.ascontiguousarray(X[:, :n_pcs])
    batch = np.asarray(batch)
    if batch.shape[0] != X.shape[0]:
        raise ValueError(f"batch has {batch.shape[0]} labels for {X.shape[0]} cells")
    _, codes, counts = batch_codes(batch)
    dev = torch.device(device) if device is not None else torch.device("cuda",
                                                                       torch.cuda.current_device())
    Xd = torch.from_numpy(X).to(dev)
    cd = torch.from_numpy(codes).to(dev)
    res = bbknn_device(Xd, cd, counts, neighbors_within_batch, trim, precision=precision)
    torch.cuda.current_stream(dev).synchronize()
    dist, conn = graph_to_host(res, X.shape[0])
    return dist, conn, int(res["K"])
