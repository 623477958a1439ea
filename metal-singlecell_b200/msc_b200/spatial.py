"""Spatial (2-D / 3-D) neighbour search on the GPU: metalsinglecell's uniform-grid index
(``neighbors._knn_grid`` / ``neighbors._radius_grid``, neighbors.py:143-417) and
``spatial.spatial_neighbors`` (spatial.py:13-44), through the C ABI (``msc_spatial_*``).

Every row is exact under one arithmetic: the float32 squared distance of float32 differences,
summed axis by axis without fused multiply-add (the reference grid kernel's, neighbors.py:180-183),
the correctly rounded float32 square root as the distance, self first, then (distance, index)
order.  The reference redoes the rows its completeness test rejects with a different (FP64,
centred) arithmetic (neighbors.py:420-462); here the device search expands its rings of cells
until the row is provably complete, so no row takes another path.

Requests the grid kernels do not take — coordinates of other than 2 or 3 dimensions, more than
``SPATIAL_MAX_K`` neighbours — go to the exact kNN of ``msc_b200.neighbors`` (FP64 ranking, the
same (distance, index) order), as the reference sends them to its exact brute force
(neighbors.py:350-351).
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .neighbors import Workspace, _stream, _torch


def _device(torch, device):
    return torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())


def knn_grid_device(coords, k: int, workspace: Workspace | None = None):
    """``(idx int32 (n, k), dist float32 (n, k), stats int64 (8,))`` on the device for float32
    coordinates ``coords`` (n, 2|3) on the device; asynchronous on the current stream."""
    torch = _torch()
    lib = _lib.load()
    X = coords.contiguous()
    if X.dtype != torch.float32 or not X.is_cuda or X.dim() != 2:
        raise ValueError("coords must be a 2-D float32 CUDA tensor")
    n, d = X.shape
    if not 1 <= k <= n:
        raise ValueError(f"k={k} must be in [1, n={n}]")
    dev = X.device
    idx = torch.empty((n, k), dtype=torch.int32, device=dev)
    dist = torch.empty((n, k), dtype=torch.float32, device=dev)
    stats = torch.zeros(_lib.SP_STATS_LEN, dtype=torch.int64, device=dev)
    nbytes = lib.msc_spatial_knn_workspace_bytes(n, d, k)
    ws = (workspace or Workspace(dev)).get(nbytes)
    _lib.check(lib.msc_spatial_knn(X.data_ptr(), n, d, k, idx.data_ptr(), dist.data_ptr(),
                                   stats.data_ptr(), ws.data_ptr(), ws.numel(),
                                   _stream(torch, dev)), "msc_spatial_knn")
    return idx, dist, stats


def radius_grid_device(coords, radius: float, min_radius: float = 0.0,
                       workspace: Workspace | None = None):
    """``(indptr int64 (n+1,), cols int32 (nnz,), dist float32 (nnz,), stats)`` on the device:
    every other point with min_radius² ≤ d² ≤ radius², columns ascending in every row.  Reads
    nnz back once (an 8-byte copy) between the count and the fill pass."""
    torch = _torch()
    lib = _lib.load()
    X = coords.contiguous()
    if X.dtype != torch.float32 or not X.is_cuda or X.dim() != 2:
        raise ValueError("coords must be a 2-D float32 CUDA tensor")
    n, d = X.shape
    dev = X.device
    if n == 0:
        z = torch.zeros(1, dtype=torch.int64, device=dev)
        return (z, torch.zeros(0, dtype=torch.int32, device=dev),
                torch.zeros(0, dtype=torch.float32, device=dev),
                torch.zeros(_lib.SP_STATS_LEN, dtype=torch.int64, device=dev))
    st = _stream(torch, dev)
    indptr = torch.empty(n + 1, dtype=torch.int64, device=dev)
    stats = torch.zeros(_lib.SP_STATS_LEN, dtype=torch.int64, device=dev)
    nbytes = lib.msc_spatial_radius_workspace_bytes(n, d)
    ws = (workspace or Workspace(dev)).get(nbytes)
    _lib.check(lib.msc_spatial_radius_count(X.data_ptr(), n, d, float(radius), float(min_radius),
                                            indptr.data_ptr(), stats.data_ptr(), ws.data_ptr(),
                                            ws.numel(), st), "msc_spatial_radius_count")
    nnz = int(indptr[n].item())
    _lib.check_spatial_stats(stats.cpu().numpy())
    cols = torch.empty(nnz, dtype=torch.int32, device=dev)
    dist = torch.empty(nnz, dtype=torch.float32, device=dev)
    sbytes = lib.msc_spatial_radius_scratch_bytes(nnz)
    scratch = torch.empty(max(sbytes, 256), dtype=torch.uint8, device=dev)
    _lib.check(lib.msc_spatial_radius_fill(n, d, float(radius), float(min_radius),
                                           indptr.data_ptr(), nnz, cols.data_ptr(),
                                           dist.data_ptr(), ws.data_ptr(), ws.numel(),
                                           scratch.data_ptr(), scratch.numel(), st),
               "msc_spatial_radius_fill")
    return indptr, cols, dist, stats


def edge_lengths_device(coords64, indptr, cols):
    """FP64 Euclidean length of every CSR edge from float64 coordinates on the device."""
    torch = _torch()
    lib = _lib.load()
    X = coords64.contiguous()
    n, d = X.shape
    out = torch.empty(cols.numel(), dtype=torch.float64, device=X.device)
    if cols.numel():
        _lib.check(lib.msc_spatial_edge_lengths(X.data_ptr(), n, d, indptr.data_ptr(),
                                                cols.data_ptr(), out.data_ptr(),
                                                _stream(torch, X.device)),
                   "msc_spatial_edge_lengths")
    return out


def knn_lists_device(coords, k: int, workspace: Workspace | None = None):
    """``(idx int32 (n, k), dist float32 (n, k))`` on the device: the grid search where it
    applies (d ∈ {2, 3}, k ≤ SPATIAL_MAX_K), else the exact kNN of ``msc_b200.neighbors``."""
    n, d = coords.shape
    if d in (2, 3) and k <= _lib.SPATIAL_MAX_K:
        idx, dist, stats = knn_grid_device(coords, k, workspace)
        _torch().cuda.current_stream(coords.device).synchronize()
        _lib.check_spatial_stats(stats.cpu().numpy())
        return idx, dist
    from .neighbors import knn_device
    idx, dist, stats = knn_device(coords, k, workspace=workspace)
    _torch().cuda.current_stream(coords.device).synchronize()
    _lib.check_stats(stats.cpu().numpy())
    return idx, dist


def _knn_grid(coords: np.ndarray, k: int, min_n: int = 4_000, device=None):
    """Exact self-inclusive kNN of 2-D / 3-D points: ``(idx int64 (n, k), dist float32 (n, k))``,
    self first, (distance, index) order — metalsinglecell ``_knn_grid`` (neighbors.py:333-417).
    ``min_n`` is accepted for the reference's signature; the grid serves every n here."""
    torch = _torch()
    X = np.ascontiguousarray(coords, dtype=np.float32)
    n = X.shape[0]
    if not 1 <= k <= n:
        raise ValueError(f"k={k} must be in [1, n={n}]")
    idx, dist = knn_lists_device(torch.from_numpy(X).to(_device(torch, device)), k)
    return idx.cpu().numpy().astype(np.int64), dist.cpu().numpy()


def _radius_grid(coords: np.ndarray, radius: float, min_radius: float = 0.0, device=None):
    """All other points within ``radius`` (and at least ``min_radius``) of each point:
    ``(indptr int64, indices int32, distances float32)`` of an (n, n) CSR — metalsinglecell
    ``_radius_grid`` (neighbors.py:255-330).  Columns come ascending in every row (the
    reference writes them in its cell-walk order: the same matrix)."""
    X = np.ascontiguousarray(coords, dtype=np.float32)
    n, d = X.shape
    if n == 0:
        return np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0, np.float32)
    if d not in (2, 3):
        raise ValueError(f"radius search expects 2-D or 3-D coordinates, got {d}-D")
    torch = _torch()
    indptr, cols, dist, _ = radius_grid_device(torch.from_numpy(X).to(_device(torch, device)),
                                               radius, min_radius)
    return indptr.cpu().numpy(), cols.cpu().numpy(), dist.cpu().numpy()


def spatial_neighbors(coords, n_neighs: int = 6, symmetric: bool = False, device=None):
    """Binary spatial kNN adjacency (metalsinglecell ``spatial.spatial_neighbors``,
    spatial.py:13-44): the directed n_neighs-NN graph, self excluded, as a float32 CSR; with
    ``symmetric=True`` the undirected union (A + Aᵀ > 0)."""
    import scipy.sparse as sp
    coords = np.asarray(coords)
    n = coords.shape[0]
    idx, _ = _knn_grid(np.asarray(coords, dtype=np.float32), n_neighs + 1, device=device)
    rows = np.repeat(np.arange(n), n_neighs)
    A = sp.csr_matrix((np.ones(rows.size, np.float32), (rows, idx[:, 1:].ravel())), shape=(n, n))
    if symmetric:
        A = ((A + A.T) > 0).astype(np.float32)
    return A.tocsr()
