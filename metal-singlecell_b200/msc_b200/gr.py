"""Spatial graph builders (squidpy's ``gr.spatial_neighbors_knn`` / ``_radius`` / ``_grid`` /
``_delaunay`` contract), as metalsinglecell's ``gr`` provides them (gr.py:19-368): the first three
on the GPU grid search of ``msc_b200.spatial``, the Delaunay triangulation on SciPy's Qhull (as
the reference has it) with the edge lengths on the GPU.

The search and the FP64 edge lengths run on the device; the tail the reference runs on the host
with SciPy — percentile pruning on the distances, ``set_diag``, the adjacency transform, the
block-diagonal assembly of per-library graphs (gr.py:81-147) — runs on the host here too, with
the same operations, so the two CSR matrices equal the reference's for the same neighbour lists.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np

from . import spatial as _sp
from .neighbors import _torch


class SpatialNeighborsResult(NamedTuple):
    """What the builders return under ``copy=True`` (gr.py:150-154)."""

    connectivities: object
    distances: object


def _coords(adata, spatial_key):
    """float64 coordinates as stored, for edge lengths (gr.py:19-29)."""
    if spatial_key not in adata.obsm:
        raise KeyError(f"no adata.obsm[{spatial_key!r}] with spatial coordinates")
    return np.ascontiguousarray(adata.obsm[spatial_key], dtype=np.float64)


def _library_groups(adata, library_key):
    """Row indices per library, in category order, empty categories skipped (gr.py:107-120)."""
    if library_key is None:
        return None
    if library_key not in adata.obs:
        raise KeyError(f"no adata.obs[{library_key!r}] to group libraries by")
    col = adata.obs[library_key]
    import pandas as pd
    if not isinstance(getattr(col, "dtype", None), pd.CategoricalDtype):
        raise TypeError(f"adata.obs[{library_key!r}] must be categorical "
                        f"(squidpy requires it); got {getattr(col, 'dtype', type(col))}")
    codes = np.asarray(col.cat.codes if hasattr(col, "cat") else col.codes)
    groups = [np.flatnonzero(codes == c) for c in range(len(col.dtype.categories))]
    return [g for g in groups if g.size]


def _keep(M, keep):
    """The entries of CSR ``M`` where ``keep`` holds and the value is non-zero."""
    import scipy.sparse as sp
    ok = np.asarray(keep, bool) & (M.data != 0)
    rows = np.repeat(np.arange(M.shape[0]), np.diff(M.indptr))[ok]
    indptr = np.zeros(M.shape[0] + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=M.shape[0]), out=indptr[1:])
    return sp.csr_matrix((M.data[ok], M.indices[ok], indptr), shape=M.shape)


def _transform(adj, transform):
    """None | 'spectral' (D^-1/2 A D^-1/2, D the column degrees, zero degree → zero scale) |
    'cosine' (row cosine similarity), gr.py:37-57."""
    import scipy.sparse as sp
    if transform in (None, "none"):
        return adj
    if transform == "spectral":
        deg = np.asarray(adj.sum(axis=0)).ravel()
        scale = np.zeros_like(deg)
        np.divide(1.0, np.sqrt(deg), out=scale, where=deg > 0)
        D = sp.diags(scale)
        return (D @ adj @ D).tocsr()
    if transform == "cosine":
        from sklearn.metrics.pairwise import cosine_similarity
        return sp.csr_matrix(cosine_similarity(adj, dense_output=False))
    raise NotImplementedError(f"transform={transform!r} is not implemented "
                              f"(expected None, 'spectral' or 'cosine')")


def _finish(adj, dst, transform, set_diag, percentile):
    """percentile prune on the distances → set_diag → distances without diagonal and zeros →
    transform (gr.py:81-104)."""
    import scipy.sparse as sp
    adj, dst = sp.csr_matrix(adj), sp.csr_matrix(dst)
    if percentile is not None and dst.nnz:
        keep = dst.data <= np.percentile(dst.data, percentile)
        adj, dst = _keep(adj, keep), _keep(dst, keep)
    if set_diag:
        adj = adj.maximum(sp.identity(adj.shape[0], format="csr", dtype=adj.dtype)).tocsr()
    rows = np.repeat(np.arange(dst.shape[0]), np.diff(dst.indptr))
    dst = _keep(dst, dst.indices != rows)
    return _transform(adj, transform), dst


def _assemble(coords64, groups, build, transform, set_diag, percentile):
    """One graph per library, finished on its own, combined block-diagonally and returned in
    observation order (gr.py:123-147)."""
    import scipy.sparse as sp
    if groups is None:
        return _finish(*build(coords64), transform, set_diag, percentile)
    parts = [_finish(*build(np.ascontiguousarray(coords64[g])), transform, set_diag, percentile)
             for g in groups]
    adj = sp.block_diag([p[0] for p in parts], format="csr")
    dst = sp.block_diag([p[1] for p in parts], format="csr")
    order = np.concatenate(groups) if groups else np.zeros(0, np.int64)
    if np.any(np.diff(order) < 0):
        back = np.argsort(order)
        adj, dst = adj[back][:, back], dst[back][:, back]
    return adj.tocsr(), dst.tocsr()


def _write(adata, adj, dst, params, key_added, transform, copy):
    """squidpy's slots, or the pair under ``copy`` (gr.py:157-168)."""
    if copy:
        return SpatialNeighborsResult(adj, dst)
    ck, dk = f"{key_added}_connectivities", f"{key_added}_distances"
    adata.obsp[ck] = adj
    adata.obsp[dk] = dst
    adata.uns[f"{key_added}_neighbors"] = {"connectivities_key": ck, "distances_key": dk,
                                           "params": {**params, "transform": transform}}
    return None


def knn_edges(x64: np.ndarray, n_neighs: int, device=None):
    """``(indptr int64, cols int32, lengths float64)`` of the directed n_neighs-NN graph of the
    float64 coordinates ``x64`` (search on their float32 rounding, lengths in FP64): the edge
    list of gr._knn_edges (gr.py:186-195) with the lengths of gr._edge_lengths."""
    torch = _torch()
    dev = _sp._device(torch, device)
    n = x64.shape[0]
    if not 0 < n_neighs < n:
        raise ValueError(f"n_neighs={n_neighs} must be in [1, n - 1 = {n - 1}]")
    x64d = torch.from_numpy(np.ascontiguousarray(x64, np.float64)).to(dev)
    idx, _ = _sp.knn_lists_device(x64d.float(), n_neighs + 1)
    cols = idx[:, 1:].contiguous().view(-1)
    indptr = torch.arange(n + 1, dtype=torch.int64, device=dev) * n_neighs
    length = _sp.edge_lengths_device(x64d, indptr, cols)
    return indptr.cpu().numpy(), cols.cpu().numpy(), length.cpu().numpy()


def radius_edges(x64: np.ndarray, lo: float, hi: float, device=None):
    """``(indptr int64, cols int32, lengths float64)`` of every pair with lo ≤ distance ≤ hi
    (float32 test as ``_radius_grid``), lengths in FP64."""
    torch = _torch()
    dev = _sp._device(torch, device)
    if x64.shape[1] not in (2, 3):
        raise ValueError(f"radius search expects 2-D or 3-D coordinates, got {x64.shape[1]}-D")
    x64d = torch.from_numpy(np.ascontiguousarray(x64, np.float64)).to(dev)
    indptr, cols, _, _ = _sp.radius_grid_device(x64d.float(), hi, lo)
    length = _sp.edge_lengths_device(x64d, indptr, cols)
    return indptr.cpu().numpy(), cols.cpu().numpy(), length.cpu().numpy()


def knn_edges_f32(x64: np.ndarray, n_neighs: int, device=None):
    """``(cols int32 (n·n_neighs,), dist float32)``: each point's n_neighs nearest other points
    and their float32 grid distances (the lists the lattice builder corrects by the median)."""
    torch = _torch()
    dev = _sp._device(torch, device)
    n = x64.shape[0]
    if not 0 < n_neighs < n:
        raise ValueError(f"n_neighs={n_neighs} must be in [1, n - 1 = {n - 1}]")
    x32 = torch.from_numpy(np.ascontiguousarray(x64, np.float64)).to(dev).float()
    idx, dist = _sp.knn_lists_device(x32, n_neighs + 1)
    return (idx[:, 1:].contiguous().view(-1).cpu().numpy(),
            dist[:, 1:].contiguous().view(-1).cpu().numpy())


def _with_diag(M):
    """1.0 on the diagonal of a 0/1 (or ring-valued, diagonal ≤ 1) CSR."""
    import scipy.sparse as sp
    return M.maximum(sp.identity(M.shape[0], format="csr", dtype=M.dtype)).tocsr()


def _without_diag(M):
    rows = np.repeat(np.arange(M.shape[0]), np.diff(M.indptr))
    return _keep(M, M.indices != rows)


def _rings(adj, n_rings: int):
    """Breadth-first ring index of every point reachable within ``n_rings`` steps of the
    graph (the point itself at 1 with its direct neighbours, then 2, 3, ...): squidpy's grid
    convention, where the distances hold the ring, not a length."""
    import scipy.sparse as sp
    step = _with_diag(adj).astype(bool).astype(np.float32)
    reached = step.copy()
    level = step.copy()
    frontier = step
    for r in range(2, n_rings + 1):
        nxt = (frontier @ step).astype(bool).tocsr()
        fresh = (nxt.astype(np.int8) - nxt.multiply(reached.astype(bool)).astype(np.int8)).tocsr()
        fresh.eliminate_zeros()
        if fresh.nnz == 0:
            break
        fresh = fresh.astype(np.float32)
        frontier = fresh
        reached = (reached + fresh).tocsr()
        fresh.data[:] = float(r)
        level = (level + fresh).tocsr()
    return sp.csr_matrix(level)


def _delaunay(x32: np.ndarray):
    """Symmetric 0/1 adjacency of the Delaunay triangulation (SciPy's Qhull, as gr.py:303-310
    builds it from the float32 working coordinates)."""
    import scipy.sparse as sp
    from scipy.spatial import Delaunay
    tri = Delaunay(np.asarray(x32, dtype=np.float64))
    indptr, indices = tri.vertex_neighbor_vertices
    n = x32.shape[0]
    return sp.csr_matrix((np.ones(indices.size, np.float32), indices, indptr), shape=(n, n))


def spatial_neighbors_grid(adata, *, n_neighs: int = 6, n_rings: int = 1, delaunay: bool = False,
                           spatial_key: str = "spatial", library_key: str | None = None,
                           transform: str | None = None, set_diag: bool = False,
                           key_added: str = "spatial", copy: bool = False, device=None):
    """Lattice spatial graph (gr.py:257-300), the Visium / Stereo-seq mode: the n_neighs-NN
    graph without the edges longer than 1.3 × the median kNN distance (squidpy's lattice
    correction; or the Delaunay triangulation), expanded to ``n_rings`` rings; binary
    connectivities, distances holding the ring index."""
    import scipy.sparse as sp

    def build(x64):
        n = x64.shape[0]
        x32 = x64.astype(np.float32)
        if delaunay:
            adj = _delaunay(x32)
        else:
            cols, dist = knn_edges_f32(x64, n_neighs, device)
            rows = np.repeat(np.arange(n), n_neighs)
            keep = dist < np.median(dist) * 1.3
            adj = sp.csr_matrix((np.ones(int(keep.sum()), np.float32), (rows[keep], cols[keep])),
                                shape=(n, n))
        if n_rings > 1:
            lv = _rings(adj, n_rings)
            lv = _with_diag(lv) if set_diag else _without_diag(lv)
            lv.eliminate_zeros()
            dst = lv.copy()
            adj = lv.copy()
            adj.data[:] = 1.0
        else:
            if set_diag:
                adj = _with_diag(adj)
            dst = adj.copy()
        return adj, dst

    adj, dst = _assemble(_coords(adata, spatial_key), _library_groups(adata, library_key), build,
                         transform, set_diag, None)
    return _write(adata, adj, dst, {"coord_type": "grid", "n_neighbors": n_neighs,
                                    "n_rings": n_rings, "delaunay": delaunay},
                  key_added, transform, copy)


def delaunay_edges(x64: np.ndarray, device=None):
    """``(rows, cols, lengths float64)`` of the Delaunay triangulation of the float64
    coordinates (SciPy's Qhull, gr.py:313-320, 355-357), lengths on the device."""
    import scipy.sparse as sp
    from scipy.spatial import Delaunay
    torch = _torch()
    dev = _sp._device(torch, device)
    n = x64.shape[0]
    indptr, indices = Delaunay(np.asarray(x64, dtype=np.float64)).vertex_neighbor_vertices
    A = sp.csr_matrix((np.ones(indices.size, np.float32), indices, indptr), shape=(n, n)).tocoo()
    # COO of the CSR: rows ascending, columns in stored order within a row
    ip = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(A.row, minlength=n), out=ip[1:])
    length = _sp.edge_lengths_device(torch.from_numpy(np.ascontiguousarray(x64, np.float64)).to(dev),
                                     torch.from_numpy(ip).to(dev),
                                     torch.from_numpy(A.col.astype(np.int32)).to(dev))
    return A.row, A.col, length.cpu().numpy()


def spatial_neighbors_delaunay(adata, *, radius=None, spatial_key: str = "spatial",
                               library_key: str | None = None, percentile: float | None = None,
                               transform: str | None = None, set_diag: bool = False,
                               key_added: str = "spatial", copy: bool = False, device=None):
    """Delaunay spatial graph (gr.py:323-368): the triangulation (SciPy's Qhull, as the
    reference and squidpy use), optionally pruned to edges of length within ``radius`` (a
    maximum or a (min, max) interval); binary connectivities, FP64 edge lengths."""
    import scipy.sparse as sp
    stored = radius
    if radius is not None:
        lo, hi = ((0.0, float(radius)) if np.isscalar(radius)
                  else (float(min(radius)), float(max(radius))))
        stored = (lo, hi)

    def build(x64):
        n = x64.shape[0]
        rows, cols, dist = delaunay_edges(x64, device)
        if radius is not None:
            keep = (dist >= lo) & (dist <= hi)
            rows, cols, dist = rows[keep], cols[keep], dist[keep]
        return (sp.csr_matrix((np.ones(dist.size, np.float32), (rows, cols)), shape=(n, n)),
                sp.csr_matrix((dist, (rows, cols)), shape=(n, n)))

    adj, dst = _assemble(_coords(adata, spatial_key), _library_groups(adata, library_key), build,
                         transform, set_diag, percentile)
    return _write(adata, adj, dst, {"coord_type": "generic", "radius": stored},
                  key_added, transform, copy)


def _pair(n, indptr, cols, length):
    import scipy.sparse as sp
    return (sp.csr_matrix((np.ones(length.size, np.float32), cols, indptr), shape=(n, n)),
            sp.csr_matrix((length, cols, indptr), shape=(n, n)))


def spatial_neighbors_knn(adata, *, n_neighs: int = 6, spatial_key: str = "spatial",
                          library_key: str | None = None, percentile: float | None = None,
                          transform: str | None = None, set_diag: bool = False,
                          key_added: str = "spatial", copy: bool = False, device=None):
    """Directed k-NN spatial graph (gr.py:198-225): ``n_neighs`` edges per observation, self
    excluded, the nearest in (float32 distance, index) order; binary connectivities, FP64
    Euclidean distances.  ``library_key`` builds one graph per section."""
    def build(x64):
        return _pair(x64.shape[0], *knn_edges(x64, n_neighs, device))

    adj, dst = _assemble(_coords(adata, spatial_key), _library_groups(adata, library_key), build,
                         transform, set_diag, percentile)
    return _write(adata, adj, dst, {"coord_type": "generic", "n_neighbors": n_neighs},
                  key_added, transform, copy)


def spatial_neighbors_radius(adata, *, radius, spatial_key: str = "spatial",
                             library_key: str | None = None, percentile: float | None = None,
                             transform: str | None = None, set_diag: bool = False,
                             key_added: str = "spatial", copy: bool = False, device=None):
    """Fixed-radius spatial graph (gr.py:228-255): every pair within ``radius`` (a maximum, or
    a ``(min, max)`` interval); binary connectivities, FP64 Euclidean distances."""
    if np.isscalar(radius):
        lo, hi = 0.0, float(radius)
    else:
        lo, hi = float(min(radius)), float(max(radius))

    def build(x64):
        return _pair(x64.shape[0], *radius_edges(x64, lo, hi, device))

    adj, dst = _assemble(_coords(adata, spatial_key), _library_groups(adata, library_key), build,
                         transform, set_diag, percentile)
    return _write(adata, adj, dst, {"coord_type": "generic", "radius": radius},
                  key_added, transform, copy)


def spatial_neighbors(adata, n_neighs: int = 6, coord_type: str | None = None, n_rings: int = 1,
                      delaunay: bool = False, radius=None, spatial_key: str = "spatial",
                      library_key: str | None = None, transform: str | None = None,
                      set_diag: bool = False, percentile: float | None = None,
                      key_added: str = "spatial", copy: bool = False, device=None):
    """The deprecated single entry point (gr.py:371-411, squidpy's ``gr.spatial_neighbors``):
    warns, then dispatches to the mode builders.  ``coord_type`` None means 'grid' when
    ``uns['spatial']`` exists, else 'generic'; 'grid' rejects ``percentile``; with
    ``delaunay=True`` a scalar ``radius`` is ignored and a (min, max) tuple applied — the legacy
    behaviour code written against this entry point expects."""
    import warnings
    warnings.warn("gr.spatial_neighbors is deprecated (squidpy removes it in 1.9). Use "
                  "spatial_neighbors_knn / spatial_neighbors_radius / spatial_neighbors_delaunay"
                  " / spatial_neighbors_grid.", FutureWarning, stacklevel=2)
    if coord_type is None:
        coord_type = "grid" if "spatial" in adata.uns else "generic"
    common = dict(spatial_key=spatial_key, library_key=library_key, transform=transform,
                  set_diag=set_diag, key_added=key_added, copy=copy, device=device)
    if coord_type == "grid":
        if percentile is not None:
            raise ValueError("'percentile' is not supported for grid coordinates")
        return spatial_neighbors_grid(adata, n_neighs=n_neighs, n_rings=n_rings,
                                      delaunay=delaunay, **common)
    if coord_type != "generic":
        raise ValueError(f"coord_type must be 'grid', 'generic' or None, got {coord_type!r}")
    if delaunay:
        return spatial_neighbors_delaunay(adata, radius=radius if isinstance(radius, tuple)
                                          else None, percentile=percentile, **common)
    if radius is not None:
        return spatial_neighbors_radius(adata, radius=radius, percentile=percentile, **common)
    return spatial_neighbors_knn(adata, n_neighs=n_neighs, percentile=percentile, **common)
