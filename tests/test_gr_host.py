"""Host logic of the spatial graph builders (``msc_b200.gr``) on the CPU: the device search is
replaced by the oracle's (oracle/spatial.py), so the tail the builders run on the host —
percentile pruning, set_diag, the transforms, per-library assembly, the squidpy slots — is
checked against the reference's own ``gr`` code (tests/golden/reference_spatial.npz, bit for bit)
without a GPU.  The GPU lane runs the same cases through the device search
(tests/test_gpu_spatial.py)."""
import json
from pathlib import Path

import numpy as np
import pandas as pd
import pytest
import scipy.sparse as sp

from oracle import spatial as osp
from msc_b200 import gr, AnnDataLite

G = Path(__file__).resolve().parent / "golden"


def _oracle_knn_edges(x64, n_neighs, device=None):
    n = x64.shape[0]
    if not 0 < n_neighs < n:
        raise ValueError("n_neighs out of range")
    rows, cols, _ = osp.knn_edges(x64.astype(np.float32), n_neighs)
    indptr = np.arange(n + 1, dtype=np.int64) * n_neighs
    return indptr, cols.astype(np.int32), osp.edge_lengths_f64(x64, rows, cols)


def _oracle_radius_edges(x64, lo, hi, device=None):
    indptr, cols, _ = osp.grid_radius(x64.astype(np.float32), hi, lo)
    rows = np.repeat(np.arange(x64.shape[0]), np.diff(indptr))
    return indptr, cols, osp.edge_lengths_f64(x64, rows, cols)


def _oracle_knn_edges_f32(x64, n_neighs, device=None):
    _, cols, dist = osp.knn_edges(x64.astype(np.float32), n_neighs)
    return cols.astype(np.int32), dist


def _host_delaunay_edges(x64, device=None):
    import scipy.sparse as sp
    from scipy.spatial import Delaunay
    n = x64.shape[0]
    ip, ind = Delaunay(np.asarray(x64, dtype=np.float64)).vertex_neighbor_vertices
    A = sp.csr_matrix((np.ones(ind.size, np.float32), ind, ip), shape=(n, n)).tocoo()
    return A.row, A.col, osp.edge_lengths_f64(x64, A.row, A.col)


@pytest.fixture
def oracle_search(monkeypatch):
    monkeypatch.setattr(gr, "delaunay_edges", _host_delaunay_edges)
    monkeypatch.setattr(gr, "knn_edges", _oracle_knn_edges)
    monkeypatch.setattr(gr, "knn_edges_f32", _oracle_knn_edges_f32)
    monkeypatch.setattr(gr, "radius_edges", _oracle_radius_edges)


def golden_cases():
    g = np.load(G / "reference_spatial.npz")
    for c in range(int(g["n_cases"])):
        kind, name, kw = json.loads(str(g[f"c{c}_case"]))
        if isinstance(kw.get("radius"), list):
            kw["radius"] = tuple(kw["radius"])
        lib = g[f"{name}_library"] if f"{name}_library" in g else None
        yield c, kind, g[f"{name}_coords"], lib, kw, g


def adata_for(xy, lib):
    obs = {}
    if lib is not None:
        obs["library"] = pd.Categorical.from_codes(lib, ["s0", "s1", "s2"][:max(3, lib.max() + 1)])
    return AnnDataLite(obs=obs, obsm={"spatial": xy}, n_obs=xy.shape[0])


def assert_same(M, g, c, tag):
    M = sp.csr_matrix(M)
    M.sort_indices()
    np.testing.assert_array_equal(M.indptr, g[f"c{c}_{tag}_indptr"])
    np.testing.assert_array_equal(M.indices, g[f"c{c}_{tag}_indices"])
    ref = g[f"c{c}_{tag}_data"]
    assert M.data.dtype == ref.dtype, (c, tag)
    np.testing.assert_array_equal(M.data, ref)


def test_builders_equal_reference_gr(oracle_search):
    n = 0
    for c, kind, xy, lib, kw, g in golden_cases():
        fn = {"knn": gr.spatial_neighbors_knn, "radius": gr.spatial_neighbors_radius,
              "grid": gr.spatial_neighbors_grid, "delaunay": gr.spatial_neighbors_delaunay}[kind]
        extra = {"library_key": "library"} if lib is not None else {}
        res = fn(adata_for(xy, lib), copy=True, **kw, **extra)
        assert isinstance(res, gr.SpatialNeighborsResult)
        assert_same(res.connectivities, g, c, "adj")
        assert_same(res.distances, g, c, "dst")
        n += 1
    assert n == 22


def test_slots_and_params(oracle_search):
    xy = np.random.default_rng(0).uniform(0, 500, (300, 2))
    a = adata_for(xy, None)
    assert gr.spatial_neighbors_knn(a, n_neighs=5, transform="spectral") is None
    assert set(a.obsp) == {"spatial_connectivities", "spatial_distances"}
    assert a.uns["spatial_neighbors"] == {
        "connectivities_key": "spatial_connectivities", "distances_key": "spatial_distances",
        "params": {"coord_type": "generic", "n_neighbors": 5, "transform": "spectral"}}
    gr.spatial_neighbors_radius(a, radius=(10.0, 60.0), key_added="ring")
    assert a.uns["ring_neighbors"]["params"] == {"coord_type": "generic", "radius": (10.0, 60.0),
                                                 "transform": None}
    D = a.obsp["ring_distances"]
    assert D.data.min() >= 10.0 - 1e-3 and D.data.max() <= 60.0 + 1e-3


def test_errors(oracle_search):
    xy = np.random.default_rng(1).uniform(0, 100, (50, 2))
    with pytest.raises(KeyError):
        gr.spatial_neighbors_knn(AnnDataLite(obsm={"xy": xy}, n_obs=50))
    with pytest.raises(KeyError):
        gr.spatial_neighbors_knn(adata_for(xy, None), library_key="missing")
    bad = AnnDataLite(obs={"library": np.zeros(50, int)}, obsm={"spatial": xy}, n_obs=50)
    with pytest.raises(TypeError):
        gr.spatial_neighbors_knn(bad, library_key="library")
    with pytest.raises(NotImplementedError):
        gr.spatial_neighbors_knn(adata_for(xy, None), transform="laplacian")
    with pytest.raises(ValueError):
        gr.spatial_neighbors_knn(adata_for(xy, None), n_neighs=50)


def test_deprecated_entry_point_dispatches(oracle_search):
    xy = np.random.default_rng(4).uniform(0, 1000, (400, 2))

    def same(a, b):
        for x, y in zip(a, b):
            x, y = sp.csr_matrix(x), sp.csr_matrix(y)
            x.sort_indices()
            y.sort_indices()
            assert (x != y).nnz == 0 and x.data.dtype == y.data.dtype

    a = adata_for(xy, None)
    with pytest.warns(FutureWarning):
        r = gr.spatial_neighbors(a, n_neighs=5, copy=True)
    same(r, gr.spatial_neighbors_knn(a, n_neighs=5, copy=True))
    with pytest.warns(FutureWarning):
        r = gr.spatial_neighbors(a, radius=80.0, copy=True)
    same(r, gr.spatial_neighbors_radius(a, radius=80.0, copy=True))
    with pytest.warns(FutureWarning):                  # a scalar radius is ignored with delaunay
        r = gr.spatial_neighbors(a, delaunay=True, radius=10.0, copy=True)
    same(r, gr.spatial_neighbors_delaunay(a, copy=True))
    with pytest.warns(FutureWarning):                  # a tuple radius is applied
        r = gr.spatial_neighbors(a, delaunay=True, radius=(0.0, 60.0), copy=True)
    same(r, gr.spatial_neighbors_delaunay(a, radius=(0.0, 60.0), copy=True))
    g = adata_for(xy, None)
    g.uns["spatial"] = {}                              # Visium-style: grid inferred
    with pytest.warns(FutureWarning):
        r = gr.spatial_neighbors(g, n_neighs=6, n_rings=2, copy=True)
    same(r, gr.spatial_neighbors_grid(g, n_neighs=6, n_rings=2, copy=True))
    with pytest.warns(FutureWarning), pytest.raises(ValueError):
        gr.spatial_neighbors(g, percentile=90.0)
    with pytest.warns(FutureWarning), pytest.raises(ValueError):
        gr.spatial_neighbors(a, coord_type="hexagonal")
