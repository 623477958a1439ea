"""Parity of the spatial grid search (``msc_spatial_*`` through the C ABI) with the CPU oracle
(oracle/spatial.py), and of the spatial graph builders with the reference's own ``gr`` code
(tests/golden/reference_spatial.npz).

The bar is bit-exact: kNN indices (self first, (distance, index) order) and float32 distances;
radius CSR structure (columns ascending) and float32 distances; FP64 edge lengths; the builders'
two CSR matrices, dtypes included.  Cases: the reference's hex lattice (exact ties), jittered
lattices, clustered points with far outliers (rings beyond the first), an elongated bounding
box (coarsened cells), 3-D clouds with duplicates, Xenium-scale coordinates, collinear and
coincident points, the smallest sizes, and the widest k.
"""
import json
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import spatial as osp
from msc_b200 import spatial as msp, gr, _lib, AnnDataLite

pytestmark = pytest.mark.gpu

G = Path(__file__).resolve().parent / "golden"


def lattice(side, jitter=0.0, seed=0):
    r, c = np.divmod(np.arange(side * side), side)
    xy = np.c_[c * 100.0 + (r % 2) * 50.0, r * 86.6]
    if jitter:
        xy = xy + np.random.default_rng(seed).normal(0, jitter, xy.shape)
    return xy.astype(np.float32)


def case(name):
    rng = np.random.default_rng(11)
    if name == "lattice":
        return lattice(40)
    if name == "jitter":
        return lattice(40, 1.0)
    if name == "clusters":
        return np.vstack([rng.normal(0, 1, (3000, 2)), rng.normal(50, 5, (800, 2)),
                          rng.uniform(-500, 500, (40, 2))]).astype(np.float32)
    if name == "elongated":
        return np.c_[rng.uniform(0, 1e5, 4000), rng.uniform(0, 1, 4000)].astype(np.float32)
    if name == "vol":
        return rng.uniform(0, 50, (6000, 3)).astype(np.float32)
    if name == "int3d_dups":
        X = np.round(rng.uniform(0, 30, (3000, 3))).astype(np.float32)
        X[2000:2100] = X[:100]
        return X
    if name == "xenium":
        return (lattice(30, 0.5) + 2e5).astype(np.float32)
    if name == "collinear":
        return np.c_[np.arange(700), np.zeros(700)].astype(np.float32)
    if name == "coincident":
        return np.ones((50, 2), np.float32)
    raise KeyError(name)


def knn_device(X, k):
    import torch
    idx, dist, stats = msp.knn_grid_device(torch.from_numpy(X).cuda(), k)
    torch.cuda.synchronize()
    st = stats.cpu().numpy()
    _lib.check_spatial_stats(st)
    return idx.cpu().numpy(), dist.cpu().numpy(), st


@pytest.mark.parametrize("name,k", [
    ("lattice", 7), ("lattice", 11), ("jitter", 12), ("clusters", 16), ("elongated", 9),
    ("vol", 20), ("int3d_dups", 65), ("int3d_dups", 2), ("xenium", 8), ("collinear", 5),
    ("coincident", 10), ("jitter", 33), ("vol", 64),
])
def test_knn_equals_oracle(name, k):
    X = case(name)
    gi, gd, st = knn_device(X, k)
    oi, od = osp.grid_knn(X, k)
    np.testing.assert_array_equal(gi, oi.astype(np.int32), err_msg="indices")
    np.testing.assert_array_equal(gd, od, err_msg="distances")
    assert st[_lib.SP_STAT_CELLS] >= 1 and st[_lib.SP_STAT_EVALS] > 0
    if name == "clusters":
        assert st[_lib.SP_STAT_EXPANDED] > 0          # the outliers needed more rings


def test_knn_smallest_sizes():
    for n in (1, 2, 3, 33):
        X = np.random.default_rng(n).uniform(0, 10, (n, 2)).astype(np.float32)
        for k in sorted({1, n}):
            gi, gd, _ = knn_device(X, k)
            oi, od = osp.grid_knn(X, k)
            np.testing.assert_array_equal(gi, oi.astype(np.int32))
            np.testing.assert_array_equal(gd, od)


def radius_device(X, r, rlo=0.0):
    import torch
    ip, c, d, st = msp.radius_grid_device(torch.from_numpy(X).cuda(), r, rlo)
    torch.cuda.synchronize()
    _lib.check_spatial_stats(st.cpu().numpy())
    return ip.cpu().numpy(), c.cpu().numpy(), d.cpu().numpy()


def reference_radius_inputs():
    rng = np.random.RandomState(0)
    return [(rng.uniform(0, 100, (3000, 2)).astype(np.float32), 6.0),
            ((rng.normal(size=(3000, 2)) * [30, 3]).astype(np.float32), 4.0),
            (rng.uniform(0, 50, (2000, 3)).astype(np.float32), 7.0)]


@pytest.mark.parametrize("i", [0, 1, 2])
def test_radius_reference_inputs(i):
    """The reference's own radius known-answer inputs (tests/test_spatial_neighbors.py:363-375)."""
    X, r = reference_radius_inputs()[i]
    ip, c, d = radius_device(X, r)
    oip, oc, od = osp.grid_radius(X, r)
    np.testing.assert_array_equal(ip, oip)
    np.testing.assert_array_equal(c, oc)
    np.testing.assert_array_equal(d, od)


@pytest.mark.parametrize("name,r,rlo", [
    ("lattice", 150.0, 0.0), ("jitter", 200.0, 130.0), ("clusters", 0.5, 0.0),
    ("elongated", 40.0, 0.0), ("vol", 7.0, 2.0), ("int3d_dups", 2.0, 0.0), ("xenium", 101.0, 0.0),
    ("collinear", 1.0, 0.0), ("coincident", 0.0, 0.0), ("coincident", 1.0, 0.5),
])
def test_radius_equals_oracle(name, r, rlo):
    X = case(name)
    ip, c, d = radius_device(X, r, rlo)
    oip, oc, od = osp.grid_radius(X, r, rlo)
    np.testing.assert_array_equal(ip, oip)
    np.testing.assert_array_equal(c, oc)
    np.testing.assert_array_equal(d, od)


def test_host_mirrors():
    X = case("jitter")
    idx, dist = msp._knn_grid(X, 7)
    oi, od = osp.grid_knn(X, 7)
    assert idx.dtype == np.int64 and dist.dtype == np.float32
    np.testing.assert_array_equal(idx, oi)
    ip, c, d = msp._radius_grid(X, 120.0)
    assert ip.dtype == np.int64 and c.dtype == np.int32 and d.dtype == np.float32
    oip, oc, od = osp.grid_radius(X, 120.0)
    np.testing.assert_array_equal(c, oc)
    A = msp.spatial_neighbors(X, n_neighs=6)
    assert (np.diff(A.indptr) == 6).all() and A.diagonal().sum() == 0
    S = msp.spatial_neighbors(X, n_neighs=6, symmetric=True)
    assert (abs(S - S.T) > 0).nnz == 0
    # requests the grid does not take go to the exact kNN (4-D coordinates, k above 65)
    X4 = np.random.default_rng(2).uniform(0, 1, (500, 4)).astype(np.float32)
    i4, _ = msp._knn_grid(X4, 5)
    assert (i4[:, 0] == np.arange(500)).all()
    with pytest.raises(ValueError):
        msp._radius_grid(X4, 0.1)


def test_edge_lengths_fp64():
    import torch
    xy = case("xenium").astype(np.float64) + np.random.default_rng(3).uniform(0, 1e-3, (900, 2))
    ip, c, _ = osp.grid_radius(xy.astype(np.float32), 120.0)
    L = msp.edge_lengths_device(torch.from_numpy(xy).cuda(), torch.from_numpy(ip).cuda(),
                                torch.from_numpy(c).cuda()).cpu().numpy()
    rows = np.repeat(np.arange(900), np.diff(ip))
    np.testing.assert_array_equal(L, osp.edge_lengths_f64(xy, rows, c))


def test_builders_equal_reference_gr():
    import pandas as pd
    g = np.load(G / "reference_spatial.npz")
    for c in range(int(g["n_cases"])):
        kind, name, kw = json.loads(str(g[f"c{c}_case"]))
        if isinstance(kw.get("radius"), list):
            kw["radius"] = tuple(kw["radius"])
        xy = g[f"{name}_coords"]
        obs, extra = {}, {}
        if f"{name}_library" in g:
            obs["library"] = pd.Categorical.from_codes(g[f"{name}_library"], ["s0", "s1", "s2"])
            extra["library_key"] = "library"
        a = AnnDataLite(obs=obs, obsm={"spatial": xy}, n_obs=xy.shape[0])
        fn = {"knn": gr.spatial_neighbors_knn, "radius": gr.spatial_neighbors_radius,
              "grid": gr.spatial_neighbors_grid, "delaunay": gr.spatial_neighbors_delaunay}[kind]
        res = fn(a, copy=True, **kw, **extra)
        for tag, M in (("adj", res.connectivities), ("dst", res.distances)):
            M = sp.csr_matrix(M)
            M.sort_indices()
            np.testing.assert_array_equal(M.indptr, g[f"c{c}_{tag}_indptr"], err_msg=f"{c}{tag}")
            np.testing.assert_array_equal(M.indices, g[f"c{c}_{tag}_indices"], err_msg=f"{c}{tag}")
            assert M.data.dtype == g[f"c{c}_{tag}_data"].dtype
            np.testing.assert_array_equal(M.data, g[f"c{c}_{tag}_data"], err_msg=f"{c}{tag}")


def test_errors_and_nonfinite():
    import torch
    X = case("jitter").copy()
    X[5, 1] = np.nan
    _, _, stats = msp.knn_grid_device(torch.from_numpy(X).cuda(), 5)
    torch.cuda.synchronize()
    with pytest.raises(ValueError):
        _lib.check_spatial_stats(stats.cpu().numpy())
    with pytest.raises(ValueError):
        msp.radius_grid_device(torch.from_numpy(X).cuda(), 10.0)
    with pytest.raises(ValueError):
        msp.knn_grid_device(torch.from_numpy(case("jitter")).cuda(), 0)


def test_full_size_slide():
    """1,000,000 spots of the bench's synthetic slide, k = 7 and a 10 µm radius (~7M edges):
    properties that
    hold at any size, and bit-exact rows against the oracle on 128 seeded spots (each scanned
    against all 1M)."""
    import torch
    import bench
    xy = bench.spatial_slide(1_000_000).astype(np.float32)
    n = xy.shape[0]
    gi, gd, st = knn_device(xy, 7)
    assert (gi[:, 0] == np.arange(n)).all() and (gd[:, 0] == 0).all()
    assert gi.min() >= 0 and gi.max() < n
    assert (np.diff(gd, axis=1) >= 0).all()
    s = np.sort(gi, axis=1)
    assert (np.diff(s, axis=1) > 0).all()
    rows = np.sort(np.random.default_rng(20261204).choice(n, 128, replace=False))
    oi, od = osp.grid_knn(xy, 7, rows=rows)
    np.testing.assert_array_equal(gi[rows], oi.astype(np.int32))
    np.testing.assert_array_equal(gd[rows], od)
    ip, c, d = radius_device(xy, 10.0)
    A = sp.csr_matrix((d, c, ip), shape=(n, n))
    assert A.has_sorted_indices and A.diagonal().sum() == 0
    assert (abs(A - A.T) > 0).nnz == 0                    # symmetric, distances bit-equal
    assert d.max() <= 10.0
