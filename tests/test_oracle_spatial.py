"""The spatial oracle (oracle/spatial.py) against the reference's own known-answer criteria for
its uniform-grid index, run here with sklearn as the independent exact search:

* ``tests/test_spatial_neighbors.py:363-375``: the radius search gives exactly sklearn's
  ``radius_neighbors_graph`` pattern (diagonal removed) on three seeded inputs — 2-D uniform,
  2-D anisotropic normal, 3-D uniform;
* ``:378-387``: distances survive Visium/Xenium-scale coordinates (273 ± 1e-3);
* ``:33-47``: kNN sets equal sklearn's except where two candidates are exactly equidistant,
  on the reference's hex lattice (ties by construction) and a jittered one;
* the rules the oracle states: self first, (float32 distance, index) order, ascending columns,
  the annulus ``(min_radius, radius)``.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import spatial as osp


def lattice(side=40, jitter=0.0, seed=0):
    """The reference test's Visium-like hex lattice (spacing 100), optionally jittered."""
    r, c = np.divmod(np.arange(side * side), side)
    xy = np.c_[c * 100.0 + (r % 2) * 50.0, r * 86.6]
    if jitter:
        xy = xy + np.random.default_rng(seed).normal(0, jitter, xy.shape)
    return xy


def tie_free_differences(idx_a, idx_b, coords):
    """Rows whose neighbour sets differ for a reason other than an exact distance tie."""
    bad = 0
    for i in range(idx_a.shape[0]):
        sa, sb = set(idx_a[i]), set(idx_b[i])
        if sa == sb:
            continue
        da = [np.linalg.norm(coords[i] - coords[j]) for j in sa - sb]
        db = [np.linalg.norm(coords[i] - coords[j]) for j in sb - sa]
        if not (da and db and abs(max(da) - max(db)) < 1e-9):
            bad += 1
    return bad


def reference_radius_inputs():
    rng = np.random.RandomState(0)
    return [(rng.uniform(0, 100, (3000, 2)).astype(np.float32), 6.0),
            ((rng.normal(size=(3000, 2)) * [30, 3]).astype(np.float32), 4.0),
            (rng.uniform(0, 50, (2000, 3)).astype(np.float32), 7.0)]


def test_radius_matches_sklearn_exactly():
    from sklearn.neighbors import NearestNeighbors
    for X, r in reference_radius_inputs():
        A = osp.radius_csr(X, r)
        ours = sp.csr_matrix((np.ones_like(A.data), A.indices, A.indptr), shape=A.shape)
        ref = NearestNeighbors(radius=r).fit(X).radius_neighbors_graph(mode="connectivity")
        ref.setdiag(0)
        ref.eliminate_zeros()
        assert (abs(ours - ref) > 0).nnz == 0
        assert A.has_sorted_indices and A.indices.dtype == np.int32
        assert A.data.dtype == np.float32 and A.data.max() <= r


def test_radius_annulus_and_distances():
    X = lattice(20, jitter=2.0).astype(np.float32)
    D = osp.radius_csr(X, 200.0)
    assert (abs(D - D.T) > 0).nnz == 0                      # symmetric, values included
    Db = osp.radius_csr(X, 200.0, 130.0)                    # drops the first shell
    assert 0 < Db.nnz < D.nnz
    assert Db.data.min() >= 130.0 - 1e-4 and Db.data.max() <= 200.0 + 1e-4
    exact = np.sqrt(((X[D.nonzero()[0]].astype(np.float64)
                      - X[D.indices].astype(np.float64)) ** 2).sum(1))
    assert np.abs(D.data - exact).max() <= 1e-4 * exact.max()


def test_distances_survive_large_coordinates():
    base = np.array([[9237.0, 15447.0], [9510.0, 15447.0], [9237.0, 15720.0]])
    for offset in (0.0, 20_000.0, 200_000.0):
        X = np.ascontiguousarray(base + offset, dtype=np.float32)
        _, d = osp.grid_knn(X, 2)
        assert abs(d[0, 1] - 273.0) < 1e-3, (offset, d[0, 1])
        _, _, dr = osp.grid_radius(X, 300.0)
        assert np.all(np.abs(dr - 273.0) < 1e-3)


@pytest.mark.parametrize("jitter", [0.0, 1.0])
def test_knn_matches_sklearn_up_to_ties(jitter):
    from sklearn.neighbors import NearestNeighbors
    xy = lattice(25, jitter=jitter)
    X = xy.astype(np.float32)
    idx, dist = osp.grid_knn(X, 7)
    assert (idx[:, 0] == np.arange(X.shape[0])).all() and (dist[:, 0] == 0).all()
    _, ref = NearestNeighbors(n_neighbors=6).fit(X).kneighbors()
    assert tie_free_differences(idx[:, 1:], ref, xy) == 0
    rows, cols, d = osp.knn_edges(X, 6)
    assert np.array_equal(cols.reshape(-1, 6), idx[:, 1:])


def test_knn_order_and_ties_3d():
    rng = np.random.default_rng(7)
    X = np.round(rng.uniform(0, 20, (1500, 3))).astype(np.float32)   # integer grid: many ties
    X[1000:1010] = X[0:10]                                            # coincident points
    idx, dist = osp.grid_knn(X, 12)
    n = X.shape[0]
    assert (idx[:, 0] == np.arange(n)).all()
    d2 = osp.sq_dist_f32(X, X)
    for i in range(0, n, 37):
        s = np.sqrt(d2[i])
        s[i] = -1
        o = np.lexsort((np.arange(n), s))[:12]
        assert np.array_equal(idx[i], o)
        assert np.array_equal(dist[i], np.maximum(s[o], 0).astype(np.float32))
    assert (dist[1000:1010, 1] == 0).all() and (idx[1000:1010, 1] == np.arange(10)).all()


def test_edge_cases():
    X = np.zeros((5, 2), np.float32)                        # all coincident
    idx, dist = osp.grid_knn(X, 5)
    assert (idx == np.array([[i] + [j for j in range(5) if j != i] for i in range(5)])).all()
    assert (dist == 0).all()
    ip, c, d = osp.grid_radius(X, 1.0)
    assert (np.diff(ip) == 4).all() and (d == 0).all()
    ip, c, d = osp.grid_radius(X, 1.0, 0.5)                 # annulus excludes distance 0
    assert ip[-1] == 0 and c.size == 0
    ip, c, d = osp.grid_radius(np.zeros((0, 2), np.float32), 1.0)
    assert ip.tolist() == [0] and c.size == 0
    with pytest.raises(ValueError):
        osp.grid_knn(X, 6)
    with pytest.raises(ValueError):
        osp.knn_edges(X, 5)


def test_knn_rows_subset_equals_full():
    X = np.random.default_rng(9).uniform(0, 100, (2000, 2)).astype(np.float32)
    full_i, full_d = osp.grid_knn(X, 9)
    rows = np.array([0, 5, 1999, 777, 5])
    i, d = osp.grid_knn(X, 9, rows=rows)
    np.testing.assert_array_equal(i, full_i[rows])
    np.testing.assert_array_equal(d, full_d[rows])
