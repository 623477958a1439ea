"""The oracle against golden vectors produced by the reference's own code
(tests/golden/make_golden.py runs metalsinglecell's NumPy-expressible neighbour functions).

* ``_knn_gpu`` (neighbors.py:82-132) at k = 33, 50 on the reference's test input: the reference
  ranks on fp16 (recall ~0.99 by its own test), then recomputes fp32 distances.  The exact oracle
  must contain it (recall ≥ 0.99, self first) and agree to fp32 precision on every neighbour both
  place at the same position.
* mlx-vis ``_fuzzy_simplicial_set`` (_vendor/mlx_vis/umap.py:199-271): ρ must be identical and σ
  within the bisection tolerance (1e-5 relative on the sum ⇒ ~1e-5 on σ), wherever that function
  and umap-learn share semantics (ρ > 1e-8, no mean-distance floor).
* ``neighbors`` (neighbors.py:727-760) with the exact oracle's lists standing in for its Metal
  kNN: the distances CSR its own lines build (neighbors.py:755-759) must equal the oracle's
  ``distances_csr`` bit for bit, stored zero distances of duplicate cells included.
* ``_trim_graph`` (neighbors.py:465-488) on batch-balanced connectivities at several trims:
  the oracle's ``trim_graph`` must give the same CSR bit for bit.
* ``gr.spatial_neighbors_knn`` / ``gr.spatial_neighbors_radius`` (gr.py:198-255) with the
  oracle's grid search in place of the Metal grid kernels: the oracle's restatement of the
  builders (edge selection, FP64 edge lengths, percentile / set_diag / transform, per-library
  blocks) must give the same two CSR matrices bit for bit, 13 cases.
"""
from pathlib import Path

import numpy as np
import pytest

import scipy.sparse as sp

import oracle
from oracle import bbknn as obb

G = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("k", [33, 50])
def test_oracle_vs_reference_knn(k):
    g = np.load(G / "reference_knn_500x20.npz")
    X, ri, rd = g["X"], g[f"idx_k{k}"], g[f"dist_k{k}"]
    idx, d2, dist = oracle.knn_exact(X, k)
    assert (ri[:, 0] == np.arange(500)).all() and (idx[:, 0] == np.arange(500)).all()
    recall = np.mean([len(set(idx[i]) & set(ri[i])) / k for i in range(500)])
    assert recall >= 0.99
    same = idx == ri
    assert same.mean() >= 0.99
    rel = np.abs(dist[same] - rd[same]) / np.maximum(rd[same], 1e-30)
    assert rel.max() < 1e-6
    # the reference's lists are ascending, like the oracle's
    assert (np.diff(rd, axis=1) >= 0).all()


def test_oracle_vs_reference_rho_sigma():
    g = np.load(G / "reference_rho_sigma.npz")
    sigma, rho = oracle.smooth_knn_dist(g["knn_dist"], float(g["k"]))
    ok = g["rho"] > 1e-8
    assert ok.all()
    assert np.array_equal(rho, g["rho"])
    rel = np.abs(sigma - g["sigma"]) / g["sigma"]
    assert rel.max() < 1e-5


def test_oracle_trim_vs_reference():
    g = np.load(G / "reference_trim.npz")
    checked = 0
    for c in range(int(g["n_cases"])):
        ip = g[f"c{c}_indptr"]
        n = ip.size - 1
        A = sp.csr_matrix((g[f"c{c}_data"], g[f"c{c}_indices"], ip), shape=(n, n))
        for t in g[f"c{c}_trims"]:
            R = obb.trim_graph(A, int(t))
            assert R.data.dtype == np.float32
            np.testing.assert_array_equal(R.indptr, g[f"c{c}_t{t}_indptr"])
            np.testing.assert_array_equal(R.indices, g[f"c{c}_t{t}_indices"])
            np.testing.assert_array_equal(R.data, g[f"c{c}_t{t}_data"])
            checked += 1
    # the cases trim hard, lightly and not at all, and drop stored zeros
    assert checked == 12


def test_oracle_distances_csr_vs_reference():
    g = np.load(G / "reference_distances_csr.npz")
    X, k = g["X"], int(g["k"])
    n = X.shape[0]
    idx, _, dist = oracle.knn_exact(X, k)
    np.testing.assert_array_equal(idx, g["knn_idx"])
    np.testing.assert_array_equal(dist, g["knn_dist"])
    D = oracle.distances_csr(idx, dist, n)
    assert D.data.dtype == np.float32
    np.testing.assert_array_equal(D.indptr, g["indptr"])
    np.testing.assert_array_equal(D.indices, g["indices"])
    np.testing.assert_array_equal(D.data, g["data"])
    assert D.nnz == n * (k - 1) and (D.data == 0).sum() == 20     # 10 duplicate pairs, both ways


def _spatial_cases():
    import json
    g = np.load(G / "reference_spatial.npz")
    for c in range(int(g["n_cases"])):
        kind, name, kw = json.loads(str(g[f"c{c}_case"]))
        if "radius" in kw and isinstance(kw["radius"], list):
            kw["radius"] = tuple(kw["radius"])
        lib = g[f"{name}_library"] if f"{name}_library" in g else None
        yield c, kind, g[f"{name}_coords"], lib, kw, g


def test_oracle_spatial_graphs_vs_reference():
    """The reference's own gr.spatial_neighbors_knn / _radius (run with the oracle's search in
    place of its Metal grid kernels) against the oracle's restatement of the whole builder:
    adjacency and distances bit for bit, dtypes included."""
    from oracle import spatial as osp
    checked = 0
    for c, kind, xy, lib, kw, g in _spatial_cases():
        if kind in ("grid", "delaunay"):
            continue                 # the lattice and Delaunay builders: checked on the product side
        fn = osp.spatial_neighbors_knn if kind == "knn" else osp.spatial_neighbors_radius
        adj, dst = fn(xy, library=lib, **kw)
        for tag, M in (("adj", adj), ("dst", dst)):
            M = sp.csr_matrix(M)
            M.sort_indices()
            np.testing.assert_array_equal(M.indptr, g[f"c{c}_{tag}_indptr"], err_msg=f"{c} {tag}")
            np.testing.assert_array_equal(M.indices, g[f"c{c}_{tag}_indices"], err_msg=f"{c} {tag}")
            ref = g[f"c{c}_{tag}_data"]
            assert M.data.dtype == ref.dtype, (c, tag, M.data.dtype, ref.dtype)
            np.testing.assert_array_equal(M.data, ref, err_msg=f"{c} {tag}")
        checked += 1
    assert checked == 13


def test_oracle_umap_edges_vs_reference():
    # the reference's own _prune_weak_edges + tocoo + _make_epochs_per_sample (embedding.py)
    import scipy.sparse as sp
    from oracle import handoff
    g = np.load(G / "reference_umap_edges.npz")
    n = g["indptr"].size - 1
    C = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(n, n))
    for e in g["epochs"]:
        o = handoff.umap_edges(C, int(e))
        np.testing.assert_array_equal(o["rows"], g[f"e{e}_rows"])
        np.testing.assert_array_equal(o["cols"], g[f"e{e}_cols"])
        np.testing.assert_array_equal(o["weights"], g[f"e{e}_weights"])
        np.testing.assert_array_equal(o["epochs_per_sample"], g[f"e{e}_eps"])
        assert o["indptr"][-1] == o["rows"].size
        np.testing.assert_array_equal(np.diff(o["indptr"]), np.bincount(o["rows"], minlength=n))
