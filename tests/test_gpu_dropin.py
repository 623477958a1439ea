"""The drop-in calls themselves on the GPU, end to end: ``msc_b200.pp.neighbors(adata)``
(metalsinglecell pp.py:753-788) and ``msc_b200.neighbors.neighbors(X_pca)`` (host NumPy in,
SciPy CSR out; neighbors.py:727-760), checked against the oracle bit for bit.

These run the whole public path — the AnnData slots, the representation choice and ``n_pcs``
truncation, the host upload, the CUDA graph, the host CSR conversion with its int32 index arrays —
where the other GPU tests enter at the device-level functions.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from msc_b200 import AnnDataLite, neighbors as nbm, pp, synth

pytestmark = pytest.mark.gpu


def _same_csr(got, ref, what):
    assert isinstance(got, sp.csr_matrix), what
    assert got.dtype == np.float32, what
    assert got.indptr.dtype == np.int32 and got.indices.dtype == np.int32, what
    assert got.shape == ref.shape and got.nnz == ref.nnz, what
    np.testing.assert_array_equal(got.indptr, ref.indptr, err_msg=what)
    np.testing.assert_array_equal(got.indices, ref.indices, err_msg=what)
    np.testing.assert_array_equal(got.data, ref.data, err_msg=what)


@pytest.fixture(scope="module")
def plain():
    X, p = synth.plain_10k()
    return X, p, oracle.neighbors_graph(X, p["n_neighbors"])


def test_neighbors_host_in_scipy_out(plain):
    X, p, ref = plain
    dist, conn = nbm.neighbors(X, n_neighbors=p["n_neighbors"])
    _same_csr(dist, ref["distances"], "distances")
    _same_csr(conn, ref["connectivities"], "connectivities")


def test_knn_host_call(plain):
    X, p, ref = plain
    for backend in ("nndescent", "ivf", "pynndescent"):
        idx, dist = nbm._knn(X, p["n_neighbors"], backend=backend)
        assert idx.dtype == np.int32 and dist.dtype == np.float32
        np.testing.assert_array_equal(idx, ref["idx"].astype(np.int32))
        np.testing.assert_array_equal(dist, ref["dist"])
    with pytest.raises(ValueError):
        nbm._knn(X, p["n_neighbors"], backend="annoy")


def test_pp_neighbors_default_slots(plain):
    X, p, ref = plain
    rng = np.random.default_rng(1)
    a = AnnDataLite(X=rng.standard_normal((X.shape[0], 80)).astype(np.float32),
                    obsm={"X_pca": X})
    assert pp.neighbors(a, n_neighbors=p["n_neighbors"]) is None
    _same_csr(a.obsp["distances"], ref["distances"], "obsp['distances']")
    _same_csr(a.obsp["connectivities"], ref["connectivities"], "obsp['connectivities']")
    assert a.uns["neighbors"] == {"connectivities_key": "connectivities",
                                  "distances_key": "distances",
                                  "params": {"n_neighbors": p["n_neighbors"], "method": "umap",
                                             "random_state": 0, "metric": "euclidean"}}
    assert pp.connectivities(a) is a.obsp["connectivities"]


def test_pp_neighbors_copy_key_added_n_pcs():
    X = synth.gaussian_mixture(4000, 50, 10, seed=21)
    a = AnnDataLite(X=np.zeros((4000, 60), np.float32), obsm={"X_pca": X})
    b = pp.neighbors(a, 12, 30, key_added="pcs30", copy=True)
    assert b is not a and not a.obsp and not a.uns
    ref = oracle.neighbors_graph(np.ascontiguousarray(X[:, :30]), 12)
    _same_csr(b.obsp["pcs30_distances"], ref["distances"], "pcs30 distances")
    _same_csr(b.obsp["pcs30_connectivities"], ref["connectivities"], "pcs30 connectivities")
    assert b.uns["pcs30"]["params"] == {"n_neighbors": 12, "method": "umap", "random_state": 0,
                                        "metric": "euclidean", "n_pcs": 30}
    assert pp.connectivities(b, "pcs30") is b.obsp["pcs30_connectivities"]


@pytest.mark.parametrize("metric,method", [("cosine", "umap"), ("euclidean", "gauss")])
def test_pp_neighbors_metric_and_method(metric, method):
    X = synth.gaussian_mixture(3000, 20, 8, seed=22, normalize=metric == "cosine")
    a = AnnDataLite(X=X)                           # 20 variables: the graph is built on .X
    pp.neighbors(a, 10, metric=metric, method=method)
    ref = oracle.neighbors_graph(X, 10, metric=metric, method=method)
    _same_csr(a.obsp["distances"], ref["distances"], "distances")
    _same_csr(a.obsp["connectivities"], ref["connectivities"], "connectivities")
    assert a.uns["neighbors"]["params"]["metric"] == metric
    assert a.uns["neighbors"]["params"]["method"] == method


def test_pp_neighbors_use_rep_and_errors():
    X = synth.gaussian_mixture(2000, 16, 6, seed=23)
    a = AnnDataLite(X=np.zeros((2000, 100), np.float32), obsm={"X_emb": X})
    pp.neighbors(a, 8, use_rep="X_emb")
    ref = oracle.neighbors_graph(X, 8)
    _same_csr(a.obsp["connectivities"], ref["connectivities"], "use_rep connectivities")
    assert a.uns["neighbors"]["params"]["use_rep"] == "X_emb"
    with pytest.raises(ValueError, match="Did not find X_nope"):
        pp.neighbors(a, 8, use_rep="X_nope")
    with pytest.raises(NotImplementedError):
        pp.neighbors(a, 8, use_rep="X_emb", metric="manhattan")
    with pytest.raises(ValueError):                 # 100 variables and no X_pca: run PCA first
        pp.neighbors(a, 8)
