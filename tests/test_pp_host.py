"""Host logic of ``pp.neighbors``: slots, key_added, uns params, copy semantics, representation
choice and errors — the contract of metalsinglecell pp.py:722-788 and tl.py:14-21.  The compute
call is replaced by the CPU oracle here (no GPU in this lane); the GPU lane runs the real one."""
import numpy as np
import pytest

import oracle
from msc_b200 import pp, AnnDataLite


@pytest.fixture
def fake_compute(monkeypatch):
    calls = []

    def _nb(rep, n_neighbors=15, random_state=0, metric="euclidean", method="umap",
            precision="bf16x3"):
        calls.append((rep.shape, n_neighbors, metric, method))
        g = oracle.neighbors_graph(rep, n_neighbors, metric=metric, method=method)
        return g["distances"], g["connectivities"]

    monkeypatch.setattr(pp, "_nb", _nb)
    return calls


def adata(n=120, d=50, n_vars=None):
    rng = np.random.default_rng(0)
    X_pca = rng.standard_normal((n, d)).astype(np.float32)   # 50 PCs: scanpy keeps X_pca
    return AnnDataLite(X=rng.standard_normal((n, n_vars or 80)).astype(np.float32),
                       obsm={"X_pca": X_pca})


def test_default_slots(fake_compute):
    a = adata()
    assert pp.neighbors(a, n_neighbors=10) is None
    assert set(a.obsp) == {"distances", "connectivities"}
    assert a.uns["neighbors"] == {"connectivities_key": "connectivities",
                                  "distances_key": "distances",
                                  "params": {"n_neighbors": 10, "method": "umap",
                                             "random_state": 0, "metric": "euclidean"}}
    assert fake_compute[0] == ((120, 50), 10, "euclidean", "umap")
    assert a.obsp["distances"].nnz == 120 * 9


def test_key_added_redirects_all_three_slots(fake_compute):
    a = adata()
    pp.neighbors(a, n_neighbors=5, key_added="small")
    assert "small_connectivities" in a.obsp and "small_distances" in a.obsp
    assert a.uns["small"]["connectivities_key"] == "small_connectivities"
    assert pp.connectivities(a, "small") is a.obsp["small_connectivities"]
    with pytest.raises(ValueError):
        pp.connectivities(a, "neighbors")


def test_copy_semantics(fake_compute):
    a = adata()
    b = pp.neighbors(a, n_neighbors=6, copy=True)
    assert b is not a and "connectivities" in b.obsp and "connectivities" not in a.obsp


def test_n_pcs_truncates_and_is_recorded(fake_compute):
    a = adata()
    pp.neighbors(a, 8, 12)                       # n_pcs positional, as in scanpy
    assert fake_compute[0][0] == (120, 12)
    assert a.uns["neighbors"]["params"]["n_pcs"] == 12


def test_use_rep(fake_compute):
    a = adata()
    a.obsm["X_harmony"] = a.obsm["X_pca"][:, :7].copy()
    pp.neighbors(a, 5, use_rep="X_harmony")
    assert fake_compute[0][0] == (120, 7)
    assert a.uns["neighbors"]["params"]["use_rep"] == "X_harmony"
    with pytest.raises(ValueError, match="Did not find"):
        pp.neighbors(a, 5, use_rep="X_missing")
    pp.neighbors(a, 5, use_rep="X")
    assert fake_compute[-1][0] == (120, 80)


def test_narrow_object_uses_X_and_wide_without_pca_raises(fake_compute):
    a = AnnDataLite(X=np.random.default_rng(1).standard_normal((50, 30)).astype(np.float32))
    pp.neighbors(a, 5)
    assert fake_compute[0][0] == (50, 30)
    b = AnnDataLite(X=np.zeros((50, 60), np.float32))
    with pytest.raises(ValueError, match="X_pca"):
        pp.neighbors(b, 5)


def test_metric_and_method(fake_compute):
    a = adata()
    pp.neighbors(a, 5, metric="cosine", method="gauss")
    assert a.uns["neighbors"]["params"]["metric"] == "cosine"
    assert a.uns["neighbors"]["params"]["method"] == "gauss"
    with pytest.raises(NotImplementedError):
        pp.neighbors(a, 5, metric="manhattan")
    with pytest.raises(ValueError):
        pp.neighbors(a, 5, method="rapids")


@pytest.fixture
def fake_bbknn(monkeypatch):
    from oracle import bbknn as obb
    calls = []

    def _bb(X, batch, neighbors_within_batch=3, n_pcs=50, trim=None, random_state=0,
            precision="fp16"):
        calls.append((X.shape, neighbors_within_batch, n_pcs, trim))
        dist, conn, K, _ = obb.bbknn(X, batch, neighbors_within_batch, n_pcs, trim)
        return dist, conn, K

    monkeypatch.setattr(pp, "_bbknn", _bb)
    return calls


def bb_adata(n=150, d=20):
    rng = np.random.default_rng(3)
    return AnnDataLite(X=rng.standard_normal((n, 30)).astype(np.float32),
                       obs={"batch": np.array(["x", "y", "z"])[rng.integers(0, 3, n)],
                            "donor": np.array(["d1", "d2"])[rng.integers(0, 2, n)]},
                       obsm={"X_pca": rng.standard_normal((n, d)).astype(np.float32)})


def test_bbknn_slots_and_params(fake_bbknn):
    a = bb_adata()
    assert pp.bbknn(a) is None
    assert set(a.obsp) == {"distances", "connectivities"}
    u = a.uns["neighbors"]
    assert u["connectivities_key"] == "connectivities" and u["distances_key"] == "distances"
    p = u["params"]
    # n_neighbors = neighbors_within_batch x batches (the combined width)
    assert p["n_neighbors"] == 9 and p["method"] == "umap" and p["metric"] == "euclidean"
    assert p["use_rep"] == "X_pca" and p["n_pcs"] == 50
    assert p["bbknn"]["trim"] == 90
    assert fake_bbknn[-1] == ((150, 20), 3, 50, None)
    assert pp.connectivities(a) is a.obsp["connectivities"]


def test_bbknn_options_and_copy(fake_bbknn):
    a = bb_adata()
    b = pp.bbknn(a, batch_key="donor", neighbors_within_batch=4, n_pcs=10, trim=5, copy=True)
    assert not a.obsp and b.uns["neighbors"]["params"]["n_neighbors"] == 8
    assert b.uns["neighbors"]["params"]["bbknn"]["trim"] == 5
    assert fake_bbknn[-1] == ((150, 20), 4, 10, 5)
    with pytest.raises(ValueError):
        pp.bbknn(a, use_rep="X_umap")
    with pytest.raises(KeyError):
        pp.bbknn(a, batch_key="sample")
