"""The precision configuration at its stated size: 200,000 cells × 50 PCs, 50 anisotropic
clusters with Dirichlet sizes, rows L2-normalised; cosine, n_neighbors=30, over-fetch k'=48.

* every candidate form — the plain FP32 SIMT scan, the three-term BF16 tensor-core form and the
  default one-term FP16 form (each with k'=48 and the exact FP32/FP64 re-rank) — gives the same
  whole kNN lists, bit for bit, and each equals the oracle's exact FP64 lists on 1,024 seeded rows;
* the pruned tensor-core scan equals the full scan for both 16-bit forms;
* the whole graph of the default form (the oracle's ρ/σ, memberships, fuzzy union and distances
  CSR run on the host over the GPU's lists) equals the GPU's CSR matrices bit for bit.
"""
import os

import numpy as np
import pytest

import oracle
from msc_b200 import neighbors as nbm, synth, _lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2():
    X, p = synth.precision_200k()
    rows = np.sort(np.random.default_rng(20261204).choice(X.shape[0], 1024, replace=False))
    ridx, _, rdist = oracle.knn_exact(X, p["n_neighbors"], metric=p["metric"], rows=rows)
    return X, p, rows, ridx.astype(np.int32), rdist


def _knn(X, p, precision, prune=True):
    import torch
    old = os.environ.get("MSC_B200_PRUNE")
    os.environ["MSC_B200_PRUNE"] = "1" if prune else "0"
    try:
        Xd = torch.from_numpy(X).cuda()
        idx, dist, stats = nbm.knn_device(Xd, p["n_neighbors"], metric=p["metric"],
                                          precision=precision, kprime=p["kprime"])
        torch.cuda.synchronize()
        return idx.cpu().numpy(), dist.cpu().numpy(), stats.cpu().numpy()
    finally:
        if old is None:
            del os.environ["MSC_B200_PRUNE"]
        else:
            os.environ["MSC_B200_PRUNE"] = old


@pytest.fixture(scope="module")
def forms(c2):
    X, p, *_ = c2
    return {prec: _knn(X, p, prec) for prec in ("fp32", "bf16x3", "fp16")}


@pytest.mark.parametrize("precision", ["fp32", "bf16x3", "fp16"])
def test_c2_rows_match_oracle(c2, forms, precision):
    X, p, rows, ridx, rdist = c2
    idx, dist, stats = forms[precision]
    assert int(stats[_lib.STAT_TIMEOUT]) == 0 and int(stats[_lib.STAT_NONFINITE]) == 0
    assert int(stats[_lib.STAT_CERTIFIED]) + int(stats[_lib.STAT_RESCANNED]) >= X.shape[0]
    np.testing.assert_array_equal(idx[rows], ridx, err_msg=f"{precision}: indices")
    np.testing.assert_array_equal(dist[rows], rdist, err_msg=f"{precision}: distances")


def test_c2_forms_give_one_graph(forms):
    ref_i, ref_d, _ = forms["fp32"]
    for prec in ("bf16x3", "fp16"):
        np.testing.assert_array_equal(forms[prec][0], ref_i, err_msg=f"{prec} vs fp32: indices")
        np.testing.assert_array_equal(forms[prec][1], ref_d, err_msg=f"{prec} vs fp32: distances")


@pytest.mark.parametrize("precision", ["bf16x3", "fp16"])
def test_c2_pruned_equals_full_scan(c2, forms, precision):
    X, p, *_ = c2
    fi, fd, fs = _knn(X, p, precision, prune=False)
    assert int(fs[_lib.STAT_TIMEOUT]) == 0
    np.testing.assert_array_equal(forms[precision][0], fi, err_msg="pruned vs full: indices")
    np.testing.assert_array_equal(forms[precision][1], fd, err_msg="pruned vs full: distances")


def test_c2_whole_graph_matches_oracle(c2):
    import torch
    X, p, rows, ridx, rdist = c2
    n, k = X.shape[0], p["n_neighbors"]
    res = nbm.neighbors_device(torch.from_numpy(X).cuda(), k, metric=p["metric"],
                               method=p["method"], kprime=p["kprime"])
    dist_csr, conn_csr = nbm.graph_to_host(res, n, k)
    idx = res["knn_idx"].cpu().numpy()
    dist = res["knn_dist"].cpu().numpy()
    np.testing.assert_array_equal(idx[rows], ridx)
    sigma, rho = oracle.smooth_knn_dist(dist, k)
    w = oracle.membership_strengths(idx, dist, sigma, rho)
    for what, got, ref in (("connectivities", conn_csr, oracle.fuzzy_union(idx, w, n)),
                           ("distances", dist_csr, oracle.distances_csr(idx, dist, n))):
        assert got.nnz == ref.nnz, what
        np.testing.assert_array_equal(got.indptr.astype(np.int64), ref.indptr.astype(np.int64))
        np.testing.assert_array_equal(got.indices, ref.indices.astype(np.int32), what)
        np.testing.assert_array_equal(got.data, ref.data, what)
