"""Parity of the batch-balanced graph (``msc_bbknn_*`` + the fuzzy-set stages, through the C ABI)
with the CPU oracle (oracle/bbknn.py), and of the GPU trimming with the reference's own
``_trim_graph`` (tests/golden/reference_trim.npz).

The bar is bit-exact: every cell's combined list (indices and float32 distances in (distance,
index) order), the distances CSR, the untrimmed connectivities and the trimmed ones.  Cases cover
the reference's own tiny-batch input (tests/test_postfix_fixes.py:186-193), uneven batches, wide
lists that the certificate cannot prove for every cell (the FP64 scan finishes them), lists too
wide for the candidate kernel (FP64 scan only), coincident cells across batches, and both
tensor-core precisions.
"""
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import bbknn as obb
from msc_b200 import bbknn as bbm, synth, pp, AnnDataLite, _lib

pytestmark = pytest.mark.gpu

G = Path(__file__).resolve().parent / "golden"


def _case(name):
    if name == "tiny_batch":
        X = np.random.default_rng(0).standard_normal((60, 10)).astype(np.float32)
        return X, np.array(["a"] * 40 + ["b"] * 2 + ["c"] * 18), 3
    if name == "uneven":
        X = synth.gaussian_mixture(12_000, 30, 12, seed=31, sizes="lognormal", noise_frac=0.01)
        sizes = np.array([0.55, 0.25, 0.12, 0.06, 0.02])
        return X, np.random.default_rng(32).choice(5, X.shape[0], p=sizes), 3
    if name == "wide":
        X = synth.gaussian_mixture(6_000, 50, 8, seed=33)
        return X, np.random.default_rng(34).integers(0, 3, X.shape[0]), 20
    if name == "widest_candidates":
        X = synth.gaussian_mixture(3_000, 16, 5, seed=35)
        return X, np.random.default_rng(36).integers(0, 2, X.shape[0]), 60
    if name == "fp64_only":
        X = synth.gaussian_mixture(2_000, 12, 4, seed=37)
        return X, np.random.default_rng(38).integers(0, 2, X.shape[0]), 64
    if name == "one_cell_batch":
        X = np.random.default_rng(44).standard_normal((2_000, 8)).astype(np.float32)
        return X, np.array([0] * 1_999 + [1]), 4
    if name == "one_per_batch":
        X = synth.gaussian_mixture(5_000, 12, 5, seed=45)
        return X, np.random.default_rng(46).integers(0, 3, X.shape[0]), 1
    if name == "forty_batches":
        X = synth.gaussian_mixture(4_000, 10, 8, seed=47)
        return X, np.random.default_rng(48).integers(0, 40, X.shape[0]), 3
    if name == "coincident":
        X = np.random.default_rng(39).standard_normal((3_000, 20)).astype(np.float32)
        X[2000:2300] = X[0:300]                        # copies of batch-0 cells in batch 2
        return X, np.repeat([0, 1, 2], 1000), 5
    raise KeyError(name)


def _csr_equal(a, b, what):
    a, b = sp.csr_matrix(a), sp.csr_matrix(b)
    a.sort_indices()
    b.sort_indices()
    np.testing.assert_array_equal(a.indptr, b.indptr, err_msg=f"{what}: indptr")
    np.testing.assert_array_equal(a.indices, b.indices, err_msg=f"{what}: indices")
    np.testing.assert_array_equal(a.data, b.data, err_msg=f"{what}: data")
    assert a.data.dtype == np.float32


def _device_graph(X, batch, kwb, precision, trim=None):
    import torch
    _, codes, counts = bbm.batch_codes(batch)
    res = bbm.bbknn_device(torch.from_numpy(X).cuda(), torch.from_numpy(codes).cuda(), counts,
                           kwb, trim, precision=precision)
    torch.cuda.synchronize()
    return res


@pytest.mark.parametrize("name,precision", [
    ("tiny_batch", "fp16"), ("uneven", "fp16"), ("uneven", "bf16x3"), ("wide", "fp16"),
    ("widest_candidates", "fp16"), ("fp64_only", "fp16"), ("coincident", "fp16"),
    ("one_cell_batch", "fp16"), ("one_per_batch", "fp16"), ("forty_batches", "fp16"),
])
def test_bbknn_equals_oracle(name, precision):
    X, batch, kwb = _case(name)
    n = X.shape[0]
    res = _device_graph(X, batch, kwb, precision)
    stats = res["stats"].cpu().numpy()
    assert int(stats[_lib.STAT_TIMEOUT]) == 0 and int(stats[_lib.STAT_NONFINITE]) == 0
    rdist, rconn, K, inter = obb.bbknn(X, batch, kwb)
    assert res["K"] == K
    np.testing.assert_array_equal(res["knn_idx"].cpu().numpy(), inter["idx"].astype(np.int32),
                                  err_msg="combined lists: indices")
    np.testing.assert_array_equal(res["knn_dist"].cpu().numpy(), inter["dist"],
                                  err_msg="combined lists: distances")
    np.testing.assert_array_equal(res["sigma"].cpu().numpy(), inter["sigma"], err_msg="sigma")
    np.testing.assert_array_equal(res["rho"].cpu().numpy(), inter["rho"], err_msg="rho")
    union = bbm._csr_to_host(res["union_indptr"], res["union_indices"], res["union_data"], n)
    _csr_equal(union, inter["untrimmed"], "untrimmed connectivities")
    dist, conn = bbm.graph_to_host(res, n)
    _csr_equal(dist, rdist, "distances")
    _csr_equal(conn, rconn, "trimmed connectivities")
    # every cell was certified or scanned exactly
    if name == "fp64_only":
        assert int(stats[_lib.STAT_PRECISION]) == -1
    assert int(stats[_lib.STAT_CERTIFIED]) + int(stats[_lib.STAT_RESCANNED]) >= n


def test_bbknn_trims_like_oracle_at_small_trims():
    X, batch, kwb = _case("uneven")
    for t in (4, 9, 15):
        res = _device_graph(X, batch, kwb, "fp16", trim=t)
        _, conn = bbm.graph_to_host(res, X.shape[0])
        _, rconn, _, _ = obb.bbknn(X, batch, kwb, trim=t)
        _csr_equal(conn, rconn, f"trim={t}")


def test_gpu_trim_equals_reference_function():
    g = np.load(G / "reference_trim.npz")
    for c in range(int(g["n_cases"])):
        ip = g[f"c{c}_indptr"]
        n = ip.size - 1
        A = sp.csr_matrix((g[f"c{c}_data"], g[f"c{c}_indices"], ip), shape=(n, n))
        for t in g[f"c{c}_trims"]:
            R = bbm.trim_graph(A, int(t))
            np.testing.assert_array_equal(R.indptr, g[f"c{c}_t{t}_indptr"])
            np.testing.assert_array_equal(R.indices, g[f"c{c}_t{t}_indices"])
            np.testing.assert_array_equal(R.data, g[f"c{c}_t{t}_data"])


def test_pp_bbknn_writes_the_reference_slots():
    X, batch, kwb = _case("tiny_batch")
    a = AnnDataLite(obs={"batch": batch}, obsm={"X_pca": X})
    pp.bbknn(a, batch_key="batch")
    rdist, rconn, K, _ = obb.bbknn(X, batch, 3)
    _csr_equal(a.obsp["distances"], rdist, "obsp distances")
    _csr_equal(a.obsp["connectivities"], rconn, "obsp connectivities")
    assert a.obsp["connectivities"].indices.dtype == np.int32
    assert a.uns["neighbors"]["params"]["n_neighbors"] == K == 8
