"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

The bar is bit-exact: neighbour indices and their order, float32 distances, the distances CSR and
the connectivities CSR (structure and float32 values) must equal the oracle's.  The design makes
that possible: candidates are certified or re-scanned, the boundary is resolved in FP64 with the
oracle's (distance, index) order, and the fuzzy-set arithmetic is fixed to the same float32
operations (see oracle/graph.py).  The stated tolerance of the path (1e-5 relative on distances
and connectivities) is therefore checked in its strongest form, equality.
"""
import numpy as np
import pytest

import oracle
from msc_b200 import neighbors as nbm, synth, _lib

pytestmark = pytest.mark.gpu

PRECISIONS = ["fp32", "bf16x3", "fp16", "bf16"]


def run_graph(X, k, metric="euclidean", method="umap", precision="bf16x3", kprime=0):
    import torch
    Xd = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
    res = nbm.neighbors_device(Xd, k, metric=metric, method=method, precision=precision,
                               kprime=kprime)
    torch.cuda.synchronize()
    dist, conn = nbm.graph_to_host(res, X.shape[0], k)
    stats = res["stats"].cpu().numpy()
    return res["knn_idx"].cpu().numpy(), res["knn_dist"].cpu().numpy(), dist, conn, stats


def assert_csr_equal(a, b, what):
    assert a.shape == b.shape, what
    assert np.array_equal(np.asarray(a.indptr, np.int64), np.asarray(b.indptr, np.int64)), \
        f"{what}: indptr differs"
    assert np.array_equal(a.indices, b.indices), f"{what}: indices differ"
    if not np.array_equal(a.data, b.data):
        diff = np.abs(a.data.astype(np.float64) - b.data)
        rel = diff / np.maximum(np.abs(b.data), 1e-30)
        raise AssertionError(f"{what}: {int((diff > 0).sum())} values differ, "
                             f"max rel {rel.max():.3e}")


def check_against_oracle(X, k, metric="euclidean", method="umap", precision="bf16x3", kprime=0):
    gi, gd, gdist, gconn, stats = run_graph(X, k, metric, method, precision, kprime)
    ref = oracle.neighbors_graph(X, k, metric=metric, method=method)
    assert int(stats[_lib.STAT_TIMEOUT]) == 0
    n = X.shape[0]
    assert int(stats[_lib.STAT_CERTIFIED]) + int(stats[_lib.STAT_RESCANNED]) >= n
    np.testing.assert_array_equal(gi, ref["idx"].astype(np.int32), err_msg="knn indices")
    np.testing.assert_array_equal(gd, ref["dist"], err_msg="knn distances")
    assert_csr_equal(gdist, ref["distances"], "distances CSR")
    assert_csr_equal(gconn, ref["connectivities"], "connectivities CSR")
    return stats


@pytest.mark.parametrize("precision", PRECISIONS)
def test_plain_10k_bit_exact(mixture_10k, precision):
    """The plain 10,000 × 50 workload (euclidean, k=15, umap) against the oracle."""
    X, p = mixture_10k
    stats = check_against_oracle(X, 15, precision=precision)
    if precision in ("fp32", "bf16x3", "fp16"):
        # the certificate should hold for (almost) every row at these precisions
        assert int(stats[_lib.STAT_RESCANNED]) <= X.shape[0] // 100


@pytest.mark.parametrize("precision", ["fp32", "bf16x3", "fp16"])
@pytest.mark.parametrize("k", [1, 2, 15, 33, 50, 65, 100])
def test_reference_knn_case_all_k(precision, k):
    """The reference's own kNN known-answer case (tests/test_postfix_fixes.py:108-121:
    500×20 N(0,1), default_rng(0), k ∈ {15, 33, 50}), extended to more k: exact here."""
    rng = np.random.default_rng(0)
    X = rng.standard_normal((500, 20)).astype(np.float32)
    check_against_oracle(X, k, precision=precision)
    # and the reference test's own criterion: recall >= 0.99 vs NumPy brute force
    idx, _ = nbm._knn(X, k, precision=precision)
    D = np.sqrt(((X[:, None, :] - X[None, :, :]) ** 2).sum(-1))
    ref = np.argsort(D, axis=1)[:, :k]
    recall = np.mean([len(set(idx[i]) & set(ref[i])) / k for i in range(X.shape[0])])
    assert idx.shape == (500, k) and recall >= 0.99


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_coincident_points(precision):
    """The reference's coincident-cells case (tests/test_postfix_fixes.py:197-207: 60×10 N(0,1)
    plus 5 exact duplicates, k=10): finite connectivities — and here identical to the oracle."""
    rng = np.random.default_rng(0)
    X = rng.standard_normal((60, 10)).astype(np.float32)
    Xd = np.vstack([X, X[:5]]).astype(np.float32)
    check_against_oracle(Xd, 10, precision=precision)
    _, conn = nbm.neighbors(Xd, n_neighbors=10, precision=precision)
    assert np.isfinite(conn.data).all()


@pytest.mark.parametrize("precision", ["fp16", "bf16x3"])
def test_distances_csr_equals_reference_golden(precision):
    """The distances CSR that the reference's own ``neighbors`` builds (neighbors.py:755-759) on
    an input with 10 duplicated cells (tests/golden/reference_distances_csr.npz): stored zero
    distances included, bit for bit."""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "reference_distances_csr.npz")
    X, k = g["X"], int(g["k"])
    gi, gd, gdist, _, _ = run_graph(X, k, precision=precision)
    np.testing.assert_array_equal(gi, g["knn_idx"].astype(np.int32))
    np.testing.assert_array_equal(gd, g["knn_dist"])
    np.testing.assert_array_equal(np.asarray(gdist.indptr, np.int64), g["indptr"])
    np.testing.assert_array_equal(np.asarray(gdist.indices, np.int64), g["indices"])
    np.testing.assert_array_equal(gdist.data, g["data"])


def test_many_duplicates_hub():
    """A large group of identical cells: ties at distance 0 resolved by index, hub rows with
    in-degree above the warp tier of the fuzzy union."""
    rng = np.random.default_rng(3)
    X = rng.standard_normal((3000, 16)).astype(np.float32)
    X[:600] = X[0]
    check_against_oracle(X, 15, precision="bf16x3")


@pytest.mark.parametrize("precision", ["fp32", "bf16x3", "fp16"])
def test_cosine_small(precision):
    X, p = synth.precision_200k(n=6000)
    check_against_oracle(X, 30, metric="cosine", precision=precision, kprime=48)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_gauss(precision):
    X = synth.gaussian_mixture(4000, 30, 12, seed=11)
    check_against_oracle(X, 15, method="gauss", precision=precision)


@pytest.mark.parametrize("n,d", [(1, 5), (2, 3), (129, 7), (257, 64), (300, 100), (1000, 128)])
def test_shapes(n, d):
    rng = np.random.default_rng(n * 1000 + d)
    X = rng.standard_normal((n, d)).astype(np.float32)
    k = min(n, 15)
    for precision in ("fp32", "bf16x3"):
        check_against_oracle(X, k, precision=precision)


def test_errors():
    import torch
    X = torch.zeros((10, 5), device="cuda")
    with pytest.raises(ValueError):
        nbm.neighbors_device(X, 11)                       # k > n
    with pytest.raises(NotImplementedError):
        nbm.neighbors_device(X, 3, metric="manhattan")
    Xn = torch.full((64, 4), float("nan"), device="cuda")
    res = nbm.neighbors_device(Xn, 5)
    torch.cuda.synchronize()
    with pytest.raises(ValueError):
        _lib.check_stats(res["stats"].cpu().numpy())


def test_bounded_wait_gives_up_without_hanging():
    """Failure detection without a GPU fault: a device wait on a barrier nothing arrives at gives
    up after its bound, the kernel returns an error status, and the context stays usable."""
    import torch
    lib = _lib.load()
    out = torch.zeros(3, dtype=torch.int32, device="cuda")
    _lib.check(lib.msc_selftest_wait_timeout(50_000_000, out.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    gave_up, flag, ms = out.cpu().tolist()
    assert gave_up == 1 and flag == 1 and 40 <= ms < 5000
    # the context still works
    X = synth.gaussian_mixture(2000, 20, 5, seed=3)
    check_against_oracle(X, 10, precision="bf16x3")


def _tile(bn, stages, cb, epi, pair=0):
    return bn | (stages << 12) | (cb << 20) | ((epi == 8) << 27) | (pair << 28)


@pytest.mark.parametrize("precision,kprime", [("bf16x3", 0), ("fp16", 32), ("bf16x3", 48)])
def test_candidate_tile_configs_agree(monkeypatch, precision, kprime):
    """Every candidate-kernel configuration (key tile rows, K-atom stages, selector buffer, four or
    eight epilogue warps, single CTAs or CTA pairs) gives the oracle's graph: 20,000 × 50, two
    clusters of unequal size so that tiles are ragged."""
    X = synth.gaussian_mixture(20000, 50, 2, seed=23)
    ref = oracle.neighbors_graph(X, 15)
    tried = 0
    for code in (_tile(256, 4, 16, 4), _tile(256, 2, 16, 8), _tile(128, 4, 16, 8),
                 _tile(64, 3, 32, 8), _tile(64, 2, 16, 4), _tile(256, 5, 16, 8, 1),
                 _tile(256, 4, 32, 4, 1), _tile(128, 6, 16, 8, 1), _tile(64, 4, 16, 4, 1)):
        monkeypatch.setenv("MSC_B200_TILE_CONFIG", hex(code))
        try:
            gi, gd, _, gconn, stats = run_graph(X, 15, precision=precision, kprime=kprime)
        except ValueError:
            continue                     # the configuration does not fit this operand width
        tried += 1
        assert int(stats[_lib.STAT_TIMEOUT]) == 0
        np.testing.assert_array_equal(gi, ref["idx"].astype(np.int32), err_msg=hex(code))
        np.testing.assert_array_equal(gd, ref["dist"], err_msg=hex(code))
        assert_csr_equal(gconn, ref["connectivities"], f"connectivities {hex(code)}")
    assert tried >= (5 if kprime <= 32 else 1)     # 64-entry lists fit fewer configurations


@pytest.mark.parametrize("precision,kprime", [("fp16", 0), ("bf16", 14), ("fp16", 14)])
def test_refine_pass(precision, kprime):
    """One-term FP16/BF16 candidates: rows whose certificate fails re-run through the BF16x3
    candidate kernel (MSC_STAT_REFINED), and only rows failing that too take the FP64 scan.
    k' = k-1 (no over-fetch) sends many rows through the refine pass; the graph must still be
    the oracle's, bit for bit."""
    X = synth.gaussian_mixture(30000, 50, 12, seed=31, sizes="lognormal")
    stats = check_against_oracle(X, 15, precision=precision, kprime=kprime)
    refined = int(stats[_lib.STAT_REFINED])
    assert int(stats[_lib.STAT_RESCANNED]) <= refined
    if kprime == 14:
        assert refined > 0
