"""Key-tile pruning of the tensor-core scan (prune.cu) changes nothing in the result.

Pruning skips (query tile, key tile) pairs whose bounding balls prove that no key of the tile can
enter a query row's candidate list.  Its correctness is a pure equality: the pruned and the full
scan must give the same neighbours and distances bit for bit, and both must match the oracle.
The inputs are clustered with uniform noise cells (the rows that pruning moves to the end of the
sample), large enough that most key tiles are skipped.
"""
import os

import numpy as np
import pytest

import oracle
from msc_b200 import neighbors as nbm, synth, _lib

pytestmark = pytest.mark.gpu


def _knn(X, k, precision, metric="euclidean", prune=True):
    import torch
    old = os.environ.get("MSC_B200_PRUNE")
    os.environ["MSC_B200_PRUNE"] = "1" if prune else "0"
    try:
        Xd = torch.from_numpy(X).cuda()
        idx, dist, stats = nbm.knn_device(Xd, k, metric=metric, precision=precision)
        torch.cuda.synchronize()
        return idx.cpu().numpy(), dist.cpu().numpy(), stats.cpu().numpy()
    finally:
        if old is None:
            del os.environ["MSC_B200_PRUNE"]
        else:
            os.environ["MSC_B200_PRUNE"] = old


def _visited_fraction(X, k, precision, metric="euclidean"):
    import ctypes
    import torch
    lib = _lib.load()
    lib.msc_profile_enable(1)
    try:
        _knn(X, k, precision, metric)
        cnt = (ctypes.c_ulonglong * 16)()
        _lib.check(lib.msc_profile_counters(cnt, 16))
    finally:
        lib.msc_profile_enable(0)
    torch.cuda.synchronize()
    return cnt[10] / max(cnt[11], 1)


CASES = [
    # n, d, clusters, noise, k, metric, precision
    (60_000, 50, 40, 0.01, 15, "euclidean", "fp16"),
    (60_000, 50, 40, 0.01, 15, "euclidean", "bf16x3"),
    (50_000, 30, 25, 0.03, 30, "euclidean", "fp16"),
    (40_000, 50, 20, 0.00, 15, "cosine", "fp16"),
]


@pytest.mark.parametrize("n,d,c,noise,k,metric,precision", CASES)
def test_pruned_equals_full_scan_and_oracle(n, d, c, noise, k, metric, precision):
    X = synth.gaussian_mixture(n, d, c, seed=11, sizes="lognormal", noise_frac=noise,
                               normalize=metric == "cosine")
    pi, pd, ps = _knn(X, k, precision, metric, prune=True)
    fi, fd, fs = _knn(X, k, precision, metric, prune=False)
    assert int(ps[_lib.STAT_TIMEOUT]) == 0 and int(fs[_lib.STAT_TIMEOUT]) == 0
    np.testing.assert_array_equal(pi, fi, err_msg="pruned vs full scan: indices")
    np.testing.assert_array_equal(pd, fd, err_msg="pruned vs full scan: distances")
    rows = np.sort(np.random.default_rng(5).choice(n, 1500, replace=False))
    ridx, _, rdist = oracle.knn_exact(X, k, metric=metric, rows=rows)
    np.testing.assert_array_equal(pi[rows], ridx.astype(np.int32), err_msg="oracle: indices")
    np.testing.assert_array_equal(pd[rows], rdist, err_msg="oracle: distances")
    frac = _visited_fraction(X, k, precision, metric)
    assert frac < 0.6, f"pruning kept {frac:.2f} of the far key tiles"


def test_fp32_form_under_the_same_plan_equals_its_full_scan():
    # MSC_B200_PRUNE_FP32=1: the plain FP32 SIMT form runs the same near pass, outlier partition
    # and pruning plan as the tensor-core forms (the comparison of the forms at equal pruning)
    X = synth.gaussian_mixture(60_000, 50, 40, seed=12, sizes="lognormal", noise_frac=0.01)
    fi, fd, fs = _knn(X, 15, "fp32", prune=False)
    old = os.environ.get("MSC_B200_PRUNE_FP32")
    os.environ["MSC_B200_PRUNE_FP32"] = "1"
    try:
        pi, pd, ps = _knn(X, 15, "fp32", prune=True)
        frac = _visited_fraction(X, 15, "fp32")
    finally:
        if old is None:
            del os.environ["MSC_B200_PRUNE_FP32"]
        else:
            os.environ["MSC_B200_PRUNE_FP32"] = old
    assert int(ps[_lib.STAT_TIMEOUT]) == 0
    np.testing.assert_array_equal(pi, fi, err_msg="pruned vs full FP32 scan: indices")
    np.testing.assert_array_equal(pd, fd, err_msg="pruned vs full FP32 scan: distances")
    rows = np.sort(np.random.default_rng(6).choice(X.shape[0], 1000, replace=False))
    ridx, _, rdist = oracle.knn_exact(X, 15, rows=rows)
    np.testing.assert_array_equal(pi[rows], ridx.astype(np.int32))
    np.testing.assert_array_equal(pd[rows], rdist)
    assert frac < 0.6, f"pruning kept {frac:.2f} of the far key tiles"


def test_ordered_walk_equals_full_scan():
    # MSC_B200_ORDERED=1: far tiles nearest ball first, walks ended once every row's radius is
    # passed; the lists must equal the full scan's and the oracle's
    X = synth.gaussian_mixture(60_000, 50, 40, seed=13, sizes="lognormal", noise_frac=0.01)
    fi, fd, _ = _knn(X, 15, "fp16", prune=False)
    old = os.environ.get("MSC_B200_ORDERED")
    os.environ["MSC_B200_ORDERED"] = "1"
    try:
        oi, od, os_ = _knn(X, 15, "fp16", prune=True)
    finally:
        if old is None:
            del os.environ["MSC_B200_ORDERED"]
        else:
            os.environ["MSC_B200_ORDERED"] = old
    assert int(os_[_lib.STAT_TIMEOUT]) == 0
    np.testing.assert_array_equal(oi, fi, err_msg="ordered vs full scan: indices")
    np.testing.assert_array_equal(od, fd, err_msg="ordered vs full scan: distances")
    rows = np.sort(np.random.default_rng(7).choice(X.shape[0], 1000, replace=False))
    ridx, _, rdist = oracle.knn_exact(X, 15, rows=rows)
    np.testing.assert_array_equal(oi[rows], ridx.astype(np.int32))
    np.testing.assert_array_equal(od[rows], rdist)


def test_point_test_equals_full_scan():
    # MSC_B200_POINT_TEST=1: kept pairs whose every key is separated from the query tile's ball
    # are dropped from the plan; the lists must equal the full scan's and the oracle's, and the
    # plan must keep fewer far tiles than without the test
    X = synth.gaussian_mixture(60_000, 50, 40, seed=17, sizes="lognormal", noise_frac=0.01)
    fi, fd, _ = _knn(X, 15, "fp16", prune=False)
    base = _visited_fraction(X, 15, "fp16")
    old = os.environ.get("MSC_B200_POINT_TEST")
    os.environ["MSC_B200_POINT_TEST"] = "1"
    try:
        pi, pd, ps = _knn(X, 15, "fp16", prune=True)
        frac = _visited_fraction(X, 15, "fp16")
    finally:
        if old is None:
            del os.environ["MSC_B200_POINT_TEST"]
        else:
            os.environ["MSC_B200_POINT_TEST"] = old
    assert int(ps[_lib.STAT_TIMEOUT]) == 0
    np.testing.assert_array_equal(pi, fi, err_msg="point test vs full scan: indices")
    np.testing.assert_array_equal(pd, fd, err_msg="point test vs full scan: distances")
    rows = np.sort(np.random.default_rng(8).choice(X.shape[0], 1000, replace=False))
    ridx, _, rdist = oracle.knn_exact(X, 15, rows=rows)
    np.testing.assert_array_equal(pi[rows], ridx.astype(np.int32))
    np.testing.assert_array_equal(pd[rows], rdist)
    assert frac < base, f"point test kept {frac:.3f} of the far tiles, {base:.3f} without"
