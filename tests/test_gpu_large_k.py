"""Exact kNN beyond 129 neighbours (``msc_knn`` alone, up to MSC_MAX_K_KNN = 513): every row takes
the FP64 scan with a 256- or 512-entry warp list.  scrublet needs it: its ``_knn`` call
(preprocess.py:280-306) asks for k_adj + 1 = round(round(0.5·√n)·(1 + r)) + 1 neighbours over the
observed and simulated cells, which passes 129 from n = 7,226 cells at r = 2.  Bit-exact against
the oracle."""
import numpy as np
import pytest

import oracle
from msc_b200 import neighbors as nbm, synth, _lib

pytestmark = pytest.mark.gpu


def _knn(X, k):
    import torch
    idx, dist, stats = nbm.knn_device(torch.from_numpy(X).cuda(), k)
    torch.cuda.synchronize()
    return idx.cpu().numpy(), dist.cpu().numpy(), stats.cpu().numpy()


@pytest.mark.parametrize("k", [130, 257, 513])
def test_large_k_equals_oracle(k):
    X = synth.gaussian_mixture(3000, 20, 6, seed=41)
    X[100:110] = X[0:10]                                 # exact duplicates: ties by index
    idx, dist, st = _knn(X, k)
    assert int(st[_lib.STAT_RESCANNED]) == 3000 and int(st[_lib.STAT_TIMEOUT]) == 0
    ridx, _, rdist = oracle.knn_exact(X, k)
    np.testing.assert_array_equal(idx, ridx.astype(np.int32))
    np.testing.assert_array_equal(dist, rdist)


def test_scrublet_shaped_call():
    rng = np.random.default_rng(7)
    n, r = 10_000, 2
    obs = synth.gaussian_mixture(n, 30, 10, seed=43)
    pairs = rng.integers(0, n, (r * n, 2))
    sim = (0.5 * (obs[pairs[:, 0]] + obs[pairs[:, 1]])).astype(np.float32)
    X = np.vstack([obs, sim])
    n_neighbors = int(round(0.5 * np.sqrt(n)))
    k = int(round(n_neighbors * (1.0 + r))) + 1            # 151
    assert k > _lib.MAX_K
    idx, dist, _ = _knn(X, k)
    rows = np.sort(rng.choice(X.shape[0], 400, replace=False))
    ridx, _, rdist = oracle.knn_exact(X, k, rows=rows)
    np.testing.assert_array_equal(idx[rows], ridx.astype(np.int32))
    np.testing.assert_array_equal(dist[rows], rdist)
    # the statistic scrublet takes from the list: simulated neighbours per observed cell
    n_doublet = (idx[:n, 1:] >= n).sum(axis=1)
    assert n_doublet.min() >= 0 and n_doublet.max() <= k - 1
