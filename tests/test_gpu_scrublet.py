"""The second caller of the kNN boundary: scrublet's ``_knn`` call (metalsinglecell
preprocess.py:280-306).  Scrublet embeds the observed cells together with n_sim = r·n simulated
doublets and asks ``_knn`` for k_adj + 1 neighbours of every row, k_adj = round(k·(1 + n_sim/n))
with k = round(0.5·√n) (:283-287, :299); the score of a cell is the smoothed fraction of
simulated cells among its neighbours (:300-305).

Here: the same call through ``msc_b200.neighbors._knn`` on a synthetic 30-PC embedding whose
simulated doublets are midpoints of random observed pairs, bit-identical to the oracle (indices
and distances), so the doublet scores are identical too; up to k_adj + 1 = 214 (n = 20,000,
r = 2; ``msc_knn`` serves k ≤ 513, n ≤ ~116k at r = 2), and one request above that width, which
is refused as unsupported.
"""
import numpy as np
import pytest

import oracle
from msc_b200 import neighbors as nbm, synth

pytestmark = pytest.mark.gpu


def scrublet_embedding(n, r=2.0, seed=0):
    X = synth.gaussian_mixture(n, 30, 10, seed=seed)
    rng = np.random.default_rng(seed + 1)
    n_sim = int(round(n * r))
    a, b = rng.integers(0, n, n_sim), rng.integers(0, n, n_sim)
    sim = 0.5 * (X[a] + X[b]) + rng.normal(0, 0.05, (n_sim, 30)).astype(np.float32)
    return np.vstack([X, sim]).astype(np.float32), n_sim


def k_adj_of(n, n_sim):
    k = int(round(0.5 * np.sqrt(n)))
    return int(round(k * (1.0 + n_sim / max(n, 1))))


def scores(knn_idx, n, k_adj, rho=0.05, r=2.0):
    n_doublet = (knn_idx[:, 1:] >= n).sum(axis=1)
    q = (n_doublet + 1.0) / (k_adj + 2.0)
    return (q * rho / r) / (q * rho / r + (1 - q) * (1 - rho) + 1e-12)


@pytest.mark.parametrize("n", [3000, 7225, 7226, 20000])
def test_scrublet_knn_call_equals_oracle(n):
    X, n_sim = scrublet_embedding(n)
    k_adj = k_adj_of(n, n_sim)
    assert k_adj + 1 == {3000: 82, 7225: 127, 7226: 130, 20000: 214}[n]
    idx, dist = nbm._knn(X, k_adj + 1, random_state=0)
    ridx, _, rdist = oracle.knn_exact(X, k_adj + 1)
    np.testing.assert_array_equal(idx, ridx.astype(np.int32))
    np.testing.assert_array_equal(dist, rdist)
    np.testing.assert_array_equal(scores(idx, n, k_adj), scores(ridx, n, k_adj))


def test_scrublet_above_the_supported_width_is_refused():
    n = 116_282                       # round(0.5·√n) = 171: k_adj + 1 = 514
    X, n_sim = scrublet_embedding(n)
    k_adj = k_adj_of(n, n_sim)
    assert k_adj + 1 == 514
    with pytest.raises(NotImplementedError):
        nbm._knn(X, k_adj + 1)


def test_scrublet_knn_call_at_30k_cells():
    # a typical sample: n = 30,000 observed cells and 60,000 simulated doublets, k_adj + 1 = 262
    n = 30_000
    X, n_sim = scrublet_embedding(n, seed=3)
    k_adj = k_adj_of(n, n_sim)
    assert k_adj + 1 == 262
    idx, dist = nbm._knn(X, k_adj + 1, random_state=0)
    assert idx.shape == (X.shape[0], k_adj + 1)
    assert (idx[:, 0] == np.arange(X.shape[0])).all()
    rows = np.sort(np.random.default_rng(30).choice(X.shape[0], 1000, replace=False))
    ridx, _, rdist = oracle.knn_exact(X, k_adj + 1, rows=rows)
    np.testing.assert_array_equal(idx[rows], ridx.astype(np.int32))
    np.testing.assert_array_equal(dist[rows], rdist)
    # the doublet score of a sampled observed cell is that of the oracle's list
    obs = rows[rows < n]
    np.testing.assert_array_equal(scores(idx[obs], n, k_adj),
                                  scores(ridx[: obs.size], n, k_adj))
