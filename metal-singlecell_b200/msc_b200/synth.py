"""Seeded synthetic PCA embeddings shaped like the workloads this library is measured on.

No public single-cell dataset ships with this repository, so the embeddings are Gaussian mixtures
drawn with ``numpy.random.default_rng(seed)``.  They have the shapes, cluster structure and value
ranges of the workloads the reference's neighbour step is benchmarked on (50 PCs of a few thousand
to a million cells; the reference's own large run is a 1.3M-cell atlas, README.md:89-90).

Every generator returns C-contiguous float32 ``(n, d)`` arrays.  Rows are shuffled, because cells
in a real ``AnnData`` are not sorted by cluster.
"""

from __future__ import annotations

import numpy as np


def gaussian_mixture(n: int, d: int, n_clusters: int, *, seed: int, centre_scale: float = 5.0,
                     sizes: str = "equal", size_sigma: float = 1.0, anisotropic: bool = False,
                     noise_frac: float = 0.0, normalize: bool = False,
                     shuffle: bool = True) -> np.ndarray:
    """Mixture of ``n_clusters`` Gaussians in ``d`` dimensions.

    * centres ~ N(0, centre_scale²) per dimension;
    * within-cluster spread N(0, 1), or with ``anisotropic`` a per-cluster per-dimension scale
      drawn from LogNormal(0, 0.5);
    * cluster sizes: ``equal``, ``lognormal`` (∝ LogNormal(0, size_sigma)) or ``dirichlet``
      (Dirichlet(α=1)·n);
    * ``noise_frac`` of the cells uniform over the bounding box of the centres;
    * ``normalize`` L2-normalises every row (the cosine workload).
    """
    rng = np.random.default_rng(seed)
    n_noise = int(round(n * noise_frac))
    n_mix = n - n_noise
    if sizes == "equal":
        w = np.full(n_clusters, 1.0 / n_clusters)
    elif sizes == "lognormal":
        w = rng.lognormal(0.0, size_sigma, n_clusters)
        w /= w.sum()
    elif sizes == "dirichlet":
        w = rng.dirichlet(np.ones(n_clusters))
    else:
        raise ValueError(f"unknown sizes={sizes!r}")
    counts = np.floor(w * n_mix).astype(np.int64)
    counts[np.argsort(-w)[: n_mix - counts.sum()]] += 1      # hand out the remainder
    centres = rng.normal(0.0, centre_scale, (n_clusters, d))
    parts = []
    for c in range(n_clusters):
        if counts[c] == 0:
            continue
        scale = rng.lognormal(0.0, 0.5, d) if anisotropic else 1.0
        parts.append(centres[c] + rng.standard_normal((counts[c], d)) * scale)
    if n_noise:
        lo, hi = centres.min(0), centres.max(0)
        parts.append(rng.uniform(lo, hi, (n_noise, d)))
    X = np.concatenate(parts).astype(np.float32)
    if shuffle:
        X = X[rng.permutation(X.shape[0])]
    if normalize:
        nrm = np.sqrt((X.astype(np.float64) ** 2).sum(1, keepdims=True))
        X = (X / np.maximum(nrm, 1e-30)).astype(np.float32)
    return np.ascontiguousarray(X)


# The five measured workloads.  Each returns (X or list of X, parameters).

def plain_10k(seed: int = 0):
    """10,000 cells × 50 PCs, 20 equal clusters; euclidean, k=15, umap."""
    X = gaussian_mixture(10_000, 50, 20, seed=seed, sizes="equal")
    return X, dict(n_neighbors=15, metric="euclidean", method="umap")


def precision_200k(seed: int = 1, n: int = 200_000):
    """200,000 cells × 50 PCs, 50 anisotropic clusters, Dirichlet sizes, rows L2-normalised;
    cosine, k=30, over-fetch k'=48."""
    X = gaussian_mixture(n, 50, 50, seed=seed, sizes="dirichlet", anisotropic=True,
                         normalize=True)
    return X, dict(n_neighbors=30, metric="cosine", method="umap", kprime=48)


def scale_1m3(seed: int = 2, n: int = 1_300_000):
    """1,300,000 cells × 50 PCs, 200 clusters with LogNormal(σ=1) sizes, 1% uniform noise;
    euclidean, k=15, umap."""
    X = gaussian_mixture(n, 50, 200, seed=seed, sizes="lognormal", size_sigma=1.0,
                         noise_frac=0.01)
    return X, dict(n_neighbors=15, metric="euclidean", method="umap")


def batch_sizes(n_samples: int = 256, seed: int = 3, lo: int = 2_000, hi: int = 100_000):
    """Cell counts of the batching workload: round(LogNormal(ln 11000, 0.9)) clipped to [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.clip(np.round(rng.lognormal(np.log(11_000), 0.9, n_samples)), lo, hi).astype(np.int64)


def batch_samples(n_samples: int = 256, seed: int = 3, d: int = 30, sizes=None):
    """The batching workload: ``n_samples`` independent embeddings of 30 PCs, each a mixture of
    10-40 clusters; euclidean, k=15.  Returns the concatenated rows and per-sample offsets."""
    rng = np.random.default_rng(seed + 1000)
    ns = batch_sizes(n_samples, seed) if sizes is None else np.asarray(sizes, np.int64)
    parts = []
    for s, ns_ in enumerate(ns):
        ncl = int(rng.integers(10, 41))
        parts.append(gaussian_mixture(int(ns_), d, ncl, seed=seed * 100_003 + s,
                                      sizes="lognormal", size_sigma=0.5))
    offsets = np.zeros(len(ns) + 1, np.int64)
    offsets[1:] = np.cumsum(ns)
    return np.ascontiguousarray(np.concatenate(parts)), offsets, dict(n_neighbors=15,
                                                                     metric="euclidean")


def serving_requests(rate_hz: float, n_requests: int, seed: int = 5, lo: int = 1_000,
                     hi: int = 500_000, median: int = 20_000, sigma: float = 1.0):
    """Poisson arrivals of neighbour-graph requests.

    Each request: cells ~ LogNormal(ln median, sigma) clipped to [lo, hi], PCs ∈ {30, 50, 100},
    k ∈ {10, 15, 30}, metric ∈ {euclidean, cosine}.  Returns a list of dicts with the arrival
    time (seconds from the start), the shape and parameters, and a per-request data seed.
    """
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n_requests))
    out = []
    for i in range(n_requests):
        n = int(np.clip(round(rng.lognormal(np.log(median), sigma)), lo, hi))
        out.append(dict(arrival=float(t[i]), n=n, d=int(rng.choice([30, 50, 100])),
                        k=int(rng.choice([10, 15, 30])),
                        metric=str(rng.choice(["euclidean", "cosine"])),
                        seed=int(rng.integers(0, 2**31 - 1))))
    return out


def request_embedding(req: dict) -> np.ndarray:
    """The embedding of one serving request (seeded, 10-40 cluster mixture)."""
    rng = np.random.default_rng(req["seed"])
    X = gaussian_mixture(req["n"], req["d"], int(rng.integers(10, 41)), seed=req["seed"],
                         sizes="lognormal", size_sigma=0.5,
                         normalize=req["metric"] == "cosine")
    return X
