"""UMAP edge preparation on the device (``msc_umap_edges`` through ``neighbors.umap_edges``):
weak-edge pruning, the kept graph in CSR order and epochs-per-sample, on a graph the GPU built,
bit for bit against the oracle's restatement — which the reference's own ``_prune_weak_edges`` and
``_make_epochs_per_sample`` (embedding.py:123-137, 255-267) pin on the CPU."""
import numpy as np
import pytest

from oracle import handoff
from msc_b200 import neighbors as nbm, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,k,epochs", [(8000, 15, None), (8000, 15, 3), (12000, 30, 200),
                                        (600, 10, 5000)])
def test_umap_edges_match_oracle(n, k, epochs):
    import torch
    X = synth.gaussian_mixture(n, 30, 9, seed=n + k, sizes="lognormal", noise_frac=0.02)
    res = nbm.neighbors_device(torch.from_numpy(X).cuda(), k)
    _, conn = nbm.graph_to_host(res, n, k)
    got = nbm.umap_edges(res, n, epochs)
    e = got["n_epochs"]
    assert e == (epochs if epochs is not None else (500 if n <= 10_000 else 200))
    ref = handoff.umap_edges(conn, e)
    for key in ("indptr", "rows", "cols", "weights", "epochs_per_sample"):
        np.testing.assert_array_equal(got[key].cpu().numpy(), ref[key], err_msg=key)
