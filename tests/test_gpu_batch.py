"""Batched path: many samples in one persistent launch (+ CUDA graph, + autotuned tiles) must give
exactly the per-sample results, which must equal the oracle."""
import numpy as np
import pytest

import oracle
from msc_b200 import synth, batch, _lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cohort():
    sizes = [5000, 2000, 3300, 129, 257, 4096, 2500, 6000, 1000, 700]
    X, offsets, p = synth.batch_samples(len(sizes), seed=21, d=30, sizes=sizes)
    return X, offsets


def oracle_cohort(X, offsets, k, samples):
    out = {}
    for s in samples:
        a, b = offsets[s], offsets[s + 1]
        idx, d2, dist = oracle.knn_exact(X[a:b], k)
        out[s] = (idx + a, dist)
    return out


@pytest.mark.parametrize("precision", ["bf16x3", "fp16", "fp32"])
def test_batched_equals_per_sample_and_oracle(cohort, precision):
    import torch
    X, offsets = cohort
    Xd = torch.from_numpy(X).cuda()
    bk = batch.BatchedKnn(offsets, X.shape[1], 15, precision=precision)
    idx, dist = bk.run(Xd)
    stats = bk.check()
    assert int(stats[_lib.STAT_TIMEOUT]) == 0
    li, ld = batch.per_sample_loop(Xd, offsets, 15, precision=precision)
    torch.cuda.synchronize()
    assert torch.equal(idx, li) and torch.equal(dist, ld)
    ref = oracle_cohort(X, offsets, 15, [0, 3, 4, 9])
    gi, gd = idx.cpu().numpy(), dist.cpu().numpy()
    for s, (ri, rd) in ref.items():
        a, b = offsets[s], offsets[s + 1]
        assert np.array_equal(gi[a:b], ri.astype(np.int32)), f"sample {s}"
        assert np.array_equal(gd[a:b], rd), f"sample {s}"
    # neighbours never leave their sample
    sample_of = np.repeat(np.arange(len(offsets) - 1), np.diff(offsets))
    assert (sample_of[gi] == sample_of[:, None]).all()


def test_graph_capture_replay_is_identical(cohort):
    import torch
    X, offsets = cohort
    Xd = torch.from_numpy(X).cuda()
    bk = batch.BatchedKnn(offsets, X.shape[1], 15)
    idx0, dist0 = [t.clone() for t in bk.run(Xd)]
    bk.capture(Xd)
    bk.idx.zero_()
    bk.replay()
    torch.cuda.synchronize()
    assert torch.equal(bk.idx, idx0) and torch.equal(bk.dist, dist0)
    # replay with new contents in the same buffer
    Xd2 = Xd.flip(0).contiguous()
    Xd.copy_(Xd2)
    bk.replay()
    ref = batch.BatchedKnn(offsets, X.shape[1], 15)
    ri, rd = ref.run(Xd)
    torch.cuda.synchronize()
    assert torch.equal(bk.idx, ri) and torch.equal(bk.dist, rd)


def test_autotune_picks_a_valid_config(cohort, tmp_path, monkeypatch):
    import torch
    monkeypatch.setenv("MSC_B200_TUNE_CACHE", str(tmp_path / "tiles.json"))
    X, offsets = cohort
    Xd = torch.from_numpy(X).cuda()
    r = batch.autotune(Xd, offsets, 15, reps=1,
                       configs=[batch.tile_code(256, 3, 32), batch.tile_code(128, 2, 16),
                                batch.tile_code(64, 4, 32), batch.tile_code(32, 2, 16)])
    assert r["tile_config"] and len(r["table"]) >= 3
    bk = batch.BatchedKnn(offsets, X.shape[1], 15, tile_config=r["tile_config"])
    idx, dist = bk.run(Xd)
    ref = batch.BatchedKnn(offsets, X.shape[1], 15)
    ri, rd = ref.run(Xd)
    torch.cuda.synchronize()
    assert torch.equal(idx, ri) and torch.equal(dist, rd)
    assert batch.autotune(Xd, offsets, 15)["cached"]
