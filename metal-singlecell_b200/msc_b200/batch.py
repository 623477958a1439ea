"""Many independent samples in one persistent launch, captured in a CUDA graph.

A cohort of samples (one embedding per sample, neighbours searched only within a sample) is laid out
as one row-concatenated matrix with offsets.  ``BatchedKnn`` plans it once
(``msc_batched_prepare``: sample table into the workspace), then every run enqueues one pipeline
whose persistent candidate kernel takes 128-row query tiles of all samples from one work list.
Samples are packed largest first, so the round-robin tile assignment balances the SMs.
``capture()`` records that pipeline in a CUDA graph, and ``replay()`` relaunches it with no host
work.  ``autotune()`` times the candidate kernel's tile configurations (key tile rows, pipeline
depth, selector buffer) on the actual cohort and keeps the fastest.

The reference has no batched path.  Its closest relative is bbknn's per-batch loop of brute-force
calls (metalsinglecell neighbors.py:516-539); ``per_sample_loop`` is that pattern on this
library's kernels and is the baseline the batched launch is measured against.
"""

from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

from . import _lib
from .neighbors import _torch, _ids, knn_device, Workspace, DEFAULT_PRECISION

_TILE_CACHE: dict[str, int] = {}


def tile_code(bn: int, stages: int, cb: int, epi: int = 4, pair: int = 0) -> int:
    """Candidate-kernel tile configuration: key tile rows, K-atom stages, selector buffer,
    epilogue warps (4 or 8) and CTA pairs (1: two-CTA clusters, 256-row query tiles)."""
    return (int(bn) | (int(stages) << 12) | (int(cb) << 20) | (int(epi == 8) << 27)
            | (int(bool(pair)) << 28))


def decode_tile_code(code: int):
    return {"bn": code & 0xFFF, "stages": (code >> 12) & 0xFF, "cb": (code >> 20) & 0x7F,
            "epi": 8 if (code >> 27) & 1 else 4, "pair": (code >> 28) & 1}


class BatchedKnn:
    """Exact kNN of every sample of a cohort in one persistent launch."""

    def __init__(self, offsets, d: int, n_neighbors: int = 15, *, metric: str = "euclidean",
                 precision: str = DEFAULT_PRECISION, kprime: int = 0, tile_config: int = 0,
                 device=None):
        torch = _torch()
        self.lib = _lib.load()
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        self.S = len(self.offsets) - 1
        self.n = int(self.offsets[-1])
        self.d, self.k = int(d), int(n_neighbors)
        self.mid, _, self.pid = _ids(metric, "umap", precision)
        self.kprime = int(kprime)
        self.tile_config = int(tile_config)
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        off = self.offsets.ctypes.data
        nbytes = self.lib.msc_batched_workspace_bytes(off, self.S, self.d, self.k, self.mid,
                                                      self.pid, self.kprime)
        if nbytes == 0:
            _lib.check(self.lib.msc_batched_prepare(off, self.S, self.d, self.k, self.mid,
                                                    self.pid, self.kprime, None, 0, None),
                       "msc_batched_prepare")
            raise ValueError("msc_batched: invalid arguments")
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        st = torch.cuda.current_stream(self.device)
        _lib.check(self.lib.msc_batched_prepare(off, self.S, self.d, self.k, self.mid, self.pid,
                                                self.kprime, self.ws.data_ptr(), nbytes,
                                                st.cuda_stream), "msc_batched_prepare")
        self.idx = torch.empty((self.n, self.k), dtype=torch.int32, device=self.device)
        self.dist = torch.empty((self.n, self.k), dtype=torch.float32, device=self.device)
        self.stats = torch.zeros(_lib.STATS_LEN, dtype=torch.int64, device=self.device)
        self.graph = None
        self._X = None

    def run(self, X):
        """Enqueue the whole cohort on the current stream (no host sync)."""
        torch = _torch()
        if X.shape != (self.n, self.d) or X.dtype != torch.float32 or not X.is_cuda:
            raise ValueError(f"X must be a CUDA float32 ({self.n}, {self.d}) tensor")
        X = X.contiguous()
        self._X = X
        st = torch.cuda.current_stream(self.device)
        _lib.check(self.lib.msc_batched_knn(X.data_ptr(), self.offsets.ctypes.data, self.S,
                                            self.d, self.k, self.mid, self.pid, self.kprime,
                                            self.tile_config, self.idx.data_ptr(),
                                            self.dist.data_ptr(), self.stats.data_ptr(),
                                            self.ws.data_ptr(), self.ws.numel(), st.cuda_stream),
                   "msc_batched_knn")
        return self.idx, self.dist

    def capture(self, X):
        """Record the pipeline for ``X`` (whose storage must stay alive) in a CUDA graph."""
        torch = _torch()
        self.run(X)                                   # un-captured first run: lazy set-up
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run(X)
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            raise RuntimeError("capture() first")
        self.graph.replay()
        return self.idx, self.dist

    def check(self):
        torch = _torch()
        torch.cuda.synchronize(self.device)
        s = self.stats.cpu().numpy()
        _lib.check_stats(s)
        return s


def per_sample_loop(X, offsets, n_neighbors: int = 15, *, metric: str = "euclidean",
                    precision: str = DEFAULT_PRECISION, kprime: int = 0,
                    workspace: Workspace | None = None, out=None):
    """The baseline: one full kNN pipeline launch per sample (bbknn's loop pattern)."""
    torch = _torch()
    offsets = np.asarray(offsets, np.int64)
    ws = workspace or Workspace(X.device)
    if out is None:
        out = (torch.empty((X.shape[0], n_neighbors), dtype=torch.int32, device=X.device),
               torch.empty((X.shape[0], n_neighbors), dtype=torch.float32, device=X.device))
    for s in range(len(offsets) - 1):
        a, b = int(offsets[s]), int(offsets[s + 1])
        idx, dist, _ = knn_device(X[a:b], n_neighbors, metric=metric, precision=precision,
                                  kprime=kprime, workspace=ws)
        out[0][a:b] = idx + a          # local → global row indices
        out[1][a:b] = dist
    return out


def _cache_file() -> Path:
    return Path(os.environ.get("MSC_B200_TUNE_CACHE",
                               Path.home() / ".cache" / "msc_b200" / "tiles.json"))


def autotune(X, offsets, n_neighbors: int = 15, *, metric: str = "euclidean",
             precision: str = DEFAULT_PRECISION, kprime: int = 0, reps: int = 3,
             configs=None, use_cache: bool = True, verbose: bool = False) -> dict:
    """Time the candidate kernel's tile configurations on this cohort; return the fastest.

    Returns ``{"tile_config": code, "ms": best_ms, "table": [(code, ms), ...]}``.  Invalid
    configurations (shared memory does not fit) are skipped.  Results are cached per
    (GPU, d, k, k', precision, metric, cohort size class).
    """
    torch = _torch()
    offsets = np.asarray(offsets, np.int64)
    n, d = X.shape
    sizes = np.diff(offsets)
    key = json.dumps([torch.cuda.get_device_name(X.device), int(d), int(n_neighbors),
                      int(kprime), precision, metric, int(len(sizes)),
                      int(np.log2(max(sizes.max(), 1))), int(np.log2(max(n, 1)))])
    if use_cache:
        if key in _TILE_CACHE:
            return {"tile_config": _TILE_CACHE[key], "cached": True}
        f = _cache_file()
        if f.exists():
            try:
                disk = json.loads(f.read_text())
                if key in disk:
                    _TILE_CACHE[key] = int(disk[key])
                    return {"tile_config": int(disk[key]), "cached": True}
            except Exception:
                pass
    if configs is None:
        configs = [tile_code(bn, st, cb, ep, pr) for pr in (1, 0) for ep in (8, 4)
                   for bn in (256, 128, 64) for st in (2, 3, 4, 6) for cb in (16,)]
    table = []
    for code in configs:
        try:
            bk = BatchedKnn(offsets, d, n_neighbors, metric=metric, precision=precision,
                            kprime=kprime, tile_config=code, device=X.device)
            bk.run(X)
            torch.cuda.synchronize(X.device)
        except (ValueError, NotImplementedError):
            continue
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            bk.run(X)
        e1.record()
        torch.cuda.synchronize(X.device)
        ms = e0.elapsed_time(e1) / reps
        table.append((code, ms))
        if verbose:
            print(f"  tile {decode_tile_code(code)}: {ms:.3f} ms", flush=True)
        del bk
    if not table:
        raise RuntimeError("autotune: no valid tile configuration")
    best = min(table, key=lambda t: t[1])
    _TILE_CACHE[key] = best[0]
    if use_cache:
        try:
            f = _cache_file()
            f.parent.mkdir(parents=True, exist_ok=True)
            disk = json.loads(f.read_text()) if f.exists() else {}
            disk[key] = best[0]
            f.write_text(json.dumps(disk))
        except Exception:
            pass
    return {"tile_config": best[0], "ms": best[1], "table": table, "cached": False}
