"""The UMAP layout's edge preparation on the host.  TEST INFRASTRUCTURE ONLY (the checker of the
device-side ``msc_umap_edges``).

Restates metalsinglecell ``embedding.umap``'s first steps on a connectivities CSR:
``_prune_weak_edges`` (embedding.py:255-267) keeps an entry when w >= max(w) / n_epochs, the
division in float32 (NumPy 2 keeps a float32 scalar divided by a Python float in float32); the
kept graph is taken as COO in CSR order (embedding.py:115); ``_make_epochs_per_sample``
(embedding.py:123-137) gives each kept edge n_epochs / (n_epochs · (w / max w)) in FP64, or -1
when that count is not positive.  Pinned bit for bit by ``tests/golden/reference_umap_edges.npz``,
which the reference's own two functions produced.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def umap_edges(conn: sp.csr_matrix, n_epochs: int) -> dict:
    C = sp.csr_matrix(conn)
    data = np.asarray(C.data, np.float32)
    n = C.shape[0]
    if data.size == 0:
        empty = np.zeros(0)
        return {"indptr": np.zeros(n + 1, np.int64), "rows": empty.astype(np.int32),
                "cols": empty.astype(np.int32), "weights": empty.astype(np.float32),
                "epochs_per_sample": empty}
    wmax = data.max()
    thr = np.float32(wmax / np.float32(max(n_epochs, 1)))
    keep = data >= thr
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(C.indptr))[keep]
    kept_per_row = np.add.reduceat(keep.astype(np.int64), C.indptr[:-1]) if n else np.zeros(0)
    kept_per_row = np.where(np.diff(C.indptr) > 0, kept_per_row, 0)
    indptr = np.concatenate([[0], np.cumsum(kept_per_row)]).astype(np.int64)
    w = data[keep]
    w64 = w.astype(np.float64)
    n_samples = float(n_epochs) * (w64 / np.float64(wmax))
    eps = np.full(w.size, -1.0)
    pos = n_samples > 0
    with np.errstate(over="ignore", divide="ignore"):
        eps[pos] = float(n_epochs) / n_samples[pos]
    return {"indptr": indptr, "rows": rows, "cols": C.indices[keep].astype(np.int32),
            "weights": w, "epochs_per_sample": eps}
