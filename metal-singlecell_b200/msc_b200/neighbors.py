"""Neighbour graph on a PCA embedding — the compute layer under ``pp.neighbors``.

Mirrors metalsinglecell ``neighbors.py``:

* ``neighbors(X_pca, n_neighbors, random_state, approx)`` → ``(distances, connectivities)`` SciPy
  CSR matrices (neighbors.py:727-760);
* ``_knn(X_pca, n_neighbors, random_state, approx)`` → ``(indices, dists)`` of shape (n, k), self
  first, ascending (neighbors.py:698-724);
* ``bbknn(X_pca, batch, neighbors_within_batch, n_pcs, trim, random_state)`` and
  ``_trim_graph(conn, trim)`` (neighbors.py:491-559, 465-488), implemented in ``msc_b200.bbknn``.

Everything runs on one GPU through the C ABI of ``libmsc_b200.so``; PyTorch only provides the
device buffers and the current stream.  Unlike the reference, the kNN is exact at every size (no
approximate NNDescent branch above 30k cells, no fp16 ranking loss): candidates from the tensor
cores are re-ranked exactly and every row is certified or re-scanned, so ``approx`` is accepted
for signature compatibility and ignored.
"""

from __future__ import annotations

import numpy as np

from . import _lib

# FP16 candidates on the tensor cores (as the reference ranks on an fp16 Gram matrix,
# neighbors.py:114-119), exact FP32/FP64 re-rank, BF16x3 refine of the rows the FP16 certificate
# cannot prove, FP64 scan of whatever is left: the fastest exact path at 50 PCs
DEFAULT_PRECISION = "fp16"


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("msc_b200 needs a CUDA device (B200); none is visible")
    return torch


def _stream(torch, device):
    return torch.cuda.current_stream(device).cuda_stream


def _ids(metric, method, precision):
    if metric not in _lib.METRIC:
        raise NotImplementedError(f"metric={metric!r} is not implemented (euclidean, cosine)")
    if method not in _lib.METHOD:
        raise ValueError(f"method={method!r} must be 'umap' or 'gauss'")
    if precision not in _lib.PRECISION:
        raise ValueError(f"precision={precision!r} must be one of {sorted(_lib.PRECISION)}")
    return _lib.METRIC[metric], _lib.METHOD[method], _lib.PRECISION[precision]


class Workspace:
    """A reusable device scratch buffer (grown on demand; with ``pow2``, to the next power of two,
    so that a user of many sizes re-allocates only a few times)."""

    def __init__(self, device=None, pow2: bool = False):
        self.device = device
        self.pow2 = pow2
        self.buf = None

    def get(self, nbytes: int):
        torch = _torch()
        if self.buf is None or self.buf.numel() < nbytes:
            size = max(int(nbytes), 256)
            if self.pow2:
                size = 1 << (size - 1).bit_length()
            self.buf = torch.empty(size, dtype=torch.uint8, device=self.device)
        return self.buf


def neighbors_device(X, n_neighbors: int = 15, *, metric: str = "euclidean",
                     method: str = "umap", precision: str = DEFAULT_PRECISION, kprime: int = 0,
                     workspace: Workspace | None = None, out: dict | None = None) -> dict:
    """The whole graph on device tensors, enqueued on the current stream (no host sync).

    ``X`` is a CUDA float32 (n, d) tensor.  Returns a dict of CUDA tensors: ``knn_idx`` (n,k)
    int32, ``knn_dist`` (n,k) float32, ``dist_indptr/indices/data`` (distances CSR),
    ``conn_indptr/indices/data`` (connectivities CSR; capacity 2n(k-1), valid length
    ``conn_indptr[n]``) and ``stats`` (int64[8], see ``_lib.STAT_*``).
    """
    torch = _torch()
    lib = _lib.load()
    if X.dtype != torch.float32 or not X.is_cuda or X.dim() != 2:
        raise ValueError("X must be a 2-D float32 CUDA tensor")
    X = X.contiguous()
    n, d = X.shape
    k = int(n_neighbors)
    mid, meth, pid = _ids(metric, method, precision)
    nbytes = lib.msc_neighbors_workspace_bytes(n, d, k, mid, meth, pid, int(kprime))
    if nbytes == 0:
        # re-run the argument checks for the message
        _lib.check(lib.msc_neighbors(0, n, d, k, mid, meth, pid, int(kprime), *([0] * 10), 0, 0),
                   "msc_neighbors")
        raise ValueError("msc_neighbors: invalid arguments")
    ws = (workspace or Workspace(X.device)).get(nbytes)
    dev = X.device
    m = max(k - 1, 0)
    o = out if out is not None else {}
    def buf(name, shape, dtype):
        t = o.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=dev)
            o[name] = t
        return t
    knn_idx = buf("knn_idx", (n, k), torch.int32)
    knn_dist = buf("knn_dist", (n, k), torch.float32)
    d_ptr = buf("dist_indptr", (n + 1,), torch.int64)
    d_ind = buf("dist_indices", (max(n * m, 1),), torch.int32)
    d_dat = buf("dist_data", (max(n * m, 1),), torch.float32)
    c_ptr = buf("conn_indptr", (n + 1,), torch.int64)
    c_ind = buf("conn_indices", (max(2 * n * m, 1),), torch.int32)
    c_dat = buf("conn_data", (max(2 * n * m, 1),), torch.float32)
    stats = buf("stats", (_lib.STATS_LEN,), torch.int64)
    rc = lib.msc_neighbors(X.data_ptr(), n, d, k, mid, meth, pid, int(kprime),
                           knn_idx.data_ptr(), knn_dist.data_ptr(), d_ptr.data_ptr(),
                           d_ind.data_ptr(), d_dat.data_ptr(), c_ptr.data_ptr(),
                           c_ind.data_ptr(), c_dat.data_ptr(), stats.data_ptr(), ws.data_ptr(),
                           ws.numel(), _stream(torch, dev))
    _lib.check(rc, "msc_neighbors")
    return o


def knn_device(X, n_neighbors: int = 15, *, metric: str = "euclidean",
               precision: str = DEFAULT_PRECISION, kprime: int = 0,
               workspace: Workspace | None = None):
    """Exact kNN on device tensors: ``(knn_idx int32 (n,k), knn_dist float32 (n,k), stats)``."""
    torch = _torch()
    lib = _lib.load()
    if X.dtype != torch.float32 or not X.is_cuda or X.dim() != 2:
        raise ValueError("X must be a 2-D float32 CUDA tensor")
    X = X.contiguous()
    n, d = X.shape
    k = int(n_neighbors)
    mid, _, pid = _ids(metric, "umap", precision)
    nbytes = lib.msc_knn_workspace_bytes(n, d, k, mid, pid, int(kprime))
    if nbytes == 0:
        _lib.check(lib.msc_knn(0, n, d, k, mid, pid, int(kprime), 0, 0, 0, 0, 0, 0), "msc_knn")
        raise ValueError("msc_knn: invalid arguments")
    ws = (workspace or Workspace(X.device)).get(nbytes)
    idx = torch.empty((n, k), dtype=torch.int32, device=X.device)
    dist = torch.empty((n, k), dtype=torch.float32, device=X.device)
    stats = torch.zeros(_lib.STATS_LEN, dtype=torch.int64, device=X.device)
    rc = lib.msc_knn(X.data_ptr(), n, d, k, mid, pid, int(kprime), idx.data_ptr(),
                     dist.data_ptr(), stats.data_ptr(), ws.data_ptr(), ws.numel(),
                     _stream(torch, X.device))
    _lib.check(rc, "msc_knn")
    return idx, dist, stats


class HostGraphState:
    """Buffers reused by ``neighbors_host`` across calls of one shape: device input and outputs,
    the workspace, pinned host outputs, a copy stream and the distances-ready event."""

    def __init__(self, n: int, d: int, k: int, device=None):
        torch = _torch()
        self.shape = (int(n), int(d), int(k))
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.dev_out: dict = {}
        self.workspace = Workspace(self.device)
        self.copy_stream = torch.cuda.Stream(device=self.device)
        # torch creates an event's CUDA handle at its first record: record once now, so that the
        # handle passed to msc_neighbors_ex exists (a wait on a never-recorded event would not
        # wait at all)
        self.ready = torch.cuda.Event()
        self.ready.record(torch.cuda.current_stream(self.device))
        m = max(int(k) - 1, 0)
        pin = lambda numel, dt: torch.empty(max(numel, 1), dtype=dt).pin_memory()
        self.host = {"dist_indptr": pin(n + 1, torch.int64),
                     "dist_indices": pin(n * m, torch.int32),
                     "dist_data": pin(n * m, torch.float32),
                     "conn_indptr": pin(n + 1, torch.int64),
                     "conn_indices": pin(2 * n * m, torch.int32),
                     "conn_data": pin(2 * n * m, torch.float32),
                     "stats": pin(_lib.STATS_LEN, torch.int64)}
        self.X = torch.empty((int(n), int(d)), dtype=torch.float32, device=self.device)


def neighbors_host(Xh, n_neighbors: int = 15, *, metric: str = "euclidean",
                   method: str = "umap", precision: str = DEFAULT_PRECISION, kprime: int = 0,
                   state: HostGraphState | None = None) -> dict:
    """The whole graph from a host embedding to host CSR matrices, with the copies overlapped.

    ``Xh`` is a float32 (n, d) CPU tensor (pinned for an asynchronous upload).  The graph runs
    through ``msc_neighbors_ex``; as soon as the kNN lists and the distances CSR are final its
    event fires, and a second stream copies the distances CSR to the host while the
    connectivities are computed; the connectivities follow once their size is known.  Returns the
    pinned host tensors of ``state.host`` with ``conn_nnz``: the distances CSR is
    ``dist_indptr`` / ``dist_indices`` / ``dist_data``, the connectivities the first ``conn_nnz``
    entries of ``conn_indices`` / ``conn_data`` with ``conn_indptr``."""
    torch = _torch()
    lib = _lib.load()
    n, d = int(Xh.shape[0]), int(Xh.shape[1])
    k = int(n_neighbors)
    st = state if state is not None else HostGraphState(n, d, k)
    if st.shape != (n, d, k):
        raise ValueError(f"state was made for {st.shape}, not {(n, d, k)}")
    mid, meth, pid = _ids(metric, method, precision)
    nbytes = lib.msc_neighbors_workspace_bytes(n, d, k, mid, meth, pid, int(kprime))
    if nbytes == 0:
        _lib.check(lib.msc_neighbors(0, n, d, k, mid, meth, pid, int(kprime), *([0] * 10), 0, 0),
                   "msc_neighbors")
        raise ValueError("msc_neighbors: invalid arguments")
    ws = st.workspace.get(nbytes)
    if not st.ready.cuda_event:
        raise RuntimeError("neighbors_host: the distances-ready event has no CUDA handle")
    main = torch.cuda.current_stream(st.device)
    st.X.copy_(Xh, non_blocking=True)
    o = st.dev_out
    def buf(name, shape, dtype):
        t = o.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=st.device)
            o[name] = t
        return t
    m = max(k - 1, 0)
    knn_idx, knn_dist = buf("knn_idx", (n, k), torch.int32), buf("knn_dist", (n, k), torch.float32)
    d_ptr, d_ind = buf("dist_indptr", (n + 1,), torch.int64), buf("dist_indices", (max(n * m, 1),), torch.int32)
    d_dat = buf("dist_data", (max(n * m, 1),), torch.float32)
    c_ptr = buf("conn_indptr", (n + 1,), torch.int64)
    c_ind = buf("conn_indices", (max(2 * n * m, 1),), torch.int32)
    c_dat = buf("conn_data", (max(2 * n * m, 1),), torch.float32)
    stats = buf("stats", (_lib.STATS_LEN,), torch.int64)
    rc = lib.msc_neighbors_ex(st.X.data_ptr(), n, d, k, mid, meth, pid, int(kprime),
                              knn_idx.data_ptr(), knn_dist.data_ptr(), d_ptr.data_ptr(),
                              d_ind.data_ptr(), d_dat.data_ptr(), c_ptr.data_ptr(),
                              c_ind.data_ptr(), c_dat.data_ptr(), stats.data_ptr(), ws.data_ptr(),
                              ws.numel(), main.cuda_stream, st.ready.cuda_event)
    _lib.check(rc, "msc_neighbors_ex")
    h = st.host
    with torch.cuda.stream(st.copy_stream):
        st.copy_stream.wait_event(st.ready)
        h["dist_indptr"].copy_(d_ptr, non_blocking=True)
        h["dist_indices"][: n * m].copy_(d_ind[: n * m], non_blocking=True)
        h["dist_data"][: n * m].copy_(d_dat[: n * m], non_blocking=True)
    h["stats"].copy_(stats, non_blocking=True)
    h["conn_indptr"].copy_(c_ptr, non_blocking=True)
    main.synchronize()
    _lib.check_stats(h["stats"].numpy())
    nnz = int(h["conn_indptr"][n])
    h["conn_indices"][:nnz].copy_(c_ind[:nnz], non_blocking=True)
    h["conn_data"][:nnz].copy_(c_dat[:nnz], non_blocking=True)
    main.synchronize()
    st.copy_stream.synchronize()
    return dict(h, conn_nnz=nnz)


def _index_dtype(n: int, nnz: int):
    return np.int32 if max(n, nnz) < 2 ** 31 else np.int64


def graph_to_host(res: dict, n: int, k: int):
    """Device result of ``neighbors_device`` → (distances CSR, connectivities CSR) on the host,
    in SciPy's canonical layout with int32 index arrays (what SciPy itself produces for
    nnz < 2³¹, as the reference's ``csr_matrix`` calls do)."""
    import scipy.sparse as sp
    torch = _torch()
    stats = res["stats"].cpu().numpy()
    _lib.check_stats(stats)
    nnz = int(stats[_lib.STAT_CONN_NNZ])
    m = max(k - 1, 0)
    # SciPy's own choice of index type: int32 while every index and nnz fit, else int64
    d_ptr = res["dist_indptr"].cpu().numpy().astype(_index_dtype(n, n * m))
    d_ind = res["dist_indices"][: n * m].cpu().numpy()
    d_dat = res["dist_data"][: n * m].cpu().numpy()
    c_ptr = res["conn_indptr"].cpu().numpy().astype(_index_dtype(n, nnz))
    c_ind = res["conn_indices"][:nnz].cpu().numpy()
    c_dat = res["conn_data"][:nnz].cpu().numpy()
    dist = sp.csr_matrix((d_dat, d_ind, d_ptr), shape=(n, n))
    conn = sp.csr_matrix((c_dat, c_ind, c_ptr), shape=(n, n))
    del torch
    return dist, conn


def csr_device(res: dict, n: int, which: str = "connectivities"):
    """``(indptr int64 (n+1,), indices int32 (nnz,), data float32 (nnz,))`` of a device result of
    ``neighbors_device`` (``which`` = "connectivities" or "distances"), as views of its buffers
    trimmed to the valid length.  Reading that length is one 8-byte device-to-host copy."""
    if which not in ("connectivities", "distances"):
        raise ValueError(f"which={which!r} must be 'connectivities' or 'distances'")
    pre = "conn_" if which == "connectivities" else "dist_"
    indptr = res[pre + "indptr"]
    nnz = int(indptr[n].item())
    return indptr, res[pre + "indices"][:nnz], res[pre + "data"][:nnz]


def to_torch_csr(res: dict, n: int, which: str = "connectivities"):
    """The graph as a ``torch.sparse_csr_tensor`` on the result's device, sharing its buffers:
    GPU consumers take it without a host round trip."""
    import torch
    indptr, indices, data = csr_device(res, n, which)
    if indices.numel() < 2 ** 31:          # 32-bit row pointers: the column indices stay shared
        indptr = indptr.to(torch.int32)
    else:
        indices = indices.to(torch.int64)
    import warnings
    with warnings.catch_warnings():                # torch's notes on sparse CSR support
        warnings.filterwarnings("ignore", message="Sparse invariant checks are implicitly")
        warnings.filterwarnings("ignore", message="Sparse CSR tensor support is in beta")
        return torch.sparse_csr_tensor(indptr, indices, data, size=(n, n),
                                       check_invariants=False)


def graph_arrays(res: dict, n: int, which: str = "connectivities") -> dict:
    """The layout of the reference's graph container (``Graph.from_scipy``,
    graph/csr_graph.py:15-40: ``indptr``, ``indices``, ``weights``, ``edge_src`` = the source row of
    every edge, ``n``) built on the device from a ``neighbors_device`` result, for the graph
    consumers (Leiden, UMAP epochs) that the reference feeds through a host CSR."""
    import torch
    indptr, indices, data = csr_device(res, n, which)
    if indices.numel() >= 2 ** 32:
        raise ValueError("the graph container's uint32 row pointers hold at most 2^32 - 1 edges")
    deg = indptr[1:] - indptr[:-1]
    src = torch.repeat_interleave(torch.arange(n, device=indptr.device, dtype=torch.int32), deg)
    # the container keeps its row pointers as uint32 (csr_graph.py:32); torch's uint32 type has
    # few operators, so the words are taken as they lie: an int64 value below 2^32 has that
    # uint32 value as its low (first, little-endian) word
    lo = indptr.view(torch.int32).view(n + 1, 2)[:, 0].contiguous().view(torch.uint32)
    return {"indptr": lo, "indices": indices, "weights": data, "edge_src": src, "n": n}


def umap_edges(res: dict, n: int, n_epochs: int | None = None, *, stream=None) -> dict:
    """The edge list the UMAP layout samples, prepared on the device from a ``neighbors_device``
    result (metalsinglecell embedding.py:100-116, 123-137, 255-267): edges with weight below
    max(w) / n_epochs dropped, the kept graph as COO in CSR order, and each edge's sampling period
    ``epochs_per_sample`` (FP64; -1 never sampled).  ``n_epochs`` defaults as the reference's
    ``umap`` does: 500 up to 10,000 cells, else 200.

    Returns device tensors ``indptr`` (the kept graph's int64 row pointers), ``rows``, ``cols``
    (int32), ``weights`` (float32), ``epochs_per_sample`` (float64) and ``n_epochs``."""
    torch = _torch()
    lib = _lib.load()
    if n_epochs is None:
        n_epochs = 500 if n <= 10_000 else 200
    indptr = res["conn_indptr"]
    dev = indptr.device
    cap = max(int(res["conn_indices"].numel()), 1)
    out_ptr = torch.empty(n + 1, dtype=torch.int64, device=dev)
    rows = torch.empty(cap, dtype=torch.int32, device=dev)
    cols = torch.empty(cap, dtype=torch.int32, device=dev)
    w = torch.empty(cap, dtype=torch.float32, device=dev)
    eps = torch.empty(cap, dtype=torch.float64, device=dev)
    nbytes = lib.msc_umap_edges_workspace_bytes(n)
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    st = _stream(torch, dev) if stream is None else stream
    _lib.check(lib.msc_umap_edges(indptr.data_ptr(), res["conn_indices"].data_ptr(),
                                  res["conn_data"].data_ptr(), n, int(n_epochs),
                                  out_ptr.data_ptr(), rows.data_ptr(), cols.data_ptr(),
                                  w.data_ptr(), eps.data_ptr(), ws.data_ptr(), nbytes, st),
               "msc_umap_edges")
    m = int(out_ptr[n].item())
    return {"indptr": out_ptr, "rows": rows[:m], "cols": cols[:m], "weights": w[:m],
            "epochs_per_sample": eps[:m], "n_epochs": int(n_epochs)}


_HOST_STATE: dict = {}           # the buffers of the last shape the host-level call saw


def _host_state(n: int, d: int, k: int, device) -> HostGraphState:
    key = (n, d, k, str(device))
    st = _HOST_STATE.get(key)
    if st is None:
        _HOST_STATE.clear()                    # keep one shape's pinned buffers at most
        st = HostGraphState(n, d, k, device=device)
        _HOST_STATE[key] = st
    return st


_STAGE_BYTES = 32 << 20              # pinned staging chunk of the upload
_DOWN_CHUNK = 8 << 20                # entries per chunk of the connectivities download


def _upload(torch, st: HostGraphState, X: np.ndarray):
    """Copy a pageable host embedding into ``st.X`` through two pinned staging chunks: the host
    copy of one chunk (multi-threaded) overlaps the DMA of the other, at pinned-copy speed."""
    if getattr(st, "stage", None) is None:
        st.stage = [torch.empty(_STAGE_BYTES, dtype=torch.uint8).pin_memory() for _ in range(2)]
        st.stage_ev = [None, None]
    src = torch.from_numpy(X).view(-1).view(torch.uint8)
    dst = st.X.view(-1).view(torch.uint8)
    main = torch.cuda.current_stream(st.device)
    total = src.numel()
    for c, off in enumerate(range(0, total, _STAGE_BYTES)):
        b = c & 1
        m = min(_STAGE_BYTES, total - off)
        if st.stage_ev[b] is not None:
            st.stage_ev[b].synchronize()           # its previous chunk has left the buffer
        st.stage[b][:m].copy_(src[off:off + m])
        dst[off:off + m].copy_(st.stage[b][:m], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(main)
        st.stage_ev[b] = ev


def _owned(torch, t, count: int, dtype):
    """A new NumPy array holding the first ``count`` elements of pinned tensor ``t``."""
    out = np.empty(count, dtype=dtype)
    if count:
        torch.from_numpy(out).copy_(t[:count])          # multi-threaded host copy
    return out


def _graph_host(X: np.ndarray, k: int, metric: str, method: str, precision: str, kprime: int,
                st: HostGraphState):
    """The drop-in's path: upload, graph, and both matrices back as SciPy CSR owning their arrays.
    The distances CSR is final before the connectivities are computed (``msc_neighbors_ex``
    records an event there): it is copied to pinned memory on a second stream and from there into
    its NumPy arrays while the GPU still computes the connectivities."""
    import scipy.sparse as sp
    torch = _torch()
    lib = _lib.load()
    n, d = X.shape
    mid, meth, pid = _ids(metric, method, precision)
    nbytes = lib.msc_neighbors_workspace_bytes(n, d, k, mid, meth, pid, int(kprime))
    ws = st.workspace.get(nbytes)
    main = torch.cuda.current_stream(st.device)
    _upload(torch, st, X)
    o = st.dev_out

    def buf(name, shape, dtype):
        t = o.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=st.device)
            o[name] = t
        return t
    m = max(k - 1, 0)
    knn_idx, knn_dist = buf("knn_idx", (n, k), torch.int32), buf("knn_dist", (n, k), torch.float32)
    d_ptr = buf("dist_indptr", (n + 1,), torch.int64)
    d_ind = buf("dist_indices", (max(n * m, 1),), torch.int32)
    d_dat = buf("dist_data", (max(n * m, 1),), torch.float32)
    c_ptr = buf("conn_indptr", (n + 1,), torch.int64)
    c_ind = buf("conn_indices", (max(2 * n * m, 1),), torch.int32)
    c_dat = buf("conn_data", (max(2 * n * m, 1),), torch.float32)
    stats = buf("stats", (_lib.STATS_LEN,), torch.int64)
    _lib.check(lib.msc_neighbors_ex(st.X.data_ptr(), n, d, k, mid, meth, pid, int(kprime),
                                    knn_idx.data_ptr(), knn_dist.data_ptr(), d_ptr.data_ptr(),
                                    d_ind.data_ptr(), d_dat.data_ptr(), c_ptr.data_ptr(),
                                    c_ind.data_ptr(), c_dat.data_ptr(), stats.data_ptr(),
                                    ws.data_ptr(), ws.numel(), main.cuda_stream,
                                    st.ready.cuda_event), "msc_neighbors_ex")
    h = st.host
    cs = st.copy_stream
    with torch.cuda.stream(cs):
        cs.wait_event(st.ready)
        h["dist_indptr"].copy_(d_ptr, non_blocking=True)
        h["dist_indices"][: n * m].copy_(d_ind[: n * m], non_blocking=True)
        h["dist_data"][: n * m].copy_(d_dat[: n * m], non_blocking=True)
    h["stats"].copy_(stats, non_blocking=True)
    h["conn_indptr"].copy_(c_ptr, non_blocking=True)
    cs.synchronize()                              # the distances are on the host; the GPU goes on
    d_ptr_h = h["dist_indptr"].numpy().astype(_index_dtype(n, n * m))
    dist = sp.csr_matrix((_owned(torch, h["dist_data"], n * m, np.float32),
                          _owned(torch, h["dist_indices"], n * m, np.int32), d_ptr_h),
                         shape=(n, n))
    main.synchronize()
    _lib.check_stats(h["stats"].numpy())
    nnz = int(h["conn_indptr"][n])
    # the connectivities in chunks: every chunk's download is queued at once on the copy stream,
    # and each chunk is copied into the NumPy arrays as soon as it has arrived, while the later
    # chunks are still in flight
    c_data = np.empty(nnz, np.float32)
    c_indices = np.empty(nnz, np.int32)
    chunks = []
    with torch.cuda.stream(cs):
        for off in range(0, nnz, _DOWN_CHUNK):
            m = min(_DOWN_CHUNK, nnz - off)
            h["conn_indices"][off:off + m].copy_(c_ind[off:off + m], non_blocking=True)
            h["conn_data"][off:off + m].copy_(c_dat[off:off + m], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(cs)
            chunks.append((off, m, ev))
    for off, m, ev in chunks:
        ev.synchronize()
        torch.from_numpy(c_indices[off:off + m]).copy_(h["conn_indices"][off:off + m])
        torch.from_numpy(c_data[off:off + m]).copy_(h["conn_data"][off:off + m])
    conn = sp.csr_matrix((c_data, c_indices,
                          h["conn_indptr"].numpy().astype(_index_dtype(n, nnz))), shape=(n, n))
    return dist, conn


def neighbors(X_pca: np.ndarray, n_neighbors: int = 15, random_state: int = 0,
              approx: bool | None = None, *, metric: str = "euclidean", method: str = "umap",
              precision: str = DEFAULT_PRECISION, kprime: int = 0, device=None):
    """Distance + connectivity graphs of a PCA embedding (metalsinglecell neighbors.py:727-760).

    Returns ``(distances, connectivities)`` as SciPy CSR matrices: ``distances`` holds the k-1
    nearest other cells of every row (explicit zeros kept for coincident cells, as SciPy keeps
    them in the reference), ``connectivities`` the symmetric fuzzy graph (method='umap') or the
    Gaussian-kernel graph (method='gauss').  ``random_state`` and ``approx`` are accepted for
    compatibility; the graph is exact and deterministic.

    The embedding is uploaded through pinned staging chunks, the graph built on the GPU, and the
    distances matrix copied back and assembled on the host while the connectivities are still
    being computed.  Device and pinned buffers of the last shape are kept for the next call of
    that shape.
    """
    torch = _torch()
    X = np.ascontiguousarray(X_pca, dtype=np.float32)
    if X.ndim != 2:
        raise ValueError("X_pca must be 2-D")
    n, d = X.shape
    k = int(n_neighbors)
    dev = torch.device(device) if device is not None else torch.device("cuda",
                                                                       torch.cuda.current_device())
    # argument errors are raised before any buffer of this shape is made
    mid, meth, pid = _ids(metric, method, precision)
    lib = _lib.load()
    if lib.msc_neighbors_workspace_bytes(n, d, k, mid, meth, pid, int(kprime)) == 0:
        _lib.check(lib.msc_neighbors(0, n, d, k, mid, meth, pid, int(kprime), *([0] * 10), 0, 0),
                   "msc_neighbors")
        raise ValueError("msc_neighbors: invalid arguments")
    st = _host_state(n, d, k, dev)
    with torch.cuda.device(dev):
        return _graph_host(X, k, metric, method, precision, kprime, st)


def _knn(X_pca: np.ndarray, n_neighbors: int, random_state: int = 0,
         approx: bool | None = None, backend: str = "nndescent", *, metric: str = "euclidean",
         precision: str = DEFAULT_PRECISION, kprime: int = 0, device=None):
    """Exact kNN ``(indices int32 (n,k), dists float32 (n,k))``, self first, ascending by
    (distance, index) — the contract of metalsinglecell ``_knn`` (neighbors.py:698-724), also
    used by scrublet there.  ``backend`` names the reference's approximate engines; all of them
    are replaced by the exact path here."""
    if backend not in ("nndescent", "ivf", "pynndescent"):
        raise ValueError(f"unknown kNN backend {backend!r} (nndescent|ivf|pynndescent)")
    torch = _torch()
    X = np.ascontiguousarray(X_pca, dtype=np.float32)
    dev = torch.device(device) if device is not None else torch.device("cuda",
                                                                       torch.cuda.current_device())
    idx, dist, stats = knn_device(torch.from_numpy(X).to(dev), n_neighbors, metric=metric,
                                  precision=precision, kprime=kprime)
    torch.cuda.current_stream(dev).synchronize()
    _lib.check_stats(stats.cpu().numpy())
    return idx.cpu().numpy(), dist.cpu().numpy()


def bbknn(X_pca: np.ndarray, batch, neighbors_within_batch: int = 3, n_pcs: int | None = 50,
          trim: int | None = None, random_state: int = 0, **kw):
    """Batch-balanced kNN graph (neighbors.py:491-559); see ``msc_b200.bbknn.bbknn``."""
    from .bbknn import bbknn as _impl
    return _impl(X_pca, batch, neighbors_within_batch, n_pcs, trim, random_state, **kw)


def _trim_graph(conn, trim):
    """Each cell's ``trim`` strongest connectivities (neighbors.py:465-488), on the GPU; see
    ``msc_b200.bbknn.trim_graph``."""
    from .bbknn import trim_graph as _impl
    return _impl(conn, trim)
