"""ctypes binding of the C ABI declared in ``include/msc_b200.h``.

The library is loaded from the package directory (``libmsc_b200.so``, built by
``msc_b200._build``).  There is no CPU fallback: if the library is missing every compute call
raises.  Status codes map onto the exceptions the reference raises for the same conditions
(``ValueError`` for bad arguments, ``NotImplementedError`` for unsupported requests — cf.
metalsinglecell pp.py:768-769, neighbors.py:724).
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int32, c_int64, c_size_t, c_void_p, c_char_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmsc_b200.so"

MSC_OK, MSC_ERR_INVALID_ARG, MSC_ERR_WORKSPACE, MSC_ERR_TIMEOUT, MSC_ERR_CUDA, \
    MSC_ERR_UNSUPPORTED = range(6)

METRIC = {"euclidean": 0, "cosine": 1}
PRECISION = {"fp32": 0, "bf16x3": 1, "fp16": 2, "bf16": 3}
METHOD = {"umap": 0, "gauss": 1}

STAT_NONFINITE, STAT_TIMEOUT, STAT_CERTIFIED, STAT_REFINED, STAT_RESCANNED, STAT_FP64_TIES, \
    STAT_CONN_NNZ, STAT_PRECISION = range(8)
STATS_LEN = 8
MAX_K = 129
MAX_K_KNN = 513
MAX_D = 128
BBKNN_MAX_WIDTH = 128
NOALLOC_MAX_CELLS = 65536
NOALLOC_MAX_ENTRIES = 1 << 20

SP_STAT_NONFINITE, SP_STAT_STATUS, SP_STAT_CELLS, SP_STAT_CHUNKS, SP_STAT_EVALS, \
    SP_STAT_EXPANDED, SP_STAT_RING, SP_STAT_CELL_SIDE = range(8)
SP_STATS_LEN = 8
SPATIAL_MAX_K = 65

P = c_void_p
I32, I64, SZ, F32, F64 = c_int32, c_int64, c_size_t, c_float, c_double

# name -> (restype, argtypes); mirrors include/msc_b200.h
SIGNATURES = {
    "msc_version": (I32, []),
    "msc_last_error": (c_char_p, []),
    "msc_launch_count": (ctypes.c_longlong, []),
    "msc_profile_enable": (I32, [I32]),
    "msc_profile_read": (I32, [P, I32]),
    "msc_profile_counters": (I32, [P, I32]),
    "msc_selftest_wait_timeout": (I32, [I64, P, P]),
    "msc_neighbors_workspace_bytes": (SZ, [I64, I32, I32, I32, I32, I32, I32]),
    "msc_neighbors": (I32, [P, I64, I32, I32, I32, I32, I32, I32, P, P, P, P, P, P, P, P, P, P,
                            SZ, P]),
    "msc_neighbors_ex": (I32, [P, I64, I32, I32, I32, I32, I32, I32, P, P, P, P, P, P, P, P, P,
                               P, SZ, P, P]),
    "msc_knn_workspace_bytes": (SZ, [I64, I32, I32, I32, I32, I32]),
    "msc_knn": (I32, [P, I64, I32, I32, I32, I32, I32, P, P, P, P, SZ, P]),
    "msc_batched_workspace_bytes": (SZ, [P, I32, I32, I32, I32, I32, I32]),
    "msc_batched_prepare": (I32, [P, I32, I32, I32, I32, I32, I32, P, SZ, P]),
    "msc_batched_knn": (I32, [P, P, I32, I32, I32, I32, I32, I32, I32, P, P, P, P, SZ, P]),
    "msc_smooth_knn_dist": (I32, [P, I64, I32, F32, P, P, P, SZ, P]),
    "msc_membership": (I32, [P, P, P, P, I64, I32, P, P]),
    "msc_fuzzy_union_workspace_bytes": (SZ, [I64, I32]),
    "msc_fuzzy_union": (I32, [P, P, I64, I32, P, P, P, P, P, SZ, P]),
    "msc_fuzzy_union_noalloc": (I32, [P, P, I64, I32, P, P, P, P, P]),
    "msc_gauss_workspace_bytes": (SZ, [I64, I32]),
    "msc_gauss_connectivities": (I32, [P, P, I64, I32, P, P, P, P, P, SZ, P]),
    "msc_distances_csr": (I32, [P, P, I64, I32, P, P, P, P]),
    "msc_umap_edges_workspace_bytes": (SZ, [I64]),
    "msc_umap_edges": (I32, [P, P, P, I64, I32, P, P, P, P, P, P, SZ, P]),
    "msc_bbknn_width": (I32, [P, I32, I32]),
    "msc_bbknn_workspace_bytes": (SZ, [I64, I32, P, I32, I32, I32]),
    "msc_bbknn_knn": (I32, [P, I64, I32, P, P, I32, I32, I32, P, P, P, P, SZ, P]),
    "msc_bbknn_distances_workspace_bytes": (SZ, [I64]),
    "msc_bbknn_distances_csr": (I32, [P, P, I64, I32, P, P, P, P, SZ, P]),
    "msc_trim_graph_workspace_bytes": (SZ, [I64]),
    "msc_trim_graph": (I32, [P, P, P, I64, I32, P, P, P, P, SZ, P]),
    "msc_spatial_knn_workspace_bytes": (SZ, [I64, I32, I32]),
    "msc_spatial_knn": (I32, [P, I64, I32, I32, P, P, P, P, SZ, P]),
    "msc_spatial_radius_workspace_bytes": (SZ, [I64, I32]),
    "msc_spatial_radius_count": (I32, [P, I64, I32, F64, F64, P, P, P, SZ, P]),
    "msc_spatial_radius_scratch_bytes": (SZ, [I64]),
    "msc_spatial_radius_fill": (I32, [I64, I32, F64, F64, P, I64, P, P, P, SZ, P, SZ, P]),
    "msc_spatial_edge_lengths": (I32, [P, I64, I32, P, P, P, P]),
}

_lib = None


def load():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"msc_b200 CUDA library missing ({LIB_PATH}); build it with "
                "`python -m msc_b200._build` — there is no CPU fallback")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def last_error() -> str:
    msg = load().msc_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str = "msc_b200") -> None:
    if status == MSC_OK:
        return
    msg = f"{what}: {last_error()}"
    if status == MSC_ERR_INVALID_ARG:
        raise ValueError(msg)
    if status == MSC_ERR_WORKSPACE:
        raise MemoryError(msg)
    if status == MSC_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(f"{msg} (status {status})")


def check_stats(stats) -> None:
    """Device-side failures recorded in the stats block (read after the stream completed)."""
    if int(stats[STAT_TIMEOUT]):
        raise RuntimeError("msc_b200: a device-side wait timed out; results are invalid")
    if int(stats[STAT_NONFINITE]):
        raise ValueError(f"msc_b200: input holds {int(stats[STAT_NONFINITE])} non-finite values")


def check_spatial_stats(stats) -> None:
    """Device-side failures of the spatial search (read after the stream completed)."""
    if int(stats[SP_STAT_NONFINITE]):
        raise ValueError(f"msc_b200: coordinates hold {int(stats[SP_STAT_NONFINITE])} "
                         "non-finite values")
    if int(stats[SP_STAT_STATUS]):
        raise RuntimeError(f"msc_b200: spatial grid plan failed (status "
                           f"{int(stats[SP_STAT_STATUS])})")


def ptr(t) -> int:
    """Device (or host) address of a torch tensor / numpy array, 0 for None."""
    if t is None:
        return 0
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data
