"""The C-ABI library loads and exports every entry point ``include/msc_b200.h`` declares; host-side
argument checks answer with the documented status codes.  No compute calls: runs without a GPU."""
import ctypes
import re
from pathlib import Path

import pytest

from msc_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "msc_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(msc_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), f"{name} declared in msc_b200.h but not exported"
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_constants():
    lib = _lib.load()
    assert lib.msc_version() >= 10000
    text = HEADER.read_text()
    for name, val in [("MSC_STATS_LEN", _lib.STATS_LEN), ("MSC_MAX_K", _lib.MAX_K),
                      ("MSC_MAX_D", _lib.MAX_D), ("MSC_STAT_CONN_NNZ", _lib.STAT_CONN_NNZ)]:
        assert re.search(rf"#define {name}\s+{val}\b", text), name


@pytest.mark.parametrize("n,d,k,metric,prec,kprime,code", [
    (10, 5, 11, 0, 1, 0, _lib.MSC_ERR_INVALID_ARG),      # k > n
    (10, 0, 3, 0, 1, 0, _lib.MSC_ERR_INVALID_ARG),       # d = 0
    (10, 129, 3, 0, 1, 0, _lib.MSC_ERR_INVALID_ARG),     # d > MSC_MAX_D
    (10, 5, 0, 0, 1, 0, _lib.MSC_ERR_INVALID_ARG),       # k = 0
    (1000, 30, 514, 0, 1, 0, _lib.MSC_ERR_UNSUPPORTED),  # k above MSC_MAX_K_KNN: unsupported
    (10, 5, 3, 7, 1, 0, _lib.MSC_ERR_INVALID_ARG),       # metric
    (10, 5, 3, 0, 9, 0, _lib.MSC_ERR_INVALID_ARG),       # precision
    (100, 5, 30, 0, 1, 20, _lib.MSC_ERR_INVALID_ARG),    # kprime < k-1
    (100, 5, 3, 0, 1, 65, _lib.MSC_ERR_INVALID_ARG),     # kprime > 64
    (10, 5, 3, 0, 1, 0, _lib.MSC_ERR_INVALID_ARG),       # NULL pointers
])
def test_argument_checks(n, d, k, metric, prec, kprime, code):
    lib = _lib.load()
    rc = lib.msc_knn(None, n, d, k, metric, prec, kprime, None, None, None, None, 0, None)
    assert rc == code
    assert _lib.last_error()
    with pytest.raises((ValueError, NotImplementedError)):
        _lib.check(rc)


def test_spatial_argument_checks():
    """The spatial entry points refuse bad requests before anything reaches a device: the
    address below is never dereferenced, since every case fails a host-side check first."""
    lib = _lib.load()
    F, big = 4096, 1 << 40
    E = _lib
    cases = [
        (lib.msc_spatial_knn(F, 100, 4, 5, F, F, F, F, big, None), E.MSC_ERR_UNSUPPORTED),  # 4-D
        (lib.msc_spatial_knn(F, 100, 2, 0, F, F, F, F, big, None), E.MSC_ERR_INVALID_ARG),  # k=0
        (lib.msc_spatial_knn(F, 100, 2, 101, F, F, F, F, big, None), E.MSC_ERR_INVALID_ARG),
        (lib.msc_spatial_knn(F, 100, 2, 66, F, F, F, F, big, None), E.MSC_ERR_UNSUPPORTED),
        (lib.msc_spatial_knn(None, 100, 2, 5, F, F, F, F, big, None), E.MSC_ERR_INVALID_ARG),
        (lib.msc_spatial_knn(F, 100, 2, 5, F, F, F, F, 16, None), E.MSC_ERR_WORKSPACE),
        (lib.msc_spatial_knn(F, 0, 2, 1, F, F, F, F, big, None), E.MSC_ERR_INVALID_ARG),
        (lib.msc_spatial_radius_count(F, 100, 2, -1.0, 0.0, F, F, F, big, None),
         E.MSC_ERR_INVALID_ARG),
        (lib.msc_spatial_radius_count(F, 100, 2, 1.0, 2.0, F, F, F, big, None),
         E.MSC_ERR_INVALID_ARG),                                                       # min > max
        (lib.msc_spatial_radius_count(F, 100, 2, float("inf"), 0.0, F, F, F, big, None),
         E.MSC_ERR_INVALID_ARG),
        (lib.msc_spatial_radius_count(F, 100, 3, 1.0, 0.0, F, F, F, 16, None),
         E.MSC_ERR_WORKSPACE),
        (lib.msc_spatial_radius_fill(100, 2, 1.0, 0.0, F, -1, F, F, F, big, F, big, None),
         E.MSC_ERR_INVALID_ARG),                                                       # nnz < 0
        (lib.msc_spatial_radius_fill(100, 2, 1.0, 0.0, F, 10, F, F, F, big, F, 8, None),
         E.MSC_ERR_WORKSPACE),                                                         # scratch
        (lib.msc_spatial_edge_lengths(F, 100, 4, F, F, F, None), E.MSC_ERR_INVALID_ARG),
    ]
    for i, (rc, code) in enumerate(cases):
        assert rc == code, (i, rc, _lib.last_error())
    text = HEADER.read_text()
    for name, val in [("MSC_SPATIAL_MAX_K", _lib.SPATIAL_MAX_K),
                      ("MSC_SP_STATS_LEN", _lib.SP_STATS_LEN),
                      ("MSC_SP_STAT_EXPANDED", _lib.SP_STAT_EXPANDED),
                      ("MSC_SP_STAT_CELL_SIDE", _lib.SP_STAT_CELL_SIDE)]:
        assert re.search(rf"#define {name}\s+{val}\b", text), name
    assert lib.msc_spatial_knn_workspace_bytes(1_000_000, 2, 7) > 0
    assert lib.msc_spatial_radius_scratch_bytes(0) >= 0


def test_workspace_queries_are_host_only():
    lib = _lib.load()
    a = lib.msc_neighbors_workspace_bytes(1_300_000, 50, 15, 0, 0, 1, 0)     # BF16x3
    b = lib.msc_neighbors_workspace_bytes(1_300_000, 50, 15, 0, 0, 2, 0)     # FP16 (+ refine)
    c = lib.msc_neighbors_workspace_bytes(1_300_000, 50, 15, 0, 0, 0, 0)     # FP32
    # FP16 carries the BF16x3 refine operands on top of its own, FP32 has the narrowest rows
    assert b > a > c > 0
    assert b < 4e9            # the whole scale workload fits a few GB of the 180 GB
    assert lib.msc_neighbors_workspace_bytes(10, 5, 11, 0, 0, 1, 0) == 0
    off = (ctypes.c_int64 * 4)(0, 100, 300, 350)
    assert lib.msc_batched_workspace_bytes(off, 3, 30, 15, 0, 1, 0) > 0
    bad = (ctypes.c_int64 * 3)(0, 10, 300)             # sample 0 smaller than k
    assert lib.msc_batched_workspace_bytes(bad, 2, 30, 15, 0, 1, 0) == 0
    assert lib.msc_fuzzy_union_workspace_bytes(1000, 15) > 0


def test_status_mapping():
    with pytest.raises(ValueError):
        _lib.check(_lib.MSC_ERR_INVALID_ARG)
    with pytest.raises(MemoryError):
        _lib.check(_lib.MSC_ERR_WORKSPACE)
    with pytest.raises(NotImplementedError):
        _lib.check(_lib.MSC_ERR_UNSUPPORTED)
    with pytest.raises(RuntimeError):
        _lib.check(_lib.MSC_ERR_TIMEOUT)
    with pytest.raises(RuntimeError):
        _lib.check_stats([0, 1, 0, 0, 0, 0, 0, 0])
    with pytest.raises(ValueError):
        _lib.check_stats([3, 0, 0, 0, 0, 0, 0, 0])


def test_knn_alone_reaches_large_k():
    lib = _lib.load()
    assert lib.msc_knn_workspace_bytes(3000, 20, _lib.MAX_K_KNN, 0, 2, 0) > 0
    assert lib.msc_knn_workspace_bytes(3000, 20, _lib.MAX_K_KNN + 1, 0, 2, 0) == 0
    assert lib.msc_knn_workspace_bytes(100, 20, 101, 0, 2, 0) == 0          # k > n
    # the whole graph keeps its own limit
    assert lib.msc_neighbors_workspace_bytes(3000, 20, _lib.MAX_K + 1, 0, 0, 2, 0) == 0
    assert re.search(rf"#define MSC_MAX_K_KNN\s+{_lib.MAX_K_KNN}\b", HEADER.read_text())


def test_bbknn_argument_checks():
    lib = _lib.load()
    C = lambda *v: (ctypes.c_int64 * len(v))(*v)
    inv = _lib.MSC_ERR_INVALID_ARG
    assert lib.msc_bbknn_width(C(40, 2, 18), 3, 3) == 3 + 2 + 3
    assert lib.msc_bbknn_workspace_bytes(60, 10, C(40, 2, 18), 3, 3, 2) > 0
    assert lib.msc_bbknn_workspace_bytes(60, 10, C(40, 2, 17), 3, 3, 2) == 0   # counts != n
    assert lib.msc_bbknn_workspace_bytes(60, 10, C(40, 0, 20), 3, 3, 2) == 0   # an empty batch
    assert lib.msc_bbknn_workspace_bytes(600, 10, C(300, 300), 2, 65, 2) == 0  # K = 130 > 128
    assert lib.msc_bbknn_workspace_bytes(600, 10, C(300, 300), 2, 64, 2) > 0   # K = 128
    assert lib.msc_bbknn_workspace_bytes(60, 129, C(60), 1, 3, 2) == 0         # d > MSC_MAX_D
    assert lib.msc_bbknn_workspace_bytes(60, 10, C(60), 1, 0, 2) == 0          # k = 0
    assert lib.msc_bbknn_workspace_bytes(60, 10, C(60), 1, 3, 9) == 0          # precision
    assert lib.msc_bbknn_knn(None, 60, 10, None, C(40, 2, 18), 3, 3, 2, None, None, None, None,
                             0, None) == inv
    assert "X" in _lib.last_error()
    assert lib.msc_bbknn_distances_csr(None, None, 10, 129, None, None, None, None, 0,
                                       None) == inv
    assert lib.msc_trim_graph(None, None, None, 10, 0, None, None, None, None, 0, None) == inv
    assert lib.msc_bbknn_distances_workspace_bytes(1000) > 0
    assert lib.msc_trim_graph_workspace_bytes(1000) > 0
    text = HEADER.read_text()
    assert re.search(rf"#define MSC_BBKNN_MAX_WIDTH\s+{_lib.BBKNN_MAX_WIDTH}\b", text)


def test_no_alloc_limits_match_the_header_and_fit_its_array():
    # the fixed array of msc_fuzzy_union_noalloc is 20 MiB; the workspace the union needs at the
    # corners of the accepted region must fit in it, or accepted calls would be refused
    lib = _lib.load()
    text = HEADER.read_text()
    assert re.search(rf"#define MSC_NOALLOC_MAX_CELLS\s+{_lib.NOALLOC_MAX_CELLS}\b", text)
    assert re.search(rf"#define MSC_NOALLOC_MAX_ENTRIES\s+{_lib.NOALLOC_MAX_ENTRIES}\b", text)
    for n, k in ((_lib.NOALLOC_MAX_CELLS, _lib.NOALLOC_MAX_ENTRIES // _lib.NOALLOC_MAX_CELLS),
                 (_lib.NOALLOC_MAX_ENTRIES // _lib.MAX_K, _lib.MAX_K),
                 (_lib.NOALLOC_MAX_CELLS, 2)):
        assert 0 < lib.msc_fuzzy_union_workspace_bytes(n, k) <= 20 << 20, (n, k)
