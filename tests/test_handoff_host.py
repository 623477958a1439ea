"""Device-resident hand-off of the graph (``csr_device``, ``to_torch_csr``, ``graph_arrays`` in
``msc_b200.neighbors``): views of a ``neighbors_device`` result as a torch CSR tensor and in the
layout of the reference's graph container (graph/csr_graph.py:15-40), checked here on CPU
tensors shaped like a device result (the views do not depend on the device)."""
import numpy as np
import pytest
import torch

import oracle
from msc_b200 import neighbors as nbm


@pytest.fixture
def result():
    X = np.random.default_rng(2).standard_normal((300, 8)).astype(np.float32)
    g = oracle.neighbors_graph(X, 10)
    C, D = g["connectivities"], g["distances"]
    cap = 2 * 300 * 9
    res = {"conn_indptr": torch.from_numpy(C.indptr.astype(np.int64)),
           "conn_indices": torch.zeros(cap, dtype=torch.int32),
           "conn_data": torch.zeros(cap, dtype=torch.float32),
           "dist_indptr": torch.from_numpy(D.indptr.astype(np.int64)),
           "dist_indices": torch.from_numpy(D.indices.astype(np.int32)),
           "dist_data": torch.from_numpy(D.data)}
    res["conn_indices"][:C.nnz] = torch.from_numpy(C.indices.astype(np.int32))
    res["conn_data"][:C.nnz] = torch.from_numpy(C.data)
    return res, C, D


def test_csr_views_and_torch_tensor(result):
    res, C, D = result
    ip, ind, dat = nbm.csr_device(res, 300)
    assert ind.numel() == C.nnz and dat.numel() == C.nnz
    assert dat.data_ptr() == res["conn_data"].data_ptr()          # a view, no copy
    T = nbm.to_torch_csr(res, 300)
    assert T.col_indices().data_ptr() == res["conn_indices"].data_ptr()
    np.testing.assert_array_equal(T.to_dense().numpy(), C.toarray())
    Td = nbm.to_torch_csr(res, 300, "distances")
    np.testing.assert_array_equal(Td.to_dense().numpy(), D.toarray())
    with pytest.raises(ValueError):
        nbm.csr_device(res, 300, "weights")


def test_graph_container_layout(result):
    res, C, _ = result
    g = nbm.graph_arrays(res, 300)
    assert g["n"] == 300 and g["indptr"].dtype == torch.uint32     # csr_graph.py:32
    np.testing.assert_array_equal(g["indptr"].numpy(), C.indptr)
    np.testing.assert_array_equal(g["indices"].numpy(), C.indices)
    np.testing.assert_array_equal(g["weights"].numpy(), C.data)
    # Graph.from_scipy: edge_src = np.repeat(arange(n), diff(indptr))
    np.testing.assert_array_equal(g["edge_src"].numpy(),
                                  np.repeat(np.arange(300, dtype=np.int32), np.diff(C.indptr)))
