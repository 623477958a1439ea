"""The device-resident hand-off on a real result: the torch CSR tensor and the graph-container
arrays of ``neighbors_device`` equal the host CSR matrices of the same call."""
import numpy as np
import pytest

from msc_b200 import neighbors as nbm, synth

pytestmark = pytest.mark.gpu


def test_handoff_matches_host_graph():
    import torch
    X = synth.gaussian_mixture(5000, 20, 8, seed=51)
    res = nbm.neighbors_device(torch.from_numpy(X).cuda(), 15)
    torch.cuda.synchronize()
    dist, conn = nbm.graph_to_host(res, 5000, 15)
    T = nbm.to_torch_csr(res, 5000)
    assert T.is_cuda and T.values().data_ptr() == res["conn_data"].data_ptr()
    np.testing.assert_array_equal(T.crow_indices().cpu().numpy(), conn.indptr)
    np.testing.assert_array_equal(T.col_indices().cpu().numpy(), conn.indices)
    np.testing.assert_array_equal(T.values().cpu().numpy(), conn.data)
    g = nbm.graph_arrays(res, 5000)
    np.testing.assert_array_equal(g["edge_src"].cpu().numpy(),
                                  np.repeat(np.arange(5000), np.diff(conn.indptr)))
    D = nbm.to_torch_csr(res, 5000, "distances")
    np.testing.assert_array_equal(D.values().cpu().numpy(), dist.data)
