"""``neighbors_host`` (host in, host out, the distances CSR copied out on a second stream while the
connectivities are computed) returns exactly the graph of ``neighbors_device``."""
import numpy as np
import pytest

from msc_b200 import neighbors as nbm, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", ["umap", "gauss"])
def test_overlapped_host_call_equals_device_call(method):
    import torch
    X = synth.gaussian_mixture(20_000, 30, 12, seed=61)
    n, k = X.shape[0], 15
    ref = nbm.neighbors_device(torch.from_numpy(X).cuda(), k, method=method)
    torch.cuda.synchronize()
    dist, conn = nbm.graph_to_host(ref, n, k)
    st = nbm.HostGraphState(n, X.shape[1], k)
    Xh = torch.from_numpy(X).pin_memory()
    for _ in range(3):                                   # reused state, same answer every time
        h = nbm.neighbors_host(Xh, k, method=method, state=st)
        nnz = h["conn_nnz"]
        m = n * (k - 1)
        np.testing.assert_array_equal(h["dist_indptr"].numpy(), dist.indptr)
        np.testing.assert_array_equal(h["dist_indices"][:m].numpy(), dist.indices)
        np.testing.assert_array_equal(h["dist_data"][:m].numpy(), dist.data)
        np.testing.assert_array_equal(h["conn_indptr"].numpy(), conn.indptr)
        np.testing.assert_array_equal(h["conn_indices"][:nnz].numpy(), conn.indices)
        np.testing.assert_array_equal(h["conn_data"][:nnz].numpy(), conn.data)
