"""msc_b200 — the single-cell neighbour graph (``msc.pp.neighbors``) on NVIDIA B200.

A drop-in for metalsinglecell's ``pp.neighbors`` path: exact kNN from fused tcgen05 distance +
top-k kernels, UMAP fuzzy connectivities (or the gauss kernel) and the distances CSR, all on one
GPU through the C ABI in ``include/msc_b200.h``.

    import msc_b200 as msc
    msc.pp.neighbors(adata, n_neighbors=15)
    msc.pp.bbknn(adata, batch_key="batch")      # batch-balanced graph

``msc_b200.gr`` / ``msc_b200.spatial`` carry the spatial (2-D / 3-D) kNN and radius graphs on a
uniform-grid search.
"""

from . import pp, neighbors, bbknn, synth, spatial, gr, _lib
from .anndata_lite import AnnDataLite

__version__ = "0.1.0"

__all__ = ["pp", "neighbors", "bbknn", "synth", "spatial", "gr", "AnnDataLite", "__version__"]
