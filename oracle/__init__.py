"""CPU oracle for the ``pp.neighbors`` path.  TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy/SciPy on the host, what the reference computes for
``msc.pp.neighbors`` (metalsinglecell ``pp.py:753-788`` → ``neighbors.py:727-760``):

* ``knn.knn_exact`` — exact k nearest neighbours, self first, then the k-1 nearest other
  cells ordered by (FP64 squared distance, index) — the tie rule of ``neighbors.py:457-461``;
  returned distances are float32 ``sqrt`` of the FP64 squared distance (``neighbors.py:129-131``).
* ``graph.smooth_knn_dist`` / ``graph.membership_strengths`` / ``graph.fuzzy_union`` — the
  umap-learn 0.5.12 ``fuzzy_simplicial_set`` the reference calls at ``neighbors.py:742-753``
  (umap-learn is a third-party dependency, ``pyproject.toml:36``, absent here; its published
  algorithm is restated).
* ``graph.distances_csr`` — the distances graph exactly as ``neighbors.py:755-759`` builds it.
* ``graph.gauss_connectivities`` — the locally scaled Gaussian kernel (Haghverdi et al. 2016)
  for ``method='gauss'``, which the reference does not implement.
* ``bbknn.bbknn`` / ``bbknn.trim_graph`` — the batch-balanced graph of ``pp.bbknn``
  (``pp.py:809-833`` → ``neighbors.py:491-559``, trimming ``neighbors.py:465-488``), the next
  caller of the same kNN and fuzzy-set steps.
* ``spatial.grid_knn`` / ``spatial.grid_radius`` / ``spatial.knn_edges`` — the uniform-grid
  spatial kNN and radius search of 2-D/3-D coordinates (``neighbors.py:143-417``, used by
  ``gr.py:186-255``), pinned against sklearn by the reference's own known-answer criteria.
* ``handoff.umap_edges`` — the UMAP layout's edge preparation (weak-edge pruning and
  epochs-per-sample, ``embedding.py:100-137, 255-267``), the first consumer of the graph.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import this
package, and only as the checker.  The product (``metal-singlecell_b200/``) never imports it.

Pinning: ``bbknn.trim_graph`` and ``handoff.umap_edges`` equal the reference's own
``_trim_graph`` and ``_prune_weak_edges`` / ``_make_epochs_per_sample`` bit for bit on the fixtures
of ``tests/golden/make_golden.py``.  The kNN restatement is pinned by the reference's own known-answer tests
(``tests/test_postfix_fixes.py:108-121``, 500×20 recall vs NumPy brute force;
``tests/test_postfix_fixes.py:197-207``, coincident points stay finite) and by fixtures generated
from the reference's NumPy-expressible code (``tests/golden/make_golden.py``).  Connectivity
VALUES have no reference test or golden vector (umap-learn and scanpy are absent):
**parity unpinned** for the fuzzy-set and gauss values; the oracle states their arithmetic exactly
and the CUDA path is checked bit-for-bit against it.
"""

from .knn import knn_exact, l2_normalize_rows, sq_dist_f64
from .graph import (smooth_knn_dist, membership_strengths, fuzzy_union, distances_csr,
                    gauss_connectivities, neighbors_graph, exp_f32)

__all__ = ["knn_exact", "l2_normalize_rows", "sq_dist_f64", "smooth_knn_dist",
           "membership_strengths", "fuzzy_union", "distances_csr", "gauss_connectivities",
           "neighbors_graph", "exp_f32"]
