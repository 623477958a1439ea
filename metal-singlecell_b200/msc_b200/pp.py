"""AnnData-facing drop-ins for ``msc.pp.neighbors`` (metalsinglecell pp.py:722-788) and
``msc.pp.bbknn`` (pp.py:809-833).

``neighbors(adata, n_neighbors=15, n_pcs=None, *, use_rep=None, metric='euclidean',
method='umap', key_added=None, random_state=0, copy=False)`` writes the same slots as the
reference: ``obsp['distances']`` / ``obsp['connectivities']`` (or ``f'{key_added}_…'``) and
``uns['neighbors']`` (or ``uns[key_added]``) = ``{connectivities_key, distances_key, params}``,
which graph consumers resolve through ``neighbors_key`` (tl.py:14-21).  Additions over the
reference: ``method='gauss'`` and ``metric='cosine'`` (the reference raises for the latter,
pp.py:768-769), and a ``precision`` keyword selecting the tensor-core candidate form.
"""

from __future__ import annotations

import numpy as np

from .neighbors import neighbors as _nb, DEFAULT_PRECISION
from .bbknn import bbknn as _bbknn

# Width below which scanpy builds the graph on ``.X`` itself rather than on a PCA (the default
# component count of its settings object).
_WIDE = 50


def _as_f32(M):
    """A dense float32 array of ``M``, which may be a SciPy sparse matrix."""
    if hasattr(M, "toarray") and not isinstance(M, np.ndarray):
        M = M.toarray()
    return np.asarray(M, dtype=np.float32)


def _choose_representation(adata, use_rep, n_pcs):
    """The embedding the graph is built on, with the name it is recorded under (pp.py:722-745).

    * ``use_rep`` given: ``'X'`` selects ``.X``; any other name must be a key of ``.obsm``, else
      ``ValueError`` with the reference's message.
    * ``use_rep`` absent: ``.X`` when ``n_pcs == 0`` or the object has at most 50 variables;
      otherwise ``obsm['X_pca']``, which must hold at least ``n_pcs`` (default 50) components.
      The reference computes that PCA itself when it is missing (pp.py:735-737); PCA is a
      preprocessing step outside this library, so here the caller is asked to run it first.
    """
    if use_rep == "X":
        return _as_f32(adata.X), "X"
    if use_rep is not None:
        if use_rep not in adata.obsm:
            raise ValueError(f"Did not find {use_rep} in .obsm.keys(). "
                             f"You need to compute it first.")
        return _as_f32(adata.obsm[use_rep]), use_rep
    if n_pcs == 0 or adata.n_vars <= _WIDE:
        return _as_f32(adata.X), None
    pcs = adata.obsm["X_pca"] if "X_pca" in adata.obsm else None
    if pcs is None or pcs.shape[1] < (n_pcs or _WIDE):
        raise ValueError("obsm['X_pca'] with enough components is missing: run PCA "
                         "(e.g. msc.pp.pca) before pp.neighbors")
    return _as_f32(pcs), "X_pca"


def neighbors(adata, n_neighbors: int = 15, n_pcs: int | None = None, *,
              use_rep: str | None = None, metric: str = "euclidean", method: str = "umap",
              key_added: str | None = None, random_state: int = 0, copy: bool = False,
              precision: str = DEFAULT_PRECISION):
    """kNN graph (``sc.pp.neighbors``); writes ``obsp['distances']``/``['connectivities']`` and
    ``uns['neighbors']`` (pp.py:753-788).  Returns ``None``, or the modified copy if ``copy``.

    ``key_added`` renames all three slots (``f'{key}_distances'``, ``f'{key}_connectivities'``,
    ``uns[key]``).  ``uns[...]['params']`` holds ``n_neighbors``, ``method``, ``random_state`` and
    ``metric`` always, and ``use_rep`` / ``n_pcs`` only when the caller passed them."""
    if metric not in ("euclidean", "cosine"):
        raise NotImplementedError(f"metric={metric!r} is not implemented (euclidean, cosine)")
    if method not in ("umap", "gauss"):
        raise ValueError(f"method={method!r} must be 'umap' or 'gauss'")
    target = adata.copy() if copy else adata
    rep, _ = _choose_representation(target, use_rep, n_pcs)
    if n_pcs is not None:
        rep = rep[:, :n_pcs]          # only the leading n_pcs columns take part
    dist, conn = _nb(rep, n_neighbors=n_neighbors, random_state=random_state, metric=metric,
                     method=method, precision=precision)
    prefix = "" if key_added is None else f"{key_added}_"
    slots = {"connectivities_key": prefix + "connectivities",
             "distances_key": prefix + "distances"}
    target.obsp[slots["distances_key"]] = dist
    target.obsp[slots["connectivities_key"]] = conn
    params = dict(n_neighbors=n_neighbors, method=method, random_state=random_state,
                  metric=metric)
    params.update({name: val for name, val in (("use_rep", use_rep), ("n_pcs", n_pcs))
                   if val is not None})
    target.uns["neighbors" if key_added is None else key_added] = {**slots, "params": params}
    return target if copy else None


def _obs_column(adata, key):
    col = adata.obs[key]
    return col.to_numpy() if hasattr(col, "to_numpy") else np.asarray(col)


def bbknn(adata, batch_key: str = "batch", *, use_rep: str = "X_pca",
          neighbors_within_batch: int = 3, n_pcs: int | None = 50, trim: int | None = None,
          random_state: int = 0, copy: bool = False, precision: str = DEFAULT_PRECISION):
    """Batch-balanced kNN (``sc.external.pp.bbknn``); writes ``obsp['distances']`` /
    ``['connectivities']`` and ``uns['neighbors']`` with ``n_neighbors`` = the width of the
    combined lists, ``neighbors_within_batch`` × the batch count for batches of at least that
    size (pp.py:809-833).  Returns ``None``, or the modified copy if ``copy``."""
    adata = adata.copy() if copy else adata
    if use_rep not in adata.obsm:
        raise ValueError(f"Did not find {use_rep} in .obsm.keys(). You need to compute it first.")
    dist, conn, n_neighbors = _bbknn(np.asarray(adata.obsm[use_rep], dtype=np.float32),
                                     _obs_column(adata, batch_key),
                                     neighbors_within_batch=neighbors_within_batch, n_pcs=n_pcs,
                                     trim=trim, random_state=random_state, precision=precision)
    adata.obsp["distances"] = dist
    adata.obsp["connectivities"] = conn
    adata.uns["neighbors"] = {
        "connectivities_key": "connectivities", "distances_key": "distances",
        "params": {"n_neighbors": n_neighbors, "method": "umap", "metric": "euclidean",
                   "random_state": random_state, "use_rep": use_rep, "n_pcs": n_pcs,
                   "bbknn": {"trim": 10 * n_neighbors if trim is None else trim,
                             "computation": "cuda"}}}
    return adata if copy else None


def connectivities(adata, neighbors_key: str = "neighbors"):
    """The connectivity graph, resolved through ``uns[neighbors_key]`` as the reference's graph
    consumers do (tl.py:14-21)."""
    key = "connectivities"
    if neighbors_key in adata.uns:
        key = adata.uns[neighbors_key].get("connectivities_key", key)
    if key not in adata.obsp:
        raise ValueError(f"run pp.neighbors first (no adata.obsp[{key!r}])")
    return adata.obsp[key]
