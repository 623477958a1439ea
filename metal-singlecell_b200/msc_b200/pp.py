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

_N_PCS_DEFAULT = 50            # scanpy's settings.N_PCS


def _dense(X):
    import scipy.sparse as sp
    return X.toarray() if sp.issparse(X) else np.asarray(X)


def _choose_representation(adata, use_rep, n_pcs):
    """scanpy's representation rule as the reference applies it (pp.py:722-745): ``.X`` when
    ``n_pcs == 0`` or the object has at most 50 variables, ``X_pca`` otherwise, ``obsm[use_rep]``
    when given (``'X'`` = ``.X``).  Computing a missing PCA (pp.py:735-737) is a preprocessing step
    outside this library: run PCA first."""
    if use_rep is None and n_pcs == 0:
        return np.asarray(_dense(adata.X), dtype=np.float32), None
    if use_rep is None:
        if adata.n_vars > _N_PCS_DEFAULT:
            if "X_pca" not in adata.obsm or adata.obsm["X_pca"].shape[1] < (n_pcs or _N_PCS_DEFAULT):
                raise ValueError("obsm['X_pca'] with enough components is missing: run PCA "
                                 "(e.g. msc.pp.pca) before pp.neighbors")
            return np.asarray(adata.obsm["X_pca"], dtype=np.float32), "X_pca"
        return np.asarray(_dense(adata.X), dtype=np.float32), None
    if use_rep == "X":
        return np.asarray(_dense(adata.X), dtype=np.float32), "X"
    if use_rep not in adata.obsm:
        raise ValueError(f"Did not find {use_rep} in .obsm.keys(). "
                         f"You need to compute it first.")
    return np.asarray(adata.obsm[use_rep], dtype=np.float32), use_rep


def neighbors(adata, n_neighbors: int = 15, n_pcs: int | None = None, *,
              use_rep: str | None = None, metric: str = "euclidean", method: str = "umap",
              key_added: str | None = None, random_state: int = 0, copy: bool = False,
              precision: str = DEFAULT_PRECISION):
    """kNN graph (``sc.pp.neighbors``); writes ``obsp['distances']``/``['connectivities']`` and
    ``uns['neighbors']`` (pp.py:753-788).  Returns ``None``, or the modified copy if ``copy``."""
    if metric not in ("euclidean", "cosine"):
        raise NotImplementedError(f"metric={metric!r} is not implemented (euclidean, cosine)")
    if method not in ("umap", "gauss"):
        raise ValueError(f"method={method!r} must be 'umap' or 'gauss'")
    adata = adata.copy() if copy else adata
    rep, _ = _choose_representation(adata, use_rep, n_pcs)
    if n_pcs is not None:                            # scanpy truncates the rep to the first n_pcs
        rep = rep[:, :n_pcs]
    dist, conn = _nb(rep, n_neighbors=n_neighbors, random_state=random_state, metric=metric,
                     method=method, precision=precision)
    ck = "connectivities" if key_added is None else f"{key_added}_connectivities"
    dk = "distances" if key_added is None else f"{key_added}_distances"
    adata.obsp[dk] = dist
    adata.obsp[ck] = conn
    params = {"n_neighbors": n_neighbors, "method": method,
              "random_state": random_state, "metric": metric}
    if use_rep is not None:            # scanpy records only what the caller asked for
        params["use_rep"] = use_rep
    if n_pcs is not None:
        params["n_pcs"] = n_pcs
    adata.uns["neighbors" if key_added is None else key_added] = {
        "connectivities_key": ck, "distances_key": dk, "params": params}
    return adata if copy else None


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
