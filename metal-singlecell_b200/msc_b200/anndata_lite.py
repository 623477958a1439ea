"""A minimal AnnData stand-in: the slots ``pp.neighbors`` and ``pp.bbknn`` read and write.

``pp.neighbors`` and ``pp.bbknn`` work on any object exposing ``X``, ``n_obs``, ``n_vars``,
``obs`` (per-cell columns), ``obsm``, ``obsp``, ``uns`` and ``copy()`` — a real ``anndata.AnnData``
included; the spatial builders also read ``obs`` (a mapping or DataFrame of per-observation
columns).  This class provides exactly that for environments without anndata.
"""

from __future__ import annotations

import copy as _copy


class AnnDataLite:
    def __init__(self, X=None, *, obs=None, obsm=None, obsp=None, uns=None, n_obs=None,
                 n_vars=None):
        self.X = X
        self.obs = obs if obs is not None else {}
        self.obsm = dict(obsm or {})
        self.obsp = dict(obsp or {})
        self.uns = dict(uns or {})
        if n_obs is None:
            if X is not None:
                n_obs = X.shape[0]
            elif self.obsm:
                n_obs = next(iter(self.obsm.values())).shape[0]
            else:
                n_obs = 0
        self.n_obs = int(n_obs)
        self.n_vars = int(n_vars if n_vars is not None else (X.shape[1] if X is not None else 0))

    @property
    def shape(self):
        return (self.n_obs, self.n_vars)

    def copy(self):
        return _copy.deepcopy(self)

    def __repr__(self):
        return (f"AnnDataLite(n_obs={self.n_obs}, n_vars={self.n_vars}, obs={list(self.obs)}, "
                f"obsm={list(self.obsm)}, obsp={list(self.obsp)}, uns={list(self.uns)})")
