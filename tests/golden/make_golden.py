"""Generate golden vectors by running the reference's own code (metalsinglecell) on the CPU.

The reference needs Apple's `mlx`, which cannot exist here.  The parts of its neighbour path that
use only array arithmetic are run under a small NumPy stand-in for ``mlx.core`` (the module below
maps every ``mx.*`` call those functions make onto its NumPy equivalent):

* ``neighbors._knn_gpu`` (neighbors.py:82-132) for k = 33 and 50 on the reference's own test
  input (tests/test_postfix_fixes.py:108-121: 500×20 N(0,1), default_rng(0)).  For k > 32 the
  reference selects with ``mx.argpartition`` (neighbors.py:66-68), so every step it takes —
  fp16 rescaled Gram ranking, argpartition, fp32 direct-difference recompute, host sort — is the
  reference's code.  (k ≤ 32 goes through a Metal kernel and is not run.)
* the vendored mlx-vis ``UMAP._fuzzy_simplicial_set`` (_vendor/mlx_vis/umap.py:199-271) on an
  exact kNN graph: the per-row ρ and the bisection σ are captured from its ``mx.eval`` calls.

* ``neighbors.neighbors`` (neighbors.py:727-760) with the exact oracle's kNN lists in place of its
  Metal kNN and the oracle's fuzzy set in place of umap-learn: the distances CSR its own code
  builds (neighbors.py:755-759), on an input with duplicate cells (stored zero distances);
* ``neighbors._trim_graph`` (neighbors.py:465-488), pure SciPy, run as is on batch-balanced
  connectivities built by the oracle (the reference test's tiny-batch input,
  tests/test_postfix_fixes.py:186-193, and a 3-batch mixture) and on a random symmetric graph
  that stores explicit zeros, at several trims;
* ``gr.spatial_neighbors_knn`` / ``_radius`` / ``_grid`` / ``_delaunay`` (gr.py:198-368) with the
  oracle's grid kNN and radius search (oracle/spatial.py) in place of the Metal grid kernels: the edge
  selection, FP64 edge lengths, the lattice median correction and ring expansion, the
  percentile / set_diag / transform tail and the per-library blocks are the reference's code,
  on jittered and exact hex lattices, a 3-D point cloud and interleaved sections;
* the UMAP layout's edge preparation ``embedding._prune_weak_edges`` and
  ``_make_epochs_per_sample`` (embedding.py:100-137, 255-267), pure NumPy/SciPy, run as is on
  connectivities built by the oracle, at several epoch counts.

Run from the repository root, naming the reference project's ``src`` directory (the one that
holds the ``metalsinglecell`` package), as an argument or in ``MSC_REFERENCE_SRC``:

    python tests/golden/make_golden.py <reference>/src

Writes tests/golden/reference_knn_500x20.npz, reference_rho_sigma.npz, reference_distances_csr.npz,
reference_trim.npz, reference_spatial.npz and reference_umap_edges.npz.
"""
import os
import sys
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
sys.path.insert(0, str(Path(__file__).resolve().parents[2] / "metal-singlecell_b200"))


def numpy_mlx():
    """A stand-in ``mlx.core`` backed by NumPy; ``captured`` records every ``eval`` argument."""
    mx = types.ModuleType("mlx.core")
    mx.captured = []
    mx.float16, mx.float32, mx.int32, mx.uint32, mx.int64 = (np.float16, np.float32, np.int32,
                                                              np.uint32, np.int64)

    def array(x, dtype=None):
        a = np.array(x)
        if dtype is not None:
            a = a.astype(dtype)
        elif a.dtype == np.float64:
            a = a.astype(np.float32)             # MLX's default float type
        return a

    def eval_(*args):
        mx.captured.append([np.array(a) for a in args])

    mx.array = array
    mx.eval = eval_
    mx.sum = lambda a, axis=None: np.sum(a, axis=axis, dtype=a.dtype)
    mx.max = lambda a, axis=None: np.max(a, axis=axis)
    mx.min = lambda a, axis=None: np.min(a, axis=axis)
    mx.maximum = lambda a, b: np.maximum(a, np.asarray(b, dtype=np.asarray(a).dtype))
    mx.where = lambda c, a, b: np.where(c, a, b).astype(np.result_type(
        np.asarray(a).dtype, np.asarray(b).dtype) if np.asarray(a).dtype != np.float64
        else np.float32)
    mx.full = lambda shape, v: np.full(shape, v, dtype=np.float32)
    mx.ones = lambda shape: np.ones(shape, dtype=np.float32)
    mx.exp = np.exp
    mx.abs = np.abs
    mx.all = np.all
    mx.argpartition = lambda a, kth, axis=-1: np.argpartition(a, kth, axis=axis)
    mx.argsort = lambda a, axis=-1: np.argsort(a, axis=axis)
    mx.compile = lambda f: f                     # decorators in the vendored module
    pkg = types.ModuleType("mlx")
    pkg.core = mx
    sys.modules["mlx"] = pkg
    sys.modules["mlx.core"] = mx
    return mx


def reference_src(argv) -> Path:
    """The reference's ``src`` directory: the first argument, else ``MSC_REFERENCE_SRC``."""
    src = argv[1] if len(argv) > 1 else os.environ.get("MSC_REFERENCE_SRC")
    if not src:
        sys.exit("usage: make_golden.py <reference src directory> (or set MSC_REFERENCE_SRC)")
    src = Path(src)
    if not (src / "metalsinglecell").is_dir():
        sys.exit(f"{src} holds no metalsinglecell package")
    return src


def main():
    ref = reference_src(sys.argv)
    mx = numpy_mlx()
    sys.path.insert(0, str(ref))
    from metalsinglecell import neighbors as ref_nb
    from metalsinglecell._vendor.mlx_vis.umap import UMAP as RefUMAP

    rng = np.random.default_rng(0)
    X = rng.standard_normal((500, 20)).astype(np.float32)
    out = {"X": X}
    for k in (33, 50):
        idx, dist = ref_nb._knn_gpu(X, k)
        out[f"idx_k{k}"] = np.asarray(idx, np.int64)
        out[f"dist_k{k}"] = np.asarray(dist, np.float32)
    np.savez_compressed(OUT / "reference_knn_500x20.npz", **out)

    import oracle
    from msc_b200 import synth
    Xg = synth.gaussian_mixture(400, 12, 6, seed=17)
    k = 15
    idx, d2, dist = oracle.knn_exact(Xg, k)
    self = types.SimpleNamespace(n_neighbors=k, n_epochs=200)
    mx.captured.clear()
    try:
        RefUMAP._fuzzy_simplicial_set(self, idx.astype(np.int32), dist, Xg.shape[0])
    except Exception:
        pass            # only the captured ρ and σ are needed; the later symmetrisation may not run
    rho = np.asarray(mx.captured[0][0], np.float32)
    sigma = np.asarray([c[0] for c in mx.captured if c[0].shape == rho.shape][-1], np.float32)
    np.savez_compressed(OUT / "reference_rho_sigma.npz", X=Xg, knn_idx=idx, knn_dist=dist,
                        rho=rho, sigma=sigma, k=k)

    # the reference's own neighbors() (neighbors.py:727-760) builds the distances graph from the
    # kNN lists: its kNN engine (Metal) and umap-learn are absent, so the lists come from the
    # exact oracle and the fuzzy set from the oracle's restatement (its output is not stored:
    # that would pin the oracle against itself); the distances CSR is the reference's code.
    # Input with exact duplicates, so that zero distances are stored explicitly.
    Xd = np.random.default_rng(5).standard_normal((300, 12)).astype(np.float32)
    Xd[250:260] = Xd[0:10]
    kd = 10

    def _knn_exact(X, k, random_state=0, approx=None):
        i, _, dd = oracle.knn_exact(X, k)
        return i, dd

    def _fss(X, n_neighbors, random_state, metric, knn_indices, knn_dists, **kw):
        sg, rh = oracle.smooth_knn_dist(knn_dists, float(n_neighbors))
        w = oracle.membership_strengths(knn_indices, knn_dists, sg, rh)
        return oracle.fuzzy_union(knn_indices, w, knn_indices.shape[0]), sg, rh

    umap_pkg, umap_mod = types.ModuleType("umap"), types.ModuleType("umap.umap_")
    umap_mod.fuzzy_simplicial_set = _fss
    umap_pkg.umap_ = umap_mod
    sys.modules.setdefault("umap", umap_pkg)
    sys.modules.setdefault("umap.umap_", umap_mod)
    saved_knn = ref_nb._knn
    ref_nb._knn = _knn_exact
    try:
        Dref, _ = ref_nb.neighbors(Xd, kd)
    finally:
        ref_nb._knn = saved_knn
    Dref = Dref.tocsr()
    ki, _, kdist = oracle.knn_exact(Xd, kd)
    np.savez_compressed(OUT / "reference_distances_csr.npz", X=Xd, k=kd, knn_idx=ki,
                        knn_dist=kdist, indptr=Dref.indptr.astype(np.int64),
                        indices=Dref.indices.astype(np.int64), data=Dref.data)

    # the reference's _trim_graph on batch-balanced connectivities: the reference test's own
    # tiny-batch input (tests/test_postfix_fixes.py:186-193) and a 3-batch mixture, several trims
    from oracle import bbknn as obb
    r0 = np.random.default_rng(0)
    cases = [(r0.standard_normal((60, 10)).astype(np.float32),
              np.array(["a"] * 40 + ["b"] * 2 + ["c"] * 18), 3, (0, 4, 6, 30)),
             (synth.gaussian_mixture(500, 16, 5, seed=23),
              np.random.default_rng(29).choice(np.array(["p", "q", "r"]), 500), 5, (8, 12, 20, 150))]
    trim_out = {}
    for c, (Xc, bc, kwb, trims) in enumerate(cases):
        _, _, K, inter = obb.bbknn(Xc, bc, neighbors_within_batch=kwb)
        conn = inter["untrimmed"].tocsr()
        trim_out[f"c{c}_indptr"] = conn.indptr.astype(np.int64)
        trim_out[f"c{c}_indices"] = conn.indices.astype(np.int64)
        trim_out[f"c{c}_data"] = conn.data.astype(np.float32)
        trim_out[f"c{c}_trims"] = np.asarray(trims, np.int64)
        for t in trims:
            R = ref_nb._trim_graph(conn, t).tocsr()
            R.sort_indices()
            trim_out[f"c{c}_t{t}_indptr"] = R.indptr.astype(np.int64)
            trim_out[f"c{c}_t{t}_indices"] = R.indices.astype(np.int64)
            trim_out[f"c{c}_t{t}_data"] = R.data.astype(np.float32)
    # and a symmetric random graph that stores explicit zeros (the reference drops them)
    import scipy.sparse as sp
    Z = sp.random(300, 300, density=0.08, random_state=2, format="csr", dtype=np.float32)
    Z = (Z + Z.T).tocsr()
    Z.data[np.random.default_rng(1).random(Z.nnz) < 0.1] = 0.0
    c = len(cases)
    trim_out[f"c{c}_indptr"] = Z.indptr.astype(np.int64)
    trim_out[f"c{c}_indices"] = Z.indices.astype(np.int64)
    trim_out[f"c{c}_data"] = Z.data.astype(np.float32)
    trim_out[f"c{c}_trims"] = np.asarray((3, 5, 8, 12), np.int64)
    for t in (3, 5, 8, 12):
        R = ref_nb._trim_graph(Z, t).tocsr()
        R.sort_indices()
        trim_out[f"c{c}_t{t}_indptr"] = R.indptr.astype(np.int64)
        trim_out[f"c{c}_t{t}_indices"] = R.indices.astype(np.int64)
        trim_out[f"c{c}_t{t}_data"] = R.data.astype(np.float32)
    np.savez_compressed(OUT / "reference_trim.npz", n_cases=len(cases) + 1, **trim_out)

    # the reference's spatial graph builders (gr.py:198-255: edge selection, FP64 edge lengths,
    # the percentile / set_diag / transform tail gr.py:81-104, per-library blocks gr.py:107-147)
    # with the oracle's grid kNN and radius search standing in for the Metal grid kernels
    from metalsinglecell import gr as ref_gr
    from oracle import spatial as osp
    spatial_golden(ref_nb, ref_gr, osp)
    umap_edges_golden()
    print("wrote", sorted(p.name for p in OUT.glob("reference_*.npz")))


def spatial_inputs():
    """Seeded coordinate sets of the spatial cases (float64, as ``adata.obsm['spatial']``)."""
    def lattice(side, jitter, seed):
        r, c = np.divmod(np.arange(side * side), side)
        xy = np.c_[c * 100.0 + (r % 2) * 50.0, r * 86.6]
        return xy + np.random.default_rng(seed).normal(0, jitter, xy.shape)
    lat = lattice(25, 1.0, 0)
    vol = np.random.default_rng(3).uniform(0, 50, (800, 3))
    two = np.vstack([lattice(16, 1.0, 1), lattice(16, 1.0, 2)])
    perm = np.random.default_rng(4).permutation(two.shape[0])
    lib = np.repeat([0, 2], 256)[perm]                   # category 1 unused; interleaved order
    hexl = lattice(30, 0.0, 0)                            # an exact Visium-like lattice
    fine = lattice(16, 0.0, 0) * 0.5 + np.array([5000.0, 0.0])   # a section at half the spacing
    both = np.vstack([lattice(16, 0.0, 0), fine])
    perm2 = np.random.default_rng(5).permutation(both.shape[0])
    lib2 = np.repeat([0, 1], 256)[perm2]
    return {"lat": (lat, None), "vol": (vol, None), "two": (two[perm], lib),
            "hex": (hexl, None), "hexlib": (both[perm2], lib2)}


SPATIAL_CASES = [
    ("knn", "lat", {"n_neighs": 6}),
    ("knn", "lat", {"n_neighs": 6, "set_diag": True}),
    ("knn", "lat", {"n_neighs": 6, "transform": "spectral"}),
    ("knn", "lat", {"n_neighs": 6, "transform": "cosine"}),
    ("knn", "lat", {"n_neighs": 10, "percentile": 80.0}),
    ("knn", "two", {"n_neighs": 6}),
    ("knn", "vol", {"n_neighs": 8}),
    ("radius", "lat", {"radius": 150.0}),
    ("radius", "lat", {"radius": (90.0, 150.0)}),
    ("radius", "lat", {"radius": 150.0, "percentile": 50.0}),
    ("radius", "lat", {"radius": 150.0, "set_diag": True, "transform": "spectral"}),
    ("radius", "two", {"radius": 120.0}),
    ("radius", "vol", {"radius": 7.0}),
    ("grid", "hex", {"n_neighs": 6}),
    ("grid", "hex", {"n_neighs": 6, "n_rings": 2}),
    ("grid", "hex", {"n_neighs": 6, "n_rings": 3, "set_diag": True}),
    ("grid", "hex", {"n_neighs": 6, "transform": "spectral"}),
    ("grid", "hexlib", {"n_neighs": 6, "n_rings": 2}),
    ("grid", "hex", {"delaunay": True}),
    ("grid", "hex", {"delaunay": True, "n_rings": 2, "set_diag": True}),
    ("delaunay", "lat", {}),
    ("delaunay", "two", {"radius": (20.0, 150.0), "percentile": 90.0, "transform": "spectral"}),
]


def spatial_golden(ref_nb, ref_gr, osp):
    import json
    import pandas as pd
    out = {}
    inputs = spatial_inputs()
    for name, (xy, lib) in inputs.items():
        out[f"{name}_coords"] = xy
        if lib is not None:
            out[f"{name}_library"] = lib
    saved = ref_nb._knn_grid, ref_nb._radius_grid
    ref_nb._knn_grid = lambda coords, k, min_n=4_000: osp.grid_knn(coords, k)
    ref_nb._radius_grid = lambda coords, radius, min_radius=0.0: osp.grid_radius(
        coords, radius, min_radius)
    try:
        for c, (kind, name, kw) in enumerate(SPATIAL_CASES):
            xy, lib = inputs[name]
            obs = pd.DataFrame(index=[str(i) for i in range(xy.shape[0])])
            extra = {}
            if lib is not None:
                obs["library"] = pd.Categorical.from_codes(lib, ["s0", "s1", "s2"])
                extra["library_key"] = "library"
            adata = types.SimpleNamespace(obsm={"spatial": xy}, obs=obs, obsp={}, uns={})
            fn = {"knn": ref_gr.spatial_neighbors_knn, "radius": ref_gr.spatial_neighbors_radius,
                  "grid": ref_gr.spatial_neighbors_grid,
                  "delaunay": ref_gr.spatial_neighbors_delaunay}[kind]
            adj, dst = fn(adata, copy=True, **kw, **extra)
            out[f"c{c}_case"] = np.array(json.dumps([kind, name, kw]))
            for tag, M in (("adj", adj), ("dst", dst)):
                M = M.tocsr()
                M.sort_indices()
                out[f"c{c}_{tag}_indptr"] = M.indptr.astype(np.int64)
                out[f"c{c}_{tag}_indices"] = M.indices.astype(np.int64)
                out[f"c{c}_{tag}_data"] = M.data
    finally:
        ref_nb._knn_grid, ref_nb._radius_grid = saved
    np.savez_compressed(OUT / "reference_spatial.npz", n_cases=len(SPATIAL_CASES), **out)


def umap_edges_golden():
    """The reference UMAP's edge preparation (embedding.py:100-137, 255-267) run as is on
    connectivities the oracle builds: `_prune_weak_edges` at several n_epochs, the kept graph as
    COO (embedding.py:115) and `_make_epochs_per_sample` of its weights.  Pure NumPy/SciPy."""
    import oracle
    from metalsinglecell import embedding as ref_emb
    out = {}
    X = oracle_input_mixture()
    C = oracle.neighbors_graph(X, 15)["connectivities"]
    # the lowest weights of this graph (~1e-3) sit between max/1000 and max/200, so the epochs
    # below drop some edges (200, 500) or none (3)
    cases = (3, 200, 500, 5000)
    out["indptr"] = C.indptr.astype(np.int64)
    out["indices"] = C.indices.astype(np.int64)
    out["data"] = C.data.astype(np.float32)
    out["epochs"] = np.asarray(cases, np.int64)
    for e in cases:
        G = ref_emb._prune_weak_edges(C, e)
        coo = G.tocoo()
        out[f"e{e}_rows"] = coo.row.astype(np.int64)
        out[f"e{e}_cols"] = coo.col.astype(np.int64)
        out[f"e{e}_weights"] = coo.data.astype(np.float32)
        out[f"e{e}_eps"] = ref_emb._make_epochs_per_sample(np.asarray(coo.data, np.float64), e)
    np.savez_compressed(OUT / "reference_umap_edges.npz", **out)


def oracle_input_mixture():
    """2,000 cells × 10 dims from 6 Gaussian clusters (seeded), for the UMAP edge golden."""
    rng = np.random.default_rng(77)
    centres = rng.normal(0, 4, (6, 10))
    lab = rng.integers(0, 6, 2000)
    return (centres[lab] + rng.standard_normal((2000, 10))).astype(np.float32)


if __name__ == "__main__":
    main()
