#!/usr/bin/env python
"""Benchmark of the neighbour-graph path (``pp.neighbors``) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload scale|plain|precision|batch|serve|bbknn]
                    [--precision fp16|bf16x3|bf16|fp32]

A step = one full graph (exact kNN → distances CSR → UMAP connectivities) of the workload's
synthetic embedding.  Default workload: 1,300,000 cells × 50 PCs, 200-cluster Gaussian mixture with
lognormal sizes and 1% noise cells, euclidean, k=15, method='umap'; default path: FP16
tensor-core candidates with key-tile pruning, exact re-rank (BF16x3 refine, FP64 at the boundary).

value   cells/s with the embedding resident in HBM (whole job: N replicas × cells / max time);
e2e     the same through the public call with host buffers: pinned host → device copy of the
        embedding and device → host copy of both CSR matrices inside the timed region;
roofline: the main tensor-core candidate launch, 2·d·128·256 FLOP per (query tile, key tile) pair
        it computes (near + kept far tiles) over its event-timed duration, against the measured
        sustained dense BF16 peak (MEASURED_PEAKS.json); dense_equivalent_tflops divides 2·d·n²;
cpu_baseline: the CPU oracle port on this host's cores, on a bounded sample of query rows;
fp32_form: the plain FP32 SIMT form of the same exact graph (full scan);
bf16x3_form: the three-term BF16 tensor-core form of the same exact graph.

With --impl reference the CPU implementation alone runs (rank 0), on bounded samples.
Multi-GPU (torchrun): every rank builds its own full graph (replicas; the path runs on one GPU).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for p in (ROOT, ROOT / "metal-singlecell_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import numpy as np

METRIC = "kNN-graph cells/s at 1.3M×50 k=15, BF16+rerank vs FP32 GPU; serve p50/p99 ms"
FORM_STEPS = 3            # graphs timed for each comparison form
# DRAM bytes (read + written) of one main-scan launch of the candidate kernel, from a one-pass
# ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of this bench's own command; a
# profiler cannot run inside the timed bench, so the figure is carried here with its source
MAIN_SCAN_TRAFFIC = {
    "scale:fp16": (4_517_000_000,
                   "copied from a one-pass ncu capture of knn_tc_kernel's main-scan launch at "
                   "1.3M cells (4.255 GB read + 0.262 GB written): ncu --metrics "
                   "gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum "
                   "--clock-control none -k regex:knn_tc -c 3 python bench.py --steps 1 "
                   "--warmup 1 --skip-cpu --skip-fp32 --skip-configs (the second launch)"),
}


def workload(name: str, n: int | None = None):
    from msc_b200 import synth
    if name == "scale":
        X, p = synth.scale_1m3(n=n or 1_300_000)
        return X, p, (f"scale: {X.shape[0]:,} cells x 50 PCs, 200 clusters (lognormal sizes), "
                      "1% noise")
    if name == "plain":
        X, p = synth.plain_10k()
        return X, p, "plain: 10,000 cells x 50 PCs, 20 equal clusters"
    if name == "precision":
        X, p = synth.precision_200k()
        return X, p, "precision: 200,000 cells x 50 PCs, 50 anisotropic clusters, cosine"
    raise SystemExit(f"unknown workload {name}")


def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples of this GPU during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                   "-lms", "200"]
            if self.uuid:
                cmd += ["-i", self.uuid]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


class Replicas:
    """One process per GPU, each building its own full graph (the path runs on one GPU, so the
    ranks are independent replicas with no collective on the data path): a barrier on both sides
    of the timed region, per-rank times combined as their max, and the whole-job rate
    world × cells / time.  RANK / WORLD_SIZE / MASTER_* come from the environment (torchrun)."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 600.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.backend = backend
        self.device = device
        if self.world > 1:
            import torch.distributed as dist
            from datetime import timedelta
            kw = {"device_id": device} if backend == "nccl" and device is not None else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch
        import torch.distributed as dist
        dev = self.device if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def rate(self, cells_per_rank: int, seconds: float) -> float:
        return self.world * cells_per_rank / seconds

    def close(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


def cpu_baseline(X, k, metric, budget_s: float = 15.0):
    """Oracle port on the host: exact kNN of a seeded sample of query rows against the whole
    embedding, plus the per-row ρ/σ and membership stages; cells/s = rows / time."""
    import oracle
    cores = len(os.sched_getaffinity(0))
    rng = np.random.default_rng(1234)
    n = X.shape[0]
    m = int(min(n, 256))
    t_total, rows = 0.0, 0
    while t_total < budget_s and rows < n:
        q = np.sort(rng.choice(n, m, replace=False))
        t0 = time.perf_counter()
        idx, d2, dist = oracle.knn_exact(X, k, metric=metric, rows=q, threads=cores)
        sigma, rho = oracle.smooth_knn_dist(dist, float(k))
        oracle.membership_strengths(idx - q[:, None] + np.arange(m)[:, None], dist, sigma, rho)
        t_total += time.perf_counter() - t0
        rows += m
        m = int(min(n, max(m, rows * 2)))  # grow the sample until the budget is spent
        if t_total > budget_s * 0.5:
            break
    return {"value": rows / t_total, "unit": "cells/s", "cores": cores, "kind": "port",
            "sample": f"{rows} seeded query rows of the {n}-cell embedding (exact kNN against all "
                      f"{n} cells + rho/sigma + memberships), {t_total:.1f} s on {cores} threads"}


def error_vs_fp64(X, idx, dist, k, metric, n_rows: int = 512, seed: int = 20261204):
    """Distance error of the returned float32 distances against the FP64 oracle on a seeded
    sample of rows, and whether those rows' neighbour lists equal the oracle's exactly."""
    import oracle
    n = X.shape[0]
    rows = np.sort(np.random.default_rng(seed).choice(n, min(n_rows, n), replace=False))
    ridx, rd2, _ = oracle.knn_exact(X, k, metric=metric, rows=rows,
                                    threads=len(os.sched_getaffinity(0)))
    exact = rd2 * 0.5 if metric == "cosine" else np.sqrt(rd2)
    got = np.asarray(dist[rows], np.float64)
    nz = exact > 0
    rel = np.abs(got[nz] - exact[nz]) / exact[nz]
    same = (np.asarray(idx[rows]) == ridx).all(axis=1)
    return {"rows": int(rows.size), "rows_identical_to_oracle": int(same.sum()),
            "max_rel_error": float(rel.max()) if rel.size else 0.0,
            "mean_rel_error": float(rel.mean()) if rel.size else 0.0,
            "bound": 2.0 ** -24,
            "note": "float32 distance vs FP64 sqrt of the FP64 squared distance (cosine: d2/2); "
                    "target 1e-5 relative"}


def events_ms(torch, fn, reps: int, warm: int = 1) -> float:
    """Mean device time of ``fn`` over ``reps`` calls, CUDA events on the current stream."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def config_leg(name: str, uuid, steps: int = 5):
    """One configuration of the workload list at its stated size: the default form, the
    three-term BF16 form and the plain FP32 form of the same exact graph, each timed over
    ``steps`` graphs with its own clock record, the forms' kNN lists compared with each other,
    and the distance error against the FP64 oracle on sampled rows."""
    import torch
    from msc_b200 import neighbors as nbm, _lib
    X, p, desc = workload(name)
    n = X.shape[0]
    k, metric, method = p["n_neighbors"], p["metric"], p.get("method", "umap")
    kprime = p.get("kprime", 0)
    Xd = torch.from_numpy(X).cuda()
    out = {"workload": desc, "n_neighbors": k, "metric": metric, "method": method,
           "kprime": int(kprime) or "auto", "forms": {}}
    lists = {}
    for prec in ("fp16", "bf16x3", "fp32"):
        ws, buf = nbm.Workspace(Xd.device), {}

        def step():
            return nbm.neighbors_device(Xd, k, metric=metric, method=method, precision=prec,
                                        kprime=kprime, workspace=ws, out=buf)
        res = step()
        torch.cuda.synchronize()
        _lib.check_stats(res["stats"].cpu().numpy())
        with ClockSampler(uuid) as clk:
            ms = events_ms(torch, step, steps, warm=1)
        lists[prec] = (res["knn_idx"].clone(), res["knn_dist"].clone())
        out["forms"][prec] = {"ms_per_graph": ms, "cells_per_s": n / (ms / 1000.0),
                              "steps": steps, "clocks": clk.summary()}
    ref_i, ref_d = lists["fp32"]
    out["forms_identical"] = all(bool(torch.equal(i, ref_i) and torch.equal(d, ref_d))
                                 for i, d in lists.values())
    out["speedup_fp16_over_fp32"] = out["forms"]["fp32"]["ms_per_graph"] / \
        out["forms"]["fp16"]["ms_per_graph"]
    out["speedup_bf16x3_over_fp32"] = out["forms"]["fp32"]["ms_per_graph"] / \
        out["forms"]["bf16x3"]["ms_per_graph"]
    idx, dist = (t.cpu().numpy() for t in lists["fp16"])
    out["error_vs_fp64"] = error_vs_fp64(X, idx, dist, k, metric)
    del Xd, lists
    torch.cuda.empty_cache()
    return out


def batch_leg(uuid, n_samples: int = 64, steps: int = 5):
    """The batching configuration, reduced to ``n_samples`` samples: one persistent launch under
    a captured CUDA graph with autotuned tiles against the per-sample launch loop."""
    import torch
    from msc_b200 import batch, synth, _lib
    X, offsets, p = synth.batch_samples(n_samples, seed=3, d=30)
    n, d = X.shape
    k = p["n_neighbors"]
    Xd = torch.from_numpy(X).cuda()
    loop_out = batch.per_sample_loop(Xd, offsets, k)
    tune = batch.autotune(Xd, offsets, k, reps=1, use_cache=False)
    bt = batch.BatchedKnn(offsets, d, k, tile_config=tune["tile_config"])
    bt.capture(Xd)
    with ClockSampler(uuid) as clk:
        loop_ms = events_ms(torch, lambda: batch.per_sample_loop(Xd, offsets, k, out=loop_out),
                            steps)
        graph_ms = events_ms(torch, bt.replay, steps)
    stats = bt.check()
    sizes = np.diff(offsets)
    same = bool(torch.equal(bt.idx, loop_out[0]) and torch.equal(bt.dist, loop_out[1]))
    out = {"workload": f"{len(sizes)} samples, {n:,} cells (min {int(sizes.min())}, max "
                       f"{int(sizes.max())}), 30 PCs, k=15, euclidean (the 256-sample "
                       f"configuration's first {n_samples} samples)",
           "graph_ms": graph_ms, "cells_per_s": n / (graph_ms / 1000.0),
           "per_sample_loop_ms": loop_ms, "speedup_vs_loop": loop_ms / graph_ms,
           "identical_to_loop": same, "tile": batch.decode_tile_code(tune["tile_config"]),
           "certified": int(stats[_lib.STAT_CERTIFIED]),
           "rescanned": int(stats[_lib.STAT_RESCANNED]), "steps": steps,
           "clocks": clk.summary()}
    del Xd, bt, loop_out
    torch.cuda.empty_cache()
    return out


def serve_leg(uuid, args, load_fracs=(0.5, 0.7, 0.85), pool_size: int = 64):
    """The serving configuration: Poisson arrivals of ``args.serve_requests`` graph requests per
    load point (1k-500k cells, 30/50/100 PCs, k in {10, 15, 30}, euclidean / cosine), admitted by
    HBM budget into concurrent slots; p50 / p99 latency (arrival to the result complete in HBM
    and handed to the caller) and cells/s at arrival rates set to fractions of the batched-offline
    throughput of the same requests.  The requests cycle through ``pool_size`` distinct seeded
    embeddings (host memory), each request uploading its own."""
    import torch
    from msc_b200 import serve, synth
    spec = synth.serving_requests(1.0, args.serve_requests, seed=5)
    pool = [synth.request_embedding(r) for r in spec[:pool_size]]
    reqs_spec = [spec[i % pool_size] for i in range(len(spec))]
    data = [pool[i % pool_size] for i in range(len(spec))]
    total_cells = sum(x.shape[0] for x in data)
    budget = int(args.hbm_budget_gb * (1 << 30))

    def fresh():
        return [serve.Request(X=x, n_neighbors=r["k"], metric=r["metric"])
                for x, r in zip(data, reqs_spec)]

    # every slot stages embeddings up to the largest of the pool; one untimed pass over the
    # pool warms every shape
    pinned = max(x.nbytes for x in pool)
    # the results are released as requests complete (a consumer that takes each graph)
    serve.run_offline(fresh()[:pool_size], budget, args.slots, pinned_bytes=pinned,
                      keep_results=False)
    with ClockSampler(uuid) as clk:
        off = serve.run_offline(fresh(), budget, args.slots, pinned_bytes=pinned,
                                keep_results=False)
    off["clocks"] = clk.summary()
    mean_cells = total_cells / len(data)
    sweep = []
    for frac in load_fracs:
        rate = frac * off["cells_per_s"] / mean_cells
        rng = np.random.default_rng(7)
        arr = np.cumsum(rng.exponential(1.0 / rate, len(data))).tolist()
        with ClockSampler(uuid) as clk:
            rep = serve.run_trace(fresh(), arr, budget, args.slots, pinned_bytes=pinned,
                                  keep_results=False)
        rep.update({"load_frac_of_offline": frac, "rate_req_per_s": rate,
                    "throughput_frac_of_offline": rep["cells_per_s"] / off["cells_per_s"],
                    "clocks": clk.summary()})
        sweep.append(rep)
    kept_up = [r for r in sweep if r["failed"] == 0 and
               r["throughput_frac_of_offline"] >= 0.95 * r["load_frac_of_offline"]]
    best = max(kept_up, key=lambda r: r["load_frac_of_offline"], default=None)
    sizes = np.array([x.shape[0] for x in pool])
    return {"requests_per_point": len(data), "distinct_embeddings": pool_size,
            "cells_total_per_point": int(total_cells),
            "pool_cells": {"min": int(sizes.min()), "median": int(np.median(sizes)),
                           "max": int(sizes.max())},
            "slots": args.slots, "hbm_budget_gb": args.hbm_budget_gb,
            "distribution": "cells LogNormal(ln 20000, 1) clipped 1k-500k; PCs {30,50,100}; "
                            "k {10,15,30}; metric {euclidean, cosine}",
            "latency": "arrival -> result complete on the device and handed to the caller",
            "offline": off, "sweep": sweep,
            "sustained": None if best is None else {
                "throughput_frac_of_offline": best["throughput_frac_of_offline"],
                "load_frac_of_offline": best["load_frac_of_offline"],
                "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"]}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    X, p, desc = workload(args.workload, args.n)
    k, metric = p["n_neighbors"], p["metric"]
    for _ in range(args.warmup):
        cpu_baseline(X, k, metric, budget_s=2.0)
    vals, t0 = [], time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_baseline(X, k, metric, budget_s=args.ref_budget)["value"])
    wall = time.perf_counter() - t0
    v = float(np.median(vals))
    last = cpu_baseline(X, k, metric, budget_s=1.0)
    line = {"metric": METRIC, "value": v, "unit": "cells/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * wall / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "n_neighbors": k, "metric": metric,
                       "method": p.get("method", "umap"), "impl": "CPU oracle port (NumPy/SciPy)"},
            "cpu_baseline": {"value": v, "unit": "cells/s", "cores": last["cores"],
                             "kind": "port", "sample": last["sample"]},
            "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    from msc_b200 import neighbors as nbm, _lib

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    reps = Replicas("nccl", dev)
    world, rank = reps.world, reps.rank
    lib = _lib.load()

    X, p, desc = workload(args.workload, args.n)
    n, d = X.shape
    k, metric = p["n_neighbors"], p["metric"]
    method = p.get("method", "umap")
    kprime = args.kprime or p.get("kprime", 0)
    Xd = torch.from_numpy(X).to(dev)
    ws = nbm.Workspace(dev)
    out = {}

    def step(precision=args.precision):
        return nbm.neighbors_device(Xd, k, metric=metric, method=method, precision=precision,
                                    kprime=kprime, workspace=ws, out=out)

    barrier, max_over_ranks = reps.barrier, reps.max

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    res = step()
    torch.cuda.synchronize()
    stats = res["stats"].cpu().numpy()
    _lib.check_stats(stats)

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    st = torch.cuda.current_stream(dev)
    launches0 = lib.msc_launch_count()
    with ClockSampler(uuid) as clk:
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            step()
        e1.record(st)
        torch.cuda.synchronize()
        barrier()
    launches = lib.msc_launch_count() - launches0
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    value = reps.rate(n, ms / 1000.0)

    # per-stage times of one profiled step (events on the launching stream)
    lib.msc_profile_enable(1)
    step()
    torch.cuda.synchronize()
    import ctypes
    buf = (ctypes.c_float * 12)()
    ns = lib.msc_profile_read(buf, 12)
    lib.msc_profile_enable(0)
    stage_names = ["prep", "near_pass", "prune_plan", "candidates", "rerank_fp64",
                   "csr_rho_sigma_membership", "union"]
    stages = {stage_names[i]: round(buf[i], 3) for i in range(min(ns, len(stage_names)))}
    cnt = (ctypes.c_ulonglong * 64)()
    lib.msc_profile_counters(cnt, 64)

    def pipe(base):
        c = [int(cnt[base + i]) for i in range(16)]
        ctas = max(c[9], 1)
        nepi = c[10] / ctas if c[10] else 4.0
        return {"producer_wait_stage": c[0] / ctas, "mma_wait_keys": c[1] / ctas,
                "mma_wait_accumulator": c[2] / ctas,
                "epilogue_wait_accumulator": c[3] / ctas / nepi,
                "epilogue_loop": c[4] / ctas / nepi, "kernel": c[5] / ctas,
                "hot_chunks_per_warp": c[6] / ctas / nepi,
                "insertions_per_row": c[8] / max(n, 1), "ctas": c[9], "epilogue_warps": nepi,
                "insert_rounds_per_warp": c[11] / ctas / nepi,
                "hot_path_cycles_per_warp": c[12] / ctas / nepi,
                "far_tiles_scanned": c[13], "walks_ended_early": c[14]}
    pipeline = {"near_pass": pipe(16), "main": pipe(32), "refine": pipe(48)}
    # key tiles beyond the near ones: kept by the pruning plan / all of them
    pruning = {"far_tiles_visited": int(cnt[10]), "far_tiles_total": int(cnt[11]),
               "visited_frac": (cnt[10] / cnt[11]) if cnt[11] else None,
               "level1_failed": int(cnt[12]), "pair_stage_tiles": int(cnt[13]),
               "pair_tests": int(cnt[14])}

    pk, pk_kind = peaks()
    cand_ms = stages.get("candidates")
    # Work of the main candidate launch: the (128-row query tile, 256-key tile) pairs it computes
    # -- every query tile's near tiles (its own key tile and two either side) plus the far tiles
    # it scanned: those the pruning plan kept, minus those an ordered walk left after ending
    # early -- each 2·d·128·256 FLOP (d unpadded).  Without pruning every pair of the n×n matrix
    # is computed.
    dense_flop = 2.0 * d * float(n) * float(n)
    if cnt[11]:
        nkt = -(-n // 256)
        q = np.arange(-(-n // 128))
        diag = (128 * q) // 256
        near_tiles = int((np.minimum(nkt - 1, diag + 2) - np.maximum(0, diag - 2) + 1).sum())
        # far tiles the main scan computed: the ordered walk counts its own (it ends walks
        # early), else every tile the plan kept
        ordered = cnt[32 + 13] + cnt[32 + 14] > 0
        tile_pairs = near_tiles + int(cnt[32 + 13] if ordered else cnt[10])
        alg_flop = min(dense_flop, 2.0 * d * 128.0 * 256.0 * tile_pairs)
    else:
        tile_pairs = None
        alg_flop = dense_flop
    achieved = alg_flop / (cand_ms / 1000.0) / 1e12 if cand_ms else None
    peak = pk.get("bf16_tflops_sustained") or pk.get("bf16_tflops")
    traffic, traffic_src = MAIN_SCAN_TRAFFIC.get(f"{args.workload}:{args.precision}",
                                                 (None, None))
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "traffic_source": traffic_src,
                "kernel": "knn_tc_kernel" if args.precision != "fp32" else "knn_fp32_kernel",
                "algorithmic_flop_per_launch": alg_flop, "kernel_ms": cand_ms,
                "tile_pairs_computed": tile_pairs,
                "dense_equivalent_tflops": (dense_flop / (cand_ms / 1000.0) / 1e12)
                                           if cand_ms else None,
                "peak_kind": f"{pk_kind} bf16 sustained (kernel timed inside a full step)",
                "stage_ms": stages, "pipeline_cycles_per_cta": pipeline, "pruning": pruning}

    # e2e through the drop-in call itself (neighbors.neighbors, neighbors.py:727-760 in the
    # reference): a host NumPy embedding in, SciPy CSR matrices out; the upload, the graph, the
    # copies back (distances while the connectivities run) and the SciPy construction are all
    # inside the timed region
    m = k - 1

    def dropin_step():
        dist_csr, conn_csr = nbm.neighbors(X, k, metric=metric, method=method,
                                           precision=args.precision, kprime=kprime, device=dev)
        return conn_csr.nnz

    for _ in range(max(1, args.warmup // 2)):
        dropin_step()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nnzs = [dropin_step() for _ in range(args.steps)]
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    barrier()
    h2d = X.nbytes
    d2h = 8 * (n + 1) * 2 + n * m * 8 + nnzs[-1] * 8 + 8 * _lib.STATS_LEN
    e2e = {"value": reps.rate(n, e2e_s), "unit": "cells/s", "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "ms_per_step": 1000 * e2e_s,
           "path": "msc_b200.neighbors.neighbors(X_pca): host NumPy in, SciPy CSR out"}

    # the same through the pinned-buffer host call (neighbors_host): no pageable copies
    Xh = torch.from_numpy(X).pin_memory()
    hstate = nbm.HostGraphState(n, d, k, device=dev)

    def pinned_step():
        r = nbm.neighbors_host(Xh, k, metric=metric, method=method, precision=args.precision,
                               kprime=kprime, state=hstate)
        return r["conn_nnz"]

    pinned_step()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pinned_step()
    pin_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    barrier()
    e2e_pinned = {"value": reps.rate(n, pin_s), "unit": "cells/s", "ms_per_step": 1000 * pin_s,
                  "path": "msc_b200.neighbors.neighbors_host: pinned torch CPU tensors"}
    del hstate, Xh

    # the plain FP32 GPU form and the three-term BF16 form of the same exact graph, each over
    # FORM_STEPS graphs (the FP32 form scans every key; the 16-bit forms are pruned)
    fp32 = bf16x3 = None
    if not args.skip_fp32:
        forms = {}
        for prec in ("fp32", "bf16x3"):
            if prec == args.precision:
                continue
            fms = max_over_ranks(events_ms(torch, lambda: step(prec), FORM_STEPS, warm=1))
            forms[prec] = {"value": reps.rate(n, fms / 1000.0), "unit": "cells/s",
                           "ms_per_step": fms, "steps": FORM_STEPS}
        # the FP32 form under the same locality order, near pass and pruning plan as the 16-bit
        # forms: the gain of the 16-bit candidates alone
        os.environ["MSC_B200_PRUNE_FP32"] = "1"
        try:
            fms = max_over_ranks(events_ms(torch, lambda: step("fp32"), FORM_STEPS, warm=1))
        finally:
            del os.environ["MSC_B200_PRUNE_FP32"]
        forms["fp32_pruned"] = {"value": reps.rate(n, fms / 1000.0), "unit": "cells/s",
                                "ms_per_step": fms, "steps": FORM_STEPS,
                                "speedup_of_headline": fms / ms,
                                "pruning": "the same plan as the headline form"}
        fp32, bf16x3 = forms.get("fp32"), forms.get("bf16x3")
        if fp32:
            fp32["speedup_of_headline"] = fp32["ms_per_step"] / ms
            fp32["pruning"] = "none: every key tile of every query tile is scanned"
        if bf16x3:
            bf16x3["speedup_over_fp32_form"] = (fp32["ms_per_step"] / bf16x3["ms_per_step"]) \
                if fp32 else None

    err = None
    if rank == 0 and not args.skip_cpu:
        res = step()
        torch.cuda.synchronize()
        err = error_vs_fp64(X, res["knn_idx"].cpu().numpy(), res["knn_dist"].cpu().numpy(), k,
                            metric)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu = cpu_baseline(X, k, metric, budget_s=args.ref_budget)

    # the other configurations of the workload list, each at its stated size with its own clock
    # record (one GPU only: under torchrun every rank is a replica of the headline graph)
    configs = None
    if world == 1 and args.workload == "scale" and not args.skip_configs:
        del Xd, ws, out
        torch.cuda.empty_cache()
        configs = {"plain_10k": config_leg("plain", uuid),
                   "precision_200k": config_leg("precision", uuid),
                   "batch_64": batch_leg(uuid, args.batch_samples),
                   "bbknn_200k": bbknn_measure(200_000, 8, 3, "fp16", 3, 3, True, 0.0),
                   "serve": serve_leg(uuid, args)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": args.precision, "data": "synthetic",
                "config": {"workload": desc, "n_neighbors": k, "metric": metric,
                           "method": method, "precision": args.precision,
                           "kprime": int(kprime) or "auto",
                           "l2": "inputs larger than L2 (embedding 260 MB + packed operands)",
                           "parallelism": f"replicas x{world}"},
                "e2e": e2e, "e2e_pinned": e2e_pinned, "gpu_launches": int(launches),
                "roofline": roofline, "cpu_baseline": cpu, "fp32_form": fp32,
                "bf16x3_form": bf16x3,
                "fp32_pruned_form": forms.get("fp32_pruned") if not args.skip_fp32 else None,
                "error_vs_fp64": err, "configs": configs,
                "stats": {"certified": int(stats[_lib.STAT_CERTIFIED]),
                          "refined": int(stats[_lib.STAT_REFINED]),
                          "rescanned": int(stats[_lib.STAT_RESCANNED]),
                          "fp64_boundary_recomputes": int(stats[_lib.STAT_FP64_TIES]),
                          "conn_nnz": int(stats[_lib.STAT_CONN_NNZ])},
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    reps.close()


def run_batch(args):
    """Batching workload: 256 samples (~4M cells, 30 PCs, k=15) in one persistent launch under a
    captured CUDA graph with autotuned tiles, against a per-sample launch loop."""
    import torch
    from msc_b200 import batch, synth, _lib
    torch.cuda.set_device(0)
    X, offsets, p = synth.batch_samples(args.samples, seed=3, d=30)
    n, d = X.shape
    k = p["n_neighbors"]
    Xd = torch.from_numpy(X).cuda()

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    loop_out = batch.per_sample_loop(Xd, offsets, k)
    loop_ms = timed(lambda: batch.per_sample_loop(Xd, offsets, k, out=loop_out), args.steps)
    bk = batch.BatchedKnn(offsets, d, k)
    batched_ms = timed(lambda: bk.run(Xd), args.steps)
    tune = batch.autotune(Xd, offsets, k, reps=1, use_cache=False)
    bt = batch.BatchedKnn(offsets, d, k, tile_config=tune["tile_config"])
    bt.capture(Xd)
    graph_ms = timed(bt.replay, args.steps)
    stats = bt.check()
    same = bool(torch.equal(bt.idx, loop_out[0]) and torch.equal(bt.dist, loop_out[1]))
    sizes = np.diff(offsets)
    line = {"metric": "batching: kNN cells/s, one persistent launch + CUDA graph vs per-sample "
                      "launch loop", "value": n / (graph_ms / 1000), "unit": "cells/s",
            "n_gpus": 1, "steps": args.steps, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": f"{len(sizes)} samples, {n:,} cells (min {sizes.min()}, "
                                   f"max {sizes.max()}), 30 PCs, k=15, euclidean",
                       "precision": batch.DEFAULT_PRECISION,
                       "tile": batch.decode_tile_code(tune["tile_config"])},
            "graph_ms": graph_ms, "batched_ms": batched_ms, "per_sample_loop_ms": loop_ms,
            "speedup_vs_loop": loop_ms / graph_ms, "identical_to_loop": same,
            "autotune_table": [(batch.decode_tile_code(c), round(ms, 3))
                               for c, ms in tune.get("table", [])],
            "certified": int(stats[_lib.STAT_CERTIFIED]),
            "rescanned": int(stats[_lib.STAT_RESCANNED]),
            "algorithmic_tflops": 2.0 * d * float((sizes.astype(np.float64) ** 2).sum())
                                  / (graph_ms / 1000) / 1e12}
    print(json.dumps(line), flush=True)


def spatial_slide(n: int, seed: int = 7):
    """A Xenium-scale synthetic slide: n spots in µm on a 10 mm × 10 mm field, 70% in 12 tissue
    regions (Gaussian, σ 300-900 µm), 30% uniform background; float64 as obsm['spatial']."""
    rng = np.random.default_rng(seed)
    n_in = int(0.7 * n)
    centres = rng.uniform(1500, 8500, (12, 2))
    sig = rng.uniform(300, 900, 12)
    lab = rng.integers(0, 12, n_in)
    tissue = centres[lab] + rng.standard_normal((n_in, 2)) * sig[lab, None]
    back = rng.uniform(0, 10_000, (n - n_in, 2))
    xy = np.vstack([tissue, back])
    return xy[rng.permutation(n)]


def run_spatial(args):
    """Spatial workload: kNN (n_neighs=6 → k=7) and radius (30 µm) graphs of a 1M-spot slide on
    the uniform-grid search; device-resident rates, the end-to-end gr builder, sklearn's KD-tree
    on the host cores as the CPU baseline."""
    import torch
    from msc_b200 import spatial as msp, gr, _lib, AnnDataLite
    torch.cuda.set_device(0)
    n = args.n or 1_000_000
    xy = spatial_slide(n)
    X = torch.from_numpy(xy.astype(np.float32)).cuda()
    k, radius = 7, 30.0
    ws = msp.Workspace(X.device)

    def timed(fn, reps):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}

    def knn():
        out["knn"] = msp.knn_grid_device(X, k, ws)

    lib = _lib.load()
    l0 = lib.msc_launch_count()
    knn_ms = timed(knn, args.steps)
    launches = (lib.msc_launch_count() - l0) // (args.steps + max(args.warmup, 1))
    st = out["knn"][2].cpu().numpy()
    _lib.check_spatial_stats(st)
    rad_ms = timed(lambda: out.__setitem__("rad", msp.radius_grid_device(X, radius, 0.0, ws)),
                   args.steps)
    nnz = int(out["rad"][0][n].item())
    a = AnnDataLite(obsm={"spatial": xy}, n_obs=n)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        res = gr.spatial_neighbors_knn(a, n_neighs=k - 1, copy=True)
    e2e_s = (time.perf_counter() - t0) / args.steps
    cpu = None
    if not args.skip_cpu:
        from sklearn.neighbors import NearestNeighbors
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        NearestNeighbors(n_neighbors=k - 1, n_jobs=-1).fit(xy).kneighbors()
        cpu_s = time.perf_counter() - t0
        cpu = {"value": n / cpu_s, "unit": "spots/s", "cores": cores, "kind": "sklearn KD-tree",
               "sample": f"all {n:,} spots, n_neighbors={k - 1}, fit + kneighbors"}
    evals = int(st[_lib.SP_STAT_EVALS])
    alg_bytes = n * 16 + n * k * 8
    line = {"metric": "spatial kNN graph: spots/s (grid search, k=7, device-resident)",
            "value": n / (knn_ms / 1000), "unit": "spots/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": knn_ms, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{n:,} spots, 10 mm slide (µm), 12 tissue regions + 30% "
                                   f"background", "k": k, "radius_um": radius},
            "radius_ms": rad_ms, "radius_nnz": nnz,
            "e2e": {"value": n / e2e_s, "unit": "spots/s", "path": "gr.spatial_neighbors_knn",
                    "ms": e2e_s * 1000},
            "cells": int(st[_lib.SP_STAT_CELLS]), "chunks": int(st[_lib.SP_STAT_CHUNKS]),
            "evals_per_query": evals / n, "expanded_rows": int(st[_lib.SP_STAT_EXPANDED]),
            "achieved_gbs_algorithmic": alg_bytes / (knn_ms / 1000) / 1e9,
            "cpu_baseline": cpu, "gpu_launches": int(launches)}
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Serving workload: Poisson arrivals of graph requests (1k-500k cells, 30/50/100 PCs,
    k in {10,15,30}, euclidean/cosine); p50/p99 latency and cells/s at swept arrival rates
    against the batched-offline throughput of the same requests."""
    import torch
    from msc_b200 import serve, synth
    torch.cuda.set_device(0)
    spec = synth.serving_requests(1.0, args.requests, seed=5)
    data = [synth.request_embedding(r) for r in spec]
    total_cells = sum(x.shape[0] for x in data)
    budget = int(args.hbm_budget_gb * (1 << 30))

    def fresh():
        return [serve.Request(X=x, n_neighbors=r["k"], metric=r["metric"])
                for x, r in zip(data, spec)]

    serve.run_offline(fresh()[: min(8, len(data))], budget, args.slots)     # warm-up
    off = serve.run_offline(fresh(), budget, args.slots)
    sweep = []
    mean_cells = total_cells / len(data)
    for frac in args.load_fracs:
        rate = frac * off["cells_per_s"] / mean_cells
        rng = np.random.default_rng(7)
        arr = np.cumsum(rng.exponential(1.0 / rate, len(data))).tolist()
        rep = serve.run_trace(fresh(), arr, budget, args.slots)
        rep.update({"load_frac_of_offline": frac, "rate_req_per_s": rate,
                    "throughput_frac_of_offline": rep["cells_per_s"] / off["cells_per_s"]})
        sweep.append(rep)
    best = max((r for r in sweep if r["failed"] == 0), key=lambda r: r["cells_per_s"],
               default=None)
    line = {"metric": "serving: p50/p99 ms and cells/s vs batched offline throughput",
            "value": best["p99_ms"] if best else None, "unit": "ms (p99 at highest load swept)",
            "higher_is_better": False, "n_gpus": 1, "data": "synthetic",
            "config": {"requests": len(data), "cells_total": total_cells,
                       "slots": args.slots, "hbm_budget_gb": args.hbm_budget_gb,
                       "distribution": "cells LogNormal(ln 20000, 1) clipped 1k-500k; PCs {30,50,100}; "
                                       "k {10,15,30}; metric {euclidean, cosine}"},
            "offline": off, "sweep": sweep}
    print(json.dumps(line), flush=True)


def bbknn_workload(n: int | None, batches: int, seed: int = 41):
    """The scale embedding with uneven batch labels (Dirichlet(2) batch weights, cells drawn at
    random, so every batch spans every cluster, as batches of one tissue do)."""
    X, _, desc = workload("scale", n)
    rng = np.random.default_rng(seed)
    w = rng.dirichlet(np.full(batches, 2.0))
    batch = rng.choice(batches, X.shape[0], p=w)
    return X, batch, f"{desc}, {batches} batches (Dirichlet(2) sizes)"


def bbknn_cpu_baseline(X, batch, kwb, budget_s: float = 15.0):
    """Oracle port on the host: the exact per-batch lists of a seeded sample of query cells
    against every batch, merged by (distance, index); cells/s = query cells / time."""
    from oracle import bbknn as obb
    cores = len(os.sched_getaffinity(0))
    cats, codes = obb.batch_codes(batch)
    members = [np.flatnonzero(codes == b) for b in range(cats.size)]
    rng = np.random.default_rng(4321)
    n = X.shape[0]
    m, rows, t_total = 64, 0, 0.0
    while t_total < budget_s * 0.5 and rows < n:
        q = np.sort(rng.choice(n, m, replace=False))
        t0 = time.perf_counter()
        parts_i, parts_d = [], []
        for mem in members:
            loc, _, dd = obb.knn_cross(X[q], X[mem], min(kwb, mem.size))
            parts_i.append(mem[loc])
            parts_d.append(dd)
        idx, dist = np.concatenate(parts_i, 1), np.concatenate(parts_d, 1)
        np.lexsort((idx, dist), axis=1)
        t_total += time.perf_counter() - t0
        rows += m
        m = int(min(n, m * 2))
    return {"value": rows / t_total, "unit": "cells/s", "cores": cores, "kind": "port",
            "sample": f"{rows} seeded query cells of the {n}-cell embedding against all "
                      f"{len(members)} batches (exact per-batch lists + merge), "
                      f"{t_total:.1f} s on {cores} threads"}


def run_bbknn(args):
    line = bbknn_measure(args.n, args.batches, args.neighbors_within_batch, args.precision,
                         args.steps, args.warmup, args.skip_cpu, args.ref_budget)
    print(json.dumps(line), flush=True)


def bbknn_measure(n_cells, batches, kwb, precision, steps, warmup, skip_cpu, ref_budget):
    """Batch-balanced graph (pp.bbknn): every cell's neighbours_within_batch nearest cells of each
    batch, fuzzy set, distances graph and trimming; cells/s with the embedding resident, the kNN
    stage alone, and end to end through the host call."""
    import torch
    from msc_b200 import bbknn as bbm, neighbors as nbm, _lib
    torch.cuda.set_device(0)
    lib = _lib.load()
    X, batch, desc = bbknn_workload(n_cells, batches)
    n, d = X.shape
    _, codes, counts = bbm.batch_codes(batch)
    Xd = torch.from_numpy(X).cuda()
    cd = torch.from_numpy(codes).cuda()
    ws = nbm.Workspace(Xd.device)

    def graph():
        return bbm.bbknn_device(Xd, cd, counts, kwb, precision=precision, workspace=ws)

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, out

    for _ in range(max(warmup, 3)):
        res = graph()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(0).uuid)
    except Exception:
        uuid = None
    with ClockSampler(uuid) as cs:
        ms, res = timed(graph, steps)
    stats = res["stats"].cpu().numpy()
    _lib.check_stats(stats)
    K = res["K"]
    # the kNN stage alone (candidate launches, re-rank, FP64 scans, merge)
    cptr = np.ascontiguousarray(counts).ctypes.data
    idx = torch.empty((n, K), dtype=torch.int32, device=Xd.device)
    dist = torch.empty((n, K), dtype=torch.float32, device=Xd.device)
    st = torch.cuda.current_stream().cuda_stream
    kbytes = lib.msc_bbknn_workspace_bytes(n, d, cptr, counts.size, kwb,
                                           _lib.PRECISION[precision])
    kws = ws.get(kbytes)
    knn = lambda: _lib.check(lib.msc_bbknn_knn(Xd.data_ptr(), n, d, cd.data_ptr(), cptr,
                                               counts.size, kwb, _lib.PRECISION[precision],
                                               idx.data_ptr(), dist.data_ptr(), 0, kws.data_ptr(),
                                               kws.numel(), st), "msc_bbknn_knn")
    knn()
    knn_ms, _ = timed(knn, steps)
    # end to end through the host call (host embedding in, host CSR matrices out)
    bbm.bbknn(X, batch, kwb, n_pcs=None, precision=precision)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        dm, cm, _ = bbm.bbknn(X, batch, kwb, n_pcs=None, precision=precision)
    e2e_ms = 1000.0 * (time.perf_counter() - t0) / steps
    flop = 2.0 * d * float(n) * float(n)                  # Σ_b 2·d·n·n_b
    pk, pk_kind = peaks()
    peak = pk.get("bf16_tflops_sustained", 1400.0)
    line = {"metric": "bbknn: batch-balanced graph cells/s", "value": n / (ms / 1000),
            "unit": "cells/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": ms, "higher_is_better": True, "data": "synthetic",
            "dtype": precision,
            "config": {"workload": desc, "neighbors_within_batch": kwb, "K": K,
                       "batch_sizes": [int(c) for c in counts], "trim": res["trim"]},
            "e2e": {"value": n / (e2e_ms / 1000), "unit": "cells/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(X.nbytes + codes.nbytes),
                    "d2h_bytes_per_step": int(dm.data.nbytes + dm.indices.nbytes
                                              + dm.indptr.nbytes + cm.data.nbytes
                                              + cm.indices.nbytes + cm.indptr.nbytes)},
            "knn_stage": {"ms": knn_ms, "algorithmic_tflops": flop / (knn_ms / 1000) / 1e12,
                          "frac_of_peak": flop / (knn_ms / 1000) / 1e12 / peak,
                          "peak": peak, "peak_kind": f"{pk_kind} bf16 sustained",
                          "flop": "2·d·n·Σ n_b = 2·d·n² (every cell against every batch)"},
            "stats": {"certified": int(stats[_lib.STAT_CERTIFIED]),
                      "rescanned": int(stats[_lib.STAT_RESCANNED]),
                      "precision": int(stats[_lib.STAT_PRECISION])},
            "clocks": cs.summary()}
    if not skip_cpu:
        line["cpu_baseline"] = bbknn_cpu_baseline(X, batch, kwb, ref_budget)
    return line


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="scale",
                    choices=["scale", "plain", "precision", "batch", "serve", "bbknn",
                             "spatial"])
    ap.add_argument("--precision", default="fp16", choices=["fp16", "bf16x3", "bf16", "fp32"])
    ap.add_argument("--skip-fp32", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-configs", action="store_true",
                    help="headline graph only: no plain / precision / batching / serving legs")
    ap.add_argument("--batch-samples", type=int, default=64,
                    help="samples of the batching leg of the default run")
    ap.add_argument("--serve-requests", type=int, default=1000,
                    help="requests per load point of the serving leg of the default run")
    ap.add_argument("--ref-budget", type=float, default=15.0)
    ap.add_argument("--n", type=int, default=None, help="cells of the scale workload (profiling)")
    ap.add_argument("--samples", type=int, default=256, help="batch workload: samples")
    ap.add_argument("--requests", type=int, default=120, help="serve workload: requests")
    ap.add_argument("--slots", type=int, default=8, help="serve workload: concurrent slots")
    ap.add_argument("--hbm-budget-gb", type=float, default=64.0)
    ap.add_argument("--kprime", type=int, default=0, help="over-fetch k' (0: the library default)")
    ap.add_argument("--load-fracs", type=float, nargs="+", default=[0.3, 0.5, 0.7, 0.9])
    ap.add_argument("--batches", type=int, default=8, help="bbknn workload: batches")
    ap.add_argument("--neighbors-within-batch", type=int, default=3, help="bbknn workload")
    args = ap.parse_args(argv)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "bbknn":
        return run_bbknn(args)
    if args.workload == "spatial":
        return run_spatial(args)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
