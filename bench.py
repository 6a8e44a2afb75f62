#!/usr/bin/env python
"""Benchmark: k-NN graph build throughput (points/s) and query QPS.

Workload: N = 1,000,000 x D = 128 f32 points from a Gaussian mixture of 100
isotropic clusters (centers ~ N(0, 10^2 I), within-cluster std 1), squared
Euclidean, n_neighbors = 30, 8 RP trees, leaf size 30, <= 10 NN-Descent
iterations, delta 0.001; 10,000 queries from the same mixture, k = 10,
epsilon = 0.1.  Synthetic data (numpy seeded), generated on the host.

One step = one full index build (forest, leaf init, NN-Descent iterations,
sorted kNN rows, diversified CSR, search layout) over resident device data.
`value` = points built per second over all ranks; `e2e` = the same through
the C ABI from pinned host memory with the neighbor graph copied back.
Multi-GPU: one independent index per rank (weak scaling, no collective on the
data path); the max over ranks of the device-timed region is reported.

--impl reference: the reference's CPU algorithm (the C++ restatement under
oracle/, all host threads) on the same full workload, one build per step.
The default run also builds that oracle index once (the `cpu_baseline` leg)
and reports its recall beside the GPU's, on the same sample and queries, and
(one GPU) adds `forms`: brute-force exact kNN of the same queries against the
same rows (FP32 and the FP64 checker), the batched form (512 indices, two
warm-up calls, one timed), the serving form (10M x 96, int8 per-vector width 100 server, 2 s per
offered load) and the precision form (1M x 960 cosine, FP32 and BF16 builds,
without the oracle parity sizes) in compact runs of --workload batched /
serving / precision.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "k-NN graph build pts/sec & QPS at fixed recall@k; vs plain FP32 GPU, % roofline"
N_FULL, DIM, N_CLUSTERS, K = 1_000_000, 128, 100, 30
N_TREES, LEAF, N_ITERS, DELTA = 8, 30, 10, 0.001
N_QUERIES, QK, EPS = 10_000, 10, 0.1
# FP32 SIMT peak for context: 148 SMs x 128 FP32 lanes x 2 flops (FMA) x 1.965 GHz.
FP32_SIMT_NOMINAL_TFLOPS = 74.4
WORKLOAD = ("nndescent-build 1M x 128 f32 GMM(100 clusters, center std 10, unit std), sqeuclidean, "
            "k=30, 8 RP trees, leaf 30, <=10 iters, delta 0.001; 10k queries k=10 eps=0.1")


def gen_mixture(n, d, seed, n_clusters=N_CLUSTERS):
    rng = np.random.default_rng(seed)
    centers = rng.normal(0.0, 10.0, (n_clusters, d)).astype(np.float32)
    X = centers[rng.integers(0, n_clusters, n)]
    X += rng.standard_normal((n, d), dtype=np.float32)
    return X


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=N_FULL, help="points per rank")
    ap.add_argument("--no-recall", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="per-iteration build statistics")
    ap.add_argument("--workload", default="build", choices=["build", "batched", "serving", "precision"],
                    help="build: the 1M-point build (default); batched: many independent indices in one call; "
                         "serving: continuous-batching queries against a 10M x 96 index; precision: FP32 and "
                         "BF16 join forms at 1M x 960 cosine with distance error vs FP64")
    ap.add_argument("--serve-n", type=int, default=10_000_000, help="serving workload: index size")
    ap.add_argument("--serve-seconds", type=float, default=4.0, help="serving workload: seconds per offered load")
    ap.add_argument("--no-forms", action="store_true",
                    help="build workload: skip the compact batched and serving measurements added to the line")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "bf16"],
                    help="local-join tiles of the timed builds (the precision form is also reported beside fp32)")
    ap.add_argument("--join-tuning", default="table", choices=["table", "fixed", "retune"],
                    help="tile shape of the FP32 join: tuned table (default), fixed default shape, fresh trials")
    ap.add_argument("--items", type=int, default=512, help="batched workload: number of indices")
    ap.add_argument("--check-items", type=int, default=16,
                    help="batched workload: indices whose recall is compared with one-at-a-time builds")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks sampled with nvidia-smi during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                mx.append(float(parts[2].split()[0]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def join_traffic_per_row():
    """DRAM bytes per gathered candidate row of the join kernel, from the
    committed ncu summary (profiles/local_join_fp32.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "local_join_fp32.json")) as f:
            return float(json.load(f)["dram_bytes_per_gathered_row"])
    except (OSError, KeyError, ValueError):
        return None


def cpu_build(X, n_threads=0):
    import oracle

    t = time.perf_counter()
    ix = oracle.OracleIndex(X, n_neighbors=K, n_trees=N_TREES, leaf_size=LEAF, n_iters=N_ITERS, delta=DELTA,
                            distance_kind=oracle.SQEUCLIDEAN, correction=oracle.CORR_NONE, n_threads=n_threads)
    dt = time.perf_counter() - t
    return ix, dt


def bench_config(n, world):
    """The `config` object of both arms (identical for the same workload)."""
    return {"workload": WORKLOAD, "points_per_rank": n, "parallelism": f"replicas{world}",
            "l2": "inputs (512 MB/rank) exceed L2 (126 MB); no flush"}


def run_reference(args, rank):
    """The reference's CPU build (restated in oracle/) on the full workload:
    every step builds the whole N-point index with all host threads."""
    if rank != 0:
        return
    import oracle

    n = args.n
    X = gen_mixture(n, DIM, seed=0)
    cores = oracle.max_threads()
    for _ in range(args.warmup):
        cpu_build(X)
    times = [cpu_build(X)[1] for _ in range(args.steps)]
    total = sum(times)
    value = n * args.steps / total
    sample = f"the full workload: N={n} rows of the 100-cluster mixture per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(n, args.gpus),
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def exact_knn_torch(X_dev, Q_dev, k, chunk=512):
    """FP64 exact kNN on the GPU (recall checker only)."""
    import torch

    Xd = X_dev.double()
    xx = (Xd * Xd).sum(1)
    out = []
    for s in range(0, Q_dev.shape[0], chunk):
        q = Q_dev[s:s + chunk].double()
        d = (q * q).sum(1)[:, None] + xx[None, :] - 2.0 * (q @ Xd.T)
        out.append(torch.topk(d, k, dim=1, largest=False).indices.int().cpu())
        del d
    return torch.cat(out).numpy()


def recall(found, truth):
    k = truth.shape[1]
    hits = sum(len(set(f[f >= 0].tolist()) & set(t.tolist())) for f, t in zip(found, truth))
    return hits / (truth.shape[0] * k)


def batched_specs(n_items, seed=0):
    """Config of the batched form: N log-uniform in [2000, 200000], D from
    {32, 64, 128, 256}, 10-100 mixture clusters, metric 40% sqeuclidean / 40%
    cosine / 20% inner product, k = 15; index i uses data seed 1000 + i."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_items):
        n = int(np.exp(rng.uniform(np.log(2000), np.log(200000))))
        d = int(rng.choice([32, 64, 128, 256]))
        c = int(rng.integers(10, 101))
        u = rng.random()
        metric = "sqeuclidean" if u < 0.4 else ("cosine" if u < 0.8 else "inner_product")
        specs.append({"n": n, "d": d, "clusters": c, "metric": metric, "seed": 1000 + i})
    return specs


def run_batched(args, world, rank, local_rank, emit=True):
    """The batched form: this rank's longest-first share of the indices built
    in one rinnd_build_many call from device-resident data; timed with CUDA
    events, max over ranks; beside it the same share built one index at a time.
    Returns the line (rank 0)."""
    import datetime

    import torch
    import torch.distributed as dist

    from rinnd_b200 import _lib as L
    from rinnd_b200 import shard

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    specs = batched_specs(args.items)
    costs = [shard.build_cost(sp["n"], sp["d"], 15) for sp in specs]
    mine = shard.my_share(costs, rank, world)
    metric_of = {"sqeuclidean": (L.DIST_SQEUCLIDEAN, L.CORR_NONE, 0), "cosine": (L.DIST_ALT_COSINE, L.CORR_ALT_COSINE, 1),
                 "inner_product": (L.DIST_ALT_INNER_PRODUCT, L.CORR_ALT_IP, 1)}
    datas, params = [], []
    for i in mine:
        sp = specs[i]
        g = torch.Generator(device=dev).manual_seed(sp["seed"])
        centers = torch.randn(sp["clusters"], sp["d"], generator=g, device=dev) * 10.0
        a = torch.randint(0, sp["clusters"], (sp["n"],), generator=g, device=dev)
        datas.append((centers[a] + torch.randn(sp["n"], sp["d"], generator=g, device=dev)).contiguous())
        p = L.BuildParams()
        L.check(L.lib.rinnd_params_default(ctypes.byref(p)))
        kind, corr, ang = metric_of[sp["metric"]]
        p.n_neighbors, p.distance_kind, p.correction, p.angular = 15, kind, corr, ang
        p.random_seed, p.device = 7 + i, local_rank
        p.n_trees = int(min(max(np.floor(2.0 * np.log10(sp["n"]) + 0.5), 3), 12))
        p.precision = 1 if args.precision == "bf16" else 0
        params.append(p)
    m = len(mine)
    items = (L.BatchItem * max(m, 1))()
    for j in range(m):
        items[j].data = datas[j].data_ptr()
        items[j].n, items[j].d = datas[j].shape
        items[j].data_on_device, items[j].ld = 1, datas[j].shape[1]
        items[j].params = ctypes.addressof(params[j])
    handles = (ctypes.c_void_p * max(m, 1))()

    def options(grouped):
        o = L.BatchOptions()
        L.check(L.lib.rinnd_batch_options_default(ctypes.byref(o)))
        o.grouped = grouped
        return o

    grouped_opts, stream_opts = options(1), options(0)

    def build_batch(opts=grouped_opts):
        L.check(L.lib.rinnd_build_many_ex(items, m, ctypes.byref(opts), handles, None))
        for j in range(m):
            L.check(L.lib.rinnd_free(handles[j]))

    def one_at_a_time():
        for j in range(m):
            h = ctypes.c_void_p()
            L.check(L.lib.rinnd_build_device(ctypes.c_void_p(datas[j].data_ptr()), datas[j].shape[0],
                                             datas[j].shape[1], datas[j].shape[1], ctypes.byref(params[j]),
                                             ctypes.byref(h)))
            L.check(L.lib.rinnd_free(h))

    def timed(fn):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    for _ in range(max(args.warmup, 1)):
        build_batch()
    # builds synchronize their own streams; the host clock brackets the call
    t_batch = max(timed(build_batch) for _ in range(max(args.steps, 1)))
    t_streams = timed(lambda: build_batch(stream_opts))
    t_one = timed(one_at_a_time)

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    t_batch, t_streams, t_one = max_over_ranks(t_batch), max_over_ranks(t_streams), max_over_ranks(t_one)
    n_items, n_points = shard.gather_counts(m, int(sum(d.shape[0] for d in datas)))
    # per-index recall@15 vs FP64 exact (batched vs one at a time) on the largest checked indices of rank 0
    quality = {}
    groups = 0
    if rank == 0 and args.check_items > 0 and m > 0:
        L.check(L.lib.rinnd_build_many_ex(items, m, ctypes.byref(grouped_opts), handles, None))
        gi = L.BuildInfo()
        sizes = []
        for j in range(m):
            L.check(L.lib.rinnd_build_info_get(handles[j], ctypes.byref(gi)))
            sizes.append(gi.group_items)
        groups = int(sum(1.0 / g for g in sizes))
        diffs, rb_, ro_ = [], [], []
        for j in range(min(args.check_items, m)):
            X = datas[j]
            rows = torch.arange(min(200, X.shape[0]), device=dev)
            q = X[rows].double()
            Xd = X.double()
            sp = specs[mine[j]]
            if sp["metric"] == "sqeuclidean":
                dd = (q * q).sum(1)[:, None] + (Xd * Xd).sum(1)[None, :] - 2.0 * q @ Xd.T
            elif sp["metric"] == "cosine":
                dd = -(q / q.norm(dim=1, keepdim=True)) @ (Xd / Xd.norm(dim=1, keepdim=True)).T
            else:
                dd = -(q @ Xd.T)
            dd[torch.arange(len(rows), device=dev), rows] = float("inf")
            truth = torch.topk(dd, 15, dim=1, largest=False).indices.int().cpu().numpy()
            kb = np.empty((X.shape[0], 15), np.int32)
            kd = np.empty((X.shape[0], 15), np.float32)
            L.check(L.lib.rinnd_neighbor_graph(handles[j], L.ptr(kb), L.ptr(kd)))
            h = ctypes.c_void_p()
            L.check(L.lib.rinnd_build_device(ctypes.c_void_p(X.data_ptr()), X.shape[0], X.shape[1], X.shape[1],
                                             ctypes.byref(params[j]), ctypes.byref(h)))
            ko = np.empty((X.shape[0], 15), np.int32)
            L.check(L.lib.rinnd_neighbor_graph(h, L.ptr(ko), L.ptr(kd)))
            L.check(L.lib.rinnd_free(h))
            rb_.append(recall(kb[: len(rows)], truth))
            ro_.append(recall(ko[: len(rows)], truth))
            diffs.append(rb_[-1] - ro_[-1])
        for j in range(m):
            L.check(L.lib.rinnd_free(handles[j]))
        quality = {"checked_indices": len(diffs), "recall@15_batched_mean": float(np.mean(rb_)),
                   "recall@15_one_at_a_time_mean": float(np.mean(ro_)), "recall@15_min_diff": float(np.min(diffs))}
    if rank == 0:
        line = {
            "metric": "batched build points/s (512 independent indices, k=15)", "value": n_points / t_batch,
            "unit": "points/s", "n_gpus": world, "steps": max(args.steps, 1), "warmup": max(args.warmup, 1),
            "ms_per_step": 1000.0 * t_batch, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched: {n_items} indices, N log-uniform [2000, 200000], D in {{32,64,128,256}}, "
                                   "10-100 clusters, metric 40% sqeuclidean / 40% cosine / 20% inner product, k=15, "
                                   f"precision {args.precision}; grouped NN-Descent per (D, metric); "
                                   "longest-first over ranks",
                       "points": n_points, "parallelism": f"shards{world}", "timing": "host clock around the call, "
                       "synchronized, max over ranks (each build synchronizes its streams)"},
            "one_at_a_time": {"value": n_points / t_one, "ms": 1000.0 * t_one},
            "stream_per_index": {"value": n_points / t_streams, "ms": 1000.0 * t_streams},
            "speedup_vs_one_at_a_time": t_one / t_batch, "speedup_vs_stream_per_index": t_streams / t_batch,
            "groups": groups, "quality": quality,
        }
        if emit:
            print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return line if rank == 0 else None


PREC_D, PREC_K, PREC_SAMPLE = 960, 15, 4000
PREC_PARITY_SIZES = (20_000, 100_000)


def run_precision(args, world, rank, local_rank, emit=True, compact=False):
    """The precision workload: N x 960 rows with entries |N(0,1)|^1.5,
    L2-normalised, cosine, k=15, built with FP32 join tiles and with the BF16
    precision form (which falls back to FP32 tiles where its tensor-core join
    does not apply; `join_form` says which kernel ran).  Reports each form's
    build points/s, recall@15 against FP64 exact kNN on a seeded sample of rows,
    and the error of the reported neighbor distances against the same pairs'
    cosine distances recomputed in FP64.  Replicas on N > 1 ranks.  compact:
    without the oracle parity builds (for the default bench line).  Returns
    the line (rank 0)."""
    import datetime

    import torch
    import torch.distributed as dist

    from rinnd_b200 import _lib as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    n = args.n
    g = torch.Generator(device=dev).manual_seed(0)
    X = torch.randn(n, PREC_D, generator=g, device=dev).abs_().pow_(1.5)
    X /= X.norm(dim=1, keepdim=True)
    X = X.contiguous()
    forms_names = {L.JOIN_CHUNKED_FP32: "chunked FP32", L.JOIN_PIPELINED_FP32: "pipelined FP32",
                   L.JOIN_TENSOR_BF16: "tensor-core BF16 filter + FP32 recheck"}

    def build(prec):
        p = L.BuildParams()
        L.check(L.lib.rinnd_params_default(ctypes.byref(p)))
        p.n_neighbors, p.distance_kind, p.correction, p.angular = PREC_K, L.DIST_ALT_COSINE, L.CORR_ALT_COSINE, 1
        p.n_trees = int(min(max(np.floor(2.0 * np.log10(n) + 0.5), 3), 12))  # lib.rs:1200-1204
        p.random_seed, p.device, p.precision = 42, local_rank, prec
        h = ctypes.c_void_p()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.check(L.lib.rinnd_build_device(ctypes.c_void_p(X.data_ptr()), n, PREC_D, PREC_D, ctypes.byref(p),
                                         ctypes.byref(h)))
        torch.cuda.synchronize()
        return h, time.perf_counter() - t0

    rows = np.sort(np.random.default_rng(7).choice(n, min(PREC_SAMPLE, n), replace=False))
    truth = None
    if rank == 0 and not args.no_recall:
        Xd = X.double()
        parts = []
        for s in range(0, len(rows), 250):
            r = torch.from_numpy(rows[s:s + 250]).to(dev).long()
            dd = -(Xd[r] @ Xd.T)  # rows are unit vectors: order of 1 - cos
            dd[torch.arange(len(r), device=dev), r] = float("inf")
            parts.append(torch.topk(dd, PREC_K, dim=1, largest=False).indices.int().cpu().numpy())
        truth = np.concatenate(parts)
        del Xd

    forms = {}
    for name, prec in (("fp32", L.PRECISION_FP32), ("bf16", L.PRECISION_BF16)):
        for _ in range(max(args.warmup, 1) if name == "fp32" else 1):
            h, _t = build(prec)
            L.check(L.lib.rinnd_free(h))
        times = []
        for _ in range(max(min(args.steps, 2), 1)):
            h, t = build(prec)
            times.append(t)
            if len(times) < max(min(args.steps, 2), 1):
                L.check(L.lib.rinnd_free(h))
        t = max(times)
        if world > 1:
            tt = torch.tensor([t], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        inf = L.BuildInfo()
        L.check(L.lib.rinnd_build_info_get(h, ctypes.byref(inf)))
        entry = {"value": n * world / t, "ms_per_build": 1000.0 * t, "iterations": int(inf.iterations),
                 "join_form": forms_names.get(int(inf.join_form), str(int(inf.join_form))),
                 "ms_join_kernel": float(inf.ms_join_kernel)}
        if truth is not None:
            ki = np.empty((n, PREC_K), np.int32)
            kd = np.empty((n, PREC_K), np.float32)
            L.check(L.lib.rinnd_neighbor_graph(h, L.ptr(ki), L.ptr(kd)))
            entry["recall@15"] = recall(ki[rows], truth)
            # reported distance vs the pair's cosine distance in FP64
            ids = torch.from_numpy(ki[rows]).to(dev).long()
            ok = ids >= 0
            q = X[torch.from_numpy(rows).to(dev).long()].double()
            nb = X[ids.clamp(min=0)].double()
            exact = 1.0 - (nb * q[:, None, :]).sum(-1) / (nb.norm(dim=-1) * q.norm(dim=-1)[:, None])
            got = torch.from_numpy(kd[rows]).to(dev).double()
            err = (got - exact).abs()[ok]
            rel = err / exact.abs()[ok].clamp(min=1e-30)
            entry["distance_error_vs_fp64"] = {
                "pairs": int(err.numel()), "max_abs": float(err.max()), "p99_abs": float(torch.quantile(err, 0.99)),
                "max_rel": float(rel.max()), "p99_rel": float(torch.quantile(rel, 0.99))}
        L.check(L.lib.rinnd_free(h))
        forms[name] = entry
    # Recall on this distribution is low for any NN-Descent build (i.i.d. rows in
    # 960 dimensions have little neighborhood structure, and less the more rows
    # there are); the restatement of the reference's CPU build on the first
    # n_s rows, for each n_s in PREC_PARITY_SIZES, is the yardstick: both builds
    # see the same rows and are scored on the same seeded sample of them.
    parity = []
    if rank == 0 and not args.no_recall and not compact:
        import oracle

        for n_s in [m for m in PREC_PARITY_SIZES if m <= n]:
            Xs_d = X[:n_s].contiguous()
            Xs = Xs_d.cpu().numpy()
            rows_s = np.sort(np.random.default_rng(11).choice(n_s, min(PREC_SAMPLE // 2, n_s), replace=False))
            Xsd = Xs_d.double()
            parts = []
            for s0 in range(0, len(rows_s), 250):
                r = torch.from_numpy(rows_s[s0:s0 + 250]).to(dev).long()
                dd = -(Xsd[r] @ Xsd.T)
                dd[torch.arange(len(r), device=dev), r] = float("inf")
                parts.append(torch.topk(dd, PREC_K, dim=1, largest=False).indices.int().cpu().numpy())
            truth_s = np.concatenate(parts)
            del Xsd
            n_trees_s = int(min(max(np.floor(2.0 * np.log10(n_s) + 0.5), 3), 12))
            p = L.BuildParams()
            L.check(L.lib.rinnd_params_default(ctypes.byref(p)))
            p.n_neighbors, p.distance_kind, p.correction, p.angular = PREC_K, L.DIST_ALT_COSINE, L.CORR_ALT_COSINE, 1
            p.n_trees, p.random_seed, p.device = n_trees_s, 42, local_rank
            h = ctypes.c_void_p()
            L.check(L.lib.rinnd_build_device(ctypes.c_void_p(Xs_d.data_ptr()), n_s, PREC_D, PREC_D,
                                             ctypes.byref(p), ctypes.byref(h)))
            ks = np.empty((n_s, PREC_K), np.int32)
            kds = np.empty((n_s, PREC_K), np.float32)
            L.check(L.lib.rinnd_neighbor_graph(h, L.ptr(ks), L.ptr(kds)))
            inf_s = L.BuildInfo()
            L.check(L.lib.rinnd_build_info_get(h, ctypes.byref(inf_s)))
            L.check(L.lib.rinnd_free(h))
            t0 = time.perf_counter()
            ox = oracle.OracleIndex(Xs, n_neighbors=PREC_K, n_trees=n_trees_s, angular=True,
                                    distance_kind=oracle.ALT_COSINE, correction=oracle.CORR_ALT_COSINE)
            t_oracle = time.perf_counter() - t0
            ko = ox.neighbor_graph[0]
            parity.append({"n": n_s, "gpu_recall@15": recall(ks[rows_s], truth_s),
                           "oracle_recall@15": recall(ko[rows_s], truth_s),
                           "gpu_iterations": int(inf_s.iterations), "oracle_iterations": int(ox.iterations),
                           "recall_sample": f"{len(rows_s)} seeded rows vs FP64 exact",
                           "oracle_build_s": t_oracle, "checker": "oracle/ C++ restatement of the reference's CPU build"})
            del ox
    if rank == 0:
        line = {
            "metric": "precision form: build points/s, recall@15 and distance error vs FP64 (1M x 960 cosine, k=15)",
            "value": forms["fp32"]["value"], "unit": "points/s", "n_gpus": world, "steps": max(min(args.steps, 2), 1),
            "warmup": max(args.warmup, 1), "ms_per_step": forms["fp32"]["ms_per_build"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"precision: {n} x {PREC_D}, x = |N(0,1)|^1.5 (torch generator seed 0) "
                                   "L2-normalised rows, cosine (alternative-cosine proxy + correction), k=15, "
                                   "default trees/leaf/candidates/iterations",
                       "points_per_rank": n, "parallelism": f"replicas{world}",
                       "recall_sample": f"{len(rows)} seeded rows vs FP64 exact",
                       "timing": "host clock around the synchronized build call, max over ranks"},
            "forms": forms,
            "bf16_speedup_vs_fp32": forms["fp32"]["ms_per_build"] / forms["bf16"]["ms_per_build"],
            "parity_by_size": parity,
        }
        if emit:
            print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return line if rank == 0 else None


def run_serving(args, world, rank, local_rank, emit=True, compact=False):
    """The serving form on one GPU (replicas per rank otherwise): a 10M x 96
    index of L2-normalised Gaussian-mixture rows (1000 clusters), cosine, k=30,
    built with the BF16 join (FP32 recheck); int8 per-dimension search codes
    (sq8d) with an exact FP32 rerank behind the continuous-batching server.
    Request sizes are log-uniform in [1, 4096], k in {10, 100}, epsilon 0.1,
    arrivals Poisson at 0.5 / 0.8 / 0.95 of the measured saturated QPS.  Beside
    it, the plain FP32 search (no codes, no server) at several epsilons and
    widths, to compare throughput at equal recall@10.  compact: the per-vector
    int8 server alone (the one the value is taken from when it reaches recall
    0.95), for the summary inside the default bench line.  Returns the line."""
    import torch

    import rinnd_b200
    from rinnd_b200 import _lib as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n, d = args.serve_n, 96
    g = torch.Generator(device=dev).manual_seed(5 + rank)
    centers = torch.randn(1000, d, generator=g, device=dev) * 10.0

    def sample(m):
        out = torch.empty(m, d, device=dev)
        for s0 in range(0, m, 1 << 21):
            s1 = min(m, s0 + (1 << 21))
            a = torch.randint(0, 1000, (s1 - s0,), generator=g, device=dev)
            x = centers[a] + torch.randn(s1 - s0, d, generator=g, device=dev)
            out[s0:s1] = x / x.norm(dim=1, keepdim=True)
        return out

    X = sample(n)
    Qd = sample(60000)
    Q = Qd.cpu().numpy()
    p = L.BuildParams()
    L.check(L.lib.rinnd_params_default(ctypes.byref(p)))
    p.n_neighbors, p.distance_kind, p.correction, p.angular, p.normalize = 30, L.DIST_DIRECT_COSINE, L.CORR_NONE, 1, 1
    p.n_trees, p.precision, p.device, p.random_seed = 12, 1, local_rank, 42
    h = ctypes.c_void_p()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L.check(L.lib.rinnd_build_device(ctypes.c_void_p(X.data_ptr()), n, d, d, ctypes.byref(p), ctypes.byref(h)))
    t_build = time.perf_counter() - t0
    # exact cosine top-10 of 1000 sampled queries (FP64, the recall checker)
    ns = 1000
    qs = Qd[:ns].double()
    best_v = torch.full((ns, 10), -2.0, dtype=torch.float64, device=dev)
    best_i = torch.zeros((ns, 10), dtype=torch.int64, device=dev)
    for s0 in range(0, n, 1 << 20):
        sims = qs @ X[s0:s0 + (1 << 20)].double().T
        v, i = torch.topk(sims, 10, dim=1)
        cv = torch.cat([best_v, v], 1)
        ci = torch.cat([best_i, i + s0], 1)
        best_v, o = torch.topk(cv, 10, dim=1)
        best_i = torch.gather(ci, 1, o)
    truth = best_i.int().cpu().numpy()
    rng = np.random.default_rng(11)

    def make_requests(m):
        out = []
        for _ in range(m):
            sz = int(np.exp(rng.uniform(0, np.log(4096))))
            lo = int(rng.integers(0, len(Q) - sz))
            out.append((lo, sz, int(rng.choice([10, 100]))))
        return out

    def serve(ix, reqs, rate_qps=None):
        """Submits the requests (all at once, or Poisson at rate_qps queries/s) and collects
        them; returns (wall seconds, server stats)."""
        srv = rinnd_b200.Server(ix, quantized=True)  # default batch shape: 32768 queries, 8 in flight
        ids = []
        done = []

        def collector():
            i = 0
            while i < len(reqs):
                while i >= len(ids):
                    time.sleep(0.0002)
                srv.result(ids[i], timeout_s=120.0)
                i += 1
            done.append(time.perf_counter())

        th = threading.Thread(target=collector)
        th.start()
        mean_sz = float(np.mean([r[1] for r in reqs]))
        t_start = time.perf_counter()
        t_next = t_start
        for lo, sz, k in reqs:
            if rate_qps:
                t_next += rng.exponential(mean_sz / rate_qps)
                delay = t_next - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
            ids.append(srv.submit(Q[lo:lo + sz], k=k, epsilon=0.1))
        th.join()
        st = srv.stats()
        srv.close()
        return done[0] - t_start, st

    def serving_config(name, encoding, width, rerank):
        """Encodes the index, serves a saturated backlog and three Poisson loads
        through the continuous-batching server, and measures recall@10."""
        t0 = time.perf_counter()
        L.check(L.lib.rinnd_quantize(h, encoding))
        t_enc = time.perf_counter() - t0
        ix = rinnd_b200.RINND.__new__(rinnd_b200.RINND)
        ix._h = None
        ix._attach(h, {"n_points": n, "dim": d, "n_neighbors": 30, "metric": "cosine", "encoding": encoding,
                       "candidate_width": width, "rerank_width": rerank, "retain_fp32": True,
                       "quantize_trees": False, "leaf_budget": 1}, encode=False)
        sat_reqs = make_requests(1000)
        sat_q = sum(r[1] for r in sat_reqs)
        serve(ix, make_requests(20))  # warm-up
        t_sat, st_sat = serve(ix, sat_reqs)
        qps_sat = sat_q / t_sat
        loads = []
        for f in (0.5, 0.8, 0.95):
            rate = f * qps_sat
            mean_sz = 4095.0 / np.log(4096.0)
            m = max(20, int(args.serve_seconds * rate / mean_sz))
            reqs = make_requests(m)
            t, st = serve(ix, reqs, rate_qps=rate)
            loads.append({"offered_fraction": f, "offered_qps": rate, "achieved_qps": sum(r[1] for r in reqs) / t,
                          "requests": m, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
                          "mean_batch_queries": st["mean_batch_queries"], "peak_inflight": st["peak_inflight"]})
        srv = rinnd_b200.Server(ix, quantized=True)
        rid = srv.submit(Q[:ns], k=10, epsilon=0.1)
        qi, _ = srv.result(rid)
        srv.close()
        ix._h = None  # the handle stays with this function's caller
        return {"codes": name, "candidate_width": width, "rerank_width": rerank, "encode_s": t_enc,
                "saturated": {"qps": qps_sat, "p50_ms": st_sat["p50_ms"], "p99_ms": st_sat["p99_ms"]},
                "loads": loads, "recall@10": recall(qi, truth)}

    # the per-dimension codes the configuration names, at the widest width the
    # search takes, and the per-vector int8 codes at width 100
    servers = [] if compact else [serving_config("int8 per-dimension (sq8d)", L.Q8_PER_DIMENSION, 256, 256)]
    servers.append(serving_config("int8 per-vector (int8)", L.Q8_PER_VECTOR_COSINE, 100, 100))
    # the plain FP32 search (rinnd_query_device, 10k queries) at several operating
    # points: result width k (top 10 of it scored) and epsilon
    fp32_points = []
    for kw, eps in ((10, 0.1), (10, 0.3), (30, 0.1), (30, 0.3), (100, 0.1), (100, 0.3)):
        fi = torch.empty((10000, kw), dtype=torch.int32, device=dev)
        fd = torch.empty((10000, kw), dtype=torch.float32, device=dev)
        L.check(L.lib.rinnd_query_device(h, ctypes.c_void_p(Qd.data_ptr()), 2000, d, kw, eps, 0,
                                         ctypes.c_void_p(fi.data_ptr()), ctypes.c_void_p(fd.data_ptr()), None))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.check(L.lib.rinnd_query_device(h, ctypes.c_void_p(Qd.data_ptr()), 10000, d, kw, eps, 0,
                                         ctypes.c_void_p(fi.data_ptr()), ctypes.c_void_p(fd.data_ptr()), None))
        torch.cuda.synchronize()
        t_fp32 = time.perf_counter() - t0
        fp32_points.append({"width": kw, "epsilon": eps, "qps": 10000 / t_fp32,
                            "recall@10": recall(fi[:ns, :10].cpu().numpy(), truth)})
    for srv_cfg in servers:
        reach = [pnt for pnt in fp32_points if pnt["recall@10"] >= srv_cfg["recall@10"] - 0.005]
        srv_cfg["plain_fp32_at_equal_recall"] = max(reach, key=lambda pnt: pnt["qps"]) if reach else None
    at_target = [c for c in servers if c["recall@10"] >= 0.95]
    head = max(at_target, key=lambda c: c["saturated"]["qps"]) if at_target else servers[0]
    line = None
    if rank == 0:
        line = {
            "metric": "serving QPS and p50/p99 latency at recall@10 (10M x 96, int8 + FP32 rerank)",
            "value": head["saturated"]["qps"], "unit": "queries/s", "n_gpus": world, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8 search / f32 rerank", "data": "synthetic",
            "config": {"workload": f"serving: {n} x {d} L2-normalised GMM (1000 clusters), cosine, k=30, BF16 join + "
                                   "FP32 recheck build; int8 codes (per-dimension at width 256 and per-vector at "
                                   "width 100) with an exact FP32 rerank of the candidate list; requests "
                                   "log-uniform 1-4096 queries, k in {10, 100}, eps 0.1, Poisson arrivals; value = "
                                   "the fastest server at recall@10 >= 0.95 (else the per-dimension server)",
                       "parallelism": f"replicas{world}", "value_from": head["codes"]},
            "build_s": t_build, "servers": servers, "recall_sample_queries": ns,
            "plain_fp32_search": fp32_points,
        }
        if emit:
            print(json.dumps(line), flush=True)
    L.check(L.lib.rinnd_free(h))
    return line


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "batched":
        run_batched(args, world, rank, local_rank)
        return
    if args.workload == "serving":
        run_serving(args, world, rank, local_rank)
        return
    if args.workload == "precision":
        run_precision(args, world, rank, local_rank)
        return

    import datetime

    import torch
    import torch.distributed as dist

    from rinnd_b200 import _lib as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    n = args.n
    # data and queries: independent samples of the same mixture
    XQ = gen_mixture(n + N_QUERIES, DIM, seed=1000 * rank)
    X, Q = XQ[:n], XQ[n:]
    X_dev = torch.from_numpy(X).to(dev)
    Q_dev = torch.from_numpy(Q).to(dev)
    stream = torch.cuda.Stream(device=dev)

    p = L.BuildParams()
    L.check(L.lib.rinnd_params_default(ctypes.byref(p)))
    p.n_neighbors, p.n_trees, p.leaf_size, p.n_iters, p.delta = K, N_TREES, LEAF, N_ITERS, DELTA
    p.distance_kind, p.correction, p.random_seed, p.device = L.DIST_SQEUCLIDEAN, L.CORR_NONE, 42, local_rank
    p.verbose = int(args.verbose)
    p.precision = 1 if args.precision == "bf16" else 0
    p.join_tuning = {"table": L.TUNE_TABLE, "fixed": L.TUNE_FIXED, "retune": L.TUNE_RETUNE}[args.join_tuning]

    def build(src_ptr, on_device):
        h = ctypes.c_void_p()
        L.check(L.lib.rinnd_build_on_stream(src_ptr, on_device, n, DIM, DIM, ctypes.byref(p),
                                            ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h)))
        return h

    def info_of(h):
        inf = L.BuildInfo()
        L.check(L.lib.rinnd_build_info_get(h, ctypes.byref(inf)))
        return inf

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    xp = ctypes.c_void_p(X_dev.data_ptr())
    for _ in range(args.warmup):
        L.check(L.lib.rinnd_free(build(xp, 1)))

    # ---- timed region: K builds over resident device data ----
    launches0 = ctypes.c_uint64(0)
    launches1 = ctypes.c_uint64(0)
    infos = []
    gpu_index = local_rank
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        gpu_index = vis.split(",")[local_rank]
    barrier()
    L.lib.rinnd_kernel_launches(ctypes.byref(launches0))
    with ClockSampler(gpu_index) as clocks:
        ev = []
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h = build(xp, 1)
            e1.record(stream)
            infos.append(info_of(h))
            L.check(L.lib.rinnd_free(h))
            ev.append((e0, e1))
        barrier()
    L.lib.rinnd_kernel_launches(ctypes.byref(launches1))
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_s = max_over_ranks(sum(step_ms) / 1000.0)
    value = n * world * args.steps / total_s
    clk = clocks.summary()

    # ---- roofline of the dominant kernel (the local join, k_join_ws) ----
    # Algorithmic bytes of the join over a build: every gathered candidate row
    # (D x 4 B) plus the new/old candidate lists (2 N c x 4 B x 2) per iteration;
    # the heap row traffic belongs to k_apply_updates.  Durations: CUDA events
    # around each join launch on the build stream, summed over the timed builds.
    join_ms = sum(i.ms_join_kernel for i in infos)
    join_launches = sum(i.join_kernel_launches for i in infos)
    iters = sum(i.iterations for i in infos)
    rows = sum(i.join_rows_gathered for i in infos)
    pairs = sum(i.pairs_evaluated for i in infos)
    c = min(K, 60)
    alg_bytes = rows * DIM * 4 + iters * 2 * n * c * 4 * 2
    achieved = alg_bytes / (join_ms / 1000.0) / 1e9 if join_ms > 0 else None
    peak, peak_kind = measured_peaks()
    tpr = join_traffic_per_row()
    roofline = {
        "kernel": "k_join_ws (local join, FP32 SIMT, bulk-copy row gathers)", "bound": "hbm",
        "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
        "peak_source": peak_kind,
        "traffic": (tpr * rows / join_launches) if tpr else None,
        "algorithmic_bytes_per_launch": alg_bytes / max(join_launches, 1),
        "avg_launch_ms": join_ms / max(join_launches, 1),
        "launches_per_build": join_launches / max(len(infos), 1),
        "share_of_build": join_ms / sum(step_ms),
        "fp32_simt": {"achieved_tflops": 2.0 * DIM * pairs / (join_ms / 1000.0) / 1e12 if join_ms > 0 else None,
                      "nominal_peak_tflops": FP32_SIMT_NOMINAL_TFLOPS,
                      "flops": "2 x D per evaluated pair"},
    }

    # ---- the precision form beside the timed form (BF16 tensor-core join filter + FP32 recheck) ----
    other = "bf16" if args.precision == "fp32" else "fp32"
    p_other = L.BuildParams()
    ctypes.memmove(ctypes.byref(p_other), ctypes.byref(p), ctypes.sizeof(p))
    p_other.precision = 1 - p.precision
    p_other.verbose = 0

    def build_other():
        h2 = ctypes.c_void_p()
        L.check(L.lib.rinnd_build_on_stream(xp, 1, n, DIM, DIM, ctypes.byref(p_other),
                                            ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h2)))
        return h2

    L.check(L.lib.rinnd_free(build_other()))
    barrier()
    o_ms, o_infos, ko = [], [], None
    for _ in range(min(args.steps, 2)):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h2 = build_other()
        e1.record(stream)
        o_infos.append(info_of(h2))
        if not o_infos[:-1] and not args.no_recall:
            ko = np.empty((n, K), np.int32)
            kdo = np.empty((n, K), np.float32)
            L.check(L.lib.rinnd_neighbor_graph(h2, L.ptr(ko), L.ptr(kdo)))
        L.check(L.lib.rinnd_free(h2))
        torch.cuda.synchronize()
        o_ms.append(e0.elapsed_time(e1))
    o_s = max_over_ranks(sum(o_ms) / 1000.0)
    other_form = {"precision": other, "value": n * world * len(o_ms) / o_s, "ms_per_step": 1000.0 * o_s / len(o_ms),
                  "join_kernel_ms": [i.ms_join_kernel for i in o_infos]}

    # ---- queries (resident), QPS and recall ----
    h = build(xp, 1)
    inf = info_of(h)
    qi = torch.empty((N_QUERIES, QK), dtype=torch.int32, device=dev)
    qd = torch.empty((N_QUERIES, QK), dtype=torch.float32, device=dev)

    def run_queries():
        L.check(L.lib.rinnd_query_device(h, ctypes.c_void_p(Q_dev.data_ptr()), N_QUERIES, DIM, QK, EPS, 0,
                                         ctypes.c_void_p(qi.data_ptr()), ctypes.c_void_p(qd.data_ptr()),
                                         ctypes.c_void_p(stream.cuda_stream)))

    for _ in range(3):
        run_queries()
    torch.cuda.synchronize()
    q0 = torch.cuda.Event(enable_timing=True)
    q1 = torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for _ in range(args.steps):
        run_queries()
    q1.record(stream)
    torch.cuda.synchronize()
    q_s = max_over_ranks(q0.elapsed_time(q1) / 1000.0)
    qps = N_QUERIES * world * args.steps / q_s
    quality = {}
    if not args.no_recall:
        ki = np.empty((n, K), np.int32)
        kd = np.empty((n, K), np.float32)
        L.check(L.lib.rinnd_neighbor_graph(h, L.ptr(ki), L.ptr(kd)))
        sample = np.random.default_rng(7).choice(n, size=min(10_000, n), replace=False)
        sample.sort()
        Xd = X_dev.double()
        xx = (Xd * Xd).sum(1)
        truth = np.concatenate([_exact_rows(Xd, xx, sample[s:s + 512], K, dev)
                                for s in range(0, len(sample), 512)])
        del Xd, xx
        quality["graph_recall@30"] = recall(ki[sample], truth)
        if ko is not None:
            other_form["graph_recall@30"] = recall(ko[sample], truth)
        qtruth = exact_knn_torch(X_dev, Q_dev, QK)
        quality["query_recall@10"] = recall(qi.cpu().numpy(), qtruth)
        quality["graph_recall_sample"] = f"{len(sample)} seeded rows vs FP64 exact"
    L.check(L.lib.rinnd_free(h))

    # ---- e2e: pinned host data -> build -> neighbor graph back to host ----
    e2e = None
    if not args.no_e2e:
        X_pin = torch.from_numpy(X).pin_memory()
        out_i = torch.empty((n, K), dtype=torch.int32).pin_memory()
        out_d = torch.empty((n, K), dtype=torch.float32).pin_memory()
        hp = ctypes.c_void_p(X_pin.data_ptr())

        def e2e_step():
            hh = build(hp, 0)
            L.check(L.lib.rinnd_neighbor_graph(hh, ctypes.c_void_p(out_i.data_ptr()),
                                               ctypes.c_void_p(out_d.data_ptr())))
            return hh

        L.check(L.lib.rinnd_free(e2e_step()))
        barrier()
        ee = []
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            hh = e2e_step()
            e1.record(stream)
            L.check(L.lib.rinnd_free(hh))
            ee.append((e0, e1))
        barrier()
        e_s = max_over_ranks(sum(a.elapsed_time(b) for a, b in ee) / 1000.0)
        e2e = {"value": n * world * args.steps / e_s, "unit": "points/s", "h2d_bytes_per_step": n * DIM * 4,
               "d2h_bytes_per_step": n * K * 8}

    # ---- CPU baseline (rank 0, single GPU only): the oracle builds the same
    # full workload; its recall beside the GPU's is the parity check at scale ----
    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        import oracle

        oix, dt = cpu_build(X)
        cpu = {"value": n / dt, "unit": "points/s", "cores": oracle.max_threads(), "kind": "port",
               "sample": f"the full workload: all {n} rows of this run's mixture, same k/trees/leaf/iters "
                         "(oracle/ C++ restatement, OpenMP), one build"}
        if not args.no_recall:
            oki, _ = oix.neighbor_graph
            quality["oracle_graph_recall@30"] = recall(oki[sample], truth)
            oqi, _ = oix.query(Q, k=QK, epsilon=EPS)
            quality["oracle_query_recall@10"] = recall(oqi, qtruth)
            quality["oracle_iterations"] = oix.iterations
            quality["parity_graph_recall_gap"] = quality["graph_recall@30"] - quality["oracle_graph_recall@30"]
            quality["parity_query_recall_gap"] = quality["query_recall@10"] - quality["oracle_query_recall@10"]
        del oix

    # ---- the batched and serving forms, compact, on one GPU: their numbers in
    # this line (the full workloads: --workload batched / serving) ----
    forms = {}
    if world == 1 and rank == 0 and not args.no_forms:
        try:
            forms["brute_force"] = brute_force_form(L, X_dev, Q_dev, QK)
        except Exception as exc:  # reported in the line, the build numbers stand
            forms["brute_force"] = {"error": f"{type(exc).__name__}: {exc}"}
        del X_dev, Q_dev
        torch.cuda.empty_cache()
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup, sub.check_items, sub.precision, sub.serve_seconds = 1, 2, 4, "fp32", 2.0
        for name, fn in (("batched", lambda: run_batched(sub, 1, 0, local_rank, emit=False)),
                         ("serving", lambda: run_serving(sub, 1, 0, local_rank, emit=False, compact=True)),
                         ("precision", lambda: run_precision(sub, 1, 0, local_rank, emit=False, compact=True))):
            try:
                forms[name] = fn()
            except Exception as exc:  # reported in the line, the build numbers stand
                forms[name] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.empty_cache()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * total_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(n, world),
            "iterations_per_build": [i.iterations for i in infos],
            "clocks": clk, "e2e": e2e, "gpu_launches": int(launches1.value - launches0.value),
            "roofline": roofline, "cpu_baseline": cpu,
            "precision": args.precision, "other_precision_form": other_form,
            "query": {"qps": qps, "k": QK, "epsilon": EPS, "n_queries": N_QUERIES, **quality},
            "timed_steps_ms": {"event": step_ms, "host_total": [i.ms_total for i in infos],
                               "join_kernels": [i.ms_join_kernel for i in infos],
                               "phases": [{"forest": i.ms_forest, "leaf_init": i.ms_leaf_init,
                                           "candidates": i.ms_candidates, "join": i.ms_join,
                                           "sort": i.ms_sort, "graph": i.ms_graph} for i in infos]},
            "counters": {"pairs_evaluated": int(inf.pairs_evaluated), "pushes_accepted": int(inf.pushes_accepted),
                         "push_contention": int(inf.push_contention), "join_rows": int(inf.join_rows_gathered),
                         "iterations": int(inf.iterations), "n_leaves": int(inf.n_leaves),
                         "join_tile": {"stages": int(inf.join_tile_stages), "rows_per_item": int(inf.join_tile_rows),
                                       "ctas_per_sm": int(inf.join_tile_ctas_per_sm),
                                       "mode": args.join_tuning}},
            "phases_ms": {"forest": inf.ms_forest, "leaf_init": inf.ms_leaf_init, "iterations": inf.ms_iterations,
                          "candidates": inf.ms_candidates, "join": inf.ms_join, "sort": inf.ms_sort,
                          "graph": inf.ms_graph, "total": inf.ms_total},
            **({"forms": forms} if forms else {}),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def brute_force_form(L, X_dev, Q_dev, k):
    """Brute-force exact kNN of the build workload's queries against its rows
    (rinnd_brute_force_knn, squared Euclidean): the FP32 form (the build's join
    arithmetic), the BF16 tensor-core form (Gram-tile filter + FP32 recheck)
    and the FP64 checker, each timed after a warm-up call (synchronized host
    clock around the call); whether the BF16 form's results are the FP32
    form's bit for bit, and how many queries' id lists FP32 and FP64 agree on."""
    import torch

    nq, n, d = Q_dev.shape[0], X_dev.shape[0], X_dev.shape[1]
    out, ids, dists = {"workload": f"{nq} queries x {n} rows x {d}, k={k}, sqeuclidean, device-resident"}, {}, {}
    for name, prec in (("fp32", L.BRUTE_FP32), ("bf16", L.BRUTE_BF16), ("fp64", L.BRUTE_FP64)):
        oi = torch.empty((nq, k), dtype=torch.int32, device=X_dev.device)
        od = torch.empty((nq, k), dtype=torch.float32, device=X_dev.device)

        def call():
            L.check(L.lib.rinnd_brute_force_knn(ctypes.c_void_p(X_dev.data_ptr()), n, d, ctypes.c_void_p(Q_dev.data_ptr()),
                                                nq, d, d, k, L.DIST_SQEUCLIDEAN, prec, None, 1,
                                                ctypes.c_void_p(oi.data_ptr()), ctypes.c_void_p(od.data_ptr())))

        call()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        call()
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        ids[name] = oi.cpu().numpy()
        dists[name] = od.cpu().numpy()
        out[name] = {"ms": 1000.0 * t, "qps": nq / t, "tflops_2qnd": 2.0 * nq * n * d / t / 1e12}
    # FP32 SIMT work: a subtraction and a fused multiply-add per element pair
    out["fp32"]["fp32_simt_fraction_of_nominal"] = 3.0 * nq * n * d / (out["fp32"]["ms"] / 1000.0) / 74.4e12
    out["fp32_id_lists_equal_to_fp64"] = float(np.mean(np.all(ids["fp32"] == ids["fp64"], axis=1)))
    out["bf16_results_equal_to_fp32"] = bool(np.array_equal(ids["bf16"], ids["fp32"]) and
                                             np.array_equal(dists["bf16"].view(np.uint32), dists["fp32"].view(np.uint32)))
    out["bf16"]["speedup_vs_fp32"] = out["fp32"]["ms"] / out["bf16"]["ms"]
    return out


def _exact_rows(Xd, xx, rows, k, dev):
    """FP64 exact kNN of data rows `rows` against all of X (self excluded)."""
    import torch

    r = torch.from_numpy(np.asarray(rows)).to(dev).long()
    q = Xd[r]
    d = (q * q).sum(1)[:, None] + xx[None, :] - 2.0 * (q @ Xd.T)
    d[torch.arange(len(rows), device=dev), r] = float("inf")
    return torch.topk(d, k, dim=1, largest=False).indices.int().cpu().numpy()


if __name__ == "__main__":
    main()
