#!/usr/bin/env python
"""End-to-end HDBSCAN points/s on B200 (libhdb_b200.so).

One step = one full run of the path (NN-Descent kNN graph -> enhanced kNN
graph -> MST -> linkage tree -> condensed tree / EOM -> labels) over the whole
synthetic workload.  `value` is measured with the input already resident in
HBM; `e2e` is the same metric through the C ABI with host buffers (H2D copy of
X and D2H copy of the labels inside every timed step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload blobs_10m_d12]

N > 1 runs N independent replicas (one process per GPU, torchrun); the path
has no cross-GPU exchange, so only the timing is reduced (max over ranks).
`--impl reference` times the reference algorithm's CPU restatement (the
oracle port, all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "end-to-end HDBSCAN points/s on 1 B200: BF16-TC vs plain FP32, equal recall@k"
UNIT = "points/s"
# forms of the NN-Descent candidate distances (hdb_knn_params.precision)
PRECISIONS = {"bf16": 1, "fp32": 0, "fp16": 2}
DTYPES = {"bf16": "bf16", "fp32": "f32", "fp16": "f16"}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="blobs_20m_d128")
    ap.add_argument("--precision", choices=["fp32", "bf16", "fp16"], default=None,
                    help="form (default: bf16; fp32 for the batched workloads)")
    ap.add_argument("--instances", type=int, default=0,
                    help="batched workloads: only the first N instances (0: all)")
    ap.add_argument("--shard-instances", action="store_true",
                    help="batched workloads on N GPUs: one batch, its instances spread over the "
                         "ranks by greedy size balancing (strong scaling) instead of a seeded "
                         "copy of the batch per rank (weak scaling)")
    ap.add_argument("--loop-instances", type=int, default=256,
                    help="batched workloads: instances timed in the per-instance loop comparison")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip timing the other form (plain FP32 vs BF16-TC) and, for "
                         "batched workloads, the per-instance loop")
    ap.add_argument("--recall-queries", type=int, default=1000)
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="points in the CPU baseline sample (0: sized per workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--n", type=int, default=0,
                    help="points (0: the workload's size); blob count scales with n")
    ap.add_argument("--bare", action="store_true",
                    help="time only the K steps (no other form, recall, e2e or CPU baseline); "
                         "for profiler captures")
    args = ap.parse_args()
    if args.bare:
        args.no_compare = args.no_e2e = args.no_cpu_baseline = True
        args.recall_queries = 0
    return args


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d.get("bf16_tflops", 1590.0)), "measured"
    return 6650.0, 1590.0, "fallback"


def profiled_traffic(kernel):
    """Per-row DRAM bytes of `kernel` from the committed ncu summary (profiles/),
    or None.  Line format: TRAFFIC <kernel> bytes_per_row=<float> ..."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for name in sorted(os.listdir(pdir)):
        if not name.endswith((".md", ".txt")):
            continue
        with open(os.path.join(pdir, name)) as f:
            for line in f:
                m = re.match(rf"TRAFFIC {re.escape(kernel)} bytes_per_row=([0-9.eE+]+)", line.strip())
                if m:
                    return float(m.group(1))
    return None


def fp32_issue_roofline(stats, d, clk):
    """The FP32 local join against its FP32 issue bound: each computed pair
    (join_pairs, counted live) costs d subtractions and d fused multiply-adds,
    3 FLOP per dimension; the bound is SMs x 128 FP32 lanes x 2 FLOP x the SM
    clock sampled during the run."""
    import torch
    pairs, ms = stats.get("join_pairs", 0), stats.get("join_ms", 0.0)
    if not pairs or not ms:
        return None
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
    achieved = pairs * d * 3 / (ms / 1e3) / 1e12
    peak = sms * 128 * 2 * mhz * 1e6 / 1e12
    launches = max(1, stats.get("join_launches", 1))
    return {"kernel": "k_join (FP32 local join)", "bound": "fp32_issue",
            "achieved": round(achieved, 2), "peak": round(peak, 2), "unit": "TFLOP/s",
            "frac": round(achieved / peak, 4), "pairs_per_launch": round(pairs / launches),
            "sm_mhz": mhz, "form": stats.get("join_config")}


def tensor_roofline(n_points, d, stats, bf16_peak, iterations):
    """The tensor-core join against the measured dense BF16 peak: every tile
    (two rows' joins) is one M = N = 128 MMA chain over the padded dimensions,
    2 x 128 x 128 x dpad FLOP, about rows / 2 tiles per iteration.  join_ms
    also holds the slot-list pass before each launch."""
    ms = stats.get("join_ms", 0.0)
    if not ms:
        return None
    dpad = (d + 63) // 64 * 64
    flops = iterations * ((n_points + 1) // 2) * 2 * 128 * 128 * dpad
    achieved = flops / (ms / 1e3) / 1e12
    return {"kernel": "k_join_tc (tcgen05 Gram tiles)", "bound": "tensor",
            "achieved": round(achieved, 1), "peak": bf16_peak, "unit": "TFLOP/s",
            "frac": round(achieved / bf16_peak, 4)}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names[1:], parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def replica_workload(w, rank):
    """Each replica (rank) clusters its own seeded copy of the workload."""
    from gpu_hdbscan_b200 import synth
    return synth.Workload(**{**w.__dict__, "seed": w.seed + 1000 * rank})


def max_over_ranks(ms, device):
    """The largest per-rank duration over all ranks of the process group (the
    value itself on one rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_ranks(v, device):
    """Every rank's value of a per-rank number, in rank order (the value itself
    on one rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        out = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
        dist.all_gather(out, t)
        return [float(x.item()) for x in out]
    return [float(t.item())]


def sum_over_ranks(v, device):
    """The sum of a per-rank count over all ranks (the value itself on one rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def batch_instance_sizes(bw, count):
    """Points of every instance of a batched workload (its first `count`)."""
    from gpu_hdbscan_b200 import synth
    if isinstance(bw, synth.SplitWorkload):
        return synth.split_sizes(bw, count)
    return [n for n, _, _ in synth.batch_layout(bw, count)]


def whole_job_rate(n, steps, world, ms):
    """Points/s of the whole job: every replica clusters n points per step."""
    return n * steps * world / (ms / 1e3)


def exact_recall(X, G_ids, queries, k):
    """recall@k of G_ids[queries] against the exact FP64 kNN (torch, chunked)."""
    import torch
    q = torch.as_tensor(queries, device=X.device)
    Xq = X[q].double()
    best_d = torch.full((len(q), k), float("inf"), dtype=torch.float64, device=X.device)
    best_i = torch.zeros((len(q), k), dtype=torch.int64, device=X.device)
    chunk = 1 << 18
    for s0 in range(0, X.shape[0], chunk):
        Xc = X[s0:s0 + chunk].double()
        dd = torch.cdist(Xq, Xc).square_()
        idx = torch.arange(s0, s0 + Xc.shape[0], device=X.device)
        dd[idx[None, :] == q[:, None]] = float("inf")  # exclude the point itself
        cd = torch.cat([best_d, dd], dim=1)
        ci = torch.cat([best_i, idx[None, :].expand(len(q), -1)], dim=1)
        top = torch.topk(cd, k, dim=1, largest=False)
        best_d = top.values
        best_i = torch.gather(ci, 1, top.indices)
    got = G_ids[q].long()
    hits = (got[:, :, None] == best_i[:, None, :]).any(dim=2).sum().item()
    return hits / (len(q) * k)


def cpu_baseline_run(workload, n_sample, steps):
    """The reference algorithm on the host cores (oracle port, OpenMP over all
    available threads): NN-Descent + the _new.cu stages on a sample."""
    from gpu_hdbscan_b200 import synth
    from oracle import oracle as O

    w = workload
    X = synth.sample(w, n_sample)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ids, _ = O.nndescent(X, w.k, w.sample_num, w.iterations)
        fd = O.fix_distances(X, ids)
        O.hdbscan_from_knn(ids, fd, X, w.mpts)
        times.append(time.perf_counter() - t0)
    return {"value": n_sample * len(times) / sum(times), "unit": UNIT,
            "cores": O.num_threads(), "kind": "port",
            "sample": f"{n_sample} points drawn from the {workload.name} mixture "
                      f"(d={w.d}, k={w.k}, mpts={w.mpts}), {len(times)} run(s), oracle port "
                      f"(NN-Descent + enhanced kNNG + Kruskal + trees)"}


def default_cpu_sample(w):
    return 100_000 if w.d <= 16 else 50_000


def cpu_reference_legs(X, k, mpts):
    """The CPU path the reference validates against, timed on the host cores:
    (i) its ground-truth kNN, which it reads from exact brute-force files
    (HDBSCAN/cmake/eval.py:57) -- stood in for by scipy's cKDTree (d <= 12) or
    a blocked FP64 brute force (d > 12), and (ii) the CPU HDBSCAN its labels
    are checked against (PyPI hdbscan, prims_kdtree / EOM,
    HDBSCAN/groundtruth/groundtruth.py:115-119; not installable here) --
    stood in for by sklearn.cluster.HDBSCAN with the same min_cluster_size,
    min_samples and EOM selection.  Returns both legs in points/s."""
    import numpy as np
    n, d = X.shape
    t0 = time.perf_counter()
    if d <= 12:
        from scipy.spatial import cKDTree
        cKDTree(X).query(X, k=k + 1, workers=-1)
        knn_method = "scipy cKDTree(workers=-1), k+1 nearest per point"
    else:
        X64 = X.astype(np.float64)
        nrm = (X64 * X64).sum(1)
        for s0 in range(0, n, 2048):
            D = nrm[s0:s0 + 2048, None] + nrm[None, :] - 2.0 * (X64[s0:s0 + 2048] @ X64.T)
            np.argpartition(D, k + 1, axis=1)[:, :k + 1]
        knn_method = "blocked FP64 brute force (numpy BLAS), k+1 nearest per point"
    t1 = time.perf_counter()
    import warnings
    from sklearn.cluster import HDBSCAN
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        HDBSCAN(min_cluster_size=mpts, min_samples=mpts, cluster_selection_method="eom",
                n_jobs=-1).fit(X)
    t2 = time.perf_counter()
    return {"exact_knn": {"value": n / (t1 - t0), "unit": UNIT, "method": knn_method},
            "cpu_hdbscan": {"value": n / (t2 - t1), "unit": UNIT,
                            "method": f"sklearn.cluster.HDBSCAN(min_cluster_size={mpts}, "
                                      f"min_samples={mpts}, cluster_selection_method='eom', "
                                      "n_jobs=-1), stand-in for PyPI hdbscan prims_kdtree"},
            "knn_plus_hdbscan": {"value": n / (t2 - t0), "unit": UNIT},
            "sample_points": n, "cores": len(os.sched_getaffinity(0))}


def add_reference_legs(cb, w):
    """Adds the reference's CPU ground-truth kNN + CPU HDBSCAN legs to a CPU
    baseline record, on a sample of the workload's mixture sized to run in
    seconds (sklearn's HDBSCAN grows faster than linearly)."""
    from gpu_hdbscan_b200 import synth
    try:
        cb["legs"] = cpu_reference_legs(synth.sample(w, 20_000 if w.d <= 16 else 5_000),
                                        w.k, w.mpts)
    except Exception as e:  # report, never lose the line
        cb["legs"] = {"error": f"{type(e).__name__}: {e}"}
    return cb


def run_reference(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n_s = args.cpu_sample or default_cpu_sample(w)
    for _ in range(args.warmup):
        pass  # the CPU port has no warm-up state; warm-up steps are not repeated work
    cb = add_reference_legs(cpu_baseline_run(w, n_s, max(1, args.steps)), w)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": w.name, "n": w.n, "d": w.d, "k": w.k,
                                             "mpts": w.mpts, "sample_points": n_s},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, w):
    import torch
    import torch.distributed as dist

    import gpu_hdbscan_b200 as g
    from gpu_hdbscan_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    prec = PRECISIONS[args.precision]
    X = synth.generate_torch(replica_workload(w, rank), device=dev)
    ctx = g.Context(local)
    kw = dict(k=w.k, mpts=w.mpts, sample_num=w.sample_num, iterations=w.iterations,
              precision=prec)

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(kwx, steps, warmup):
        for _ in range(warmup):
            ctx.hdbscan(X, **kwx)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        stats = []
        ev0.record(stream)
        for _ in range(steps):
            _, st = ctx.hdbscan(X, **kwx)
            stats.append(st)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(ev0.elapsed_time(ev1), dev), stats

    clocks = ClockSampler(local)
    clocks.start()
    ms_max, stats = timed(kw, args.steps, args.warmup)
    clk = clocks.stop()
    value = whole_job_rate(w.n, args.steps, world, ms_max)
    stream = torch.cuda.current_stream()

    # the other form, for the BF16-TC vs plain FP32 comparison, and recall@32
    # of both against the exact FP64 kNN on a sample of rows
    compare = None
    if not args.no_compare:
        other = g.HDB_PREC_FP32 if prec != g.HDB_PREC_FP32 else g.HDB_PREC_BF16
        kwo = {**kw, "precision": other}
        osteps = max(1, args.steps // 2)
        oms, ostats = timed(kwo, osteps, 1)
        compare = {"form": "fp32" if other == g.HDB_PREC_FP32 else "bf16",
                   "points_per_s": round(whole_job_rate(w.n, osteps, world, oms), 1),
                   "ms_per_step": round(oms / osteps, 3), "steps": osteps,
                   "stage_ms": {s_: round(ostats[-1][f"ms_{s_}"], 3) for s_ in
                                ("knn", "graph", "mst", "tree", "total")}}
        if other == g.HDB_PREC_FP32:
            compare["issue_roofline"] = fp32_issue_roofline(ostats[-1], w.d, clk)
    recall = {}
    if args.recall_queries > 0:
        qidx = torch.randperm(w.n, generator=torch.Generator().manual_seed(7))[:args.recall_queries]
        for name_, pr in PRECISIONS.items():
            if compare is None and pr != prec:
                continue
            G = ctx.NNDescent(X, k=w.k, sample_num=w.sample_num, iterations=w.iterations,
                              precision=pr)
            ids, _ = ctx.knn_split(G)
            recall[name_] = round(exact_recall(X, ids, qidx.to(dev), w.k), 4)
            del G, ids
        torch.cuda.empty_cache()

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        Xh = X.cpu().pin_memory()
        lab = torch.empty(w.n, dtype=torch.int32).pin_memory()
        ctx.hdbscan(Xh, labels_out=lab, **kw)
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.hdbscan(Xh, labels_out=lab, **kw)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        te = max_over_ranks(e0.elapsed_time(e1), dev)
        e2e = {"value": whole_job_rate(w.n, args.steps, world, te), "unit": UNIT,
               "h2d_bytes_per_step": int(w.n * w.d * 4), "d2h_bytes_per_step": int(w.n * 4)}

    if rank == 0 and args.bare:
        print(json.dumps({"bare": True, "workload": w.name, "ms_per_step": ms_max / args.steps,
                          "stats": stats[-1]}), flush=True)
    elif rank == 0:
        hbm, _, peak_kind = measured_peaks()
        last = stats[-1]
        S = w.sample_num
        launches = max(1, last["join_launches"])
        # algorithmic bytes of the local join (per launch): staged sample rows,
        # the sample lists and counters, and each pushed candidate (inbox entry,
        # counter atomic, k-th distance read)
        if prec != g.HDB_PREC_FP32:
            tc = (w.d + 63) // 64 * 64 <= 256  # tensor-core tiles, else the mma.sync join
            jkernel = "k_join_tc" if tc else "k_join_bf16"
            row_bytes = ((w.d + 63) // 64 * 64 if tc else (w.d + 15) // 16 * 16) * 2
        else:
            jkernel, row_bytes = "k_join", w.d * 4
        join_bytes = (last["join_rows_gathered"] * row_bytes
                      + launches * w.n * (2 * 2 * S * 4 + 2 * 4 + 2 * 1)
                      + last["join_candidates"] * (8 + 4 + 4)) / launches
        join_ms = last["join_ms"] / launches
        achieved = join_bytes / (join_ms / 1e3) / 1e9
        tpr = profiled_traffic(jkernel)
        roofline = {"kernel": jkernel + " (NN-Descent local join)", "bound": "hbm",
                    "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(achieved / hbm, 4),
                    "traffic": None if tpr is None else round(tpr * w.n),
                    "peak_kind": peak_kind,
                    "algorithmic_bytes_per_launch": round(join_bytes),
                    "avg_launch_ms": round(join_ms, 4),
                    "mean_rows_gathered_per_point": round(last["join_rows_gathered"] / launches / w.n, 2)}
        cb = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cb = add_reference_legs(
                    cpu_baseline_run(w, args.cpu_sample or default_cpu_sample(w), 1), w)
            except Exception as e:  # report, never lose the GPU line
                cb = {"error": f"{type(e).__name__}: {e}"}
        line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": DTYPES[args.precision],
                "data": "synthetic",
                "config": {"workload": w.name, "n": w.n, "d": w.d, "k": w.k, "mpts": w.mpts,
                           "sample_num": w.sample_num, "iterations": w.iterations,
                           "form": args.precision, "parallelism": f"replicas{world}",
                           "l2": "inputs larger than L2 (X alone is "
                                 f"{w.n * w.d * 4 / 1e6:.0f} MB)",
                           "stage_ms": {s: round(last[f"ms_{s}"], 3) for s in
                                        ("knn", "graph", "mst", "tree", "total")},
                           "num_clusters": last["num_clusters"], "edges": last["edges"],
                           "mst_rounds": last["mst_rounds"], "knn_dropped": last["knn_dropped"],
                           "other_form": compare, "recall_at_k": recall,
                           "speedup_vs_other_form": (round(value / compare["points_per_s"], 3)
                                                     if compare else None)},
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "clocks": clk,
                "gpu_launches": int(sum(s["gpu_launches"] for s in stats))}
        # the join's compute bound beside the HBM one
        if jkernel == "k_join_tc":
            line["tensor_roofline"] = tensor_roofline(w.n, w.d, last, measured_peaks()[1],
                                                      w.iterations)
        elif jkernel == "k_join":
            line["issue_roofline"] = fp32_issue_roofline(last, w.d, clk)
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def batch_cpu_sample(bw, layout, min_points=50_000):
    """The first instances of the layout up to `min_points` points, built on
    the host (numpy) for the CPU timing (for a split workload: one piece's
    worth of points drawn from the mixture)."""
    from gpu_hdbscan_b200 import synth
    if isinstance(bw, synth.SplitWorkload):
        return [synth.sample(bw.w, min_points)]
    Xs, tot = [], 0
    for i, (n, d, b) in enumerate(layout):
        Xs.append(synth.generate(synth.batch_instance(bw, i, n, d, b)))
        tot += n
        if tot >= min_points:
            break
    return Xs


def cpu_batch_run(bw, Xs):
    """The reference algorithm per instance on the host cores (oracle port);
    an instance whose graph is disconnected is timed up to its failure, as
    the reference stops there."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    for X in Xs:
        ids, _ = O.nndescent(X, bw.k, bw.sample_num, bw.iterations)
        try:
            O.hdbscan_from_knn(ids, O.fix_distances(X, ids), X, bw.mpts)
        except RuntimeError:
            pass
    dt = time.perf_counter() - t0
    npts = sum(len(X) for X in Xs)
    return {"value": npts / dt, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": f"the first {len(Xs)} instance(s) of {bw.name} ({npts} points, d in "
                      f"{sorted({X.shape[1] for X in Xs})}, k={bw.k}, mpts={bw.mpts}), one run "
                      f"each, oracle port (NN-Descent + enhanced kNNG + Kruskal + trees)"}


def batch_reference_legs(bw, Xs):
    """The reference's CPU ground-truth kNN + CPU HDBSCAN legs on the first
    instance of the CPU sample (at most 20,000 of its points)."""
    try:
        return cpu_reference_legs(Xs[0][:20_000], bw.k, bw.mpts)
    except Exception as e:
        return {"error": f"{type(e).__name__}: {e}"}


def run_reference_batch(args, bw):
    from gpu_hdbscan_b200 import synth
    if int(os.environ.get("RANK", "0")) != 0:
        return
    layout = synth.batch_layout(bw, args.instances or None)
    Xs = batch_cpu_sample(bw, layout)
    vals = [cpu_batch_run(bw, Xs) for _ in range(max(1, args.steps))]
    cb = vals[-1]
    cb["value"] = statistics.median(v["value"] for v in vals)
    cb["legs"] = batch_reference_legs(bw, Xs)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": bw.name, "instances": len(layout),
                                             "k": bw.k, "mpts": bw.mpts},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours_batch(args, bw):
    """Many independent instances (hdb_run_batched) against a per-instance
    loop of hdb_run over the first --loop-instances of them."""
    import torch
    import torch.distributed as dist

    import gpu_hdbscan_b200 as g
    from gpu_hdbscan_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    prec = PRECISIONS[args.precision]
    count = args.instances or None
    if args.shard_instances:
        # one batch over all ranks: rank r clusters the instances the greedy
        # size balancing gives it (same seed everywhere, no exchange)
        from gpu_hdbscan_b200 import sharding
        all_sizes = batch_instance_sizes(bw, count)
        if len(all_sizes) < world:
            raise SystemExit("--shard-instances needs at least one instance per rank")
        parts = sharding.assign_instances(all_sizes, world)
        rbw = bw
        views, layout = synth.generate_batch_torch(rbw, device=dev, count=count,
                                                   indices=parts[rank])
        n_job = sum(all_sizes)
    else:
        rbw = type(bw)(**{**bw.__dict__, "seed": bw.seed + 1000 * rank})
        views, layout = synth.generate_batch_torch(rbw, device=dev, count=count)
    n_total = sum(n for n, _, _ in layout)
    if not args.shard_instances:
        n_job = n_total * world
    ctx = g.Context(local)
    kw = dict(k=bw.k, mpts=bw.mpts, sample_num=bw.sample_num, iterations=bw.iterations,
              precision=prec)
    kw_b = {**kw, "strict": False}
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    rank_ms = []

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        out = []
        e0.record(stream)
        for _ in range(steps):
            out.append(fn())
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        rank_ms[:] = all_ranks(e0.elapsed_time(e1) / steps, dev)
        return max_over_ranks(e0.elapsed_time(e1), dev), out

    clocks = ClockSampler(local)
    clocks.start()
    ms_max, outs = timed(lambda: ctx.hdbscan_batched(views, **kw_b), args.steps, args.warmup)
    clk = clocks.stop()
    per_rank_ms = [round(x, 3) for x in rank_ms]
    stats = [o[2] for o in outs]
    value = n_job * args.steps / (ms_max / 1e3)
    failed = int(sum_over_ranks(sum(1 for s_ in stats[-1]["instance_status"] if s_ != 0), dev))

    # per-instance loop (hdb_run per instance) against the batch on the same
    # instances; the loop skips the instances the batch found disconnected
    # (hdb_run stops on them, as the reference does).  --no-compare (and
    # --bare) leave it out: it launches ~1,000 kernels per instance.
    m = 0 if args.no_compare else min(args.loop_instances, len(views))
    sub = [v for v, s_ in zip(views[:m], stats[-1]["instance_status"][:m]) if s_ == 0]
    n_sub = sum(len(v) for v in sub)
    loop_failed = []

    def loop_once():
        loop_failed.clear()
        for v in sub:
            try:
                ctx.hdbscan(v, **kw)
            except g.HdbError as e:  # its own graph may fall apart where the batch's did not
                if e.status != g._lib.HDB_ERR_DISCONNECTED:
                    raise
                loop_failed.append(1)

    loop = None
    if sub:
        lms, _ = timed(loop_once, 1, 1)
        bms, _ = timed(lambda: ctx.hdbscan_batched(sub, **kw_b), 1, 1)
        loop = {"instances": len(sub), "points": n_sub,
                "loop_points_per_s": round(n_sub / (lms / 1e3), 1), "loop_ms": round(lms, 3),
                "batched_points_per_s": round(n_sub / (bms / 1e3), 1), "batched_ms": round(bms, 3),
                "speedup": round(lms / bms, 3), "loop_disconnected": len(loop_failed)}

    e2e = None
    if not args.no_e2e:
        hosts = [v.cpu() for v in views]
        try:
            hosts = [h.pin_memory() for h in hosts]
            pinned = True
        except RuntimeError:
            pinned = False
        ctx.hdbscan_batched(hosts, **kw_b)
        te, _ = timed(lambda: ctx.hdbscan_batched(hosts, **kw_b), args.steps, 0)
        e2e = {"value": n_job * args.steps / (te / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(sum(v.numel() for v in views) * 4),
               "d2h_bytes_per_step": int(n_total * 4), "pinned_inputs": pinned}
        del hosts

    if rank == 0:
        hbm, _, peak_kind = measured_peaks()
        last = stats[-1]
        S = bw.sample_num
        launches = max(1, last["join_launches"])
        per_d = {}
        for n, d, _ in layout:
            per_d[d] = per_d.get(d, 0) + n
        if prec != g.HDB_PREC_FP32:
            row_bytes = {d: ((d + 63) // 64 * 64) * 2 for d in per_d}
            jkernel = "k_join_tc"
        else:
            row_bytes = {d: d * 4 for d in per_d}
            jkernel = "k_join"
        # gathered rows are not split by d in the stats: weight the row size by points
        mean_row = sum(row_bytes[d] * c for d, c in per_d.items()) / n_total
        join_bytes = (last["join_rows_gathered"] * mean_row
                      + bw.iterations * n_total * (2 * 2 * S * 4 + 2 * 4 + 2 * 1)
                      + last["join_candidates"] * (8 + 4 + 4))
        achieved = join_bytes / (last["join_ms"] / 1e3) / 1e9
        roofline = {"kernel": jkernel + " (NN-Descent local join, all batches)", "bound": "hbm",
                    "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(achieved / hbm, 4), "traffic": None, "peak_kind": peak_kind,
                    "algorithmic_bytes_per_launch": round(join_bytes / launches),
                    "avg_launch_ms": round(last["join_ms"] / launches, 4)}
        cb = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                Xs_cpu = batch_cpu_sample(rbw, layout)
                cb = cpu_batch_run(rbw, Xs_cpu)
                cb["legs"] = batch_reference_legs(rbw, Xs_cpu)
            except Exception as e:
                cb = {"error": f"{type(e).__name__}: {e}"}
        line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
                "scaling": "strong" if args.shard_instances else "weak", "vs_baseline": None,
                "dtype": DTYPES[args.precision], "data": "synthetic",
                "config": {"workload": bw.name, "instances": len(layout), "n_total": n_total,
                           "n_job": n_job,
                           "points_per_d": {str(d): c for d, c in sorted(per_d.items())},
                           "k": bw.k, "mpts": bw.mpts, "sample_num": bw.sample_num,
                           "iterations": bw.iterations, "form": args.precision,
                           "parallelism": (f"instances{world}" if args.shard_instances
                                           else f"replicas{world}"),
                           "l2": f"inputs larger than L2 ({sum(v.numel() for v in views) * 4 / 1e9:.1f} GB)",
                           "stage_ms": {s_: round(last[f"ms_{s_}"], 3) for s_ in
                                        ("knn", "graph", "mst", "tree", "total")},
                           "num_clusters": last["num_clusters"], "edges": last["edges"],
                           "knn_dropped": last["knn_dropped"],
                           "disconnected_instances": failed, "per_instance_loop": loop,
                           "per_rank_ms_per_step": per_rank_ms,
                           "rank_points": (sharding.rank_loads(all_sizes, parts)
                                           if args.shard_instances else None),
                           "label_gather": ("not timed: the host gather of labels "
                                            "(sharding.gather_labels) runs outside the step"
                                            if args.shard_instances else None)},
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "clocks": clk,
                "gpu_launches": int(sum(s_["gpu_launches"] for s_ in stats))}
        # the join's compute bound beside the HBM one: for the FP32 join with
        # the points-weighted mean d (pairs are not counted per d); for the
        # tensor-core join when the batch has one d
        if prec == g.HDB_PREC_FP32:
            d_mean = sum(d * c for d, c in per_d.items()) / n_total
            line["issue_roofline"] = fp32_issue_roofline(last, d_mean, clk)
        elif len(per_d) == 1:
            line["tensor_roofline"] = tensor_roofline(n_total, next(iter(per_d)), last,
                                                      measured_peaks()[1], bw.iterations)
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse_args()
    from gpu_hdbscan_b200 import synth
    if args.workload in synth.BATCH_WORKLOADS or args.workload in synth.SPLIT_WORKLOADS:
        bw = synth.BATCH_WORKLOADS.get(args.workload) or synth.SPLIT_WORKLOADS[args.workload]
        if args.precision is None:
            args.precision = getattr(bw, "precision", "fp32")
        if args.impl == "reference":
            run_reference_batch(args, bw)
        else:
            run_ours_batch(args, bw)
        return
    if args.precision is None:
        args.precision = "bf16"
    w = synth.WORKLOADS[args.workload]
    if args.n and args.n != w.n:
        blobs = max(1, round(w.blobs * args.n / w.n))
        w = synth.Workload(**{**w.__dict__, "name": f"{w.name}_n{args.n}", "n": args.n,
                              "blobs": blobs})
    if args.impl == "reference":
        run_reference(args, w)
    else:
        run_ours(args, w)


if __name__ == "__main__":
    main()
