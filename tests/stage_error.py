"""Error of every distance stage of the path against exact FP64 arithmetic,
measured with the oracle on nearest-neighbour pairs drawn at the full
density of the benchmark mixtures (one whole blob of each, as the full
workload holds it), plus the FP32-versus-FP64 stability sums.

Stages and the arithmetic measured (each is bit-identical on the GPU to the
oracle function used, or bounded against it by the GPU tests):

* NN-Descent initial, join and re-rank distances: the reference's sequential
  FP32 difference sum of squares (gpuknn/nndescent.cu:1086-1093),
  ``oracle.diffsum``;
* fix_distances, the antihub clique and the Core-SG Euclidean weights: pow in
  double, float accumulation, sqrtf (build_kNNG.cu:4-13,
  calculates.cu:275-283), ``oracle.euclid_ref``; core distances and MRD
  weights select among these values without further rounding;
* BF16 / FP16 candidate distances of the tensor-core forms (search only,
  every kept neighbour is re-ranked with the FP32 sum): |a|^2 + |c|^2 - 2 a.c
  of the column-centred rows rounded to BF16, or divided by a power of two and
  rounded to FP16, evaluated exactly here; the GPU tiles stay within
  1e-5 (|a|^2 + |c|^2) of that value;
* stability: the FP32 sums of the reference's row order against FP64 sums.

Run as a script to print the table; tests/test_oracle_stage_error.py holds
the bounds.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from gpu_hdbscan_b200 import synth  # noqa: E402
from oracle import oracle  # noqa: E402


def bf16_round(x):
    """Round-to-nearest-even of float32 to bfloat16, as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def fp16_scaled(x, maxabs):
    """x / s rounded to FP16 (round to nearest even) and scaled back, with s
    the power of two that puts maxabs / s in [2^14, 2^15)."""
    s = 2.0 ** (np.floor(np.log2(maxabs)) - 14)
    return (np.asarray(x, np.float64) / s).astype(np.float16).astype(np.float64) * s


def dense_blob(name, cap, seed=7):
    """The median-size blob of a workload, drawn whole (up to `cap` points)
    with the workload's centre and sigma, and the workload's column means
    estimated from a 100k-point sample."""
    w = synth.WORKLOADS[name]
    sizes, centers, sigmas, _ = synth._layout(w, np.random.default_rng(w.seed))
    b = int(np.argsort(sizes)[len(sizes) // 2])
    rng = np.random.default_rng(seed)
    nb = int(min(sizes[b], cap))
    X = (centers[b] + rng.normal(size=(nb, w.d)) * sigmas[b]).astype(np.float32)
    mean = synth.sample(w, 100_000).astype(np.float64).mean(axis=0).astype(np.float32)
    return X, mean, int(sizes[b])


def _stats(rel):
    rel = np.asarray(rel, np.float64)
    return {"median": float(np.median(rel)), "p99": float(np.quantile(rel, 0.99)),
            "max": float(rel.max())}


def distance_errors(name, queries=100, k=32, cap=200_000, seed=7):
    X, mean, blob_size = dense_blob(name, cap, seed)
    rng = np.random.default_rng(seed + 1)
    q = rng.choice(len(X), size=min(queries, len(X)), replace=False)
    ids, _ = oracle.bruteforce_knn(X, k + 1, q)
    Xd = X.astype(np.float64)
    Xc = (X - mean).astype(np.float32)  # the GPU forms centre the FP32 rows
    maxabs = float(np.abs(Xc).max())
    Xb, Xh = bf16_round(Xc), fp16_scaled(Xc, maxabs)
    nb, nh = (Xb * Xb).sum(1), (Xh * Xh).sum(1)
    e_sum, e_sqrt, e_bf16, e_fp16, cancel = [], [], [], [], []
    for qi, row in zip(q, ids):
        for j in row:
            if j == qi:
                continue
            exact2 = float(((Xd[qi] - Xd[j]) ** 2).sum())
            if exact2 == 0.0:
                continue
            e_sum.append(abs(float(oracle.diffsum(X[qi], X[j])) - exact2) / exact2)
            e_sqrt.append(abs(float(oracle.euclid_ref(X[qi], X[j])) - np.sqrt(exact2))
                          / np.sqrt(exact2))
            vb = nb[qi] + nb[j] - 2.0 * float(Xb[qi] @ Xb[j])
            vh = nh[qi] + nh[j] - 2.0 * float(Xh[qi] @ Xh[j])
            e_bf16.append(abs(vb - exact2) / exact2)
            e_fp16.append(abs(vh - exact2) / exact2)
            cancel.append((float((Xc[qi].astype(np.float64) ** 2).sum())
                           + float((Xc[j].astype(np.float64) ** 2).sum())) / exact2)
    return {"workload": name, "blob_points": blob_size, "drawn": len(X), "pairs": len(e_sum),
            "fp32_diffsum": _stats(e_sum), "sqrt_l2": _stats(e_sqrt),
            "bf16_form": _stats(e_bf16), "fp16_form": _stats(e_fp16),
            "cancellation": _stats(cancel)}


def stability_errors(name, n=8000, k=32, mpts=32):
    """FP32 against FP64 stability sums on a sample of the mixture: the
    largest relative difference over the clusters and the labels that differ
    between the two selections."""
    X = synth.sample(synth.WORKLOADS[name], n)
    ids, _ = oracle.bruteforce_knn(X, k + 1)
    ids = np.ascontiguousarray(ids[:, 1:]).astype(np.int32)
    dist = oracle.fix_distances(X, ids)
    mst, lab32, _ = oracle.hdbscan_from_knn(ids, dist, X, mpts)
    _, lab64, _ = oracle.hdbscan_from_knn(ids, dist, X, mpts, fp64=True)
    h = oracle.linkage_tree(mst, n)
    ct = oracle.condensed_tree(h, n, mpts)
    s32, s64 = oracle.stability(ct)
    v32 = s32["lambda"].astype(np.float64)
    keep = s64 != 0
    rel = np.abs(v32[keep] - s64[keep]) / np.abs(s64[keep])
    return {"workload": name, "points": n, "clusters": int(keep.sum()),
            "stability_rel_max": float(rel.max()) if rel.size else 0.0,
            "label_diffs": int((lab32 != lab64).sum())}


WORKLOAD_NAMES = ("blobs_10m_d12", "blobs_20m_d128", "blobs_50m_d96")


def main():
    for name in WORKLOAD_NAMES:
        r = distance_errors(name)
        print(f"{name}: blob of {r['blob_points']} points ({r['drawn']} drawn), "
              f"{r['pairs']} kNN pairs")
        for key in ("fp32_diffsum", "sqrt_l2", "bf16_form", "fp16_form", "cancellation"):
            s = r[key]
            print(f"  {key:13s} median {s['median']:.3e}  p99 {s['p99']:.3e}  max {s['max']:.3e}")
        s = stability_errors(name)
        print(f"  stability FP32 vs FP64 on {s['points']} points: {s['clusters']} clusters, "
              f"max relative {s['stability_rel_max']:.3e}, {s['label_diffs']} labels differ")


if __name__ == "__main__":
    main()
