"""Seeded synthetic inputs with the shapes of the benchmark workloads.

The reference benchmarks on its own generated blobs (data/artificial/create.py)
and publishes no dataset for this path, so every workload here is a seeded
mixture of Gaussian blobs plus uniform noise in the bounding box of the blob
points, shuffled.  ``generate`` builds a workload with numpy on the host (small
sizes, tests); ``generate_torch`` builds the same distribution with a torch
generator directly on a device (the multi-GB benchmark sizes).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Workload:
    name: str
    n: int
    d: int
    blobs: int
    center_lo: float
    center_hi: float
    sigma_lo: float
    sigma_hi: float
    anisotropic: bool
    zipf_s: float  # 0 -> equal blob sizes
    noise: float
    k: int
    mpts: int
    sample_num: int
    iterations: int
    seed: int


WORKLOADS = {
    # 100k x 12, 10 isotropic blobs (sigma 1), 5 % noise, k = mpts = 32
    "blobs_100k_d12": Workload("blobs_100k_d12", 100_000, 12, 10, -10.0, 10.0, 1.0, 1.0,
                               False, 0.0, 0.05, 32, 32, 16, 6, 1),
    # 10M x 12, 100 anisotropic Zipf-sized blobs, 10 % noise
    "blobs_10m_d12": Workload("blobs_10m_d12", 10_000_000, 12, 100, -10.0, 10.0, 0.3, 2.0,
                              True, 1.1, 0.10, 32, 32, 16, 6, 2),
    # 20M x 128, 1000 blobs, sigma in [0.5, 1.5], centres in [-20, 20], 5 % noise
    "blobs_20m_d128": Workload("blobs_20m_d128", 20_000_000, 128, 1000, -20.0, 20.0, 0.5, 1.5,
                               False, 0.0, 0.05, 32, 32, 16, 6, 3),
    # 50M x 96, 200 Zipf-sized blobs, sigma in [0.2, 3.0], 8 % noise
    "blobs_50m_d96": Workload("blobs_50m_d96", 50_000_000, 96, 200, -20.0, 20.0, 0.2, 3.0,
                              False, 1.1, 0.08, 32, 32, 16, 6, 5),
}


def scaled(name: str, n: int, seed: int | None = None) -> Workload:
    """The same distribution as WORKLOADS[name] with n points."""
    w = WORKLOADS[name]
    return Workload(w.name + f"_n{n}", n, w.d, min(w.blobs, max(1, n // 200)), w.center_lo,
                    w.center_hi, w.sigma_lo, w.sigma_hi, w.anisotropic, w.zipf_s, w.noise, w.k,
                    w.mpts, w.sample_num, w.iterations, w.seed if seed is None else seed)


def _layout(w: Workload, rng: np.random.Generator):
    n_noise = int(round(w.n * w.noise))
    n_blob = w.n - n_noise
    if w.zipf_s > 0:
        p = np.arange(1, w.blobs + 1, dtype=np.float64) ** (-w.zipf_s)
    else:
        p = np.ones(w.blobs)
    p /= p.sum()
    sizes = np.floor(p * n_blob).astype(np.int64)
    sizes[: n_blob - sizes.sum()] += 1
    centers = rng.uniform(w.center_lo, w.center_hi, size=(w.blobs, w.d))
    if w.anisotropic:
        sigmas = rng.uniform(w.sigma_lo, w.sigma_hi, size=(w.blobs, w.d))
    else:
        sigmas = np.repeat(rng.uniform(w.sigma_lo, w.sigma_hi, size=(w.blobs, 1)), w.d, axis=1)
    return sizes, centers, sigmas, n_noise


def generate(w: Workload) -> np.ndarray:
    """float32 [n, d] on the host (numpy PCG64 seeded with w.seed)."""
    rng = np.random.default_rng(w.seed)
    sizes, centers, sigmas, n_noise = _layout(w, rng)
    parts = [rng.normal(centers[b], sigmas[b], size=(int(sizes[b]), w.d)) for b in range(w.blobs)]
    X = np.concatenate(parts, axis=0) if parts else np.zeros((0, w.d))
    lo, hi = X.min(axis=0), X.max(axis=0)
    noise = rng.uniform(lo, hi, size=(n_noise, w.d))
    X = np.concatenate([X, noise], axis=0).astype(np.float32)
    return X[rng.permutation(w.n)]


def sample(w: Workload, n_sample: int, seed: int = 12345) -> np.ndarray:
    """n_sample points drawn from the same mixture as `w` (same blob centres,
    sigmas and relative sizes, same noise fraction) -- a bounded sample of the
    full workload for CPU timing, without generating all of it."""
    rng = np.random.default_rng(w.seed)
    sizes, centers, sigmas, _ = _layout(w, rng)
    r2 = np.random.default_rng(seed)
    n_noise = int(round(n_sample * w.noise))
    p = sizes / max(1, sizes.sum())
    which = r2.choice(w.blobs, size=n_sample - n_noise, p=p)
    Xb = centers[which] + r2.normal(size=(len(which), w.d)) * sigmas[which]
    lo, hi = Xb.min(axis=0), Xb.max(axis=0)
    X = np.concatenate([Xb, r2.uniform(lo, hi, size=(n_noise, w.d))]).astype(np.float32)
    return X[r2.permutation(n_sample)]


def generate_torch(w: Workload, device="cuda"):
    """The same distribution built on `device` with a seeded torch generator."""
    import torch

    rng = np.random.default_rng(w.seed)
    sizes, centers, sigmas, n_noise = _layout(w, rng)
    g = torch.Generator(device=device)
    g.manual_seed(w.seed)
    X = torch.empty((w.n, w.d), dtype=torch.float32, device=device)
    row = 0
    for b in range(w.blobs):
        m = int(sizes[b])
        if m == 0:
            continue
        c = torch.as_tensor(centers[b], dtype=torch.float32, device=device)
        s = torch.as_tensor(sigmas[b], dtype=torch.float32, device=device)
        X[row:row + m].normal_(generator=g).mul_(s).add_(c)
        row += m
    lo = X[:row].amin(dim=0)
    hi = X[:row].amax(dim=0)
    X[row:].uniform_(generator=g).mul_(hi - lo).add_(lo)
    perm = torch.randperm(w.n, generator=g, device=device)
    return X[perm].contiguous()


# ---- many independent instances (hdb_run_batched) ---------------------------
@dataclass(frozen=True)
class BatchWorkload:
    name: str
    count: int         # instances
    n_lo: int          # sizes log-uniform in [n_lo, n_hi]
    n_hi: int
    dims: tuple        # d drawn uniformly from these per instance
    blobs_lo: int      # blobs per instance, uniform in [blobs_lo, blobs_hi]
    blobs_hi: int
    center_lo: float
    center_hi: float
    sigma: float
    noise: float
    k: int
    mpts: int
    sample_num: int
    iterations: int
    seed: int


BATCH_WORKLOADS = {
    # 4096 instances, n log-uniform in [1000, 200000], d in {8, 12, 32, 64},
    # 3-50 isotropic blobs (centres in [-10, 10], sigma 1) + 5 % noise each,
    # k = mpts = 16 (SAMPLE_NUM 8).  Expected total n = 4096 * 199000 / ln(200)
    # ~ 154M points (4096 times the size's geometric mean, 14142, is 58M).
    "batch_4096": BatchWorkload("batch_4096", 4096, 1000, 200_000, (8, 12, 32, 64), 3, 50,
                                -10.0, 10.0, 1.0, 0.05, 16, 16, 8, 6, 4),
}


@dataclass(frozen=True)
class SplitWorkload:
    """One workload of WORKLOADS cut into `parts` uneven consecutive pieces
    (its rows are shuffled, so each piece is a random sample of the mixture),
    each clustered on its own.  Piece sizes are log-uniform in [1, spread],
    scaled to the workload's n; `seed` seeds both the sizes and the data."""
    name: str
    base: str
    parts: int
    spread: float
    seed: int
    precision: str = "bf16"

    @property
    def w(self) -> Workload:
        return WORKLOADS[self.base]

    @property
    def count(self):
        return self.parts

    k = property(lambda self: self.w.k)
    mpts = property(lambda self: self.w.mpts)
    sample_num = property(lambda self: self.w.sample_num)
    iterations = property(lambda self: self.w.iterations)


SPLIT_WORKLOADS = {
    # 50M x 96 (200 Zipf-sized blobs, sigma in [0.2, 3.0], 8 % noise) as 64
    # uneven sub-instances, sizes spread over a factor of 20
    "blobs_50m_d96_split64": SplitWorkload("blobs_50m_d96_split64", "blobs_50m_d96", 64, 20.0, 5),
}


def split_sizes(sw: SplitWorkload, count: int | None = None):
    rng = np.random.default_rng(sw.seed)
    r = np.exp(rng.uniform(0.0, np.log(sw.spread), size=sw.parts))
    sizes = np.floor(r / r.sum() * sw.w.n).astype(np.int64)
    sizes[: sw.w.n - sizes.sum()] += 1
    return [int(x) for x in sizes[: sw.parts if count is None else count]]


def batch_layout(bw: BatchWorkload, count: int | None = None):
    """Per instance (n, d, blobs), seeded; the first `count` instances."""
    rng = np.random.default_rng(bw.seed)
    c = bw.count
    n = np.exp(rng.uniform(np.log(bw.n_lo), np.log(bw.n_hi), size=c)).astype(np.int64)
    d = rng.choice(np.asarray(bw.dims), size=c)
    b = rng.integers(bw.blobs_lo, bw.blobs_hi + 1, size=c)
    m = c if count is None else count
    return [(int(n[i]), int(d[i]), int(b[i])) for i in range(m)]


def batch_instance(bw: BatchWorkload, i: int, n: int, d: int, blobs: int) -> Workload:
    """Instance i as a single workload (its own seed)."""
    return Workload(f"{bw.name}_i{i}", n, d, blobs, bw.center_lo, bw.center_hi, bw.sigma,
                    bw.sigma, False, 0.0, bw.noise, bw.k, bw.mpts, bw.sample_num, bw.iterations,
                    bw.seed * 1_000_003 + i)


def generate_batch_torch(bw, device="cuda", count: int | None = None, indices=None):
    """The instances on `device`: one [sum n, d] array per d with the instances
    of that d back to back (in instance order), and per instance a view into
    it, in instance order.  -> (views, layout of (n, d, blobs)).  `indices`
    (ascending) keeps only those instances of the first `count`, generated
    exactly as in the whole batch; views and layout then follow `indices`."""
    import torch

    if isinstance(bw, SplitWorkload):
        sizes = split_sizes(bw, count)
        w = Workload(**{**bw.w.__dict__, "n": sum(sizes), "seed": bw.seed})
        X = generate_torch(w, device=device)
        views, row = [], 0
        for m in sizes:
            views.append(X[row:row + m])
            row += m
        layout = [(m, w.d, 0) for m in sizes]
        if indices is not None:
            views = [views[i].clone() for i in indices]
            layout = [layout[i] for i in indices]
            del X
        return views, layout
    full = batch_layout(bw, count)
    keep = list(range(len(full))) if indices is None else list(indices)
    layout = [full[i] for i in keep]
    by_d = {}
    for j, i in enumerate(keep):
        by_d.setdefault(full[i][1], []).append((j, i))
    views = [None] * len(keep)
    for d, idx in by_d.items():
        total = sum(full[i][0] for _, i in idx)
        buf = torch.empty((total, d), dtype=torch.float32, device=device)
        row = 0
        for j, i in idx:
            n, _, b = full[i]
            buf[row:row + n] = generate_torch(batch_instance(bw, i, n, d, b), device=device)
            views[j] = buf[row:row + n]
            row += n
    return views, layout
