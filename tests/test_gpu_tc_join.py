"""The BF16 tensor-core local join (TMA gather4 -> tcgen05.mma -> TMEM) through
hdb_bf16_distance_tiles, against the same arithmetic in float64 on the CPU:
rows rounded to BF16, |a|^2 + |c|^2 - 2 a.c.  Then NN-Descent on both BF16
kernels (tensor-core tiles up to d = 256, mma.sync beyond)."""
import numpy as np
import pytest

import gpu_hdbscan_b200 as g

pytestmark = pytest.mark.gpu


def bf16_round(X):
    """Round-to-nearest-even of float32 to bfloat16, returned as float64."""
    u = np.ascontiguousarray(X, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def random_tiles(rng, n, tiles, counts_choice=None):
    ids = rng.integers(0, n, size=(tiles, 128), dtype=np.int32)
    counts = rng.integers(0, 33, size=(tiles, 4), dtype=np.int32)
    if counts_choice is not None:
        counts[:] = counts_choice
    return ids, counts


def reference(Xb, ids, counts):
    """[tiles, 128, 64] float64, nan where undefined (unused rows)."""
    nrm = (Xb * Xb).sum(axis=1)
    tiles = ids.shape[0]
    out = np.full((tiles, 128, 64), np.nan)
    for t in range(tiles):
        for j in range(2):
            nn, no = counts[t, 2 * j], counts[t, 2 * j + 1]
            used = [s for s in range(64) if (s < 32 and s < nn) or (s >= 32 and s - 32 < no)]
            sl = ids[t, 64 * j:64 * j + 64]
            for r in used:
                a = sl[r]
                row = np.full(64, np.inf)
                for c in used:
                    b = sl[c]
                    row[c] = nrm[a] + nrm[b] - 2.0 * float(Xb[a] @ Xb[b])
                out[t, 64 * j + r] = row
    return out, nrm


@pytest.mark.parametrize("d", [12, 64, 100, 128, 256])
def test_distance_tiles_match_float64(ctx, d):
    rng = np.random.default_rng(100 + d)
    n, tiles = 3000, 40
    X = (rng.normal(size=(n, d)) * rng.uniform(0.2, 3.0, size=(1, d))).astype(np.float32)
    ids, counts = random_tiles(rng, n, tiles)
    counts[0] = (32, 32, 32, 32)  # full tile
    counts[1] = (0, 0, 1, 0)      # empty and single-row joins
    counts[2] = (5, 3, 31, 1)     # ragged groups of four
    out = ctx.bf16_distance_tiles(X, ids, counts).cpu().numpy().astype(np.float64)
    ref, nrm = reference(bf16_round(X), ids, counts)
    defined = ~np.isnan(ref)
    inf = np.isinf(ref) & defined
    fin = defined & ~inf
    assert np.all(np.isinf(out[inf]) & (out[inf] > 0)), "unused columns must be +inf"
    # FP32 norms and FP32 accumulation of exact BF16 products: error a few ulps
    # of the magnitude |a|^2 + |c|^2
    scale = np.zeros_like(ref)
    for t in range(tiles):
        for j in range(2):
            sl = ids[t, 64 * j:64 * j + 64]
            scale[t, 64 * j:64 * j + 64] = nrm[sl][:, None] + nrm[sl][None, :]
    err = np.abs(out[fin] - ref[fin])
    assert np.all(err <= 1e-5 * scale[fin] + 1e-6), float((err / (scale[fin] + 1e-30)).max())


def test_distance_tiles_one_value_per_pair(ctx):
    """A pair gets the same bits in both orders and in any tile position (the
    merge relies on one distance per pair to drop repeated candidates)."""
    rng = np.random.default_rng(7)
    n, d = 500, 128
    X = rng.normal(size=(n, d)).astype(np.float32) * 4
    base = rng.choice(n, size=64, replace=False).astype(np.int32)
    tiles = 6
    ids = np.zeros((tiles, 128), np.int32)
    for t in range(tiles):
        for j in range(2):
            ids[t, 64 * j:64 * j + 64] = np.roll(base, 7 * t + 13 * j)
    counts = np.full((tiles, 4), 32, np.int32)
    out = ctx.bf16_distance_tiles(X, ids, counts).cpu().numpy()
    val = {}
    for t in range(tiles):
        for j in range(2):
            sl = ids[t, 64 * j:64 * j + 64]
            for r in range(64):
                for c in range(64):
                    key = (min(sl[r], sl[c]), max(sl[r], sl[c]))
                    v = out[t, 64 * j + r, c].view(np.uint32)
                    assert val.setdefault(key, v) == v, key


def test_distance_tiles_rejects_bad_lists(ctx):
    rng = np.random.default_rng(3)
    X = rng.normal(size=(100, 16)).astype(np.float32)
    ids = np.zeros((1, 128), np.int32)
    with pytest.raises(g.HdbError, match="ARG"):
        ctx.bf16_distance_tiles(X, ids, np.array([[33, 0, 0, 0]], np.int32))
    ids[0, 3] = 100
    with pytest.raises(g.HdbError, match="ARG"):
        ctx.bf16_distance_tiles(X, ids, np.array([[4, 0, 0, 0]], np.int32))
    ids[0, 3] = 5
    ctx.bf16_distance_tiles(X, ids, np.array([[4, 0, 0, 0]], np.int32))
    with pytest.raises(g.HdbError, match="ARG"):
        ctx.bf16_distance_tiles(rng.normal(size=(100, 300)).astype(np.float32), ids,
                                np.array([[4, 0, 0, 0]], np.int32))


def test_bf16_nndescent_wide_rows_use_the_mma_sync_join(ctx, oracle):
    """Beyond 256 padded dimensions the BF16 form runs the mma.sync join; its
    graph is valid, sorted and carries the exact FP32 difference sums."""
    rng = np.random.default_rng(17)
    n, d, k = 4000, 300, 32
    centers = rng.uniform(-10, 10, size=(12, d))
    X = (centers[rng.integers(0, 12, n)] + rng.normal(size=(n, d))).astype(np.float32)
    G = ctx.NNDescent(X, k=k, sample_num=16, iterations=6, precision=g.HDB_PREC_BF16)
    ids, dist = (a.cpu().numpy() for a in ctx.knn_split(G))
    assert oracle.validate_knn(ids)
    key = dist.view(np.uint32).astype(np.uint64) << np.uint64(32) | ids.astype(np.uint64)
    assert (np.diff(key, axis=1) > 0).all()
    for i in rng.choice(n, 50, replace=False):
        for j in range(0, k, 5):
            assert np.float32(oracle.diffsum(X[i], X[ids[i, j]])).view(np.uint32) == \
                dist[i, j].view(np.uint32)
    # recall against the exact kNN, beside the plain FP32 form on the same data
    q = np.arange(0, n, 7)
    gt, _ = oracle.bruteforce_knn(X, k, q)
    G32 = ctx.NNDescent(X, k=k, sample_num=16, iterations=6, precision=g.HDB_PREC_FP32)
    ids32 = ctx.knn_split(G32)[0].cpu().numpy()
    rec16, rec32 = oracle.recall(ids[q], gt, k), oracle.recall(ids32[q], gt, k)
    assert rec16 >= rec32 - 0.01, (rec16, rec32)
