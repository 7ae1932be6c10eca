"""NN-Descent quality and the end-to-end pipeline on the GPU."""
import numpy as np
import pytest

from conftest import blobs

pytestmark = pytest.mark.gpu


def _t(x):
    return x.detach().cpu().numpy()


@pytest.mark.parametrize("n,d,k", [(5000, 12, 32), (4000, 32, 16), (3000, 3, 8)])
def test_nndescent_graph_is_valid_and_exact(ctx, oracle, n, d, k):
    X = blobs(n, d, seed=n + d)
    G = ctx.NNDescent(X, k=k, sample_num=k // 2, iterations=6)
    ids, dist = (_t(a) for a in ctx.knn_split(G))
    assert oracle.validate_knn(ids)
    # rows sorted by (distance, id) and every distance is the reference's
    # FP32 difference sum of the pair, bit for bit
    key = dist.view(np.uint32).astype(np.uint64) << np.uint64(32) | ids.astype(np.uint64)
    assert (np.diff(key, axis=1) > 0).all()
    rng = np.random.default_rng(0)
    for i in rng.choice(n, 200, replace=False):
        for j in range(k):
            ref = oracle.diffsum(X[i], X[ids[i, j]])
            assert np.float32(ref).view(np.uint32) == dist[i, j].view(np.uint32)


@pytest.mark.parametrize("n,d,k", [(20000, 12, 32), (8000, 64, 32)])
def test_nndescent_recall_matches_reference_algorithm(ctx, oracle, n, d, k):
    """Recall@k against the FP64 exact kNN within 0.5 pt of the oracle's
    restatement of the reference NN-Descent (same S, iterations)."""
    X = blobs(n, d, seed=7 + d, blobs=20)
    G = ctx.NNDescent(X, k=k, sample_num=16, iterations=6)
    ids, _ = ctx.knn_split(G)
    ids = _t(ids)
    q = np.arange(0, n, 7)
    gt, _ = oracle.bruteforce_knn(X, k, q)
    r_gpu = oracle.recall(ids[q], gt, k)
    oids, _ = oracle.nndescent(X, k, 16, 6)
    r_orc = oracle.recall(oids[q], gt, k)
    assert r_gpu >= r_orc - 0.005, (r_gpu, r_orc)


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_row_ids_of_18_bits(ctx, oracle, prec):
    """200,000 points: row ids need 18 bits, so the target sort of the
    candidate list and the row sorts of the graph stages take two 9-bit
    digit passes (every one of the 512 bins in use).  The graph is still a
    valid, exactly ranked kNN graph and the labels from it equal the
    oracle's on the same graph."""
    from gpu_hdbscan_b200 import HDB_DIST_SQUARED, HDB_PREC_BF16, HDB_PREC_FP32
    n, d, k = 200_000, 8, 16
    X = blobs(n, d, seed=41, blobs=12)
    pc = HDB_PREC_BF16 if prec == "bf16" else HDB_PREC_FP32
    G = ctx.NNDescent(X, k=k, sample_num=8, iterations=6, precision=pc)
    ids, dist = (_t(a) for a in ctx.knn_split(G))
    assert oracle.validate_knn(ids)
    key = dist.view(np.uint32).astype(np.uint64) << np.uint64(32) | ids.astype(np.uint64)
    assert (np.diff(key, axis=1) > 0).all()
    rng = np.random.default_rng(1)
    for i in rng.choice(n, 100, replace=False):
        for j in range(k):
            ref = oracle.diffsum(X[i], X[ids[i, j]])
            assert np.float32(ref).view(np.uint32) == dist[i, j].view(np.uint32)
    labels, stats = ctx.hdbscan_from_knn(G, X, k=k, mpts=k, distance=HDB_DIST_SQUARED)
    _, ref_labels, ncl = oracle.hdbscan_from_knn(ids, dist, X, k)
    np.testing.assert_array_equal(_t(labels), ref_labels)
    assert stats["num_clusters"] == ncl


@pytest.mark.parametrize("distance", ["sqrt", "squared"])
@pytest.mark.parametrize("stab", ["fp32", "fp64"])
def test_pipeline_labels_identical_on_shared_graph(ctx, oracle, distance, stab):
    """Labels of the path after the kNN graph (hdb_run_knn, the HDBSCAN/_new.cu
    flow from a finished graph) equal the oracle's on the same GPU-built graph."""
    from gpu_hdbscan_b200 import HDB_DIST_SQRT, HDB_DIST_SQUARED, HDB_STAB_FP32, HDB_STAB_FP64
    X = blobs(6000, 12, seed=21, blobs=8)
    mode = HDB_DIST_SQRT if distance == "sqrt" else HDB_DIST_SQUARED
    sm = HDB_STAB_FP32 if stab == "fp32" else HDB_STAB_FP64
    G = ctx.NNDescent(X, k=32, sample_num=16, iterations=6)
    labels, stats = ctx.hdbscan_from_knn(G, X, k=32, mpts=32, distance=mode, stability=sm)
    ids, dist = (_t(a) for a in ctx.knn_split(G))
    if distance == "sqrt":
        dist = oracle.fix_distances(X, ids)
    _, ref_labels, ncl = oracle.hdbscan_from_knn(ids, dist, X, 32, fp64=(stab == "fp64"))
    np.testing.assert_array_equal(_t(labels), ref_labels)
    assert stats["num_clusters"] == ncl
    assert ncl >= 2


def test_full_run_labels_are_consistent_with_its_own_graph_quality(ctx, oracle):
    """hdb_run end to end: clusters found on well separated blobs agree with
    the generating blobs (ARI) -- the kNN graph inside is not shared."""
    from sklearn.metrics import adjusted_rand_score
    rng = np.random.default_rng(4)
    centers = rng.uniform(-20, 20, size=(6, 12))
    lab = rng.integers(0, 6, 8000)
    X = (centers[lab] + rng.normal(size=(8000, 12))).astype(np.float32)
    labels, stats = ctx.hdbscan(X, k=32, mpts=32)
    got = labels.numpy()
    assert stats["num_clusters"] == 6
    keep = got >= 0
    assert keep.mean() > 0.8
    assert adjusted_rand_score(lab[keep], got[keep]) > 0.99


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_full_run_labels_equal_oracle_on_its_own_graph(ctx, oracle, prec):
    """hdb_run end to end (hdb_run_with_graph): the labels equal the oracle's
    HDBSCAN of the very kNN graph the same call built -- with device buffers
    and with host buffers (host_io, copies inside the call)."""
    import torch
    from gpu_hdbscan_b200 import HDB_PREC_BF16, HDB_PREC_FP32
    pc = HDB_PREC_BF16 if prec == "bf16" else HDB_PREC_FP32
    X = blobs(4000, 12, seed=3)
    Xd = torch.from_numpy(X).cuda()
    for src in (Xd, X):
        labels, st, G = ctx.hdbscan(src, k=32, mpts=32, precision=pc, want_graph=True)
        assert labels.is_cuda == (src is Xd) and G.is_cuda == (src is Xd)
        g = _t(G)
        ids = np.where(g[:, :, 1] < 0, -g[:, :, 1] - 1, g[:, :, 1]).astype(np.int32)
        assert oracle.validate_knn(ids)
        _, ref, ncl = oracle.hdbscan_from_knn(ids, oracle.fix_distances(X, ids), X, 32)
        np.testing.assert_array_equal(_t(labels), ref)
        assert st["num_clusters"] == ncl and ncl >= 2


def test_pipeline_device_and_host_io_agree(ctx):
    """hdb_run_knn on one graph gives the same labels with device and with
    host buffers."""
    import torch
    X = blobs(4000, 12, seed=3)
    Xd = torch.from_numpy(X).cuda()
    G = ctx.NNDescent(Xd, k=32, sample_num=16)
    ld, _ = ctx.hdbscan_from_knn(G, Xd)
    lh, _ = ctx.hdbscan_from_knn(G.cpu(), X)
    assert not lh.is_cuda
    np.testing.assert_array_equal(lh.numpy(), _t(ld))


def _golden_recall(name):
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                        "ref_nndescent_recall_cg.json")
    with open(path) as f:
        return json.load(f)["sets"][name]


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_recall_on_the_100k_blob_config_is_the_references(ctx, oracle, prec):
    """The 100,000 x 12 blob configuration itself (10 blobs, centres in
    [-10, 10]^12, sigma 1, 5 % noise; k = 32, S = 16, 6 iterations): recall@32
    against the exact FP64 kNN on 3,000 sampled rows is within 0.5 pt of the
    oracle's restatement (0.889, recorded beside the reference's run by
    make_ref_golden.py --nndescent-recall) or better.  The reference's own
    NN-Descent, compiled for sm_100a and run on the same data, recorded 0.0015:
    its graph stays near the random initial one, so the bound it gives is
    trivially met and the restatement is the working anchor.  The BF16 form is
    held to the restatement run in the same form (orc_nndescent_form: BF16
    candidate distances, exact re-rank) within 0.5 pt; what the form itself
    costs against FP32 at d = 12 (0.4-0.6 pt, measured) stays under 1 pt."""
    from gpu_hdbscan_b200 import HDB_PREC_BF16, HDB_PREC_FP32, synth
    ref = _golden_recall("blobs_100k_d12")
    X = synth.generate(synth.WORKLOADS["blobs_100k_d12"])
    q = np.sort(np.random.default_rng(5).choice(len(X), 3000, replace=False))
    gt, _ = oracle.bruteforce_knn(X, 32, q)
    pc = HDB_PREC_BF16 if prec == "bf16" else HDB_PREC_FP32
    ids, _ = ctx.knn_split(ctx.NNDescent(X, k=32, sample_num=16, iterations=6, precision=pc))
    r = oracle.recall(_t(ids)[q], gt, 32)
    assert r >= ref["ref_recall32"] - 0.005, (r, ref)
    if prec == "bf16":
        fids, _ = oracle.nndescent_form(X, "bf16")
        r_form = oracle.recall(fids[q], gt, 32)
        assert r >= r_form - 0.005, (r, r_form)
        assert r >= ref["oracle_recall32"] - 0.010, (r, ref)
    else:
        assert r >= ref["oracle_recall32"] - 0.005, (r, ref)


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_recall_on_a_sample_of_the_20m_x_128_distribution(ctx, oracle, prec):
    """100,000 points drawn from the 20M x 128 mixture (1,000 blobs, sigma in
    [0.5, 1.5], centres in [-20, 20]^128, 5 % noise): recall@32 on 2,000 rows
    within 0.5 pt of the oracle's restatement of the reference NN-Descent (the
    reference itself is compiled for d = 12 only)."""
    from gpu_hdbscan_b200 import HDB_PREC_BF16, HDB_PREC_FP32, synth
    X = synth.sample(synth.WORKLOADS["blobs_20m_d128"], 100_000)
    q = np.sort(np.random.default_rng(6).choice(len(X), 2000, replace=False))
    gt, _ = oracle.bruteforce_knn(X, 32, q)
    oids, _ = oracle.nndescent(X, 32, 16, 6)
    r_orc = oracle.recall(oids[q], gt, 32)
    pc = HDB_PREC_BF16 if prec == "bf16" else HDB_PREC_FP32
    ids, _ = ctx.knn_split(ctx.NNDescent(X, k=32, sample_num=16, iterations=6, precision=pc))
    r = oracle.recall(_t(ids)[q], gt, 32)
    assert r >= r_orc - 0.005, (r, r_orc)
