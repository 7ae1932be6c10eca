"""hdb_run_batched: many independent instances in shared launches.  Every
instance's labels equal the oracle's (and the single-instance GPU path's) on
the kNN graph the batch built for it, and its initial graph equals the one a
run on that instance alone starts from."""
import numpy as np
import pytest

import gpu_hdbscan_b200 as g
from conftest import blobs

pytestmark = pytest.mark.gpu


def _t(x):
    return x.detach().cpu().numpy()


def instances(seed=0):
    """Uneven sizes and dimensions, interleaved (groups by d are formed inside)."""
    spec = [(40, 3), (1500, 8), (100, 12), (3000, 3), (333, 8), (2500, 12), (17 + 1, 3),
            (800, 8), (5000, 12), (60, 8), (1200, 3)]
    out = []
    for i, (n, d) in enumerate(spec):
        # overlapping blobs for the small instances, so their exact kNN graphs
        # stay connected; separated ones where the antihub clique joins them
        spread = 2.5 if n < 500 else 10.0
        out.append(blobs(n, d, seed=seed * 100 + i, blobs=3 + i % 4, spread=spread))
    return out


@pytest.mark.parametrize("distance", ["sqrt", "squared"])
def test_batched_labels_match_oracle_per_instance(ctx, oracle, distance):
    Xs = instances()
    mode = g.HDB_DIST_SQRT if distance == "sqrt" else g.HDB_DIST_SQUARED
    labels, ncl, stats, graphs = ctx.hdbscan_batched(Xs, k=16, mpts=16, sample_num=8,
                                                     distance=mode, want_graphs=True)
    assert stats["num_clusters"] == sum(ncl)
    for X, lab, nc, G in zip(Xs, labels, ncl, graphs):
        G = G.numpy()
        ids = np.where(G[..., 1] < 0, -G[..., 1] - 1, G[..., 1]).astype(np.int32)
        assert oracle.validate_knn(ids) and ids.max() < len(X)
        dist = oracle.fix_distances(X, ids) if distance == "sqrt" else G[..., 0].view(np.float32)
        _, ref, rnc = oracle.hdbscan_from_knn(ids, dist, X, 16)
        np.testing.assert_array_equal(lab.numpy(), ref)
        assert nc == rnc


def test_batched_equals_single_instance_path_on_device(ctx):
    import torch
    Xs = [torch.from_numpy(X).cuda() for X in instances(seed=3)]
    labels, ncl, _, graphs = ctx.hdbscan_batched(Xs, k=16, mpts=8, sample_num=8, want_graphs=True)
    assert labels[0].is_cuda and graphs[0].is_cuda
    for X, lab, nc, G in zip(Xs, labels, ncl, graphs):
        ref, st = ctx.hdbscan_from_knn(G, X, k=16, mpts=8)
        np.testing.assert_array_equal(_t(lab), _t(ref))
        assert nc == st["num_clusters"]


def test_batched_initial_graph_is_the_single_instance_one(ctx):
    """With zero iterations the kNN graph is the hash-seeded initial graph:
    instance-local positions make it the one hdb_nndescent builds alone."""
    Xs = instances(seed=5)
    _, _, _, graphs = ctx.hdbscan_batched(Xs, k=16, mpts=16, sample_num=8, iterations=0,
                                          want_graphs=True)
    for X, G in zip(Xs, graphs):
        solo = _t(ctx.NNDescent(X, k=16, sample_num=8, iterations=0))
        np.testing.assert_array_equal(G.numpy(), solo)


def test_batched_contiguous_and_scattered_inputs_agree(ctx):
    """Instances that already sit back to back in one buffer are used in place;
    separate buffers are packed by a kernel -- same graphs, same labels."""
    import torch
    Xs = [X for X in instances(seed=7) if X.shape[1] == 8]
    whole = torch.from_numpy(np.concatenate(Xs)).cuda()
    views, o = [], 0
    for X in Xs:
        views.append(whole[o:o + len(X)])
        o += len(X)
    sep = [torch.from_numpy(X).cuda() for X in Xs]
    la, _, _, ga = ctx.hdbscan_batched(views, k=16, mpts=16, sample_num=8, iterations=0,
                                       want_graphs=True)
    lb, _, _, gb = ctx.hdbscan_batched(sep, k=16, mpts=16, sample_num=8, iterations=0,
                                       want_graphs=True)
    for a, b in zip(ga, gb):
        np.testing.assert_array_equal(_t(a), _t(b))
    for a, b in zip(la, lb):
        np.testing.assert_array_equal(_t(a), _t(b))


def test_batched_bf16_form(ctx, oracle):
    Xs = [blobs(n, d, seed=n, blobs=6, spread=20.0) for n, d in [(3000, 64), (1500, 32),
                                                                   (4000, 64), (900, 32)]]
    labels, ncl, _, graphs = ctx.hdbscan_batched(Xs, k=32, mpts=32, precision=g.HDB_PREC_BF16,
                                                 want_graphs=True)
    for X, lab, G in zip(Xs, labels, graphs):
        G = G.numpy()
        ids = np.where(G[..., 1] < 0, -G[..., 1] - 1, G[..., 1]).astype(np.int32)
        assert oracle.validate_knn(ids)
        _, ref, _ = oracle.hdbscan_from_knn(ids, oracle.fix_distances(X, ids), X, 32)
        np.testing.assert_array_equal(lab.numpy(), ref)


def test_batched_argument_errors(ctx):
    Xs = instances()
    with pytest.raises(g.HdbError, match="ARG"):
        ctx.hdbscan_batched(Xs + [blobs(16, 3, seed=1)], k=16, mpts=16, sample_num=8)
    with pytest.raises(g.HdbError, match="ARG"):
        ctx.hdbscan_batched(Xs, k=16, mpts=17, sample_num=8)
    labels, ncl, _ = ctx.hdbscan_batched(Xs[:2], k=16, mpts=16, sample_num=8)
    assert len(labels) == 2  # the context still works


def _two_group_graph():
    """kNN lists that stay inside two groups of 50 points; every antihub falls
    in the first group (equal degrees, ties by index), so the second group is
    unreachable: the reference stops on it with "MST montada incorretamente"
    (mst.cu:317-323)."""
    n, k = 100, 16
    ids = np.zeros((n, k), np.int32)
    for g0 in (0, 50):
        for i in range(50):
            ids[g0 + i] = [g0 + (i + s) % 50 for s in range(1, k + 1)]
    X = np.random.default_rng(0).normal(size=(n, 2)).astype(np.float32)
    G = np.zeros((n, k, 2), np.int32)
    G[..., 0] = np.ones((n, k), np.float32).view(np.int32)
    G[..., 1] = ids
    return G, X


def test_batched_disconnected_instance_fails_alone(ctx, oracle):
    """An instance with a disconnected enhanced kNN graph gets status
    HDB_ERR_DISCONNECTED and labels -1; the other instances of the batch
    complete with the oracle's labels."""
    Xs, Gs = [], []
    for i, n in enumerate((300, 0, 500, 0, 250)):
        if n == 0:
            G, X = _two_group_graph()
        else:
            X = blobs(n, 2, seed=40 + i, spread=2.5)
            G = ctx.NNDescent(X, k=16, sample_num=8).cpu().numpy()
        Xs.append(X)
        Gs.append(G)
    kw = dict(k=16, mpts=8)
    with pytest.raises(g.HdbError, match="DISCONNECTED"):
        ctx.hdbscan_batched_from_knn(Gs, Xs, **kw)
    labels, ncl, st = ctx.hdbscan_batched_from_knn(Gs, Xs, strict=False, **kw)
    D = g._lib.HDB_ERR_DISCONNECTED
    assert st["instance_status"] == [0, D, 0, D, 0]
    for i, (G, X) in enumerate(zip(Gs, Xs)):
        ids = np.where(G[..., 1] < 0, -G[..., 1] - 1, G[..., 1]).astype(np.int32)
        if st["instance_status"][i]:
            assert (labels[i].numpy() == -1).all() and ncl[i] == 0
            with pytest.raises(RuntimeError):
                oracle.hdbscan_from_knn(ids, oracle.fix_distances(X, ids), X, 8)
            continue
        _, ref, rnc = oracle.hdbscan_from_knn(ids, oracle.fix_distances(X, ids), X, 8)
        np.testing.assert_array_equal(labels[i].numpy(), ref)
        assert ncl[i] == rnc


def test_batched_from_knn_reproduces_reference_golden_labels(ctx):
    """The reference's own fixtures (tests/golden) as one batch through
    hdb_run_knn_batched: every instance's labels equal the reference's."""
    import glob
    import json
    import os
    files = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))
    if not files:
        pytest.skip("no golden fixtures")
    fx = [(dict(np.load(f)), json.load(open(f[:-4] + ".json"))) for f in files]
    batches = 0
    for mpts in sorted({v for _, m in fx for v in m["mpts"]}):
        Gs, Xs, refs = [], [], []
        for d, m in fx:
            if mpts not in m["mpts"]:
                continue
            G = np.zeros(d["ids"].shape + (2,), np.int32)
            G[..., 0] = d["dist"].view(np.int32)
            G[..., 1] = d["ids"]
            Gs.append(G)
            Xs.append(d["X"])
            refs.append(d[f"labels_{mpts}"])
        labels, _, _ = ctx.hdbscan_batched_from_knn(Gs, Xs, k=32, mpts=mpts,
                                                     distance=g.HDB_DIST_SQUARED)
        for lab, ref in zip(labels, refs):
            np.testing.assert_array_equal(lab.numpy(), ref)
        batches += len(Gs) > 1
    assert batches >= 1  # at least one mpts shared by several fixtures
