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
