"""The float MST under the tie order (weight, min id, max id) on the GPU
(hdb_mst_ordered, hdb_params.mst_gpu = HDB_MST_ID_ORDER) against the oracle's
ordered Kruskal, beside the reference's (weight, CSR edge index) order: both
trees bit for bit, the labels of the whole path, and how many tree edges the
two orders choose differently on tie-heavy and on NN-Descent graphs."""
import numpy as np
import pytest

import gpu_hdbscan_b200 as g
from conftest import blobs

pytestmark = pytest.mark.gpu


def _t(x):
    return x.detach().cpu().numpy()


def _records(mst, oracle):
    return _t(mst).copy().view(oracle.MST_EDGE).reshape(-1)


def _same(got, want):
    np.testing.assert_array_equal(got.view(np.int32), want.view(np.int32))


def test_cycle_known_answer(ctx, oracle):
    """4-cycle 0-3-1-2-0 with equal weights, rows 0: [3, 2], 1: [3, 2],
    2: [1, 0], 3: [0, 1]: the edge order closes the cycle with (1,2), the id
    order with (1,3)."""
    G = ctx.graph_from_csr(np.array([0, 2, 4, 6, 8], np.int64),
                           np.array([3, 2, 3, 2, 1, 0, 0, 1], np.int32), np.ones(8, np.float32))
    e, e_in, _ = ctx.buildMST(G, with_in_mst=True, order=g.HDB_ORDER_EDGE)
    i, i_in, _ = ctx.buildMST(G, with_in_mst=True, order=g.HDB_ORDER_IDS)
    assert _t(e).tolist() == [[0, 3, 0x3F800000], [0, 2, 0x3F800000], [1, 3, 0x3F800000]]
    assert _t(i).tolist() == [[0, 2, 0x3F800000], [0, 3, 0x3F800000], [1, 2, 0x3F800000]]
    assert _t(e_in).tolist() == [1, 1, 1, 0, 0, 0, 0, 0]
    assert _t(i_in).tolist() == [1, 1, 0, 1, 0, 0, 0, 0]


def _grid_graph(oracle, n, seed, k=16):
    rng = np.random.default_rng(seed)
    X = np.unique(rng.integers(0, 40, (n, 3)).astype(np.float32), axis=0)
    X = X[rng.permutation(len(X))]
    ids, _ = oracle.bruteforce_knn(X, k)
    ids = ids.astype(np.int32)
    return X, ids, oracle.fix_distances(X, ids)


@pytest.mark.parametrize("source", ["grid", "nndescent"])
def test_both_orders_match_the_oracle(ctx, oracle, source):
    if source == "grid":
        X, ids, dist = _grid_graph(oracle, 20000, 5)
    else:
        X = blobs(20000, 8, seed=29, blobs=12, spread=3.0)
        ids = _t(ctx.knn_split(ctx.NNDescent(X, k=32, sample_num=16))[0])
        dist = oracle.fix_distances(X, ids)
    G = ctx.buildEnhancedKNNG(ids, dist, X)
    ni, nl, ew = _t(G.nindex), _t(G.nlist), _t(G.eweight)
    plain, plain_in, _ = ctx.buildMST(G, with_in_mst=True)
    e, e_in, _ = ctx.buildMST(G, with_in_mst=True, order=g.HDB_ORDER_EDGE)
    i, i_in, rounds = ctx.buildMST(G, with_in_mst=True, order=g.HDB_ORDER_IDS)
    ref_e, ref_e_in = oracle.mst_ordered(ni, nl, ew, oracle.ORDER_EDGE)
    ref_i, ref_i_in = oracle.mst_ordered(ni, nl, ew, oracle.ORDER_IDS)
    _same(_records(plain, oracle), ref_e)
    _same(_records(e, oracle), ref_e)
    _same(_records(i, oracle), ref_i)
    np.testing.assert_array_equal(_t(plain_in).astype(bool), ref_e_in)
    np.testing.assert_array_equal(_t(e_in).astype(bool), ref_e_in)
    np.testing.assert_array_equal(_t(i_in).astype(bool), ref_i_in)
    assert 1 <= rounds <= 64
    differ = int((ref_e_in != ref_i_in).sum()) // 2
    print(f"{source}: {len(X)} points, {differ} of {len(X) - 1} MST edges differ between orders")
    if source == "grid":
        assert differ > 0


def test_run_labels_under_the_id_order(ctx, oracle):
    """hdb_run_knn with mst_gpu = HDB_MST_ID_ORDER: labels equal the oracle's
    path with its MST under (weight, min id, max id)."""
    X = blobs(6000, 8, seed=31, blobs=8, spread=3.0)
    Gk = ctx.NNDescent(X, k=32, sample_num=16)
    ids = _t(ctx.knn_split(Gk)[0])
    dist = oracle.fix_distances(X, ids)
    for order, mode in ((oracle.ORDER_EDGE, g.HDB_MST_FLOAT), (oracle.ORDER_IDS, g.HDB_MST_ID_ORDER)):
        labels, st = ctx.hdbscan_from_knn(Gk, X, k=32, mpts=16, mst_gpu=mode)
        _, ref, ncl = oracle.hdbscan_from_knn(ids, dist, X, 16, order=order)
        np.testing.assert_array_equal(_t(labels), ref)
        assert st["num_clusters"] == ncl and ncl >= 2


def test_batched_id_order_is_per_instance(ctx):
    import torch
    Xs = [torch.from_numpy(blobs(n, d, seed=n, blobs=4, spread=3.0)).cuda()
          for n, d in [(2000, 4), (900, 4), (3000, 4), (500, 4)]]
    labels, ncl, _, graphs = ctx.hdbscan_batched(Xs, k=16, mpts=8, sample_num=8,
                                                 want_graphs=True, mst_gpu=g.HDB_MST_ID_ORDER)
    for X, lab, nc, G in zip(Xs, labels, ncl, graphs):
        ref, st = ctx.hdbscan_from_knn(G, X, k=16, mpts=8, mst_gpu=g.HDB_MST_ID_ORDER)
        np.testing.assert_array_equal(_t(lab), _t(ref))
        assert nc == st["num_clusters"]


def test_order_argument_is_checked(ctx):
    G = ctx.graph_from_csr(np.array([0, 1, 2], np.int64), np.array([1, 0], np.int32),
                           np.ones(2, np.float32))
    with pytest.raises(g.HdbError):
        ctx.buildMST(G, order=2)
    with pytest.raises(g.HdbError):
        ctx.hdbscan(blobs(500, 4, seed=1), k=8, mpts=4, mst_gpu=3)
