"""KNNMerge on the GPU (hdb_knn_merge, gpuknn::KNNMerge knnmerge.cu:401-437)
against the oracle's restatement: the initial graph bit for bit, the merged
graph by recall (the merge rounds race like NN-Descent's), input checks."""
import numpy as np
import pytest

from conftest import blobs

pytestmark = pytest.mark.gpu


def _t(x):
    return x.detach().cpu().numpy()


def _subgraphs(ctx, n1, n2, d, k, seed):
    X = blobs(n1 + n2, d, seed=seed, blobs=8)
    X1, X2 = X[:n1], X[n1:]
    G1 = ctx.NNDescent(X1, k=k, sample_num=k // 2, iterations=6)
    G2 = ctx.NNDescent(X2, k=k, sample_num=k // 2, iterations=6)
    return X, X1, X2, G1, G2


def _ids(ctx, G):
    return _t(ctx.knn_split(G)[0])


@pytest.mark.parametrize("n1,n2,d,k", [(3000, 2200, 12, 32), (1500, 1700, 40, 16), (600, 400, 5, 15)])
def test_initial_graph_equals_the_oracles(ctx, oracle, n1, n2, d, k):
    """iterations = 0: the rows InitRandomBlockedKNNGraph builds (own half old,
    other set's half new), distances and order bit for bit."""
    X, X1, X2, G1, G2 = _subgraphs(ctx, n1, n2, d, k, seed=n1 + d)
    S = min(12, k // 2)
    G = ctx.KNNMerge(X1, G1, X2, G2, sample_num=S, iterations=0)
    ids, dist = (_t(a) for a in ctx.knn_split(G))
    rids, rdist = oracle.knn_merge(X1, _ids(ctx, G1), X2, _ids(ctx, G2), S, 0)
    np.testing.assert_array_equal(ids, rids)
    np.testing.assert_array_equal(dist.view(np.uint32), rdist.view(np.uint32))
    lab = _t(G)[:, :, 1]
    inb = np.arange(n1 + n2)[:, None] >= n1
    np.testing.assert_array_equal(lab >= 0, (ids >= n1) != inb)


@pytest.mark.parametrize("n1,n2,d", [(12000, 8000, 12), (5000, 6000, 64)])
def test_merged_graph_matches_the_oracles_recall(ctx, oracle, n1, n2, d):
    """11 merge rounds with 12 samples (MERGE_ITERATION, MERGE_SAMPLE_NUM):
    a valid graph with exact FP32 distances whose recall@32 against the FP64
    exact kNN is within 0.5 pt of the oracle's merge of the same subgraphs."""
    k = 32
    X, X1, X2, G1, G2 = _subgraphs(ctx, n1, n2, d, k, seed=7 + d)
    G = ctx.KNNMerge(X1, G1, X2, G2)
    ids, dist = (_t(a) for a in ctx.knn_split(G))
    assert oracle.validate_knn(ids)
    key = dist.view(np.uint32).astype(np.uint64) << np.uint64(32) | ids.astype(np.uint64)
    assert (np.diff(key, axis=1) > 0).all()
    rng = np.random.default_rng(0)
    for i in rng.choice(n1 + n2, 100, replace=False):
        for j in range(k):
            ref = oracle.diffsum(X[i], X[ids[i, j]])
            assert np.float32(ref).view(np.uint32) == dist[i, j].view(np.uint32)
    q = np.arange(0, n1 + n2, 7)
    gt, _ = oracle.bruteforce_knn(X, k, q)
    r_gpu = oracle.recall(ids[q], gt, k)
    rids, _ = oracle.knn_merge(X1, _ids(ctx, G1), X2, _ids(ctx, G2), 12, 11)
    r_orc = oracle.recall(rids[q], gt, k)
    G0 = ctx.KNNMerge(X1, G1, X2, G2, iterations=0)
    r0 = oracle.recall(_ids(ctx, G0)[q], gt, k)
    assert r_gpu >= r_orc - 0.005, (r_gpu, r_orc)
    assert r_gpu > r0 + 0.2, (r_gpu, r0)


@pytest.mark.parametrize("fault,match", [("range", "outside"), ("self", "itself"),
                                         ("repeat", "repeats")])
def test_invalid_subgraphs_are_rejected(ctx, fault, match):
    from gpu_hdbscan_b200 import HdbError, _lib
    X, X1, X2, G1, G2 = _subgraphs(ctx, 800, 700, 6, 16, seed=3)
    bad = G2.clone()
    if fault == "range":
        bad[5, 0, 1] = 700
    elif fault == "self":
        bad[5, 0, 1] = 5
    else:
        bad[5, 1, 1] = bad[5, 0, 1]
    with pytest.raises(HdbError, match=match) as e:
        ctx.KNNMerge(X1, G1, X2, bad, sample_num=6)
    assert e.value.status == _lib.HDB_ERR_ARG
    # the context stays usable
    G = ctx.KNNMerge(X1, G1, X2, G2, sample_num=6, iterations=2)
    from oracle import oracle as O
    assert O.validate_knn(_ids(ctx, G))


def test_host_inputs_give_the_device_result(ctx):
    """KNNMergeFromHost (knnmerge.cu:478-530): host arrays in, the same graph."""
    X, X1, X2, G1, G2 = _subgraphs(ctx, 900, 1000, 10, 32, seed=9)
    Gd = _t(ctx.KNNMerge(X1, G1, X2, G2, iterations=0))
    Gh = _t(ctx.KNNMerge(np.asarray(X1), _t(G1), np.asarray(X2), _t(G2), iterations=0))
    np.testing.assert_array_equal(Gd, Gh)


def test_argument_errors(ctx):
    from gpu_hdbscan_b200 import HdbError
    X, X1, X2, G1, G2 = _subgraphs(ctx, 300, 200, 4, 16, seed=2)
    with pytest.raises(HdbError, match="more than k"):
        ctx.KNNMerge(X1, G1, X2[:16], G2[:16], sample_num=6)
    with pytest.raises(HdbError):
        ctx.KNNMerge(X1, G1, X2, G2, sample_num=9)  # 2 * 9 > k
    with pytest.raises(ValueError):
        ctx.KNNMerge(X1, G1, X2[:, :3], G2)
