"""The oracle's restatement of gpuknn::KNNMerge (knnmerge.cu:401-437):
initial rows, the merge rounds and input checks, on the CPU."""
import numpy as np
import pytest

from conftest import blobs


def _sets(oracle, n1=1500, n2=1100, d=8, k=16, seed=31):
    X = blobs(n1 + n2, d, seed=seed, blobs=6)
    X1, X2 = X[:n1], X[n1:]
    i1, _ = oracle.nndescent(X1, k, k // 2, 6)
    i2, _ = oracle.nndescent(X2, k, k // 2, 6)
    return X, X1, X2, i1, i2


def test_initial_rows_follow_the_reference_layout(oracle):
    X, X1, X2, i1, i2 = _sets(oracle)
    n1, n2, k = len(X1), len(X2), i1.shape[1]
    h, r = k - k // 2, k // 2
    ids, dist = oracle.knn_merge(X1, i1, X2, i2, sample_num=6, iterations=0)
    assert oracle.validate_knn(ids)
    for row in (0, 1, n1 - 1, n1, n1 + 7, n1 + n2 - 1):
        inb = row >= n1
        local = row - n1 if inb else row
        own = (i2[local, :h] + n1) if inb else i1[local, :h]
        # the other set's ids: xorshift64star(local * r + t) % |other|, repeats advanced
        oth_n, oth_off = (n1, 0) if inb else (n2, n1)
        drawn = []
        for t in range(r):
            lab = oracle.xorshift64star(local * r + t) % oth_n
            while lab + oth_off in drawn:
                lab = (lab + 1) % oth_n
            drawn.append(lab + oth_off)
        assert sorted(ids[row].tolist()) == sorted(own.tolist() + drawn)
        key = dist[row].view(np.uint32).astype(np.uint64) << np.uint64(32) | ids[row].astype(np.uint64)
        assert (np.diff(key) > 0).all()
        for j in range(k):
            ref = oracle.diffsum(X[row], X[ids[row, j]])
            assert np.float32(ref).view(np.uint32) == dist[row, j].view(np.uint32)


def test_merge_rounds_reach_the_recall_of_a_graph_built_on_the_union(oracle):
    X, X1, X2, i1, i2 = _sets(oracle, 2500, 2000, d=12, k=32, seed=32)
    gt, _ = oracle.bruteforce_knn(X, 32)
    ids0, _ = oracle.knn_merge(X1, i1, X2, i2, 12, 0)
    ids, dist = oracle.knn_merge(X1, i1, X2, i2, 12, 11)
    assert oracle.validate_knn(ids)
    r0 = oracle.recall(ids0, gt, 32)
    r = oracle.recall(ids, gt, 32)
    iu, _ = oracle.nndescent(X, 32, 16, 6)
    ru = oracle.recall(iu, gt, 32)
    assert r0 < 0.6 and r > r0 + 0.3
    assert r >= ru - 0.01, (r, ru)


@pytest.mark.parametrize("fault", ["range", "self", "repeat"])
def test_invalid_subgraphs_are_rejected(oracle, fault):
    X, X1, X2, i1, i2 = _sets(oracle)
    bad = i2.copy()
    if fault == "range":
        bad[5, 0] = len(X2)
    elif fault == "self":
        bad[5, 0] = 5
    else:
        bad[5, 1] = bad[5, 0]
    with pytest.raises(ValueError):
        oracle.knn_merge(X1, i1, X2, bad, 6, 2)


def test_sets_need_more_than_k_points(oracle):
    X = blobs(200, 4, seed=1)
    i1, _ = oracle.nndescent(X[:100], 16, 8, 2)
    with pytest.raises(ValueError):
        oracle.knn_merge(X[:100], i1, X[100:110], np.zeros((10, 16), np.int32), 6, 2)
