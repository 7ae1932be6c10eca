"""The two tie orders of the float MST in the oracle: the reference's
(weight, CSR edge index) of cpuMST (HDBSCAN/mst/mst.cu:34-78) and
(weight, min id, max id, edge index).  A hand-built graph where they choose
different trees, the edge order against the reference's own Kruskal +
buildMST + sort_edges restatement, and the id order against a plain-Python
Kruskal on tie-heavy graphs."""
import glob
import os

import numpy as np
import pytest

# 4-cycle 0-3-1-2-0, every weight 1.  Rows list their neighbours as
# 0: [3, 2], 1: [3, 2], 2: [1, 0], 3: [0, 1] (symmetric CSR).
CYCLE = dict(nindex=np.array([0, 2, 4, 6, 8], np.int64),
             nlist=np.array([3, 2, 3, 2, 1, 0, 0, 1], np.int32),
             eweight=np.ones(8, np.float32))


def _edges(mst):
    return [(int(e["from_node"]), int(e["to_node"]), float(e["weight"])) for e in mst]


def test_cycle_known_answer(oracle):
    """The edge order takes (0,3), (0,2) and (1,3) -- row 1's entries in list
    order, so its second, (1,2), closes the cycle; the id order takes (1,2)
    before (1,3)."""
    e_mst, e_in = oracle.mst_ordered(**CYCLE, order=oracle.ORDER_EDGE)
    i_mst, i_in = oracle.mst_ordered(**CYCLE, order=oracle.ORDER_IDS)
    assert _edges(e_mst) == [(0, 3, 1.0), (0, 2, 1.0), (1, 3, 1.0)]
    assert _edges(i_mst) == [(0, 2, 1.0), (0, 3, 1.0), (1, 2, 1.0)]
    assert e_in.tolist() == [True, True, True, False, False, False, False, False]
    assert i_in.tolist() == [True, True, False, True, False, False, False, False]


def _py_kruskal_ids(nindex, nlist, ew):
    """Independent restatement: sort (w, min, max, j), union-find."""
    n = len(nindex) - 1
    cand = []
    for i in range(n):
        for j in range(nindex[i], nindex[i + 1]):
            t = int(nlist[j])
            if t > i:
                cand.append((float(ew[j]) + 0.0, i, t, j))
    cand.sort()
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    out = []
    for w, a, b, j in cand:
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[ra] = rb
            out.append((a, b, j))
    return out


def _tie_graph(oracle, n, seed):
    """kNN graph of points on a small integer grid: many equal distances, so
    many equal core distances and MRD weights."""
    rng = np.random.default_rng(seed)
    X = rng.integers(0, 7, (n, 3)).astype(np.float32) + rng.integers(0, 3, (n, 1)).astype(np.float32)
    X = np.unique(X, axis=0)
    X = X[rng.permutation(len(X))]
    k = 8
    ids, _ = oracle.bruteforce_knn(X, k)
    ids = ids.astype(np.int32)
    dist = oracle.fix_distances(X, ids)
    return X, ids, dist, oracle.enhanced_knng(ids, dist, X)[:3]


@pytest.mark.parametrize("seed", [1, 2])
def test_orders_on_a_tie_heavy_graph(oracle, seed):
    X, ids, dist, (ni, nl, ew) = _tie_graph(oracle, 400, seed)
    n = len(ni) - 1
    # edge order = the reference's Kruskal, buildMST and stable sort
    e_mst, e_in = oracle.mst_ordered(ni, nl, ew, oracle.ORDER_EDGE)
    ref_in = oracle.kruskal(ni, nl, ew)
    ref = oracle.sort_edges(oracle.build_mst(ni, nl, ew, ref_in))
    np.testing.assert_array_equal(e_in, ref_in)
    np.testing.assert_array_equal(e_mst.view(np.int32), ref.view(np.int32))
    # id order = an independent Kruskal under (w, min id, max id, j)
    i_mst, i_in = oracle.mst_ordered(ni, nl, ew, oracle.ORDER_IDS)
    want = _py_kruskal_ids(ni, nl, ew)
    assert [(int(e["from_node"]), int(e["to_node"])) for e in i_mst] == [(a, b) for a, b, _ in want]
    assert sorted(j for _, _, j in want) == np.flatnonzero(i_in).tolist()
    # any two MSTs share the weight multiset; the trees differ on ties only
    np.testing.assert_array_equal(np.sort(e_mst["weight"]), np.sort(i_mst["weight"]))
    assert len(i_mst) == n - 1
    differ = int((e_in != i_in).sum()) // 2
    assert differ > 0  # the grid's ties leave the choice open somewhere


def test_pipeline_with_the_id_order(oracle):
    """End to end from a kNN graph: the MST returned under the id order is the
    ordered Kruskal's, and the edge order reproduces the reference call."""
    X, ids, dist, (ni, nl, ew) = _tie_graph(oracle, 400, 3)
    mst_e, lab_e, ncl_e = oracle.hdbscan_from_knn(ids, dist, X, 8)
    mst_e2, lab_e2, _ = oracle.hdbscan_from_knn(ids, dist, X, 8, order=oracle.ORDER_EDGE)
    np.testing.assert_array_equal(mst_e.view(np.int32), mst_e2.view(np.int32))
    np.testing.assert_array_equal(lab_e, lab_e2)
    mst_i, lab_i, _ = oracle.hdbscan_from_knn(ids, dist, X, 8, order=oracle.ORDER_IDS)
    want, _ = oracle.mst_ordered(ni, nl, ew, oracle.ORDER_IDS)
    np.testing.assert_array_equal(mst_i.view(np.int32), want.view(np.int32))
    assert lab_i.shape == lab_e.shape


GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.rsplit("/", 1)[-1][4:-4])
def test_orders_on_the_reference_fixtures(oracle, path):
    """The edge order reproduces the reference's own sorted MST (cpuMST +
    buildMST + sort_edges output stored in the fixture); the id order spans
    the same weight multiset and differs only on tied weights."""
    g = dict(np.load(path))
    ref = next(g[k] for k in sorted(g) if k.startswith("mst_"))
    e_mst, e_in = oracle.mst_ordered(g["nindex"], g["nlist"], g["eweight"], oracle.ORDER_EDGE)
    np.testing.assert_array_equal(e_mst.view(np.int32), ref.view(np.int32))
    i_mst, i_in = oracle.mst_ordered(g["nindex"], g["nlist"], g["eweight"], oracle.ORDER_IDS)
    np.testing.assert_array_equal(np.sort(i_mst["weight"]), np.sort(ref["weight"]))
    w = g["eweight"][e_in != i_in]
    if len(w):
        # every edge the orders disagree on has a weight that at least two
        # undirected edges carry (each appears twice in the symmetric CSR)
        vals, counts = np.unique(g["eweight"], return_counts=True)
        tied = set(vals[counts > 2].tolist())
        assert all(float(x) in tied for x in w)
