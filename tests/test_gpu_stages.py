"""Stage-by-stage parity of the CUDA path against the oracle (bit-exact for
integer/index work and for the FP32 weights, which follow the reference's
own rounding)."""
import numpy as np
import pytest

from conftest import blobs

pytestmark = pytest.mark.gpu

CASES = [  # (n, d, k, seed)
    (600, 4, 8, 11),
    (3000, 12, 32, 12),
    (2500, 7, 16, 13),
]


def _knn(oracle, X, k):
    S = max(1, k // 2)
    ids, dist = oracle.nndescent(X, k, S, 6)
    return ids, dist


def _t(x):
    return x.detach().cpu().numpy()


@pytest.fixture(scope="module", params=CASES, ids=lambda c: f"n{c[0]}_d{c[1]}_k{c[2]}")
def case(request, oracle):
    n, d, k, seed = request.param
    X = blobs(n, d, seed)
    ids, dist = _knn(oracle, X, k)
    sq = dist
    fd = oracle.fix_distances(X, ids)
    return dict(X=X, ids=ids, dist=sq, fdist=fd, k=k)


def test_enhanced_knng_matches_oracle(ctx, oracle, case):
    for dist in (case["dist"], case["fdist"]):
        g = ctx.buildEnhancedKNNG(case["ids"], dist, case["X"])
        nindex, nlist, ew, ah = oracle.enhanced_knng(case["ids"], dist, case["X"])
        assert g.edges == len(nlist)
        np.testing.assert_array_equal(_t(g.antihubs), ah)
        np.testing.assert_array_equal(_t(g.nindex), nindex)
        np.testing.assert_array_equal(_t(g.nlist), nlist)
        np.testing.assert_array_equal(_t(g.eweight).view(np.uint32), ew.view(np.uint32))


def test_mst_matches_kruskal(ctx, oracle, case):
    g = ctx.buildEnhancedKNNG(case["ids"], case["fdist"], case["X"])
    mst, inm, rounds = ctx.buildMST(g, with_in_mst=True)
    nindex, nlist, ew, _ = oracle.enhanced_knng(case["ids"], case["fdist"], case["X"])
    ref_in = oracle.kruskal(nindex, nlist, ew)
    ref = oracle.sort_edges(oracle.build_mst(nindex, nlist, ew, ref_in))
    np.testing.assert_array_equal(_t(inm).astype(bool), ref_in)
    got = _t(mst).copy().view(oracle.MST_EDGE).reshape(-1)
    np.testing.assert_array_equal(got["from_node"], ref["from_node"])
    np.testing.assert_array_equal(got["to_node"], ref["to_node"])
    np.testing.assert_array_equal(got["weight"].view(np.uint32), ref["weight"].view(np.uint32))
    assert 1 <= rounds <= 64


def test_sort_edges_is_stable_by_weight(ctx, oracle):
    import torch
    rng = np.random.default_rng(5)
    m = 20000
    e = np.zeros(m, oracle.MST_EDGE)
    e["from_node"] = np.arange(m)
    e["to_node"] = rng.integers(0, 1000, m)
    e["weight"] = rng.integers(0, 50, m).astype(np.float32) / 7  # many ties
    ref = oracle.sort_edges(e)
    t = torch.from_numpy(e.view(np.int32).reshape(m, 3).copy()).cuda()
    ctx.sort_edges(t)
    got = _t(t).copy().view(oracle.MST_EDGE).reshape(-1)
    np.testing.assert_array_equal(got, ref)


def _ref_tree(oracle, case, mpts, fp64=False):
    nindex, nlist, ew, _ = oracle.enhanced_knng(case["ids"], case["fdist"], case["X"])
    ref = oracle.sort_edges(oracle.build_mst(nindex, nlist, ew, oracle.kruskal(nindex, nlist, ew)))
    n = len(case["X"])
    hier = oracle.linkage_tree(ref, n)
    cond = oracle.condensed_tree(hier, n, mpts)
    stab, s64 = oracle.stability(cond)
    labels, ncl = oracle.get_clusters(cond, stab, n, s64 if fp64 else None)
    return ref, hier, cond, stab, labels, ncl


def test_linkage_tree_matches_oracle(ctx, oracle, case):
    import torch
    ref, hier, *_ = _ref_tree(oracle, case, case["k"])
    n = len(case["X"])
    t = torch.from_numpy(ref.view(np.int32).reshape(-1, 3).copy()).cuda()
    got = _t(ctx.build_Linkage_tree(t, n)).copy().view(oracle.LINKAGE_NODE).reshape(-1)
    for f in ("left_node", "right_node", "node_size"):
        np.testing.assert_array_equal(got[f], hier[f], err_msg=f)
    np.testing.assert_array_equal(got["weight"].view(np.uint32), hier["weight"].view(np.uint32))


@pytest.mark.parametrize("mpts_div", [1, 2])
def test_condensed_tree_stability_labels_match_oracle(ctx, oracle, case, mpts_div):
    import torch
    mpts = max(2, case["k"] // mpts_div)
    ref, hier, cond, stab, labels, ncl = _ref_tree(oracle, case, mpts)
    n = len(case["X"])
    h = torch.from_numpy(hier.view(np.int32).reshape(-1, 4).copy()).cuda()
    glabels, gncl, gcond, gstab = ctx.get_clusters(h, n, mpts, want_tree=True)
    gc = _t(gcond).copy().view(oracle.CONDENSED_NODE).reshape(-1)
    order = np.lexsort((cond["child"], cond["parent"]))
    rc = cond[order]
    assert len(gc) == len(rc)
    for f in ("parent", "child", "child_size"):
        np.testing.assert_array_equal(gc[f], rc[f], err_msg=f)
    np.testing.assert_array_equal(gc["lambda_val"].view(np.uint32), rc["lambda_val"].view(np.uint32))
    gs = _t(gstab).copy().view(oracle.STABILITY).reshape(-1)
    np.testing.assert_array_equal(gs["cluster_id"], stab["cluster_id"])
    np.testing.assert_array_equal(gs["lambda"].view(np.uint32), stab["lambda"].view(np.uint32))
    assert gncl == ncl
    np.testing.assert_array_equal(_t(glabels), labels)


def test_fp64_stability_labels_match_oracle(ctx, oracle, case):
    import torch
    mpts = case["k"]
    ref, hier, cond, stab, labels, ncl = _ref_tree(oracle, case, mpts, fp64=True)
    n = len(case["X"])
    h = torch.from_numpy(hier.view(np.int32).reshape(-1, 4).copy()).cuda()
    from gpu_hdbscan_b200 import HDB_STAB_FP64
    glabels, gncl, _, _ = ctx.get_clusters(h, n, mpts, stability=HDB_STAB_FP64)
    assert gncl == ncl
    np.testing.assert_array_equal(_t(glabels), labels)


def test_fix_distances_matches_reference_rounding(ctx, oracle, case):
    got = _t(ctx.fix_distances(case["X"], case["ids"]))
    np.testing.assert_array_equal(got.view(np.uint32), case["fdist"].view(np.uint32))


@pytest.mark.parametrize("mpts", [2, 7, 300, 4000, 20000])
def test_stability_with_long_runs_of_equal_rows(ctx, oracle, mpts):
    """Large mpts makes whole subtrees fall out at one lambda, so one chain
    node contributes thousands of equal rows; the FP32 sum must still equal the
    reference's row-by-row sum bit for bit (and FP64 mode the oracle's)."""
    import torch
    n = 30000
    X = blobs(n, 5, seed=77, blobs=12, noise=0.3)
    ids, _ = oracle.nndescent(X, 16, 8, 4)
    fd = oracle.fix_distances(X, ids)
    nindex, nlist, ew, _ = oracle.enhanced_knng(ids, fd, X)
    mst = oracle.sort_edges(oracle.build_mst(nindex, nlist, ew, oracle.kruskal(nindex, nlist, ew)))
    hier = oracle.linkage_tree(mst, n)
    cond = oracle.condensed_tree(hier, n, mpts)
    stab, s64 = oracle.stability(cond)
    h = torch.from_numpy(hier.view(np.int32).reshape(-1, 4).copy()).cuda()
    from gpu_hdbscan_b200 import HDB_STAB_FP64
    for mode, ref in ((0, None), (HDB_STAB_FP64, s64)):
        labels, ncl, _, gstab = ctx.get_clusters(h, n, mpts, stability=mode, want_tree=True)
        gs = _t(gstab).copy().view(oracle.STABILITY).reshape(-1)
        np.testing.assert_array_equal(gs["lambda"].view(np.uint32), stab["lambda"].view(np.uint32))
        rl, rn = oracle.get_clusters(cond, stab, n, ref)
        assert ncl == rn
        np.testing.assert_array_equal(_t(labels), rl)
