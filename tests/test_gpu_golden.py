"""The CUDA path against golden outputs of the reference's own code
(tests/golden/ref_*.npz, made by tests/golden/make_ref_golden.py)."""
import glob
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not FILES, reason="no golden fixtures")]


@pytest.fixture(params=FILES, ids=lambda p: os.path.basename(p)[4:-4])
def golden(request):
    d = dict(np.load(request.param))
    with open(request.param[:-4] + ".json") as f:
        return d, json.load(f)


def _t(x):
    return x.detach().cpu().numpy()


def test_cuda_path_matches_reference_outputs(ctx, oracle, golden):
    import torch
    g, meta = golden
    n = meta["n"]
    G = ctx.buildEnhancedKNNG(g["ids"], g["dist"], g["X"])
    np.testing.assert_array_equal(_t(G.antihubs), g["antihubs"])
    np.testing.assert_array_equal(_t(G.nindex), g["nindex"])
    np.testing.assert_array_equal(_t(G.nlist), g["nlist"])
    np.testing.assert_array_equal(_t(G.eweight).view(np.uint32), g["eweight"].view(np.uint32))
    mst, _, _ = ctx.buildMST(G)
    got = _t(mst).copy().view(oracle.MST_EDGE).reshape(-1)
    for mpts in meta["mpts"]:
        ref = g[f"mst_{mpts}"]
        np.testing.assert_array_equal(got["from_node"], ref["from_node"])
        np.testing.assert_array_equal(got["to_node"], ref["to_node"])
        np.testing.assert_array_equal(got["weight"].view(np.uint32), ref["weight"].view(np.uint32))
        hier = _t(ctx.build_Linkage_tree(mst, n)).copy().view(oracle.LINKAGE_NODE).reshape(-1)
        rh = g[f"hier_{mpts}"]
        for f in ("left_node", "right_node", "node_size"):
            np.testing.assert_array_equal(hier[f], rh[f])
        h = torch.from_numpy(rh.view(np.int32).reshape(-1, 4).copy()).cuda()
        labels, ncl, cond, stab = ctx.get_clusters(h, n, mpts, want_tree=True)
        gc = _t(cond).copy().view(oracle.CONDENSED_NODE).reshape(-1)
        rc = g[f"cond_{mpts}"]
        rc = rc[np.lexsort((rc["child"], rc["parent"]))]
        for f in ("parent", "child", "child_size"):
            np.testing.assert_array_equal(gc[f], rc[f])
        np.testing.assert_array_equal(gc["lambda_val"].view(np.uint32), rc["lambda_val"].view(np.uint32))
        gs = _t(stab).copy().view(oracle.STABILITY).reshape(-1)
        np.testing.assert_array_equal(gs["lambda"].view(np.uint32),
                                      g[f"stab_{mpts}"]["lambda"].view(np.uint32))
        np.testing.assert_array_equal(_t(labels), g[f"labels_{mpts}"])


def test_cuda_run_from_knn_matches_reference_labels(ctx, golden):
    """hdb_run_knn (the _new.cu flow from a finished kNN graph) on the fixture's
    graph: labels equal the reference's."""
    import torch
    g, meta = golden
    n = meta["n"]
    Gk = np.zeros((n, 32, 2), np.int32)
    Gk[:, :, 0] = g["dist"].view(np.int32)
    Gk[:, :, 1] = g["ids"]
    from gpu_hdbscan_b200 import HDB_DIST_SQUARED
    for mpts in meta["mpts"]:
        labels, _ = ctx.hdbscan_from_knn(torch.from_numpy(Gk).cuda(), torch.from_numpy(g["X"]).cuda(),
                                         k=32, mpts=mpts, distance=HDB_DIST_SQUARED)
        np.testing.assert_array_equal(_t(labels), g[f"labels_{mpts}"])


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_initial_graph_matches_reference(ctx, oracle, golden, prec):
    """k_init's ids against the reference's initial graph (gpuknn::NNDescent
    with 0 iterations), and ids and distance bits against the oracle's."""
    import gpu_hdbscan_b200 as g_
    from test_oracle_golden import check_initial_graph
    g, meta = golden
    if "ref_init_ids" not in g:
        pytest.skip("the reference NN-Descent is compiled for d = 12 only")
    pc = g_.HDB_PREC_BF16 if prec == "bf16" else g_.HDB_PREC_FP32
    G = ctx.NNDescent(g["X"], k=32, sample_num=16, iterations=0, precision=pc)
    ids, dist = (_t(a) for a in ctx.knn_split(G))
    check_initial_graph(ids, g["ref_init_ids"])
    oids, odist = oracle.nndescent(g["X"], 32, 16, 0)
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(dist.view(np.uint32), odist.view(np.uint32))
