"""hdb_core_sg (build_CoreSG, core-sg.cu) against the oracle, bit for bit:
on the reference's golden kNN graphs and MSTs, and on a graph and MST built
on the GPU with squared distances."""
import glob
import json
import os

import numpy as np
import pytest

import gpu_hdbscan_b200 as g
from conftest import blobs

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))


def _t(x):
    return x.detach().cpu().numpy()


def check_same(ctx, oracle, ids, dist, X, mst):
    sg = ctx.build_CoreSG(ids, dist, X, mst)
    rn, rl, rw = oracle.core_sg(ids, dist, X, mst)
    assert sg.nodes == len(ids) and sg.edges == len(rl)
    np.testing.assert_array_equal(_t(sg.nindex), rn)
    np.testing.assert_array_equal(_t(sg.nlist), rl)
    np.testing.assert_array_equal(_t(sg.eweight).view(np.uint32), rw.view(np.uint32))


@pytest.mark.parametrize("path", FILES, ids=lambda p: os.path.basename(p)[4:-4])
def test_core_sg_on_reference_graphs(ctx, oracle, path):
    """On the reference's fixtures the GPU core-SG equals the reference's own
    (Union_kNNG_MST + update_core_sg_weights, stored by make_ref_golden.py)."""
    d = dict(np.load(path))
    check_same(ctx, oracle, d["ids"], d["dist"], d["X"], d["mst_32"])
    sg = ctx.build_CoreSG(d["ids"], d["dist"], d["X"], d["mst_32"])
    np.testing.assert_array_equal(_t(sg.nindex), d["coresg_nindex"])
    np.testing.assert_array_equal(_t(sg.nlist), d["coresg_nlist"])
    np.testing.assert_array_equal(_t(sg.eweight).view(np.uint32),
                                  d["coresg_eweight"].view(np.uint32))


def test_core_sg_on_gpu_graph_squared_distances(ctx, oracle):
    X = blobs(5000, 16, seed=9, blobs=6)
    G = ctx.NNDescent(X, k=32, sample_num=16)
    ids, dist = (_t(a) for a in ctx.knn_split(G))  # squared distances, as NN-Descent leaves them
    graph = ctx.buildEnhancedKNNG(ids, dist, X)
    mst, _, _ = ctx.buildMST(graph)
    mst_rec = _t(mst).view(oracle.MST_EDGE).reshape(-1)
    check_same(ctx, oracle, ids, dist, X, mst_rec)
    # twice in a row: the context-owned buffers are reused
    check_same(ctx, oracle, ids, dist, X, mst_rec)


def test_core_sg_rejects_bad_input(ctx, oracle):
    X = blobs(300, 4, seed=2)
    ids, _ = oracle.bruteforce_knn(X, 8)
    dist = oracle.fix_distances(X, ids)
    ni, nl, ew, _ = oracle.enhanced_knng(ids, dist, X)
    mst = oracle.sort_edges(oracle.build_mst(ni, nl, ew, oracle.kruskal(ni, nl, ew)))
    bad = mst.copy()
    bad["to_node"][5] = 300
    with pytest.raises(g.HdbError, match="ARG"):
        ctx.build_CoreSG(ids, dist, X, bad)
    bad_ids = ids.copy()
    bad_ids[3, 1] = bad_ids[3, 0]
    with pytest.raises(g.HdbError, match="ARG"):
        ctx.build_CoreSG(bad_ids, dist, X, mst)
    check_same(ctx, oracle, ids, dist, X, mst)  # the context still works
