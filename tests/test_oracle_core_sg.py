"""The oracle's Core-SG (core-sg.cu) on the reference's golden fixtures: the
kNN-plus-reverse part of every row equals the reference's own enhanced-graph
rows without the antihub clique (buildECLgraph output stored in the
fixtures), and the MST part holds the incident edges of the reference's
sorted MST in edge order, with the reference's Euclidean rounding."""
import glob
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))
pytestmark = pytest.mark.skipif(not FILES, reason="no golden fixtures")


@pytest.fixture(params=FILES, ids=lambda p: os.path.basename(p)[4:-4])
def golden(request):
    with open(request.param[:-4] + ".json") as f:
        meta = json.load(f)
    return dict(np.load(request.param)), meta


def test_core_sg_rows_follow_the_reference(oracle, golden):
    g, meta = golden
    ids, dist, X = g["ids"], g["dist"], g["X"]
    n, k = ids.shape
    mst = g[f"mst_{meta['mpts'][0]}"]
    nindex, nlist, ew = oracle.core_sg(ids, dist, X, mst)
    mdeg = np.bincount(np.concatenate([mst["from_node"], mst["to_node"]]), minlength=n)
    ah = set(g["antihubs"].tolist())
    ref_ni, ref_nl = g["nindex"], g["nlist"]
    pos = {}
    for e, (a, b) in enumerate(zip(mst["from_node"], mst["to_node"])):
        pos.setdefault(int(b), []).append(int(a))  # to_node's row takes from_node first
        pos.setdefault(int(a), []).append(int(b))
    for i in range(n):
        row = nlist[nindex[i]:nindex[i + 1]]
        ref = ref_nl[ref_ni[i]:ref_ni[i + 1]]
        nrev = len(ref) - k - (len(ah) - 1 if i in ah else 0)
        assert len(row) == k + nrev + mdeg[i]
        np.testing.assert_array_equal(row[:k + nrev], ref[:k + nrev])
        np.testing.assert_array_equal(row[k + nrev:], pos.get(i, []))
        w = ew[nindex[i]:nindex[i + 1]]
        np.testing.assert_array_equal(w[:k].view(np.uint32), dist[i].view(np.uint32))
        for t, s in enumerate(row[k:k + nrev]):
            j = int(np.nonzero(ids[s] == i)[0][0])
            assert w[k + t].view(np.uint32) == dist[s, j].view(np.uint32)
        for t, nb in enumerate(row[k + nrev:]):
            eu = np.float32(oracle.euclid_ref(X[i], X[nb]))
            assert w[k + nrev + t].view(np.uint32) == eu.view(np.uint32)
