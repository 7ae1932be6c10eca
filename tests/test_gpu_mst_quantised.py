"""The reference's mst_gpu = 1 MST (int-quantised weights: buildGPUgraph,
gpuMST, buildMST_gpu) on the GPU: against the reference's own output on the
golden fixtures, against the oracle on NN-Descent graphs (including scaled
weights beyond the int range), through hdb_run_knn / hdb_run_batched and the
hdbscan_ command line."""
import glob
import json
import os
import subprocess

import numpy as np
import pytest

import gpu_hdbscan_b200 as g
from conftest import blobs

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))


def _t(x):
    return x.detach().cpu().numpy()


def mst_records(t):
    return _t(t).copy().view(np.int32).reshape(-1, 3)


def oracle_labels(oracle, mst, n, mpts):
    """The reference's trees on a given sorted MST."""
    h = oracle.linkage_tree(mst, n)
    ct = oracle.condensed_tree(h, n, mpts)
    st, _ = oracle.stability(ct)
    return oracle.get_clusters(ct, st, n)


@pytest.mark.parametrize("path", FILES, ids=lambda p: os.path.basename(p)[4:-4])
def test_matches_reference_gpu_mst_on_golden_graphs(ctx, path):
    d = dict(np.load(path))
    G = ctx.buildEnhancedKNNG(d["ids"], d["dist"], d["X"])
    mst, _, mult, _ = ctx.buildMST_quantised(G, d["dist"])
    assert mult == int(d["mstgpu_mult"][0])
    np.testing.assert_array_equal(mst_records(mst), d["mstgpu"].view(np.int32).reshape(-1, 3))


@pytest.mark.parametrize("scale", [1.0, 1e4])
def test_matches_oracle_on_nndescent_graphs(ctx, oracle, scale):
    """scale 1e4 with tiny first distances pushes scaled weights past the int
    range (INT_MIN, as the reference's conversion gives on x86)."""
    X = blobs(4000, 6, seed=13, blobs=5, spread=3.0) * np.float32(scale)
    ids = _t(ctx.knn_split(ctx.NNDescent(X, k=32, sample_num=16))[0])
    dist = oracle.fix_distances(X, ids)
    if scale > 1:
        dist[:, 0] = np.float32(1e-6)  # multiplier 9 -> 10^9 * w overflows for w > 2.1
    G = ctx.buildEnhancedKNNG(ids, dist, X)
    mst, _, mult, _ = ctx.buildMST_quantised(G, dist)
    ref, rmult = oracle.mst_quantised(_t(G.nindex), _t(G.nlist), _t(G.eweight), dist[:, 0])
    assert mult == rmult
    got = mst_records(mst)
    np.testing.assert_array_equal(got, ref.view(np.int32).reshape(-1, 3))
    if scale > 1:
        assert (ref["weight"] < 0).any()


@pytest.mark.parametrize("distance", ["sqrt", "squared"])
def test_pipeline_labels_with_quantised_mst(ctx, oracle, distance):
    X = blobs(5000, 8, seed=17, blobs=6, spread=4.0)
    Gk = ctx.NNDescent(X, k=32, sample_num=16)
    mode = g.HDB_DIST_SQRT if distance == "sqrt" else g.HDB_DIST_SQUARED
    labels, st = ctx.hdbscan_from_knn(Gk, X, k=32, mpts=16, distance=mode, mst_gpu=1)
    ids, sq = (_t(a) for a in ctx.knn_split(Gk))
    dist = oracle.fix_distances(X, ids) if distance == "sqrt" else sq
    ni, nl, ew, _ = oracle.enhanced_knng(ids, dist, X)
    mst, mult = oracle.mst_quantised(ni, nl, ew, dist[:, 0])
    assert st["mst_multiplier"] == mult
    ref, ncl = oracle_labels(oracle, mst, len(X), 16)
    np.testing.assert_array_equal(_t(labels), ref)
    assert st["num_clusters"] == ncl


def test_batched_quantised_mst_is_per_instance(ctx):
    """Every instance takes its own multiplier, as its own run would."""
    import torch
    Xs = [torch.from_numpy(blobs(n, d, seed=n, blobs=4, spread=3.0) * np.float32(s)).cuda()
          for n, d, s in [(2000, 4, 1.0), (900, 4, 100.0), (3000, 4, 0.01), (500, 4, 1.0)]]
    labels, ncl, _, graphs = ctx.hdbscan_batched(Xs, k=16, mpts=8, sample_num=8,
                                                 want_graphs=True, mst_gpu=1)
    for X, lab, nc, G in zip(Xs, labels, ncl, graphs):
        ref, st = ctx.hdbscan_from_knn(G, X, k=16, mpts=8, mst_gpu=1)
        np.testing.assert_array_equal(_t(lab), _t(ref))
        assert nc == st["num_clusters"]


def test_cli_mst_gpu_argument(tmp_path, oracle):
    cli = os.path.join(os.path.dirname(HERE), "gpu_hdbscan_b200", "hdbscan_")
    X = blobs(3000, 5, seed=23, blobs=5, spread=4.0)
    rows = np.empty((3000, 6), np.float32)
    rows[:, 0] = np.array([5], np.int32).view(np.float32)[0]
    rows[:, 1:] = X
    vec = tmp_path / "v.fvecs"
    rows.tofile(vec)
    kg, lab, ms = tmp_path / "f.kgraph", tmp_path / "l.txt", tmp_path / "m.bin"
    r = subprocess.run([cli, "3000", "16", "1", "1", "--vectors", str(vec), "--save-fixed-kgraph",
                        str(kg), "--labels", str(lab), "--save-mst", str(ms)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(kg, np.int32).reshape(3000, 65)[:, 1:].copy()
    ids = np.where(raw[:, 1::2] < 0, -raw[:, 1::2] - 1, raw[:, 1::2]).astype(np.int32)
    dist = raw[:, 0::2].copy().view(np.float32)
    ni, nl, ew, _ = oracle.enhanced_knng(ids, dist, X)
    mst, mult = oracle.mst_quantised(ni, nl, ew, dist[:, 0])
    assert f"10^{mult}" in r.stdout
    np.testing.assert_array_equal(np.fromfile(ms, oracle.MST_EDGE).view(np.int32),
                                  mst.view(np.int32))
    ref, _ = oracle_labels(oracle, mst, 3000, 16)
    np.testing.assert_array_equal(np.loadtxt(lab, dtype=np.int32), ref)
