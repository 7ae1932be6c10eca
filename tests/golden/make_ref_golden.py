"""Generates the golden fixtures that pin the CPU oracle: runs the reference's
own code (oracle/_ref/libhdbref.so, built by oracle/ref/Makefile from the
unmodified reference sources) on small seeded inputs and stores inputs and
outputs as compressed .npz files.

Needs a GPU (the reference's tree stages allocate managed memory and launch
fill kernels).  Usage on a machine with a GPU, from the repository root:

    python tests/golden/make_ref_golden.py OUTDIR
    python tests/golden/make_ref_golden.py --add-mst-gpu OUTDIR
    python tests/golden/make_ref_golden.py --add-core-sg OUTDIR
    python tests/golden/make_ref_golden.py --nndescent-recall [--cg] OUTDIR

The second form adds the reference's mst_gpu = 1 MST (int-quantised weights,
gpuMST, buildMST_gpu) of every committed fixture's enhanced graph as
`mstgpu` / `mstgpu_mult`, leaving the fixture's other arrays as they are.
The third adds the reference's core-SG (Union_kNNG_MST + update_core_sg_weights
on the fixture's kNN graph and sorted MST) as `coresg_nindex` /
`coresg_nlist` / `coresg_eweight`, and, for the d = 12 fixture, the
reference's initial NN-Descent graph (gpuknn::NNDescent with 0 iterations) as
`ref_init_ids` / `ref_init_dist`.
The fourth runs the reference's NN-Descent (6 iterations, VEC_DIM = 12) on
d = 12 point sets up to the 100,000-point blob configuration and writes the
recall@32 of its graph, of the oracle's restatement and the rows holding a
repeated id to ref_nndescent_recall[_cg].json; --cg uses the build whose global
loads bypass L1 (oracle/ref/Makefile, libhdbref_cg.so).  Run it once per
library, each in its own process (both libraries export the same symbols).

The kNN graphs fed to the reference come from the oracle's NN-Descent (with
fix_distances applied), so every later stage sees one shared input.  The
reference NN-Descent itself (compiled with VEC_DIM = 12) is also run on the
d = 12 cases and its recall@32 against the exact FP64 kNN is recorded.
"""
import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from conftest import blobs  # noqa: E402
from oracle import oracle as O  # noqa: E402

MST_EDGE, LINK, COND, STAB = O.MST_EDGE, O.LINKAGE_NODE, O.CONDENSED_NODE, O.STABILITY

CASES = [
    # name, n, d, blobs, noise, seed, mpts list
    ("blobs_d12", 1500, 12, 6, 0.05, 101, [32, 8]),
    ("noisy_d3", 1200, 3, 4, 0.20, 102, [16, 32]),
    ("grid_ties_d2", 900, 2, 0, 0.0, 103, [32, 5]),
]


def grid_points(n, seed):
    """Integer grid points with duplicates: many equal distances and weights."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, 12, size=(n, 2)).astype(np.float32)


def load_ref(name="libhdbref.so"):
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", name), mode=C.RTLD_GLOBAL)
    P = C.c_void_p
    L.ref_enhanced_knng.restype = C.c_long
    L.ref_enhanced_knng.argtypes = [P, P, P, C.c_long, C.c_int, C.c_int, P, P, P, P, P]
    L.ref_mst_trees.restype = C.c_int
    L.ref_mst_trees.argtypes = [P, P, P, C.c_long, C.c_int, P, P, P, P, P, P, P]
    L.ref_nndescent.restype = C.c_int
    L.ref_nndescent.argtypes = [P, C.c_long, C.c_int, C.c_int, P]
    L.ref_mst_gpu.restype = C.c_int
    L.ref_mst_gpu.argtypes = [P, P, P, C.c_long, C.c_char_p, P, P]
    L.ref_core_sg.restype = C.c_long
    L.ref_core_sg.argtypes = [P, P, P, C.c_long, C.c_int, C.c_int, P, P, P, P]
    L.ref_free.argtypes = [P]
    return L


def write_kgraph(path, ids, dist):
    """The .kgraph layout (tools/filetool.hpp WriteBinaryVecs of NNDElement):
    per row int32 k, then k (float distance, int32 label) pairs."""
    n, k = ids.shape
    rows = np.empty((n, 1 + 2 * k), np.int32)
    rows[:, 0] = k
    rows[:, 1::2] = np.ascontiguousarray(dist, np.float32).view(np.int32)
    rows[:, 2::2] = ids
    rows.tofile(path)


def ref_mst_gpu(L, nindex, nlist, ew, ids, dist, outdir, name):
    """The reference's mst_gpu = 1 MST; the multiplier comes from a .kgraph
    holding the graph's distances, as build_CoreSG reads it."""
    n = len(nindex) - 1
    kg = os.path.join(outdir, f"_{name}.kgraph")
    write_kgraph(kg, ids, dist)
    mst = np.zeros(n - 1, MST_EDGE)
    mult = C.c_int(0)
    rc = L.ref_mst_gpu(p(np.ascontiguousarray(nindex, np.int64)), p(nlist), p(ew), n,
                       kg.encode(), p(mst), C.byref(mult))
    os.remove(kg)
    assert rc == 0, "reference gpuMST failed"
    return mst, mult.value


def p(a):
    return a.ctypes.data_as(C.c_void_p)


def take(L, ptr, count, ctype):
    arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(count,)).copy()
    L.ref_free(ptr)
    return arr


def run_case(L, name, n, d, nblobs, noise, seed, mpts_list, outdir):
    X = grid_points(n, seed) if nblobs == 0 else blobs(n, d, seed, blobs=nblobs, noise=noise)
    X = np.ascontiguousarray(X, np.float32)
    ids, _ = O.nndescent(X, 32, 16, 6)
    dist = O.fix_distances(X, ids)
    ids = np.ascontiguousarray(ids, np.int32)
    pn, pl, pw, pa = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    nah = C.c_int(0)
    E = L.ref_enhanced_knng(p(ids), p(dist), p(X), n, d, 32, C.byref(pn), C.byref(pl), C.byref(pw),
                            C.byref(pa), C.byref(nah))
    assert E > 0, "reference enhanced kNN graph failed"
    nindex = take(L, pn, n + 1, C.c_long).astype(np.int64)
    nlist = take(L, pl, E, C.c_int)
    ew = take(L, pw, E, C.c_float)
    ah = take(L, pa, nah.value, C.c_int)
    out = dict(X=X, ids=ids, dist=dist, nindex=nindex, nlist=nlist, eweight=ew, antihubs=ah)
    meta = {"name": name, "n": n, "d": d, "k": 32, "edges": int(E), "mpts": mpts_list}
    out["mstgpu"], mult = ref_mst_gpu(L, nindex, nlist, ew, ids, dist, outdir, name)
    out["mstgpu_mult"] = np.array([mult], np.int32)
    for mpts in mpts_list:
        mst = np.zeros(n - 1, MST_EDGE)
        hier = np.zeros(n - 1, LINK)
        labels = np.zeros(n, np.int32)
        pc, ps = C.c_void_p(), C.c_void_p()
        cs, ss = C.c_long(0), C.c_long(0)
        rc = L.ref_mst_trees(p(nindex), p(nlist), p(ew), n, mpts, p(mst), p(hier), p(labels),
                             C.byref(pc), C.byref(cs), C.byref(ps), C.byref(ss))
        assert rc == 0, "reference MST / trees failed"
        cond = take(L, pc, cs.value * 4, C.c_int).view(COND)
        stab = take(L, ps, ss.value * 2, C.c_int).view(STAB)
        out[f"mst_{mpts}"] = mst
        out[f"hier_{mpts}"] = hier
        out[f"labels_{mpts}"] = labels
        out[f"cond_{mpts}"] = cond
        out[f"stab_{mpts}"] = stab
    if d == 12:
        G = np.zeros((n, 32, 2), np.int32)
        assert L.ref_nndescent(p(X), n, d, 6, p(G)) == 0
        rids = G[:, :, 1].copy()
        rids = np.where(rids < 0, -rids - 1, rids)
        gt, _ = O.bruteforce_knn(X, 32)
        meta["ref_nndescent_recall32"] = O.recall(rids, gt, 32)
        meta["oracle_nndescent_recall32"] = O.recall(ids, gt, 32)
        out["ref_knn_ids"] = rids.astype(np.int32)
    np.savez_compressed(os.path.join(outdir, f"ref_{name}.npz"), **out)
    with open(os.path.join(outdir, f"ref_{name}.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print(name, meta, flush=True)


def add_mst_gpu(L, outdir):
    import glob
    for f in sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "ref_*.npz"))):
        d = dict(np.load(f))
        name = os.path.basename(f)[4:-4]
        d["mstgpu"], mult = ref_mst_gpu(L, d["nindex"], d["nlist"], d["eweight"], d["ids"],
                                        d["dist"], outdir, name)
        d["mstgpu_mult"] = np.array([mult], np.int32)
        np.savez_compressed(os.path.join(outdir, os.path.basename(f)), **d)
        print(name, "mst_gpu multiplier", mult, flush=True)


def ref_core_sg(L, ids, dist, X, mst):
    """The reference's core-SG rows and Euclidean weights (ref_driver.cu)."""
    n, d = X.shape
    pn, pl, pw = C.c_void_p(), C.c_void_p(), C.c_void_p()
    E = L.ref_core_sg(p(np.ascontiguousarray(ids, np.int32)), p(np.ascontiguousarray(dist, np.float32)),
                      p(np.ascontiguousarray(X, np.float32)), n, d, 32,
                      p(np.ascontiguousarray(mst, MST_EDGE)), C.byref(pn), C.byref(pl), C.byref(pw))
    assert E > 0, "reference core-SG failed"
    return (take(L, pn, n + 1, C.c_long).astype(np.int64), take(L, pl, E, C.c_int),
            take(L, pw, E, C.c_float))


def ref_graph(L, X, iterations):
    """gpuknn::NNDescent (VEC_DIM = 12) on X: (decoded ids, distances)."""
    n, d = X.shape
    G = np.zeros((n, 32, 2), np.int32)
    assert L.ref_nndescent(p(np.ascontiguousarray(X, np.float32)), n, d, iterations, p(G)) == 0
    ids = G[:, :, 1].copy()
    return np.where(ids < 0, -ids - 1, ids).astype(np.int32), G[:, :, 0].copy().view(np.float32)


def rows_with_repeats(ids):
    s = np.sort(ids, axis=1)
    return int((s[:, 1:] == s[:, :-1]).any(axis=1).sum())


def add_core_sg(L, outdir):
    import glob
    for f in sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "ref_*.npz"))):
        d = dict(np.load(f))
        name = os.path.basename(f)[4:-4]
        d["coresg_nindex"], d["coresg_nlist"], d["coresg_eweight"] = ref_core_sg(
            L, d["ids"], d["dist"], d["X"], d["mst_32"])
        if d["X"].shape[1] == 12:
            d["ref_init_ids"], d["ref_init_dist"] = ref_graph(L, d["X"], 0)
        np.savez_compressed(os.path.join(outdir, os.path.basename(f)), **d)
        print(name, "core-SG edges", len(d["coresg_nlist"]), flush=True)


def nndescent_sets():
    """d = 12 point sets for the NN-Descent comparison: the 1,500-point
    fixture, 20,000 points of 20 blobs, and the 100,000-point configuration
    (10 blobs, centres in [-10, 10]^12, sigma 1, 5 % noise)."""
    from gpu_hdbscan_b200 import synth
    fx = np.load(os.path.join(ROOT, "tests", "golden", "ref_blobs_d12.npz"))["X"]
    return [("ref_blobs_d12", fx, None),
            ("blobs_20k_d12", blobs(20000, 12, 19, blobs=20), None),
            ("blobs_100k_d12", synth.generate(synth.WORKLOADS["blobs_100k_d12"]), 3000)]


def nndescent_recall(L, outdir, tag):
    out = {"library": tag, "k": 32, "sample_num": 16, "iterations": 6, "sets": {}}
    for name, X, nq in nndescent_sets():
        X = np.ascontiguousarray(X, np.float32)
        n = len(X)
        q = np.arange(n) if nq is None else np.random.default_rng(5).choice(n, nq, replace=False)
        q = np.sort(q)
        gt, _ = O.bruteforce_knn(X, 32, q)
        rids, _ = ref_graph(L, X, 6)
        oids, _ = O.nndescent(X, 32, 16, 6)
        out["sets"][name] = {
            "n": n, "queries": "all rows" if nq is None else f"{nq} rows, default_rng(5) choice",
            "ref_recall32": O.recall(rids[q], gt, 32),
            "ref_rows_with_repeated_ids": rows_with_repeats(rids),
            "oracle_recall32": O.recall(oids[q], gt, 32)}
        print(name, out["sets"][name], flush=True)
    with open(os.path.join(outdir, f"ref_nndescent_recall{'_cg' if tag.endswith('_cg.so') else ''}.json"),
              "w") as f:
        json.dump(out, f, indent=1)


def main():
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    outdir = args[0] if args else os.path.join(ROOT, "tests", "golden")
    os.makedirs(outdir, exist_ok=True)
    O.build()
    if "--nndescent-recall" in sys.argv:
        name = "libhdbref_cg.so" if "--cg" in sys.argv else "libhdbref.so"
        nndescent_recall(load_ref(name), outdir, name)
        return
    L = load_ref()
    if "--add-mst-gpu" in sys.argv:
        add_mst_gpu(L, outdir)
        return
    if "--add-core-sg" in sys.argv:
        add_core_sg(L, outdir)
        return
    for case in CASES:
        run_case(L, *case, outdir)


if __name__ == "__main__":
    main()
