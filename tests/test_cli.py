"""The hdbscan_ command line (the reference's new.cu / _new.cu argv and file
formats): argument checks on the CPU; on the GPU, the files it writes -- the
.kgraph as NN-Descent leaves it, the .kgraph after fix_distances, the sorted
MSTedge dump and the labels -- against the oracle on the same graph."""
import os
import subprocess

import numpy as np
import pytest

from conftest import blobs

HERE = os.path.dirname(os.path.abspath(__file__))
CLI = os.path.join(os.path.dirname(HERE), "gpu_hdbscan_b200", "hdbscan_")
NND = np.dtype([("distance", "<f4"), ("label", "<i4")])

pytestmark = pytest.mark.skipif(not os.path.exists(CLI), reason="hdbscan_ not built")


def run(*args):
    return subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=600)


def write_fvecs(path, X):
    n, d = X.shape
    rows = np.empty((n, d + 1), np.float32)
    rows[:, 0] = np.array([d], np.int32).view(np.float32)[0]
    rows[:, 1:] = X
    rows.tofile(path)


def read_kgraph(path, k=32):
    raw = np.fromfile(path, np.int32).reshape(-1, 1 + 2 * k)
    assert (raw[:, 0] == k).all()  # every row: int32 k, then k NNDElements
    return raw[:, 1:].copy().view(NND).reshape(-1, k)


def decode(labels):
    return np.where(labels < 0, -labels - 1, labels).astype(np.int32)


def test_argv_checks():
    r = run(1, 2, 3)
    assert r.returncode == 1 and "NUM_VALUES NOT SETTED" in r.stdout
    r = run(100, 33, 1, 0, "--vectors", "none.fvecs")
    assert r.returncode == 1 and "k >= mpts" in r.stderr
    r = run(100, 16, 1, 0)
    assert r.returncode == 1 and "required" in r.stderr


@pytest.mark.gpu
def test_files_match_the_oracle(tmp_path, oracle):
    X = blobs(3000, 8, seed=5, blobs=6, spread=4.0)
    vec = tmp_path / "vectors.fvecs"
    write_fvecs(vec, X)
    p = {s: tmp_path / s for s in ("raw.kgraph", "fixed.kgraph", "mst.bin", "labels.txt")}
    r = run(3000, 16, 1, 0, "--vectors", vec, "--save-kgraph", p["raw.kgraph"],
            "--save-fixed-kgraph", p["fixed.kgraph"], "--save-mst", p["mst.bin"],
            "--labels", p["labels.txt"])
    assert r.returncode == 0, r.stderr
    raw = read_kgraph(p["raw.kgraph"])
    fixed = read_kgraph(p["fixed.kgraph"])
    ids = decode(raw["label"])
    assert oracle.validate_knn(ids)
    # fix_distances keeps every label_ (old/new flags included) and writes the
    # reference's sqrt-L2 bit for bit
    np.testing.assert_array_equal(fixed["label"], raw["label"])
    fd = oracle.fix_distances(X, ids)
    np.testing.assert_array_equal(fixed["distance"].view(np.uint32), fd.view(np.uint32))
    mst, labels, _ = oracle.hdbscan_from_knn(ids, fd, X, 16)
    got = np.fromfile(p["mst.bin"], oracle.MST_EDGE)
    np.testing.assert_array_equal(got.view(np.int32), mst.view(np.int32))
    np.testing.assert_array_equal(np.loadtxt(p["labels.txt"], dtype=np.int32), labels)

    # the _new.cu flow: read a finished graph -- the raw one with fix_distances
    # applied, or the fixed one as it stands -- and reach the same labels
    for extra in (["--kgraph", p["raw.kgraph"]], ["--kgraph", p["fixed.kgraph"], "--squared"]):
        out = tmp_path / "labels2.txt"
        r = run(3000, 16, 1, 0, "--vectors", vec, "--labels", out, *extra)
        assert r.returncode == 0, r.stderr
        np.testing.assert_array_equal(np.loadtxt(out, dtype=np.int32), labels)


@pytest.mark.gpu
def test_text_vectors_and_fvecs_conversion(tmp_path):
    """create.py's text layout ("N d", then the values) read as ReadTxtVecs
    does, and written back as .fvecs (PrepareVector)."""
    X = blobs(1200, 3, seed=9)
    txt = tmp_path / "vectors.txt"
    with open(txt, "w") as f:
        f.write(f"{X.shape[0]} {X.shape[1]}\n")
        for row in X:
            f.write(" ".join(repr(float(v)) for v in row) + "\n")
    fv = tmp_path / "out.fvecs"
    kg = tmp_path / "g.kgraph"
    la, lb = tmp_path / "a.txt", tmp_path / "b.txt"
    r = run(0, 8, 1, 0, "--vectors-txt", txt, "--write-fvecs", fv, "--save-kgraph", kg,
            "--labels", la)
    assert r.returncode == 0, r.stderr
    back = np.fromfile(fv, np.float32).reshape(1200, 4)
    np.testing.assert_array_equal(back[:, 1:], X)
    # the same graph (two NN-Descent runs may differ a little) from the .fvecs
    # copy: fix_distances reads the vectors again, so any change would show
    r = run(0, 8, 1, 0, "--vectors", fv, "--kgraph", kg, "--labels", lb)
    assert r.returncode == 0, r.stderr
    np.testing.assert_array_equal(np.loadtxt(la), np.loadtxt(lb))


@pytest.mark.gpu
def test_id_order_option(tmp_path, oracle):
    """--id-order: the float MST under (weight, min id, max id), its sorted dump
    and the labels equal the oracle's path in that order on the same graph."""
    X = blobs(3000, 8, seed=7, blobs=6, spread=4.0)
    vec = tmp_path / "vectors.fvecs"
    write_fvecs(vec, X)
    kg, ms, lab = tmp_path / "raw.kgraph", tmp_path / "mst.bin", tmp_path / "labels.txt"
    r = run(3000, 16, 1, 0, "--vectors", vec, "--save-kgraph", kg)
    assert r.returncode == 0, r.stderr
    r = run(3000, 16, 1, 0, "--vectors", vec, "--kgraph", kg, "--id-order", "--save-mst", ms,
            "--labels", lab)
    assert r.returncode == 0, r.stderr
    ids = decode(read_kgraph(kg)["label"])
    fd = oracle.fix_distances(X, ids)
    mst, labels, _ = oracle.hdbscan_from_knn(ids, fd, X, 16, order=oracle.ORDER_IDS)
    np.testing.assert_array_equal(np.fromfile(ms, oracle.MST_EDGE).view(np.int32),
                                  mst.view(np.int32))
    np.testing.assert_array_equal(np.loadtxt(lab, dtype=np.int32), labels)
