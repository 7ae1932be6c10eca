"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference algorithm of gorlando04/GPU_HDBSCAN stage by
stage in plain C (``oracle/hdb_oracle.c``).  Only the test-suite, the smoke
check and the CPU-baseline leg of ``bench.py`` import this module, and only to
check or time the reference algorithm -- never as the thing measured or
shipped.  Build it with ``make -C oracle`` (``__graft_entry__.build()`` does).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

MST_EDGE = np.dtype([("from_node", "<i4"), ("to_node", "<i4"), ("weight", "<f4")])
LINKAGE_NODE = np.dtype([("left_node", "<i4"), ("right_node", "<i4"), ("weight", "<f4"),
                         ("node_size", "<i4")])
CONDENSED_NODE = np.dtype([("parent", "<i4"), ("child", "<i4"), ("lambda_val", "<f4"),
                           ("child_size", "<i4")])
STABILITY = np.dtype([("cluster_id", "<i4"), ("lambda", "<f4")])

_P = C.c_void_p
_I64 = C.c_int64
_I32 = C.c_int32


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "hdb_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return path


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        sigs = {
            "orc_free": (None, [_P]),
            "orc_num_threads": (C.c_int, []),
            "orc_xorshift64star": (C.c_uint64, [C.c_uint64]),
            "orc_nndescent": (C.c_int, [_P, _I64, _I32, _I32, _I32, _I32, _P, _P]),
            "orc_nndescent_form": (C.c_int, [_P, _I64, _I32, _I32, _I32, _I32, _I32, _P, _P]),
            "orc_knn_merge": (C.c_int, [_P, _I64, _I64, _I32, _P, _P, _I32, _I32, _I32, _P, _P]),
            "orc_bruteforce_knn": (C.c_int, [_P, _I64, _I32, _I32, _P, _I64, _P, _P]),
            "orc_recall": (C.c_double, [_P, _I32, _P, _I32, _I64, _I32]),
            "orc_fix_distances": (None, [_P, _I64, _I32, _P, _I32, _P]),
            "orc_euclid_ref": (C.c_float, [_P, _P, _I32]),
            "orc_diffsum": (C.c_float, [_P, _P, _I32]),
            "orc_validate_knn": (C.c_int, [_P, _I64, _I32]),
            "orc_degrees": (None, [_P, _I64, _I32, _P]),
            "orc_select_antihubs": (_I32, [_P, _P, _I64, _I32, _P]),
            "orc_enhanced_knng": (_I64, [_P, _P, _P, _I64, _I32, _I32, _P, _P, _P, _P, _P]),
            "orc_core_sg": (_I64, [_P, _P, _P, _I64, _I32, _I32, _P, _P, _P, _P]),
            "orc_kruskal": (C.c_int, [_P, _P, _P, _I32, _I64, _P]),
            "orc_mst_ordered": (C.c_int, [_P, _P, _P, _I32, _I64, _I32, _P, _P]),
            "orc_build_mst": (C.c_int, [_P, _P, _P, _I32, _I64, _P, _P]),
            "orc_mst_quantised": (C.c_int, [_P, _P, _P, _I32, _I64, _P, _P, _P]),
            "orc_sort_edges": (None, [_P, _I64]),
            "orc_linkage_tree": (None, [_P, _I64, _P]),
            "orc_condensed_tree": (_I64, [_P, _I64, _I32, _P]),
            "orc_stability": (_I64, [_P, _I64, _P, _P]),
            "orc_get_clusters": (C.c_int, [_P, _I64, _P, _P, _I64, _I64, _P, _P]),
            "orc_hdbscan_from_knn": (C.c_int, [_P, _P, _P, _I64, _I32, _I32, _I32, _I32, _P,
                                               _P, _P]),
            "orc_hdbscan_from_knn_order": (C.c_int, [_P, _P, _P, _I64, _I32, _I32, _I32, _I32,
                                                     _I32, _P, _P, _P]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def num_threads() -> int:
    return lib().orc_num_threads()


def xorshift64star(x: int) -> int:
    return lib().orc_xorshift64star(x)


def nndescent(X, k=32, sample_num=16, iterations=6):
    X = _c(X, np.float32)
    n, d = X.shape
    ids = np.empty((n, k), np.int32)
    dist = np.empty((n, k), np.float32)
    rc = lib().orc_nndescent(_p(X), n, d, k, sample_num, iterations, _p(ids), _p(dist))
    if rc:
        raise ValueError(f"orc_nndescent failed ({rc})")
    return ids, dist


FORMS = {"fp32": 0, "bf16": 1, "fp8": 2, "fp16": 3}


def nndescent_form(X, form, k=32, sample_num=16, iterations=6):
    """NN-Descent whose local join takes candidate distances in a precision
    form ("fp32" exact, "bf16" / "fp8" / "fp16" Gram forms of the centred rows), then an
    exact FP32 re-rank of the kept neighbours (orc_nndescent_form)."""
    X = _c(X, np.float32)
    n, d = X.shape
    ids = np.empty((n, k), np.int32)
    dist = np.empty((n, k), np.float32)
    rc = lib().orc_nndescent_form(_p(X), n, d, k, sample_num, iterations, FORMS[form], _p(ids),
                                  _p(dist))
    if rc:
        raise ValueError(f"orc_nndescent_form failed ({rc})")
    return ids, dist


def knn_merge(X1, ids1, X2, ids2, sample_num=12, iterations=11):
    """gpuknn::KNNMerge (knnmerge.cu:401-437) restated: the kNN graph of the
    union of X1 and X2 (rows of X1 first, ids of X2 shifted by len(X1)) from
    ids1 [n1, k] and ids2 [n2, k], ids local to their set."""
    X1 = _c(X1, np.float32)
    X2 = _c(X2, np.float32)
    ids1 = _c(ids1, np.int32)
    ids2 = _c(ids2, np.int32)
    n1, d = X1.shape
    n2 = X2.shape[0]
    k = ids1.shape[1]
    X = np.ascontiguousarray(np.concatenate([X1, X2]))
    ids = np.empty((n1 + n2, k), np.int32)
    dist = np.empty((n1 + n2, k), np.float32)
    rc = lib().orc_knn_merge(_p(X), n1, n2, d, _p(ids1), _p(ids2), k, sample_num, iterations,
                             _p(ids), _p(dist))
    if rc:
        raise ValueError(f"orc_knn_merge failed ({rc})")
    return ids, dist


def bruteforce_knn(X, k, queries=None):
    X = _c(X, np.float32)
    n, d = X.shape
    q = None if queries is None else _c(queries, np.int64)
    nq = n if q is None else len(q)
    ids = np.empty((nq, k), np.int32)
    dist = np.empty((nq, k), np.float64)
    rc = lib().orc_bruteforce_knn(_p(X), n, d, k, _p(q), nq, _p(ids), _p(dist))
    if rc:
        raise ValueError(f"orc_bruteforce_knn failed ({rc})")
    return ids, dist


def recall(ids, gt, recall_at):
    ids = _c(ids, np.int32)
    gt = _c(gt, np.int32)
    return lib().orc_recall(_p(ids), ids.shape[1], _p(gt), gt.shape[1], ids.shape[0], recall_at)


def fix_distances(X, ids):
    X = _c(X, np.float32)
    ids = _c(ids, np.int32)
    out = np.empty(ids.shape, np.float32)
    lib().orc_fix_distances(_p(X), X.shape[0], X.shape[1], _p(ids), ids.shape[1], _p(out))
    return out


def euclid_ref(a, b):
    a = _c(a, np.float32)
    b = _c(b, np.float32)
    return lib().orc_euclid_ref(_p(a), _p(b), a.shape[0])


def diffsum(a, b):
    a = _c(a, np.float32)
    b = _c(b, np.float32)
    return lib().orc_diffsum(_p(a), _p(b), a.shape[0])


def validate_knn(ids):
    ids = _c(ids, np.int32)
    return lib().orc_validate_knn(_p(ids), ids.shape[0], ids.shape[1]) == 0


def degrees(ids):
    ids = _c(ids, np.int32)
    out = np.empty(ids.shape[0], np.int32)
    lib().orc_degrees(_p(ids), ids.shape[0], ids.shape[1], _p(out))
    return out


def select_antihubs(ids, deg=None):
    ids = _c(ids, np.int32)
    if deg is None:
        deg = degrees(ids)
    deg = _c(deg, np.int32)
    n, k = ids.shape
    out = np.empty(max(1, int(np.sqrt(n))), np.int32)
    m = lib().orc_select_antihubs(_p(ids), _p(deg), n, k, _p(out))
    return out[:m].copy()


def _take(ptr, count, ctype, np_dtype):
    if count == 0:
        lib().orc_free(ptr)
        return np.empty(0, np_dtype)
    arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(count,)).copy()
    lib().orc_free(ptr)
    return arr.view(np_dtype) if np_dtype is not None else arr


def enhanced_knng(ids, dist, X):
    """(nindex int64[n+1], nlist int32[E], eweight float32[E], antihubs int32[P])."""
    ids = _c(ids, np.int32)
    dist = _c(dist, np.float32)
    X = _c(X, np.float32)
    n, k = ids.shape
    pn, pl, pw, pa = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    nah = C.c_int32(0)
    E = lib().orc_enhanced_knng(_p(ids), _p(dist), _p(X), n, X.shape[1], k, C.byref(pn),
                                C.byref(pl), C.byref(pw), C.byref(pa), C.byref(nah))
    if E < 0:
        raise ValueError("invalid kNN graph (id out of range, self id or duplicate id)")
    nindex = _take(pn, n + 1, C.c_int64, None)
    nlist = _take(pl, E, C.c_int32, None)
    ew = _take(pw, E, C.c_float, None)
    ah = _take(pa, nah.value, C.c_int32, None)
    return nindex, nlist, ew, ah


def core_sg(ids, dist, X, mst):
    """Core-SG of a kNN graph and its sorted MST (MST_EDGE records, n-1):
    (nindex int64[n+1], nlist int32[E], eweight float32[E])."""
    ids = _c(ids, np.int32)
    dist = _c(dist, np.float32)
    X = _c(X, np.float32)
    mst = np.ascontiguousarray(mst, dtype=MST_EDGE)
    n, k = ids.shape
    if len(mst) != n - 1:
        raise ValueError("the MST must have n - 1 edges")
    pn, pl, pw = C.c_void_p(), C.c_void_p(), C.c_void_p()
    E = lib().orc_core_sg(_p(ids), _p(dist), _p(X), n, X.shape[1], k, _p(mst), C.byref(pn),
                          C.byref(pl), C.byref(pw))
    if E < 0:
        raise ValueError("invalid kNN graph (id out of range, self id or duplicate id)")
    return (_take(pn, n + 1, C.c_int64, None), _take(pl, E, C.c_int32, None),
            _take(pw, E, C.c_float, None))


def kruskal(nindex, nlist, eweight):
    nindex = _c(nindex, np.int64)
    nlist = _c(nlist, np.int32)
    eweight = _c(eweight, np.float32)
    E = len(nlist)
    inmst = np.zeros(max(E, 1), np.uint8)
    rc = lib().orc_kruskal(_p(nindex), _p(nlist), _p(eweight), len(nindex) - 1, E, _p(inmst))
    if rc:
        raise RuntimeError("graph is disconnected")
    return inmst[:E].astype(bool)


ORDER_EDGE, ORDER_IDS = 0, 1


def mst_ordered(nindex, nlist, eweight, order):
    """The float MST under a tie order (ORDER_EDGE: the reference's (weight,
    CSR edge index); ORDER_IDS: (weight, min id, max id, edge index)), listed
    in that order: (MST_EDGE[n-1], in_mst bool[edges])."""
    nindex = _c(nindex, np.int64)
    nlist = _c(nlist, np.int32)
    eweight = _c(eweight, np.float32)
    n, E = len(nindex) - 1, len(nlist)
    out = np.zeros(n - 1, MST_EDGE)
    inmst = np.zeros(max(E, 1), np.uint8)
    rc = lib().orc_mst_ordered(_p(nindex), _p(nlist), _p(eweight), n, E, order, _p(inmst),
                               _p(out))
    if rc:
        raise RuntimeError("graph is disconnected")
    return out, inmst[:E].astype(bool)


def build_mst(nindex, nlist, eweight, inmst):
    nindex = _c(nindex, np.int64)
    nlist = _c(nlist, np.int32)
    eweight = _c(eweight, np.float32)
    inmst = _c(inmst, np.uint8)
    n = len(nindex) - 1
    out = np.zeros(n - 1, MST_EDGE)
    rc = lib().orc_build_mst(_p(nindex), _p(nlist), _p(eweight), n, len(nlist), _p(inmst),
                             _p(out))
    if rc:
        raise RuntimeError("MST has the wrong number of edges")
    return out


def mst_quantised(nindex, nlist, eweight, first_dist):
    """The reference's mst_gpu = 1 MST: (sorted MST_EDGE[n-1], multiplier)."""
    nindex = _c(nindex, np.int64)
    nlist = _c(nlist, np.int32)
    eweight = _c(eweight, np.float32)
    first_dist = _c(first_dist, np.float32)
    n = len(nindex) - 1
    out = np.zeros(n - 1, MST_EDGE)
    mult = C.c_int32(0)
    rc = lib().orc_mst_quantised(_p(nindex), _p(nlist), _p(eweight), n, len(nlist), _p(first_dist),
                                 _p(out), C.byref(mult))
    if rc:
        raise RuntimeError("graph is disconnected")
    return out, mult.value


def sort_edges(edges):
    e = np.ascontiguousarray(edges.copy(), dtype=MST_EDGE)
    lib().orc_sort_edges(_p(e), len(e))
    return e


def linkage_tree(sorted_edges, n):
    e = np.ascontiguousarray(sorted_edges, dtype=MST_EDGE)
    out = np.zeros(n - 1, LINKAGE_NODE)
    lib().orc_linkage_tree(_p(e), n, _p(out))
    return out


def condensed_tree(hier, n, mpts):
    h = np.ascontiguousarray(hier, dtype=LINKAGE_NODE)
    ptr = C.c_void_p()
    m = lib().orc_condensed_tree(_p(h), n, mpts, C.byref(ptr))
    raw = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(m * 4,)).copy()
    lib().orc_free(ptr)
    return raw.view(CONDENSED_NODE)


def stability(tree, fp64=False):
    t = np.ascontiguousarray(tree, dtype=CONDENSED_NODE)
    ptr = C.c_void_p()
    p64 = C.c_void_p()
    m = lib().orc_stability(_p(t), len(t), C.byref(ptr), C.byref(p64))
    raw = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(m * 2,)).copy()
    lib().orc_free(ptr)
    s64 = np.ctypeslib.as_array(C.cast(p64, C.POINTER(C.c_double)), shape=(m,)).copy()
    lib().orc_free(p64)
    return raw.view(STABILITY), s64


def get_clusters(tree, stab, n, stab64=None):
    t = np.ascontiguousarray(tree, dtype=CONDENSED_NODE)
    s = np.ascontiguousarray(stab.copy(), dtype=STABILITY)
    s64 = None if stab64 is None else np.ascontiguousarray(stab64.copy(), dtype=np.float64)
    labels = np.empty(n, np.int32)
    ncl = C.c_int32(0)
    lib().orc_get_clusters(_p(t), len(t), _p(s), _p(s64), len(s), n, _p(labels), C.byref(ncl))
    return labels, ncl.value


def hdbscan_from_knn(ids, dist, X, mpts, fp64=False, order=None):
    """The reference call order from a given kNN graph: (sorted MST, labels).
    order=ORDER_IDS takes the MST under (weight, min id, max id)."""
    ids = _c(ids, np.int32)
    dist = _c(dist, np.float32)
    X = _c(X, np.float32)
    n, k = ids.shape
    mst = np.zeros(n - 1, MST_EDGE)
    labels = np.empty(n, np.int32)
    ncl = C.c_int32(0)
    if order is None:
        rc = lib().orc_hdbscan_from_knn(_p(ids), _p(dist), _p(X), n, X.shape[1], k, mpts,
                                        int(fp64), _p(mst), _p(labels), C.byref(ncl))
    else:
        rc = lib().orc_hdbscan_from_knn_order(_p(ids), _p(dist), _p(X), n, X.shape[1], k, mpts,
                                              int(fp64), order, _p(mst), _p(labels),
                                              C.byref(ncl))
    if rc:
        raise RuntimeError(f"orc_hdbscan_from_knn failed ({rc})")
    return mst, labels, ncl.value
