"""ctypes binding of libhdb_b200.so (include/hdb/hdb.h).

There is no fallback: if the CUDA library is missing or was built for another
GPU, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhdb_b200.so")

HDB_OK, HDB_ERR_ARG, HDB_ERR_ALLOC, HDB_ERR_CUDA, HDB_ERR_IO, HDB_ERR_TIMEOUT, \
    HDB_ERR_DISCONNECTED, HDB_ERR_INTERNAL = range(8)
STATUS_NAMES = {0: "HDB_OK", 1: "HDB_ERR_ARG", 2: "HDB_ERR_ALLOC", 3: "HDB_ERR_CUDA",
                4: "HDB_ERR_IO", 5: "HDB_ERR_TIMEOUT", 6: "HDB_ERR_DISCONNECTED",
                7: "HDB_ERR_INTERNAL"}
HDB_PREC_FP32, HDB_PREC_BF16, HDB_PREC_FP16 = 0, 1, 2
HDB_DIST_SQRT, HDB_DIST_SQUARED = 0, 1
HDB_STAB_FP32, HDB_STAB_FP64 = 0, 1
HDB_MST_FLOAT, HDB_MST_QUANTISED, HDB_MST_ID_ORDER = 0, 1, 2
HDB_ORDER_EDGE, HDB_ORDER_IDS = 0, 1

# Every symbol include/hdb/hdb.h declares.
EXPORTS = ("hdb_version", "hdb_last_error", "hdb_create", "hdb_destroy", "hdb_set_stream",
           "hdb_set_join_tiles", "hdb_nndescent", "hdb_knn_split", "hdb_fix_distances",
           "hdb_enhanced_knng", "hdb_mst",
           "hdb_sort_edges", "hdb_linkage_tree", "hdb_condense_select", "hdb_run",
           "hdb_run_with_graph", "hdb_run_knn", "hdb_sort_edges_noalloc", "hdb_bf16_distance_tiles",
           "hdb_core_sg", "hdb_run_batched", "hdb_run_knn_batched", "hdb_mst_quantised",
           "hdb_knn_merge", "hdb_mst_ordered")


class HdbError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class KnnParams(C.Structure):
    _fields_ = [("k", C.c_int32), ("sample_num", C.c_int32), ("iterations", C.c_int32),
                ("precision", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("knn", KnnParams), ("mpts", C.c_int32), ("distance", C.c_int32),
                ("stability", C.c_int32), ("host_io", C.c_int32), ("mst_gpu", C.c_int32)]


class Graph(C.Structure):
    _fields_ = [("nodes", C.c_int32), ("edges", C.c_int64), ("nindex", C.c_void_p),
                ("nlist", C.c_void_p), ("eweight", C.c_void_p), ("num_antihubs", C.c_int32),
                ("antihubs", C.c_void_p)]


class RunStats(C.Structure):
    _fields_ = [("edges", C.c_int64), ("num_antihubs", C.c_int32), ("num_clusters", C.c_int32),
                ("condensed_size", C.c_int64), ("mst_rounds", C.c_int32),
                ("knn_dropped", C.c_int64), ("ms_knn", C.c_float), ("ms_graph", C.c_float),
                ("ms_mst", C.c_float), ("ms_tree", C.c_float), ("ms_total", C.c_float),
                ("join_ms", C.c_float), ("join_launches", C.c_int32),
                ("join_rows_gathered", C.c_int64), ("join_candidates", C.c_int64),
                ("gpu_launches", C.c_int64), ("mst_multiplier", C.c_int32),
                ("join_config", C.c_int32), ("join_pairs", C.c_int64)]


class Instance(C.Structure):
    _fields_ = [("X", C.c_void_p), ("n", C.c_int64), ("d", C.c_int32),
                ("num_clusters", C.c_int32), ("labels", C.c_void_p), ("G", C.c_void_p),
                ("status", C.c_int32), ("reserved", C.c_int32)]


_L = None
_P, _I32, _I64 = C.c_void_p, C.c_int32, C.c_int64


def load(path: str = LIB_PATH):
    """Loads the library (no GPU needed) and declares every signature."""
    global _L
    if _L is not None:
        return _L
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: run `python -m gpu_hdbscan_b200.build` "
                          "(there is no CPU fallback)")
    L = C.CDLL(path)
    sig = {
        "hdb_version": (C.c_char_p, []),
        "hdb_last_error": (C.c_char_p, []),
        "hdb_create": (C.c_int, [C.POINTER(_P), _I32]),
        "hdb_destroy": (C.c_int, [_P]),
        "hdb_set_stream": (C.c_int, [_P, _P]),
        "hdb_set_join_tiles": (C.c_int, [_P, _I32]),
        "hdb_nndescent": (C.c_int, [_P, _P, _I64, _I32, C.POINTER(KnnParams), _P]),
        "hdb_knn_merge": (C.c_int, [_P, _P, _I64, _P, _P, _I64, _P, _I32,
                                    C.POINTER(KnnParams), _P]),
        "hdb_knn_split": (C.c_int, [_P, _P, _I64, _I32, _P, _P]),
        "hdb_fix_distances": (C.c_int, [_P, _P, _I64, _I32, _P, _I32, _P]),
        "hdb_enhanced_knng": (C.c_int, [_P, _P, _P, _P, _I64, _I32, _I32, C.POINTER(Graph)]),
        "hdb_mst": (C.c_int, [_P, C.POINTER(Graph), _P, _P, C.POINTER(_I32)]),
        "hdb_mst_ordered": (C.c_int, [_P, C.POINTER(Graph), _I32, _P, _P, C.POINTER(_I32)]),
        "hdb_mst_quantised": (C.c_int, [_P, C.POINTER(Graph), _P, _I32, _P, _P, C.POINTER(_I32),
                                        C.POINTER(_I32)]),
        "hdb_sort_edges": (C.c_int, [_P, _P, _I64]),
        "hdb_linkage_tree": (C.c_int, [_P, _P, _I64, _P]),
        "hdb_condense_select": (C.c_int, [_P, _P, _I64, _I32, _I32, _P, C.POINTER(_I32), _P,
                                          C.POINTER(_I64), _P, C.POINTER(_I64)]),
        "hdb_run": (C.c_int, [_P, _P, _I64, _I32, C.POINTER(Params), _P, C.POINTER(RunStats)]),
        "hdb_run_with_graph": (C.c_int, [_P, _P, _I64, _I32, C.POINTER(Params), _P, _P,
                                         C.POINTER(RunStats)]),
        "hdb_run_knn": (C.c_int, [_P, _P, _P, _I64, _I32, C.POINTER(Params), _P,
                                  C.POINTER(RunStats)]),
        "hdb_sort_edges_noalloc": (C.c_int, [_P, _I64, _P]),
        "hdb_bf16_distance_tiles": (C.c_int, [_P, _P, _I64, _I32, _P, _P, _I64, _P]),
        "hdb_core_sg": (C.c_int, [_P, _P, _P, _P, _I64, _I32, _I32, _P, C.POINTER(Graph)]),
        "hdb_run_batched": (C.c_int, [_P, C.POINTER(Instance), _I32, C.POINTER(Params),
                                      C.POINTER(RunStats)]),
        "hdb_run_knn_batched": (C.c_int, [_P, C.POINTER(Instance), _I32, C.POINTER(Params),
                                          C.POINTER(RunStats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _L = L
    return L


def check(status: int):
    if status != HDB_OK:
        raise HdbError(status, load().hdb_last_error().decode())
