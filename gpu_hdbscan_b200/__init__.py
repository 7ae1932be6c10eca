"""B200-native HDBSCAN path (libhdb_b200.so) -- Python front end.

The functions below mirror the reference's C++ stage interface, in the order
HDBSCAN/_new.cu calls them:

    NNDescent            gpuknn::NNDescent          (gpuknn/nndescent.cuh:40-42)
    fix_distances        fix_distances              (build_kNNG.cu:131-174)
    buildEnhancedKNNG    buildEnhancedKNNG          (HDBSCAN/graphs/graph.cuh:24)
    buildMST             cpuMST + buildMST          (HDBSCAN/mst/mst.cuh:64,91)
    sort_edges           sort_edges                 (HDBSCAN/merge_sort/merge_sort.cuh:30)
    build_Linkage_tree   build_Linkage_tree         (HDBSCAN/trees/tree.cuh:33)
    get_clusters         build_Condensed_tree + compute_stability + get_clusters
                                                    (HDBSCAN/trees/tree.cuh:39-45)
    hdbscan              the whole HDBSCAN/_new.cu order

Arrays are torch tensors on the context's CUDA device (PyTorch only provides
device memory and streams here; all compute is in libhdb_b200.so).  Errors
raise HdbError with the library's status and message.
"""
from __future__ import annotations

import numpy as np
import ctypes as C
from dataclasses import dataclass

from . import _lib

# hdb_instance (include/hdb/hdb.h) as a numpy record, laid out like _lib.Instance
_INSTANCE_DTYPE = np.dtype({"names": ["X", "n", "d", "num_clusters", "labels", "G", "status",
                                      "reserved"],
                            "formats": ["<u8", "<i8", "<i4", "<i4", "<u8", "<u8", "<i4", "<i4"],
                            "offsets": [0, 8, 16, 20, 24, 32, 40, 44], "itemsize": 48})
from ._lib import (HDB_DIST_SQRT, HDB_DIST_SQUARED, HDB_PREC_BF16, HDB_PREC_FP16, HDB_PREC_FP32,
                   HDB_STAB_FP32, HDB_STAB_FP64, HDB_MST_FLOAT, HDB_MST_QUANTISED,
                   HDB_MST_ID_ORDER, HDB_ORDER_EDGE, HDB_ORDER_IDS, HdbError)

__all__ = ["Context", "HdbError", "EnhancedGraph", "HDB_PREC_FP32", "HDB_PREC_BF16", "HDB_PREC_FP16",
           "HDB_DIST_SQRT", "HDB_DIST_SQUARED", "HDB_STAB_FP32", "HDB_STAB_FP64",
           "HDB_MST_FLOAT", "HDB_MST_QUANTISED", "HDB_MST_ID_ORDER", "HDB_ORDER_EDGE", "HDB_ORDER_IDS"]


def _ptr(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


@dataclass
class EnhancedGraph:
    """ECLgraph (HDBSCAN/structs/ECLgraph.h:41-47): views of context-owned memory,
    valid until the next buildEnhancedKNNG on the same context."""
    nodes: int
    edges: int
    nindex: "object"
    nlist: "object"
    eweight: "object"
    antihubs: "object"
    raw: _lib.Graph


class Context:
    """One device, one stream (libhdb_b200 hdb_ctx)."""

    def __init__(self, device: int = 0):
        import torch

        self._torch = torch
        self.L = _lib.load()
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        h = C.c_void_p()
        _lib.check(self.L.hdb_create(C.byref(h), device))
        self.h = h
        # run on torch's current stream so torch allocations order correctly
        _lib.check(self.L.hdb_set_stream(self.h, C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)))

    def set_join_tiles(self, tiles: int):
        """FP32 local join form: 1 or 2 distance tiles of 4 x 4 per lane, or 0
        to time both per shape and keep the faster (the default)."""
        _lib.check(self.L.hdb_set_join_tiles(self.h, int(tiles)))

    def close(self):
        if getattr(self, "h", None):
            self.L.hdb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- helpers ----------------------------------------------------------
    def _dev(self, t, dtype):
        torch = self._torch
        t = torch.as_tensor(t)
        return t.to(device=self.device, dtype=dtype).contiguous()

    # -- stages -----------------------------------------------------------
    def NNDescent(self, X, k=32, sample_num=16, iterations=6, precision=HDB_PREC_FP32):
        """X [n, d] float32 -> G [n, k, 2] int32 (NNDElement rows: distance bits, label)."""
        torch = self._torch
        X = self._dev(X, torch.float32)
        n, d = X.shape
        G = torch.empty((n, k, 2), dtype=torch.int32, device=self.device)
        p = _lib.KnnParams(k, sample_num, iterations, precision)
        _lib.check(self.L.hdb_nndescent(self.h, _ptr(X), n, d, C.byref(p), _ptr(G)))
        return G

    def KNNMerge(self, X1, G1, X2, G2, sample_num=12, iterations=11):
        """gpuknn::KNNMerge (knnmerge.cuh:8-12; KNNMergeFromHost :14-18 when the
        inputs are host arrays): X1 [n1, d], X2 [n2, d] float32 and their kNN
        graphs G1 [n1, k, 2], G2 [n2, k, 2] (NNDElement rows, ids local to their
        set) -> G [n1 + n2, k, 2] on the device, the rows of X1 first and the ids
        of X2 shifted by n1.  Defaults are MERGE_SAMPLE_NUM and MERGE_ITERATION."""
        torch = self._torch
        X1 = self._dev(X1, torch.float32)
        X2 = self._dev(X2, torch.float32)
        G1 = self._dev(G1, torch.int32)
        G2 = self._dev(G2, torch.int32)
        n1, d = X1.shape
        n2 = X2.shape[0]
        k = G1.shape[1]
        if X2.shape[1] != d or G2.shape[1] != k or G1.shape[0] != n1 or G2.shape[0] != n2:
            raise ValueError("KNNMerge: X1/X2 need the same d and G1/G2 the same k, one row per point")
        G = torch.empty((n1 + n2, k, 2), dtype=torch.int32, device=self.device)
        p = _lib.KnnParams(k, sample_num, iterations, HDB_PREC_FP32)
        _lib.check(self.L.hdb_knn_merge(self.h, _ptr(X1), n1, _ptr(G1), _ptr(X2), n2, _ptr(G2), d,
                                        C.byref(p), _ptr(G)))
        return G

    def knn_split(self, G):
        """G [n, k, 2] -> (ids int32 [n, k] with the old/new flag decoded, dist float32)."""
        torch = self._torch
        n, k, _ = G.shape
        ids = torch.empty((n, k), dtype=torch.int32, device=self.device)
        dist = torch.empty((n, k), dtype=torch.float32, device=self.device)
        _lib.check(self.L.hdb_knn_split(self.h, _ptr(G), n, k, _ptr(ids), _ptr(dist)))
        return ids, dist

    def fix_distances(self, X, ids):
        torch = self._torch
        X = self._dev(X, torch.float32)
        ids = self._dev(ids, torch.int32)
        n, k = ids.shape
        dist = torch.empty((n, k), dtype=torch.float32, device=self.device)
        _lib.check(self.L.hdb_fix_distances(self.h, _ptr(X), n, X.shape[1], _ptr(ids), k,
                                            _ptr(dist)))
        return dist

    def bf16_distance_tiles(self, X, ids, counts):
        """BF16 tensor-core distances of explicit slot lists (the arithmetic of
        the BF16 local join): ids [tiles, 128], counts [tiles, 4] ->
        [tiles, 128, 64] float32 (see hdb_bf16_distance_tiles)."""
        torch = self._torch
        X = self._dev(X, torch.float32)
        ids = self._dev(ids, torch.int32)
        counts = self._dev(counts, torch.int32)
        tiles = ids.shape[0]
        out = torch.empty((tiles, 128, 64), dtype=torch.float32, device=self.device)
        _lib.check(self.L.hdb_bf16_distance_tiles(self.h, _ptr(X), X.shape[0], X.shape[1],
                                                  _ptr(ids), _ptr(counts), tiles, _ptr(out)))
        return out

    def build_CoreSG(self, ids, dist, X, mst) -> EnhancedGraph:
        """Core-SG (kNN graph + MST, Euclidean weights) of ids/dist [n, k], X and
        the sorted MST (MST_EDGE records, e.g. buildMST's output)."""
        torch = self._torch
        ids = self._dev(ids, torch.int32)
        dist = self._dev(dist, torch.float32)
        X = self._dev(X, torch.float32)
        if isinstance(mst, np.ndarray) and mst.dtype.names:  # MSTedge records
            mst = mst.view(np.int32).reshape(-1, 3)
        mst = self._dev(mst, torch.int32)
        n, k = ids.shape
        g = _lib.Graph()
        _lib.check(self.L.hdb_core_sg(self.h, _ptr(ids), _ptr(dist), _ptr(X), n, X.shape[1], k,
                                      _ptr(mst), C.byref(g)))
        empty = torch.empty(0, dtype=torch.int32, device=self.device)
        return EnhancedGraph(g.nodes, g.edges, self._view(g.nindex, g.nodes + 1, torch.int64),
                             self._view(g.nlist, g.edges, torch.int32),
                             self._view(g.eweight, g.edges, torch.float32), empty, g)

    def buildEnhancedKNNG(self, ids, dist, X) -> EnhancedGraph:
        torch = self._torch
        ids = self._dev(ids, torch.int32)
        dist = self._dev(dist, torch.float32)
        X = self._dev(X, torch.float32)
        n, k = ids.shape
        g = _lib.Graph()
        _lib.check(self.L.hdb_enhanced_knng(self.h, _ptr(ids), _ptr(dist), _ptr(X), n,
                                            X.shape[1], k, C.byref(g)))
        return EnhancedGraph(g.nodes, g.edges, self._view(g.nindex, g.nodes + 1, torch.int64),
                             self._view(g.nlist, g.edges, torch.int32),
                             self._view(g.eweight, g.edges, torch.float32),
                             self._view(g.antihubs, g.num_antihubs, torch.int32), g)

    def graph_from_csr(self, nindex, nlist, eweight) -> EnhancedGraph:
        """An ECLgraph over caller arrays (nindex [n+1] int64, nlist [E] int32,
        eweight [E] float32, copied to the device), e.g. for hdb_mst on a graph
        that was not built here.  The returned object keeps the arrays alive."""
        torch = self._torch
        ni = self._dev(nindex, torch.int64)
        nl = self._dev(nlist, torch.int32)
        ew = self._dev(eweight, torch.float32)
        if ni.dim() != 1 or nl.shape != ew.shape or ni.shape[0] < 2 or int(ni[-1]) != nl.shape[0]:
            raise ValueError("graph_from_csr: inconsistent CSR arrays")
        empty = torch.empty(0, dtype=torch.int32, device=self.device)
        g = _lib.Graph(ni.shape[0] - 1, nl.shape[0], ni.data_ptr(), nl.data_ptr(), ew.data_ptr(),
                       0, None)
        return EnhancedGraph(g.nodes, g.edges, ni, nl, ew, empty, g)

    def _view(self, ptr, count, dtype):
        """Copies `count` elements of context-owned device memory into a tensor."""
        torch = self._torch
        out = torch.empty(count, dtype=dtype, device=self.device)
        if count:
            torch.cuda.synchronize(self.device)
            res = _cudart().cudaMemcpy(C.c_void_p(out.data_ptr()), C.c_void_p(ptr),
                                       C.c_size_t(count * out.element_size()), 3)
            if res != 0:
                raise HdbError(_lib.HDB_ERR_CUDA, f"cudaMemcpy failed ({res})")
        return out

    def buildMST(self, graph: EnhancedGraph, with_in_mst=False, order=None):
        """-> (mst [n-1, 3] int32 view of MSTedge sorted by (weight, edge index),
               in_mst uint8 [edges] or None, Boruvka rounds).  order=HDB_ORDER_IDS
        spans and lists the tree under (weight, min id, max id) instead
        (hdb_mst_ordered); None or HDB_ORDER_EDGE is the reference's hdb_mst."""
        torch = self._torch
        n = graph.nodes
        mst = torch.empty((n - 1, 3), dtype=torch.int32, device=self.device)
        inm = torch.empty(graph.edges, dtype=torch.uint8, device=self.device) if with_in_mst else None
        rounds = C.c_int32(0)
        if order is None:
            _lib.check(self.L.hdb_mst(self.h, C.byref(graph.raw), _ptr(inm), _ptr(mst),
                                      C.byref(rounds)))
        else:
            _lib.check(self.L.hdb_mst_ordered(self.h, C.byref(graph.raw), order, _ptr(inm),
                                              _ptr(mst), C.byref(rounds)))
        return mst, inm, rounds.value

    def buildMST_quantised(self, graph: EnhancedGraph, dist, with_in_mst=False):
        """The reference's mst_gpu = 1 MST (hdb_mst_quantised): dist [n, k] the
        kNN distances the graph was built from (its first column sets the
        scale).  -> (mst [n-1, 3] int32 view of MSTedge, in_mst or None,
        multiplier m, Boruvka rounds)."""
        torch = self._torch
        n = graph.nodes
        dist = self._dev(dist, torch.float32)
        mst = torch.empty((n - 1, 3), dtype=torch.int32, device=self.device)
        inm = torch.empty(graph.edges, dtype=torch.uint8, device=self.device) if with_in_mst else None
        rounds, mult = C.c_int32(0), C.c_int32(0)
        _lib.check(self.L.hdb_mst_quantised(self.h, C.byref(graph.raw), _ptr(dist), dist.shape[1],
                                            _ptr(inm), _ptr(mst), C.byref(mult), C.byref(rounds)))
        return mst, inm, mult.value, rounds.value

    def sort_edges(self, mst):
        """In place: stable ascending sort of MSTedge rows by weight."""
        _lib.check(self.L.hdb_sort_edges(self.h, _ptr(mst), mst.shape[0]))
        return mst

    def build_Linkage_tree(self, mst, n):
        torch = self._torch
        hier = torch.empty((n - 1, 4), dtype=torch.int32, device=self.device)
        _lib.check(self.L.hdb_linkage_tree(self.h, _ptr(mst), n, _ptr(hier)))
        return hier

    def get_clusters(self, hier, n, mpts, stability=HDB_STAB_FP32, want_tree=False):
        """-> (labels int32 [n], num_clusters, condensed [rows, 4] or None,
               stabilities [C, 2] or None)."""
        torch = self._torch
        labels = torch.empty(n, dtype=torch.int32, device=self.device)
        ncl = C.c_int32(0)
        cond = stab = None
        csize = C.c_int64(0)
        nst = C.c_int64(0)
        if want_tree:
            cap = n + 2 * (n // max(mpts, 1)) + 2
            cond = torch.empty((cap, 4), dtype=torch.int32, device=self.device)
            stab = torch.empty((cap, 2), dtype=torch.int32, device=self.device)
        _lib.check(self.L.hdb_condense_select(self.h, _ptr(hier), n, mpts, stability, _ptr(labels),
                                              C.byref(ncl), _ptr(cond), C.byref(csize), _ptr(stab),
                                              C.byref(nst)))
        if want_tree:
            cond = cond[: csize.value]
            stab = stab[: nst.value]
        return labels, ncl.value, cond, stab

    def hdbscan(self, X, k=32, mpts=32, sample_num=16, iterations=6, precision=HDB_PREC_FP32,
                distance=HDB_DIST_SQRT, stability=HDB_STAB_FP32, labels_out=None, mst_gpu=0,
                want_graph=False):
        """The whole path (hdb_run).  X on the host (numpy / CPU tensor) runs with
        host_io=1: the H2D copy of X and the D2H copy of the labels are inside
        the call.  X on the device returns device labels.  want_graph=True
        (hdb_run_with_graph) also returns the kNN graph the labels were
        computed from, [n, k, 2] NNDElement rows beside the labels:
        (labels, stats, G)."""
        torch = self._torch
        host = not (isinstance(X, torch.Tensor) and X.is_cuda)
        dev = None if host else self.device
        if host:
            X = torch.as_tensor(X, dtype=torch.float32).contiguous()
        else:
            X = X.to(torch.float32).contiguous()
        labels = labels_out if labels_out is not None else torch.empty(
            X.shape[0], dtype=torch.int32, device=dev)
        n, d = X.shape
        p = _lib.Params(_lib.KnnParams(k, sample_num, iterations, precision), mpts, distance,
                        stability, 1 if host else 0, mst_gpu)
        st = _lib.RunStats()
        if want_graph:
            G = torch.empty((n, k, 2), dtype=torch.int32, device=dev)
            _lib.check(self.L.hdb_run_with_graph(self.h, _ptr(X), n, d, C.byref(p), _ptr(labels),
                                                 _ptr(G), C.byref(st)))
            return labels, {f: getattr(st, f) for f, _ in _lib.RunStats._fields_}, G
        _lib.check(self.L.hdb_run(self.h, _ptr(X), n, d, C.byref(p), _ptr(labels), C.byref(st)))
        return labels, {f: getattr(st, f) for f, _ in _lib.RunStats._fields_}

    def hdbscan_batched(self, Xs, k=32, mpts=32, sample_num=16, iterations=6,
                        precision=HDB_PREC_FP32, distance=HDB_DIST_SQRT,
                        stability=HDB_STAB_FP32, want_graphs=False, strict=True, mst_gpu=0):
        """Independent runs of the whole path on every array of Xs in shared
        launches (hdb_run_batched).  Host arrays run with host_io=1 (copies
        inside the call); CUDA tensors give device results.
        -> (labels per instance, cluster counts, stats[, kNN graphs [n, k, 2]
        with instance-local ids]).  stats["instance_status"] holds each
        instance's status; an instance whose enhanced kNN graph is disconnected
        raises HdbError when strict, else keeps labels -1 and status
        HDB_ERR_DISCONNECTED while the others complete."""
        p = _lib.Params(_lib.KnnParams(k, sample_num, iterations, precision), mpts, distance,
                        stability, 0, mst_gpu)
        return self._batched(self.L.hdb_run_batched, Xs, None, k, p, want_graphs, strict)

    def hdbscan_batched_from_knn(self, Gs, Xs, k=32, mpts=32, distance=HDB_DIST_SQRT,
                                 stability=HDB_STAB_FP32, strict=True, mst_gpu=0):
        """The stages after the kNN graph on many instances in shared launches
        (hdb_run_knn_batched): Gs[i] [n_i, k, 2] NNDElement rows with
        instance-local ids, Xs[i] [n_i, d_i].  -> (labels, cluster counts, stats)."""
        p = _lib.Params(_lib.KnnParams(k, max(1, k // 2), 0, HDB_PREC_FP32), mpts, distance,
                        stability, 0, mst_gpu)
        return self._batched(self.L.hdb_run_knn_batched, Xs, Gs, k, p, False, strict)

    def _batched(self, fn, Xs, Gs, k, p, want_graphs, strict):
        torch = self._torch
        host = not (isinstance(Xs[0], torch.Tensor) and Xs[0].is_cuda)
        dev = None if host else self.device
        p.host_io = 1 if host else 0
        Xs = [torch.as_tensor(X, dtype=torch.float32).contiguous() if host
              else X.to(torch.float32).contiguous() for X in Xs]
        if Gs is not None:
            Gs = [torch.as_tensor(G).to(dtype=torch.int32).contiguous() if host
                  else G.to(device=self.device, dtype=torch.int32).contiguous() for G in Gs]
        # one label buffer (and one graph buffer) for all instances, split into
        # views, and the hdb_instance records filled column by column: per-call
        # host work that does not grow by a Python loop of allocations
        T = len(Xs)
        ns = np.fromiter((X.shape[0] for X in Xs), dtype=np.int64, count=T)
        off = np.zeros(T + 1, dtype=np.int64)
        np.cumsum(ns, out=off[1:])
        lab_all = torch.empty(int(off[-1]), dtype=torch.int32, device=dev)
        labels = [lab_all[int(off[i]):int(off[i + 1])] for i in range(T)]
        if want_graphs:
            g_all = torch.empty((int(off[-1]), k, 2), dtype=torch.int32, device=dev)
            graphs = [g_all[int(off[i]):int(off[i + 1])] for i in range(T)]
        else:
            graphs = Gs
        rec = np.zeros(T, dtype=_INSTANCE_DTYPE)
        rec["X"] = np.fromiter((X.data_ptr() for X in Xs), dtype=np.uint64, count=T)
        rec["n"] = ns
        rec["d"] = np.fromiter((X.shape[1] for X in Xs), dtype=np.int32, count=T)
        rec["labels"] = np.uint64(lab_all.data_ptr()) + (off[:-1] * 4).astype(np.uint64)
        if graphs is not None:
            rec["G"] = np.fromiter((G_.data_ptr() for G_ in graphs), dtype=np.uint64, count=T)
        insts = (_lib.Instance * T).from_buffer(rec)
        st = _lib.RunStats()
        rc = fn(self.h, insts, T, C.byref(p), C.byref(st))
        if rc != _lib.HDB_OK and (strict or rc != _lib.HDB_ERR_DISCONNECTED):
            _lib.check(rc)
        stats = {f: getattr(st, f) for f, _ in _lib.RunStats._fields_}
        stats["instance_status"] = rec["status"].tolist()
        ncl = rec["num_clusters"].tolist()
        if want_graphs:
            return labels, ncl, stats, graphs
        return labels, ncl, stats

    def hdbscan_from_knn(self, G, X, k=32, mpts=32, distance=HDB_DIST_SQRT,
                         stability=HDB_STAB_FP32, mst_gpu=0):
        """The stages after the kNN graph (hdb_run_knn): G [n, k, 2] NNDElement rows,
        X [n, d].  Device tensors -> device labels; host arrays -> host labels
        (host_io: copies inside the call)."""
        torch = self._torch
        host = not (isinstance(X, torch.Tensor) and X.is_cuda)
        if host:
            X = torch.as_tensor(X, dtype=torch.float32).contiguous()
            G = torch.as_tensor(G).cpu().contiguous()
            labels = torch.empty(X.shape[0], dtype=torch.int32)
        else:
            X = X.to(torch.float32).contiguous()
            G = G.to(self.device).contiguous()
            labels = torch.empty(X.shape[0], dtype=torch.int32, device=self.device)
        n, d = X.shape
        p = _lib.Params(_lib.KnnParams(k, max(1, k // 2), 0, HDB_PREC_FP32), mpts, distance,
                        stability, 1 if host else 0, mst_gpu)
        st = _lib.RunStats()
        _lib.check(self.L.hdb_run_knn(self.h, _ptr(G), _ptr(X), n, d, C.byref(p), _ptr(labels),
                                      C.byref(st)))
        return labels, {f: getattr(st, f) for f, _ in _lib.RunStats._fields_}


_CUDART = None


def _cudart():
    """The CUDA runtime, for device-to-device copies out of context-owned memory."""
    global _CUDART
    if _CUDART is None:
        import glob
        import os
        cands = ["libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so.12"]
        try:
            import nvidia.cuda_runtime as _nv  # pip CUDA runtime shipped with torch
            cands += glob.glob(os.path.join(list(_nv.__path__)[0], "lib", "libcudart.so*"))
        except Exception:
            pass
        for c in cands:
            try:
                _CUDART = C.CDLL(c)
                break
            except OSError:
                continue
        if _CUDART is None:
            raise ImportError("libcudart.so.12 not found")
        _CUDART.cudaMemcpy.restype = C.c_int
        _CUDART.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return _CUDART


def version() -> str:
    return _lib.load().hdb_version().decode()
