// Enhanced kNN graph stage (graph.cu).
#pragma once
#include "hdb_internal.cuh"

namespace hdb {

struct GraphTimes {
  cudaEvent_t after_antihubs;
};

// core[i]: distance to the k-th neighbour (calculateCoreDistance with index
// k-1, HDBSCAN/graphs/graph.cu:77), or to neighbour `col` when col >= 0.
// mode HDB_DIST_SQRT recomputes it with fix_distances' sqrt-L2 rounding;
// HDB_DIST_SQUARED reads dist[i, col].
void core_distances(Context *ctx, const float *dist, const float *X, const int32_t *ids,
                    int64_t n, int32_t d, int32_t k, int32_t mode, float *core, int32_t col = -1);

// seg: independent instances (antihubs and clique per instance); ids must
// stay inside their row's instance.  Empty for one instance.
void build_enhanced_knng(Context *ctx, const int32_t *ids, const float *core, const float *X,
                         int64_t n, int32_t d, int32_t k, hdb_graph *out, GraphTimes *times,
                         const Segments &seg = Segments{});

// Core-SG (build_CoreSG / Union_kNNG_MST, HDBSCAN/core-sg/core-sg.cu:292-571):
// the kNN graph's CSR (own ids, non-mutual reverse entries) plus the edges
// of the sorted MST, with Euclidean weights.  Output in context-owned buffers.
void build_core_sg(Context *ctx, const int32_t *ids, const float *dist, const float *X, int64_t n,
                   int32_t d, int32_t k, const hdb_mst_edge *mst, hdb_graph *out);

}  // namespace hdb
