// MST stage (mst.cu).
#pragma once
#include "hdb_internal.cuh"

namespace hdb {

// seg: independent instances -> a forest of n - seg.count edges, grouped by
// instance and sorted by (weight, edge index) inside each.
void boruvka_mst(Context *ctx, const hdb_graph *g, uint8_t *in_mst, hdb_mst_edge *mst,
                 int32_t *rounds_out, const Segments &seg = Segments{});
void sort_mst_edges(Context *ctx, hdb_mst_edge *edges, int64_t m);

}  // namespace hdb
