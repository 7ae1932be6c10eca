// MST stage (mst.cu).
#pragma once
#include "hdb_internal.cuh"

namespace hdb {

// seg: independent instances -> a forest, grouped by instance and sorted by
// (weight, edge index) inside each.  Without inst_edges every instance must be
// connected (n - seg.count edges, HDB_ERR_DISCONNECTED otherwise); with it
// (host [seg.count]) each instance's edge count is reported instead and a
// disconnected instance keeps its spanning forest.  Returns the edge count.
int64_t boruvka_mst(Context *ctx, const hdb_graph *g, uint8_t *in_mst, hdb_mst_edge *mst,
                    int32_t *rounds_out, const Segments &seg = Segments{},
                    int32_t *inst_edges = nullptr);
void sort_mst_edges(Context *ctx, hdb_mst_edge *edges, int64_t m);

}  // namespace hdb
