// Tree stage (trees.cu).
#pragma once
#include "hdb_internal.cuh"

namespace hdb {

void linkage_tree(Context *ctx, const hdb_mst_edge *mst, int64_t n, hdb_linkage_node *out);

void condense_select(Context *ctx, const hdb_linkage_node *h, int64_t n, int32_t mpts,
                     int32_t stab_mode, int32_t *labels, int32_t *num_clusters,
                     hdb_condensed_node *condensed, int64_t *condensed_size,
                     hdb_stability *stability, int64_t *num_stability);

}  // namespace hdb
