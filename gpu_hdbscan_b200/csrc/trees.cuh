// Tree stage (trees.cu).
#pragma once
#include "hdb_internal.cuh"

namespace hdb {

// seg: a forest of one tree per instance (mst holds n - seg.count edges,
// grouped by instance as boruvka_mst leaves them); node n + r for rank r.
void linkage_tree(Context *ctx, const hdb_mst_edge *mst, int64_t n, hdb_linkage_node *out,
                  const Segments &seg = Segments{});

// With seg, every tree is condensed and selected on its own: labels restart
// at 0 in each instance, inst_clusters (host, [seg.count], optional) receives
// each instance's cluster count and *num_clusters the total.  The condensed
// rows and stabilities are available for a single tree only.
void condense_select(Context *ctx, const hdb_linkage_node *h, int64_t n, int32_t mpts,
                     int32_t stab_mode, int32_t *labels, int32_t *num_clusters,
                     hdb_condensed_node *condensed, int64_t *condensed_size,
                     hdb_stability *stability, int64_t *num_stability,
                     const Segments &seg = Segments{}, int32_t *inst_clusters = nullptr);

}  // namespace hdb
