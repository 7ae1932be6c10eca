// MST stage (mst.cu).
#pragma once
#include "hdb_internal.cuh"

namespace hdb {

// seg: independent instances -> a forest, grouped by instance and sorted by
// (weight, edge index) inside each.  Without inst_edges every instance must be
// connected (n - seg.count edges, HDB_ERR_DISCONNECTED otherwise); with it
// (host [seg.count]) each instance's edge count is reported instead and a
// disconnected instance keeps its spanning forest.  Returns the edge count.
// quant (device, one per instance or one): 10^m of the reference's mst_gpu = 1
// mode (quant_scales) -- the tree under (int-quantised weight, edge index),
// written with dequantised weights in (weight, edge index) order; nullptr for
// the float weights of cpuMST.  id_order (float weights only): the tree and
// its listing under (weight, min id, max id, edge index) instead of (weight,
// edge index).
int64_t boruvka_mst(Context *ctx, const hdb_graph *g, uint8_t *in_mst, hdb_mst_edge *mst,
                    int32_t *rounds_out, const Segments &seg = Segments{},
                    int32_t *inst_edges = nullptr, const double *quant = nullptr,
                    bool id_order = false);
// The mst_gpu = 1 scale of every instance (buildGPUgraph, core-sg.cu:8-44, with
// GetMinDistanceFromKNNG's minimum): first[i * stride] is row i's first kNN
// distance; p10_dev (device) and mult_out (host, optional) get one value per
// instance (one without seg).
void quant_scales(Context *ctx, const float *first, int64_t stride, int64_t n, const Segments &seg,
                  double *p10_dev, int32_t *mult_out);
void sort_mst_edges(Context *ctx, hdb_mst_edge *edges, int64_t m);

}  // namespace hdb
