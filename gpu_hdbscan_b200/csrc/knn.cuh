// kNN graph stage (knn.cu).
#pragma once
#include "hdb_internal.cuh"

namespace hdb {

// Live measurement of the local-join kernel: summed CUDA-event time over
// its launches, rows staged in shared memory and candidates pushed.
struct JoinStats {
  double ms = 0.0;
  int64_t launches = 0, rows_gathered = 0, candidates = 0, pairs = 0;
  int32_t config = 0;  // FP32 join tile slots per lane (1 or 2); 0: a 16-bit join
};

// seg: independent instances in one run (each row's neighbours stay inside
// its instance); empty for one instance.  Every instance needs more than k rows.
void nndescent(Context *ctx, const float *X, int64_t n, int32_t d, const hdb_knn_params &p,
               hdb_nnd_element *G, int64_t *dropped_out, JoinStats *js = nullptr,
               const Segments &seg = Segments{});
// Device bytes per point that nndescent holds at its peak: X in locality
// order, the 16-bit rows, lists, samples, inboxes, the candidate list and its
// sort buffers, the graph before it is mapped back.
int64_t nndescent_bytes_per_point(int32_t d, const hdb_knn_params &p);
// Merge of the kNN graphs of two point sets into the graph of their union
// (hdb_knn_merge): FP32 join, old samples from the row's own set only.
void knn_merge(Context *ctx, const float *X1, int64_t n1, const hdb_nnd_element *G1,
               const float *X2, int64_t n2, const hdb_nnd_element *G2, int32_t d,
               const hdb_knn_params &p, hdb_nnd_element *G, int64_t *dropped_out);
// BF16 tensor-core distances for explicit slot lists (hdb_bf16_distance_tiles).
void bf16_distance_tiles(Context *ctx, const float *X, int64_t n, int32_t d, const int32_t *ids,
                         const int32_t *counts, int64_t tiles, float *out);
void knn_split(Context *ctx, const hdb_nnd_element *G, int64_t n, int32_t k, int32_t *ids,
               float *dist);
void fix_distances(Context *ctx, const float *X, int64_t n, int32_t d, const int32_t *ids,
                   int32_t k, float *dist);

}  // namespace hdb
