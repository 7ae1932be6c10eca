// extern "C" entry points of libhdb_b200 (include/hdb/hdb.h) and the
// end-to-end pipeline in the reference's HDBSCAN/_new.cu order.
#include <algorithm>
#include <map>
#include <vector>

#include "graph.cuh"
#include "hdb_internal.cuh"
#include "join_tc.cuh"
#include "knn.cuh"
#include "mst.cuh"
#include "trees.cuh"

using namespace hdb;

namespace {

Context *C(hdb_ctx *h) {
  HDB_REQUIRE(h != nullptr, HDB_ERR_ARG, "NULL context");
  HDB_CUDA(cudaSetDevice(h->c.device));
  return &h->c;
}

void require_ptr(const void *p, const char *what) {
  HDB_REQUIRE(p != nullptr, HDB_ERR_ARG, std::string("NULL pointer: ") + what);
}

void check_knn_params(const hdb_knn_params *p) {
  require_ptr(p, "params");
  HDB_REQUIRE(p->k >= 1 && p->k <= 32, HDB_ERR_ARG, "k (NEIGHB_NUM_PER_LIST) must be in [1, 32]");
  HDB_REQUIRE(p->sample_num >= 1 && 2 * p->sample_num <= p->k, HDB_ERR_ARG,
              "SAMPLE_NUM must satisfy 2*SAMPLE_NUM <= k");
  HDB_REQUIRE(p->iterations >= 0 && p->iterations <= 1000, HDB_ERR_ARG,
              "NND_ITERATION must be in [0, 1000]");
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.0f;
  HDB_CUDA(cudaEventElapsedTime(&ms, a, b));
  return ms;
}

}  // namespace

extern "C" {

HDB_API hdb_status hdb_nndescent(hdb_ctx *h, const float *X, int64_t n, int32_t d,
                                 const hdb_knn_params *params, hdb_nnd_element *G) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(X, "X");
    require_ptr(G, "G");
    check_knn_params(params);
    nndescent(ctx, X, n, d, *params, G, nullptr);
  });
}

HDB_API hdb_status hdb_knn_merge(hdb_ctx *h, const float *X1, int64_t n1,
                                 const hdb_nnd_element *G1, const float *X2, int64_t n2,
                                 const hdb_nnd_element *G2, int32_t d,
                                 const hdb_knn_params *params, hdb_nnd_element *G) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(X1, "X1");
    require_ptr(X2, "X2");
    require_ptr(G1, "G1");
    require_ptr(G2, "G2");
    require_ptr(G, "G");
    check_knn_params(params);
    knn_merge(ctx, X1, n1, G1, X2, n2, G2, d, *params, G, nullptr);
  });
}

HDB_API hdb_status hdb_knn_split(hdb_ctx *h, const hdb_nnd_element *G, int64_t n, int32_t k,
                                 int32_t *ids, float *dist) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(G, "G");
    HDB_REQUIRE(n >= 0 && k >= 1, HDB_ERR_ARG, "bad n or k");
    knn_split(ctx, G, n, k, ids, dist);
    ctx->sync();
  });
}

HDB_API hdb_status hdb_fix_distances(hdb_ctx *h, const float *X, int64_t n, int32_t d,
                                     const int32_t *ids, int32_t k, float *dist) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(X, "X");
    require_ptr(ids, "ids");
    require_ptr(dist, "dist");
    HDB_REQUIRE(n >= 0 && k >= 1 && d >= 1, HDB_ERR_ARG, "bad n, k or d");
    fix_distances(ctx, X, n, d, ids, k, dist);
    ctx->sync();
  });
}

HDB_API hdb_status hdb_bf16_distance_tiles(hdb_ctx *h, const float *X, int64_t n, int32_t d,
                                           const int32_t *ids, const int32_t *counts,
                                           int64_t tiles, float *out) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(X, "X");
    require_ptr(ids, "ids");
    require_ptr(counts, "counts");
    require_ptr(out, "out");
    HDB_REQUIRE(tiles >= 0 && tiles <= (int64_t(1) << 24), HDB_ERR_ARG, "bad tile count");
    // the slot lists are small: check them on the host before any device read
    std::vector<int32_t> hc((size_t)tiles * 4), hi((size_t)tiles * kTcTileRows);
    HDB_CUDA(cudaMemcpy(hc.data(), counts, hc.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
    HDB_CUDA(cudaMemcpy(hi.data(), ids, hi.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
    for (int64_t t = 0; t < tiles; t++)
      for (int j = 0; j < 2; j++)
        for (int h2 = 0; h2 < 2; h2++) {
          const int32_t c = hc[t * 4 + 2 * j + h2];
          HDB_REQUIRE(c >= 0 && c <= 32, HDB_ERR_ARG, "slot count outside [0, 32]");
          for (int s = 0; s < c; s++) {
            const int32_t id = hi[t * kTcTileRows + 64 * j + 32 * h2 + s];
            HDB_REQUIRE(id >= 0 && id < n, HDB_ERR_ARG, "slot id outside [0, n)");
          }
        }
    bf16_distance_tiles(ctx, X, n, d, ids, counts, tiles, out);
  });
}

HDB_API hdb_status hdb_enhanced_knng(hdb_ctx *h, const int32_t *ids, const float *dist,
                                     const float *X, int64_t n, int32_t d, int32_t k,
                                     hdb_graph *graph) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(ids, "ids");
    require_ptr(dist, "dist");
    require_ptr(X, "X");
    require_ptr(graph, "graph");
    HDB_REQUIRE(n >= 2 && k >= 1 && k <= 32 && k < n && d >= 1, HDB_ERR_ARG,
                "enhanced kNN graph: need n >= 2, 1 <= k <= 32, k < n, d >= 1");
    Buf<float> core(ctx, n);
    core_distances(ctx, dist, X, ids, n, d, k, HDB_DIST_SQUARED, core);
    build_enhanced_knng(ctx, ids, core, X, n, d, k, graph, nullptr);
  });
}

HDB_API hdb_status hdb_core_sg(hdb_ctx *h, const int32_t *ids, const float *dist, const float *X,
                               int64_t n, int32_t d, int32_t k, const hdb_mst_edge *mst,
                               hdb_graph *graph) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(ids, "ids");
    require_ptr(dist, "dist");
    require_ptr(X, "X");
    require_ptr(mst, "mst");
    require_ptr(graph, "graph");
    build_core_sg(ctx, ids, dist, X, n, d, k, mst, graph);
  });
}

HDB_API hdb_status hdb_mst(hdb_ctx *h, const hdb_graph *graph, uint8_t *in_mst, hdb_mst_edge *mst,
                           int32_t *rounds) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(graph, "graph");
    require_ptr(mst, "mst");
    boruvka_mst(ctx, graph, in_mst, mst, rounds);
  });
}

HDB_API hdb_status hdb_mst_ordered(hdb_ctx *h, const hdb_graph *graph, int32_t order,
                                   uint8_t *in_mst, hdb_mst_edge *mst, int32_t *rounds) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(graph, "graph");
    require_ptr(mst, "mst");
    HDB_REQUIRE(order == HDB_ORDER_EDGE || order == HDB_ORDER_IDS, HDB_ERR_ARG,
                "hdb_mst_ordered: unknown tie order");
    boruvka_mst(ctx, graph, in_mst, mst, rounds, Segments{}, nullptr, nullptr,
                order == HDB_ORDER_IDS);
  });
}

HDB_API hdb_status hdb_mst_quantised(hdb_ctx *h, const hdb_graph *graph, const float *dist,
                                     int32_t k, uint8_t *in_mst, hdb_mst_edge *mst,
                                     int32_t *multiplier, int32_t *rounds) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(graph, "graph");
    require_ptr(dist, "dist");
    require_ptr(mst, "mst");
    HDB_REQUIRE(k >= 1 && graph->nodes >= 2, HDB_ERR_ARG, "hdb_mst_quantised: bad k or graph");
    Buf<double> p10(ctx, 1);
    int32_t mult = 0;
    quant_scales(ctx, dist, k, graph->nodes, Segments{}, p10, &mult);
    boruvka_mst(ctx, graph, in_mst, mst, rounds, Segments{}, nullptr, p10);
    if (multiplier) *multiplier = mult;
  });
}

HDB_API hdb_status hdb_sort_edges(hdb_ctx *h, hdb_mst_edge *edges, int64_t m) {
  return guard([&] {
    Context *ctx = C(h);
    HDB_REQUIRE(m >= 0, HDB_ERR_ARG, "negative edge count");
    if (m > 0) require_ptr(edges, "edges");
    HDB_REQUIRE(m < (int64_t(1) << 32), HDB_ERR_ARG, "sort_edges: 2^32 or more edges");
    sort_mst_edges(ctx, edges, m);
  });
}

HDB_API hdb_status hdb_linkage_tree(hdb_ctx *h, const hdb_mst_edge *sorted, int64_t n,
                                    hdb_linkage_node *hierarchy) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(sorted, "sorted");
    require_ptr(hierarchy, "hierarchy");
    linkage_tree(ctx, sorted, n, hierarchy);
  });
}

HDB_API hdb_status hdb_condense_select(hdb_ctx *h, const hdb_linkage_node *hierarchy, int64_t n,
                                       int32_t mpts, int32_t stability_mode, int32_t *labels,
                                       int32_t *num_clusters, hdb_condensed_node *condensed,
                                       int64_t *condensed_size, hdb_stability *stability,
                                       int64_t *num_stability) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(hierarchy, "hierarchy");
    require_ptr(labels, "labels");
    HDB_REQUIRE(stability_mode == HDB_STAB_FP32 || stability_mode == HDB_STAB_FP64, HDB_ERR_ARG,
                "unknown stability mode");
    int32_t nc = 0;
    condense_select(ctx, hierarchy, n, mpts, stability_mode, labels, &nc, condensed,
                    condensed_size, stability, num_stability);
    if (num_clusters) *num_clusters = nc;
  });
}

}  // extern "C"

namespace {

void check_run_params(const hdb_params &p) {
  check_knn_params(&p.knn);
  HDB_REQUIRE(p.mst_gpu == HDB_MST_FLOAT || p.mst_gpu == HDB_MST_QUANTISED ||
                  p.mst_gpu == HDB_MST_ID_ORDER,
              HDB_ERR_ARG, "mst_gpu must be 0, 1 or 2");
  const int32_t k = p.knn.k;
  HDB_REQUIRE(p.mpts >= 2 && p.mpts <= k, HDB_ERR_ARG, "mpts must satisfy 2 <= mpts <= k");
  HDB_REQUIRE(p.distance == HDB_DIST_SQRT || p.distance == HDB_DIST_SQUARED, HDB_ERR_ARG,
              "unknown distance mode");
  HDB_REQUIRE(p.stability == HDB_STAB_FP32 || p.stability == HDB_STAB_FP64, HDB_ERR_ARG,
              "unknown stability mode");
}

// The stages after the kNN graph (HDBSCAN/_new.cu:243-347) on device arrays:
// ids [n, k] decoded, core [n], X [n, d] -> labels [n].  Records ev[3..5].
// first (p.mst_gpu == HDB_MST_QUANTISED only): every row's first-neighbour distance.
void run_after_knn(Context *ctx, const int32_t *ids, const float *core, const float *X, int64_t n,
                   int32_t d, int32_t k, const hdb_params &p, int32_t *labels, hdb_run_stats *st,
                   const float *first) {
  cudaStream_t s = ctx->stream;
  hdb_graph g;
  build_enhanced_knng(ctx, ids, core, X, n, d, k, &g, nullptr);
  HDB_CUDA(cudaEventRecord(ctx->ev[3], s));
  int32_t rounds = 0;
  Buf<hdb_mst_edge> mst(ctx, n - 1);
  Buf<double> p10;
  if (p.mst_gpu == HDB_MST_QUANTISED) {
    p10 = Buf<double>(ctx, 1);
    quant_scales(ctx, first, 1, n, Segments{}, p10, &st->mst_multiplier);
  }
  boruvka_mst(ctx, &g, nullptr, mst, &rounds, Segments{}, nullptr, p10.get(),
              p.mst_gpu == HDB_MST_ID_ORDER);
  HDB_CUDA(cudaEventRecord(ctx->ev[4], s));
  int32_t ncl = 0;
  {
    Buf<hdb_linkage_node> hier(ctx, n - 1);
    linkage_tree(ctx, mst, n, hier);
    condense_select(ctx, hier, n, p.mpts, p.stability, labels, &ncl, nullptr, nullptr, nullptr,
                    nullptr);
  }
  HDB_CUDA(cudaEventRecord(ctx->ev[5], s));
  st->edges = g.edges;
  st->num_antihubs = g.num_antihubs;
  st->num_clusters = ncl;
  st->mst_rounds = rounds;
}

void fill_times(Context *ctx, hdb_run_stats *st, bool with_knn) {
  cudaEvent_t *ev = ctx->ev;
  st->ms_knn = with_knn ? elapsed(ev[1], ev[2]) : 0.0f;
  st->ms_graph = elapsed(ev[2], ev[3]);
  st->ms_mst = elapsed(ev[3], ev[4]);
  st->ms_tree = elapsed(ev[4], ev[5]);
  st->ms_total = elapsed(ev[0], ev[6]);
}

// ---- hdb_run_batched: instances of one d laid back to back -----------------
// Row-major [rows, d] blocks of several instances copied into one array.
__global__ void k_pack_rows(const float *const *__restrict__ src, Segments seg, int d,
                            float *__restrict__ dst) {
  const int64_t total = seg.off[seg.count] * d;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = seg.of_point(i / d);
    dst[i] = src[t][i - seg.off[t] * d];
  }
}

__global__ void k_unpack_labels(const int32_t *__restrict__ src, Segments seg,
                                int32_t *const *__restrict__ dst) {
  const int64_t total = seg.off[seg.count];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = seg.of_point(i);
    dst[t][i - seg.off[t]] = src[i];
  }
}

__global__ void k_pack_graph(const hdb_nnd_element *const *__restrict__ src, Segments seg, int k,
                             hdb_nnd_element *__restrict__ dst) {
  const int64_t total = seg.off[seg.count] * k;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = seg.of_point(i / k);
    dst[i] = src[t][i - seg.off[t] * k];
  }
}

// Instance-local ids -> batch ids, keeping the old/new sign encoding; an id
// outside its instance becomes n (outside every instance), which the graph
// validation then rejects.
__global__ void k_global_ids(hdb_nnd_element *__restrict__ G, int k, Segments seg) {
  const int64_t n = seg.off[seg.count];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * k;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = seg.of_point(i / k);
    const int64_t base = seg.off[t], cnt = seg.off[t + 1] - base;
    const int32_t lab = G[i].label_;
    const int64_t id = lab < 0 ? -(int64_t)lab - 1 : (int64_t)lab;
    const int64_t gid = id < cnt ? base + id : n;
    G[i].label_ = (int32_t)(lab < 0 ? -gid - 1 : gid);
  }
}

// MST edges of the connected instances only, their points renumbered without
// the dropped instances' (pshift[t]: points of dropped instances before t;
// eshift[t]: their MST edges).  The edges come grouped by instance.
__global__ void k_compact_mst(const hdb_mst_edge *__restrict__ in, int64_t m, Segments seg,
                              const int32_t *__restrict__ keep, const int64_t *__restrict__ pshift,
                              const int64_t *__restrict__ eshift, hdb_mst_edge *__restrict__ out) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m;
       e += (int64_t)gridDim.x * blockDim.x) {
    hdb_mst_edge x = in[e];
    const int32_t t = seg.of_point(x.from_node);
    if (!keep[t]) continue;
    x.from_node -= (int32_t)pshift[t];
    x.to_node -= (int32_t)pshift[t];
    out[e - eshift[t]] = x;
  }
}

__global__ void k_expand_labels(const int32_t *__restrict__ kept_labels, Segments seg,
                                const int32_t *__restrict__ keep, const int64_t *__restrict__ pshift,
                                int32_t *__restrict__ labels) {
  const int64_t total = seg.off[seg.count];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = seg.of_point(i);
    labels[i] = keep[t] ? kept_labels[i - pshift[t]] : -1;
  }
}

// The stages after the kNN graph for a batch: enhanced graph, MST forest,
// then the trees of the instances whose graph is connected (the others get
// status HDB_ERR_DISCONNECTED and labels -1).  Records ev[3..5].
void batch_after_knn(Context *ctx, const int32_t *ids, const float *core, const float *X,
                     int64_t n, int32_t d, int32_t k, const hdb_params &p, int32_t *labels,
                     hdb_run_stats *st, const Segments &seg, int32_t *ncl, int32_t *status,
                     const float *first) {
  cudaStream_t s = ctx->stream;
  const int32_t T = seg.count;
  hdb_graph g;
  build_enhanced_knng(ctx, ids, core, X, n, d, k, &g, nullptr, seg);
  HDB_CUDA(cudaEventRecord(ctx->ev[3], s));
  int32_t rounds = 0;
  Buf<hdb_mst_edge> mst(ctx, n - T);
  std::vector<int32_t> iedges((size_t)T);
  Buf<double> p10;
  if (p.mst_gpu == HDB_MST_QUANTISED) {  // every instance's own scale, as its own run would take it
    p10 = Buf<double>(ctx, T);
    quant_scales(ctx, first, 1, n, seg, p10, nullptr);
  }
  const int64_t chosen = boruvka_mst(ctx, &g, nullptr, mst, &rounds, seg, iedges.data(), p10.get(),
                                     p.mst_gpu == HDB_MST_ID_ORDER);
  HDB_CUDA(cudaEventRecord(ctx->ev[4], s));
  std::vector<int32_t> keep((size_t)T);
  std::vector<int64_t> pshift((size_t)T), eshift((size_t)T), off2(1, 0);
  int64_t dp = 0, de = 0;
  for (int32_t t = 0; t < T; t++) {
    const int64_t nt = seg.host_off[t + 1] - seg.host_off[t];
    keep[t] = iedges[t] == nt - 1;
    pshift[t] = dp;
    eshift[t] = de;
    status[t] = keep[t] ? HDB_OK : HDB_ERR_DISCONNECTED;
    if (keep[t]) {
      off2.push_back(off2.back() + nt);
    } else {
      dp += nt;
      de += iedges[t];
    }
  }
  const int32_t K = (int32_t)off2.size() - 1;
  std::vector<int32_t> ncl2((size_t)K, 0);
  int32_t total_cl = 0;
  if (K == T) {
    Buf<hdb_linkage_node> hier(ctx, n - T);
    linkage_tree(ctx, mst, n, hier, seg);
    condense_select(ctx, hier, n, p.mpts, p.stability, labels, &total_cl, nullptr, nullptr,
                    nullptr, nullptr, seg, ncl2.data());
  } else {
    const int64_t n2 = off2[K];
    Buf<int32_t> dkeep(ctx, T);
    Buf<int64_t> dps(ctx, T), des(ctx, T), doff2(ctx, K + 1);
    HDB_CUDA(cudaMemcpyAsync(dkeep, keep.data(), T * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    HDB_CUDA(cudaMemcpyAsync(dps, pshift.data(), T * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    HDB_CUDA(cudaMemcpyAsync(des, eshift.data(), T * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    HDB_CUDA(cudaMemcpyAsync(doff2, off2.data(), (K + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                             s));
    Buf<int32_t> lab2(ctx, n2 > 0 ? n2 : 1);
    if (K > 0) {
      Buf<hdb_mst_edge> mst2(ctx, n2 - K);
      if (chosen > 0) {
        k_compact_mst<<<grid_for(ctx, chosen, 256), 256, 0, s>>>(mst, chosen, seg, dkeep, dps, des,
                                                                mst2); ctx->launches++;
        HDB_CHECK_LAUNCH();
      }
      Segments seg2;
      seg2.off = doff2;
      seg2.host_off = off2.data();
      seg2.count = K;
      Buf<hdb_linkage_node> hier(ctx, n2 - K);
      linkage_tree(ctx, mst2, n2, hier, seg2);
      condense_select(ctx, hier, n2, p.mpts, p.stability, lab2, &total_cl, nullptr, nullptr,
                      nullptr, nullptr, seg2, ncl2.data());
    }
    k_expand_labels<<<grid_for(ctx, n, 256), 256, 0, s>>>(lab2, seg, dkeep, dps, labels); ctx->launches++;
    HDB_CHECK_LAUNCH();
    ctx->sync();
  }
  for (int32_t t = 0, j = 0; t < T; t++) ncl[t] = keep[t] ? ncl2[j++] : 0;
  HDB_CUDA(cudaEventRecord(ctx->ev[5], s));
  st->edges = g.edges;
  st->num_antihubs = g.num_antihubs;
  st->num_clusters = total_cl;
  st->mst_rounds = rounds;
}

// Batch ids -> instance-local ids, keeping the old/new sign encoding.
__global__ void k_local_ids(hdb_nnd_element *__restrict__ G, int k, Segments seg) {
  const int64_t total = seg.off[seg.count] * k;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t base = seg.off[seg.of_point(i / k)];
    const int32_t lab = G[i].label_;
    const int32_t id = lab < 0 ? -lab - 1 : lab;
    const int32_t local = (int32_t)(id - base);
    G[i].label_ = lab < 0 ? -local - 1 : local;
  }
}

// Runs the instances `idx` (all of dimension d) as one batch.  from_knn: the
// instances' G are input kNN graphs (hdb_run_knn_batched) instead of outputs.
void run_batch_group(Context *ctx, hdb_instance *insts, const std::vector<int32_t> &idx, int32_t d,
                     const hdb_params &p, hdb_run_stats *acc, JoinStats *js_acc, bool from_knn) {
  cudaStream_t st = ctx->stream;
  cudaEvent_t *ev = ctx->ev;
  const int32_t k = p.knn.k;
  const int32_t T = (int32_t)idx.size();
  std::vector<int64_t> off((size_t)T + 1, 0);
  for (int32_t t = 0; t < T; t++) off[t + 1] = off[t] + insts[idx[t]].n;
  const int64_t n = off[T];
  HDB_REQUIRE(n < (int64_t(1) << 30), HDB_ERR_ARG,
              "hdb_run_batched: the instances of one d must hold fewer than 2^30 points");
  Buf<int64_t> doff(ctx, T + 1);
  HDB_CUDA(cudaMemcpyAsync(doff, off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  Segments seg;
  seg.off = doff;
  seg.host_off = off.data();
  seg.count = T;

  // inputs: one [n, d] array (used in place when the instances already are one)
  HDB_CUDA(cudaEventRecord(ev[1], st));
  bool contiguous = !p.host_io;
  for (int32_t t = 1; t < T && contiguous; t++)
    contiguous = insts[idx[t]].X == insts[idx[0]].X + off[t] * d;
  Buf<float> Xpack;
  const float *X = insts[idx[0]].X;
  std::vector<void *> ptrs((size_t)T);
  Buf<void *> dptrs(ctx, T);
  if (!contiguous) {
    Xpack = Buf<float>(ctx, (size_t)n * d);
    if (p.host_io) {
      for (int32_t t = 0; t < T; t++)
        HDB_CUDA(cudaMemcpyAsync(Xpack.get() + off[t] * d, insts[idx[t]].X,
                                 (size_t)(off[t + 1] - off[t]) * d * sizeof(float),
                                 cudaMemcpyHostToDevice, st));
    } else {
      for (int32_t t = 0; t < T; t++) ptrs[t] = const_cast<float *>(insts[idx[t]].X);
      HDB_CUDA(cudaMemcpyAsync(dptrs, ptrs.data(), T * sizeof(void *), cudaMemcpyHostToDevice, st));
      k_pack_rows<<<grid_for(ctx, n * d, 256), 256, 0, st>>>(
          reinterpret_cast<const float *const *>(dptrs.get()), seg, d, Xpack); ctx->launches++;
      HDB_CHECK_LAUNCH();
    }
    X = Xpack;
  }

  int64_t dropped = 0;
  JoinStats js;
  Buf<int32_t> ids(ctx, (size_t)n * k), labels(ctx, n);
  Buf<float> core(ctx, n), first;
  Buf<hdb_nnd_element> G(ctx, (size_t)n * k);
  if (from_knn) {
    if (p.host_io) {
      for (int32_t t = 0; t < T; t++)
        HDB_CUDA(cudaMemcpyAsync(G.get() + off[t] * k, insts[idx[t]].G,
                                 (size_t)(off[t + 1] - off[t]) * k * sizeof(hdb_nnd_element),
                                 cudaMemcpyHostToDevice, st));
    } else {
      for (int32_t t = 0; t < T; t++) ptrs[t] = insts[idx[t]].G;
      HDB_CUDA(cudaMemcpyAsync(dptrs, ptrs.data(), T * sizeof(void *), cudaMemcpyHostToDevice, st));
      k_pack_graph<<<grid_for(ctx, n * k, 256), 256, 0, st>>>(
          reinterpret_cast<const hdb_nnd_element *const *>(dptrs.get()), seg, k, G); ctx->launches++;
      HDB_CHECK_LAUNCH();
    }
    k_global_ids<<<grid_for(ctx, n * k, 256), 256, 0, st>>>(G, k, seg); ctx->launches++;
    HDB_CHECK_LAUNCH();
  } else {
    nndescent(ctx, X, n, d, p.knn, G, &dropped, &js, seg);
  }
  HDB_CUDA(cudaEventRecord(ev[2], st));
  {
    Buf<float> dist;
    if (p.distance == HDB_DIST_SQUARED) dist = Buf<float>(ctx, (size_t)n * k);
    knn_split(ctx, G, n, k, ids, p.distance == HDB_DIST_SQUARED ? dist.get() : nullptr);
    core_distances(ctx, dist.get(), X, ids, n, d, k, p.distance, core);
    if (p.mst_gpu == HDB_MST_QUANTISED) {
      first = Buf<float>(ctx, n);
      core_distances(ctx, dist.get(), X, ids, n, d, k, p.distance, first, 0);
    }
  }
  std::vector<int32_t> ncl((size_t)T, 0), status((size_t)T, HDB_OK);
  hdb_run_stats rs = {};
  batch_after_knn(ctx, ids, core, X, n, d, k, p, labels, &rs, seg, ncl.data(), status.data(),
                  first.get());

  // outputs
  if (p.host_io) {
    for (int32_t t = 0; t < T; t++)
      HDB_CUDA(cudaMemcpyAsync(insts[idx[t]].labels, labels.get() + off[t],
                               (off[t + 1] - off[t]) * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  } else {
    for (int32_t t = 0; t < T; t++) ptrs[t] = insts[idx[t]].labels;
    HDB_CUDA(cudaMemcpyAsync(dptrs, ptrs.data(), T * sizeof(void *), cudaMemcpyHostToDevice, st));
    k_unpack_labels<<<grid_for(ctx, n, 256), 256, 0, st>>>(
        labels, seg, reinterpret_cast<int32_t *const *>(dptrs.get())); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  bool want_graph = false;
  for (int32_t t = 0; t < T && !from_knn; t++) want_graph = want_graph || insts[idx[t]].G != nullptr;
  if (want_graph) {
    k_local_ids<<<grid_for(ctx, n * k, 256), 256, 0, st>>>(G, k, seg); ctx->launches++;
    HDB_CHECK_LAUNCH();
    for (int32_t t = 0; t < T; t++) {
      hdb_instance &in = insts[idx[t]];
      if (!in.G) continue;
      HDB_CUDA(cudaMemcpyAsync(in.G, G.get() + off[t] * k,
                               (size_t)(off[t + 1] - off[t]) * k * sizeof(hdb_nnd_element),
                               p.host_io ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
    }
  }
  ctx->sync();
  for (int32_t t = 0; t < T; t++) {
    insts[idx[t]].num_clusters = ncl[t];
    insts[idx[t]].status = status[t];
  }
  acc->edges += rs.edges;
  acc->num_antihubs += rs.num_antihubs;
  acc->num_clusters += rs.num_clusters;
  acc->mst_rounds = rs.mst_rounds > acc->mst_rounds ? rs.mst_rounds : acc->mst_rounds;
  acc->knn_dropped += dropped;
  acc->ms_knn += elapsed(ev[1], ev[2]);
  acc->ms_graph += elapsed(ev[2], ev[3]);
  acc->ms_mst += elapsed(ev[3], ev[4]);
  acc->ms_tree += elapsed(ev[4], ev[5]);
  js_acc->ms += js.ms;
  js_acc->launches += js.launches;
  js_acc->rows_gathered += js.rows_gathered;
  js_acc->candidates += js.candidates;
  js_acc->pairs += js.pairs;
  if (js.config) js_acc->config = js.config;  // the FP32 join's form (the last group's)
}

// hdb_run / hdb_run_with_graph: the whole path on one instance; G_out
// (optional) receives the kNN graph the labels were computed from.
hdb_status run_single(hdb_ctx *h, const float *X, int64_t n, int32_t d, const hdb_params *params,
                      int32_t *labels, hdb_nnd_element *G_out, hdb_run_stats *stats) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(X, "X");
    require_ptr(labels, "labels");
    require_ptr(params, "params");
    const hdb_params &p = *params;
    check_run_params(p);
    const int32_t k = p.knn.k;
    HDB_REQUIRE(n > k && d >= 1, HDB_ERR_ARG, "need n > k and d >= 1");
    cudaStream_t st = ctx->stream;
    cudaEvent_t *ev = ctx->ev;
    const int64_t launches0 = ctx->launches;
    hdb_run_stats rs = {};
    JoinStats js;
    HDB_CUDA(cudaEventRecord(ev[0], st));
    Buf<float> Xd;
    Buf<int32_t> Ld;
    const float *Xuse = X;
    int32_t *Luse = labels;
    if (p.host_io) {
      Xd = Buf<float>(ctx, (size_t)n * d);
      Ld = Buf<int32_t>(ctx, n);
      HDB_CUDA(cudaMemcpyAsync(Xd, X, (size_t)n * d * sizeof(float), cudaMemcpyHostToDevice, st));
      Xuse = Xd;
      Luse = Ld;
    }
    HDB_CUDA(cudaEventRecord(ev[1], st));
    int64_t dropped = 0;
    Buf<int32_t> ids(ctx, (size_t)n * k);
    Buf<float> core(ctx, n), first;
    {
      Buf<hdb_nnd_element> G(ctx, (size_t)n * k);
      nndescent(ctx, Xuse, n, d, p.knn, G, &dropped, &js);
      HDB_CUDA(cudaEventRecord(ev[2], st));
      if (G_out)
        HDB_CUDA(cudaMemcpyAsync(G_out, G.get(), (size_t)n * k * sizeof(hdb_nnd_element),
                                 p.host_io ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
      Buf<float> dist;
      if (p.distance == HDB_DIST_SQUARED) dist = Buf<float>(ctx, (size_t)n * k);
      knn_split(ctx, G, n, k, ids, p.distance == HDB_DIST_SQUARED ? dist.get() : nullptr);
      core_distances(ctx, dist.get(), Xuse, ids, n, d, k, p.distance, core);
      if (p.mst_gpu == HDB_MST_QUANTISED) {
        first = Buf<float>(ctx, n);
        core_distances(ctx, dist.get(), Xuse, ids, n, d, k, p.distance, first, 0);
      }
    }
    run_after_knn(ctx, ids, core, Xuse, n, d, k, p, Luse, &rs, first.get());
    if (p.host_io)
      HDB_CUDA(cudaMemcpyAsync(labels, Luse, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    HDB_CUDA(cudaEventRecord(ev[6], st));
    ctx->sync();
    if (stats) {
      rs.knn_dropped = dropped;
      fill_times(ctx, &rs, true);
      rs.join_ms = (float)js.ms;
      rs.join_launches = (int32_t)js.launches;
      rs.join_config = js.config;
      rs.join_pairs = js.pairs;
      rs.join_rows_gathered = js.rows_gathered;
      rs.join_candidates = js.candidates;
      rs.gpu_launches = ctx->launches - launches0;
      *stats = rs;
    }
  });
}

}  // namespace

extern "C" {

HDB_API hdb_status hdb_run(hdb_ctx *h, const float *X, int64_t n, int32_t d,
                           const hdb_params *params, int32_t *labels, hdb_run_stats *stats) {
  return run_single(h, X, n, d, params, labels, nullptr, stats);
}

HDB_API hdb_status hdb_run_with_graph(hdb_ctx *h, const float *X, int64_t n, int32_t d,
                                      const hdb_params *params, int32_t *labels,
                                      hdb_nnd_element *G, hdb_run_stats *stats) {
  return run_single(h, X, n, d, params, labels, G, stats);
}

}  // extern "C"

namespace {

hdb_status run_batched(hdb_ctx *h, hdb_instance *insts, int32_t count, const hdb_params *params,
                       hdb_run_stats *stats, bool from_knn) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(insts, "insts");
    require_ptr(params, "params");
    HDB_REQUIRE(count >= 1, HDB_ERR_ARG, "hdb_run_batched: need at least one instance");
    const hdb_params &p = *params;
    check_run_params(p);
    const int32_t k = p.knn.k;
    // instances grouped by d (ascending), each group in instance order
    std::map<int32_t, std::vector<int32_t>> groups;
    for (int32_t i = 0; i < count; i++) {
      hdb_instance &in = insts[i];
      require_ptr(in.X, "instance X");
      require_ptr(in.labels, "instance labels");
      if (from_knn) require_ptr(in.G, "instance G");
      HDB_REQUIRE(in.n > k && in.n < (int64_t(1) << 30) && in.d >= 1, HDB_ERR_ARG,
                  "hdb_run_batched: every instance needs k < n < 2^30 and d >= 1");
      in.status = HDB_OK;
      in.num_clusters = 0;
      groups[in.d].push_back(i);
    }
    const int64_t launches0 = ctx->launches;
    hdb_run_stats rs = {};
    JoinStats js;
    HDB_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
    // consecutive instances of one d, as many points per batch as the free
    // device memory holds (at most 2^25): 70 % of what the driver has free
    // plus the context's idle cached blocks, over the batch's bytes per point
    // at its peak (NN-Descent, or the graph / MST stages when the kNN graphs
    // are given), plus the batch's own arrays
    size_t free_b = 0, total_b = 0;
    HDB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const double avail = 0.7 * ((double)free_b + (double)ctx->cache_bytes);
    for (auto &g : groups) {
      const int64_t d = g.first;
      const int64_t graph_bpp = 40 * (int64_t)k;  // CSR + MST keys, E ~ 1.5 k per point
      const int64_t nnd_bpp = from_knn ? 0 : nndescent_bytes_per_point(g.first, p.knn);
      const int64_t bpp = std::max(nnd_bpp, graph_bpp) + 12 * (int64_t)k + 16 + 4 * d;
      const int64_t cap = std::max<int64_t>(
          int64_t(1) << 16, std::min<int64_t>(int64_t(1) << 25, (int64_t)(avail / (double)bpp)));
      // batches of about equal size, so that they reuse the same cached blocks
      // (unequal ones would free and allocate multi-GB blocks every call)
      int64_t group_points = 0;
      for (int32_t i : g.second) group_points += insts[i].n;
      const int64_t nb = (group_points + cap - 1) / cap;
      const int64_t batch_points = (group_points + nb - 1) / nb;
      std::vector<int32_t> part;
      int64_t pts = 0;
      for (int32_t i : g.second) {
        if (!part.empty() && pts + insts[i].n > batch_points) {
          run_batch_group(ctx, insts, part, g.first, p, &rs, &js, from_knn);
          part.clear();
          pts = 0;
        }
        part.push_back(i);
        pts += insts[i].n;
      }
      run_batch_group(ctx, insts, part, g.first, p, &rs, &js, from_knn);
    }
    HDB_CUDA(cudaEventRecord(ctx->ev[6], ctx->stream));
    ctx->sync();
    if (stats) {
      rs.ms_total = elapsed(ctx->ev[0], ctx->ev[6]);
      rs.join_ms = (float)js.ms;
      rs.join_launches = (int32_t)js.launches;
      rs.join_config = js.config;
      rs.join_pairs = js.pairs;
      rs.join_rows_gathered = js.rows_gathered;
      rs.join_candidates = js.candidates;
      rs.gpu_launches = ctx->launches - launches0;
      *stats = rs;
    }
    int32_t failed = 0;
    for (int32_t i = 0; i < count; i++) failed += insts[i].status != HDB_OK;
    HDB_REQUIRE(failed == 0, HDB_ERR_DISCONNECTED,
                std::to_string(failed) + " instance(s) with a disconnected enhanced kNN graph "
                "(status HDB_ERR_DISCONNECTED, labels -1); the others are complete");
  });
}

}  // namespace

extern "C" {

HDB_API hdb_status hdb_run_batched(hdb_ctx *h, hdb_instance *insts, int32_t count,
                                   const hdb_params *params, hdb_run_stats *stats) {
  return run_batched(h, insts, count, params, stats, false);
}

HDB_API hdb_status hdb_run_knn_batched(hdb_ctx *h, hdb_instance *insts, int32_t count,
                                       const hdb_params *params, hdb_run_stats *stats) {
  return run_batched(h, insts, count, params, stats, true);
}

HDB_API hdb_status hdb_run_knn(hdb_ctx *h, const hdb_nnd_element *G, const float *X, int64_t n,
                               int32_t d, const hdb_params *params, int32_t *labels,
                               hdb_run_stats *stats) {
  return guard([&] {
    Context *ctx = C(h);
    require_ptr(G, "G");
    require_ptr(X, "X");
    require_ptr(labels, "labels");
    require_ptr(params, "params");
    const hdb_params &p = *params;
    check_run_params(p);
    const int32_t k = p.knn.k;
    HDB_REQUIRE(n > k && d >= 1, HDB_ERR_ARG, "need n > k and d >= 1");
    cudaStream_t st = ctx->stream;
    cudaEvent_t *ev = ctx->ev;
    const int64_t launches0 = ctx->launches;
    hdb_run_stats rs = {};
    HDB_CUDA(cudaEventRecord(ev[0], st));
    Buf<float> Xd;
    Buf<int32_t> Ld;
    Buf<hdb_nnd_element> Gd;
    const float *Xuse = X;
    const hdb_nnd_element *Guse = G;
    int32_t *Luse = labels;
    if (p.host_io) {
      Xd = Buf<float>(ctx, (size_t)n * d);
      Gd = Buf<hdb_nnd_element>(ctx, (size_t)n * k);
      Ld = Buf<int32_t>(ctx, n);
      HDB_CUDA(cudaMemcpyAsync(Xd, X, (size_t)n * d * sizeof(float), cudaMemcpyHostToDevice, st));
      HDB_CUDA(cudaMemcpyAsync(Gd, G, (size_t)n * k * sizeof(hdb_nnd_element),
                               cudaMemcpyHostToDevice, st));
      Xuse = Xd;
      Guse = Gd;
      Luse = Ld;
    }
    HDB_CUDA(cudaEventRecord(ev[1], st));
    HDB_CUDA(cudaEventRecord(ev[2], st));
    Buf<int32_t> ids(ctx, (size_t)n * k);
    Buf<float> core(ctx, n), first;
    {
      Buf<float> dist;
      if (p.distance == HDB_DIST_SQUARED) dist = Buf<float>(ctx, (size_t)n * k);
      knn_split(ctx, Guse, n, k, ids, p.distance == HDB_DIST_SQUARED ? dist.get() : nullptr);
      core_distances(ctx, dist.get(), Xuse, ids, n, d, k, p.distance, core);
      if (p.mst_gpu == HDB_MST_QUANTISED) {
        first = Buf<float>(ctx, n);
        core_distances(ctx, dist.get(), Xuse, ids, n, d, k, p.distance, first, 0);
      }
    }
    run_after_knn(ctx, ids, core, Xuse, n, d, k, p, Luse, &rs, first.get());
    if (p.host_io)
      HDB_CUDA(cudaMemcpyAsync(labels, Luse, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    HDB_CUDA(cudaEventRecord(ev[6], st));
    ctx->sync();
    if (stats) {
      fill_times(ctx, &rs, false);
      rs.gpu_launches = ctx->launches - launches0;
      *stats = rs;
    }
  });
}

}  // extern "C"
