/*
 * hdb.h -- C ABI of the B200-native HDBSCAN path (libhdb_b200.so).
 *
 * The reference (gorlando04/GPU_HDBSCAN) has no library API: its operator
 * surface is a set of C++ functions called in the order of HDBSCAN/_new.cu
 * (kNN graph -> enhanced kNN graph -> MST -> edge sort -> linkage tree ->
 * condensed tree -> stability -> clusters), plus the compile-time parameters
 * VEC_DIM, NEIGHB_NUM_PER_LIST (k), SAMPLE_NUM and NND_ITERATION.  Every entry
 * point below replaces one of those functions; the comment above each one
 * names the reference interface (file:line) it stands in for.  Record layouts
 * are byte-identical to the reference structs so buffers can be exchanged.
 *
 * Conventions
 *  - Every call returns an hdb_status; on failure hdb_last_error() (thread
 *    local) holds a one-line message.  Nothing exits the process.
 *  - Array arguments are DEVICE pointers (cudaMalloc'd, on the context's
 *    device) unless the argument's comment says otherwise.  hdb_run also takes
 *    host pointers when hdb_params.host_io is 1.
 *  - Work is enqueued on the context's stream; every call returns after the
 *    stream has finished the call's work.
 *  - A context is single-stream and not thread safe; separate contexts are
 *    independent.  Scratch memory comes from a per-context pool that grows on
 *    demand and is released by hdb_destroy.
 */
#ifndef HDB_HDB_H
#define HDB_HDB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HDB_API __attribute__((visibility("default")))

typedef enum {
  HDB_OK = 0,
  HDB_ERR_ARG = 1,          /* invalid argument or input (the reference exit(1)s / asserts) */
  HDB_ERR_ALLOC = 2,        /* device or host allocation failed */
  HDB_ERR_CUDA = 3,         /* a CUDA runtime call failed */
  HDB_ERR_IO = 4,           /* file read/write failed */
  HDB_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
  HDB_ERR_DISCONNECTED = 6, /* the MST does not have n-1 edges ("MST montada incorretamente") */
  HDB_ERR_INTERNAL = 7
} hdb_status;

/* NNDElement, tools/nndescent_element.cuh:9-57: label_ < 0 encodes an "old"
 * neighbour as -label-1; label() decodes it.  8 bytes. */
typedef struct { float distance_; int32_t label_; } hdb_nnd_element;
/* MSTedge, HDBSCAN/structs/hdbscan_elements.cuh:40-45.  12 bytes. */
typedef struct { int32_t from_node, to_node; float weight; } hdb_mst_edge;
/* SingleLinkageNode, hdbscan_elements.cuh:50-56.  16 bytes. */
typedef struct { int32_t left_node, right_node; float weight; int32_t node_size; } hdb_linkage_node;
/* CondensedTreeNode, hdbscan_elements.cuh:59-65.  16 bytes. */
typedef struct { int32_t parent, child; float lambda_val; int32_t child_size; } hdb_condensed_node;
/* Stability, hdbscan_elements.cuh:80-84.  8 bytes. */
typedef struct { int32_t cluster_id; float lambda; } hdb_stability;

/* ECLgraph, HDBSCAN/structs/ECLgraph.h:41-47, plus the antihub list.  The
 * arrays are device memory owned by the context; they stay valid until the
 * next hdb_enhanced_knng call on the same context or hdb_destroy. */
typedef struct {
  int32_t nodes;
  int64_t edges;
  int64_t *nindex;   /* [nodes + 1] */
  int32_t *nlist;    /* [edges] */
  float *eweight;    /* [edges] mutual-reachability weights */
  int32_t num_antihubs;
  int32_t *antihubs; /* [num_antihubs], ascending */
} hdb_graph;

enum { HDB_PREC_FP32 = 0, HDB_PREC_BF16 = 1, HDB_PREC_FP16 = 2 };
enum { HDB_DIST_SQRT = 0, HDB_DIST_SQUARED = 1 };
enum { HDB_STAB_FP32 = 0, HDB_STAB_FP64 = 1 };
/* MST modes (hdb_params.mst_gpu): the reference's two, then the float MST
 * under the tie order (weight, min id, max id) of hdb_mst_ordered. */
enum { HDB_MST_FLOAT = 0, HDB_MST_QUANTISED = 1, HDB_MST_ID_ORDER = 2 };
/* Tie orders of hdb_mst_ordered. */
enum { HDB_ORDER_EDGE = 0, HDB_ORDER_IDS = 1 };

/* The compile-time parameters of gpuknn/nndescent.cuh:9-15 as run-time ones. */
typedef struct {
  int32_t k;           /* NEIGHB_NUM_PER_LIST, 1..32 (reference: 32) */
  int32_t sample_num;  /* SAMPLE_NUM, 1..k/2 (reference: 16; 2*SAMPLE_NUM <= k) */
  int32_t iterations;  /* NND_ITERATION (reference: 6) */
  int32_t precision;   /* HDB_PREC_FP32: reference difference-sum distances;
                          HDB_PREC_BF16: tensor-core candidate distances from BF16
                          rows, FP32 re-rank;
                          HDB_PREC_FP16: the same from FP16 rows scaled by one
                          power of two (3 more mantissa bits, same bytes) */
} hdb_knn_params;

typedef struct {
  hdb_knn_params knn;
  int32_t mpts;        /* min cluster size (mpts, HDBSCAN/_new.cu:163); k >= mpts >= 2 */
  int32_t distance;    /* HDB_DIST_SQRT: fix_distances applied (build_kNNG.cu:131-174);
                          HDB_DIST_SQUARED: NN-Descent's squared distances kept */
  int32_t stability;   /* HDB_STAB_FP32 (tree.cu:494-511 order) or HDB_STAB_FP64 */
  int32_t host_io;     /* hdb_run only: 1 = X and labels are host pointers */
  int32_t mst_gpu;     /* the reference's argv[4] (HDBSCAN/new.cu:38): HDB_MST_FLOAT (0) =
                          the float MST of cpuMST; HDB_MST_QUANTISED (1) = its int-quantised
                          GPU MST (hdb_mst_quantised); HDB_MST_ID_ORDER (2, not in the
                          reference) = the float MST under (weight, min id, max id) */
} hdb_params;

typedef struct {
  int64_t edges;          /* enhanced kNN graph edges (CSR entries) */
  int32_t num_antihubs;
  int32_t num_clusters;
  int64_t condensed_size;
  int32_t mst_rounds;     /* Boruvka rounds */
  int64_t knn_dropped;    /* NN-Descent candidates lost to a full inbox (normally 0) */
  float ms_knn, ms_graph, ms_mst, ms_tree, ms_total; /* device time per stage */
  /* NN-Descent local join, measured with CUDA events around each launch */
  float join_ms;                /* summed over the join launches */
  int32_t join_launches;
  int64_t join_rows_gathered;   /* sampled rows staged in shared memory, all launches */
  int64_t join_candidates;      /* candidates that passed the k-th distance filter */
  int64_t gpu_launches;         /* kernel launches issued by the call */
  int32_t mst_multiplier;       /* mst_gpu = 1: the weight scale exponent m (single runs) */
  int32_t join_config;          /* FP32 local join: 4 x 4 distance tiles per lane (1 or 2),
                                   forced (hdb_set_join_tiles) or tuned; 0 for a 16-bit join */
  int64_t join_pairs;           /* FP32 local join: distance pairs computed, all launches
                                   (the reference's new x new and new x old pairs); 0 for a
                                   16-bit join */
} hdb_run_stats;

typedef struct hdb_ctx hdb_ctx;

HDB_API const char *hdb_version(void);
HDB_API const char *hdb_last_error(void);
/* Creates a context on `device` with its own non-blocking stream. */
HDB_API hdb_status hdb_create(hdb_ctx **ctx, int32_t device);
HDB_API hdb_status hdb_destroy(hdb_ctx *ctx);
/* Run the context's work on a caller stream (cudaStream_t); NULL restores the
 * context's own stream. */
HDB_API hdb_status hdb_set_stream(hdb_ctx *ctx, void *stream);
/* FP32 local join form (no reference counterpart: the reference's join,
 * nndescent.cu:1487-1580, has one form).  tiles = 1 or 2 distance tiles of
 * 4 x 4 per lane forces that form (1: fewer registers, three blocks per SM;
 * 2: two blocks per SM, fewer passes over the staged rows); 0 (the default)
 * times both once per (device, d, k, SAMPLE_NUM, rows fit in L2) on the
 * first FP32 NN-Descent of that shape and keeps the faster for the process.
 * Both forms give the same graph. */
HDB_API hdb_status hdb_set_join_tiles(hdb_ctx *ctx, int32_t tiles);

/* gpuknn::NNDescent, gpuknn/nndescent.cuh:40-42 (nndescent.cu:2088-2199):
 * X [n, d] float32 row-major -> G [n, k] NNDElement rows sorted by ascending
 * squared L2, old/new flag sign-encoded as in the reference. */
HDB_API hdb_status hdb_nndescent(hdb_ctx *ctx, const float *X, int64_t n, int32_t d,
                                 const hdb_knn_params *params, hdb_nnd_element *G);

/* gpuknn::KNNMerge, gpuknn/knnmerge.cuh:8-12 (knnmerge.cu:401-437, with
 * NNDescentForMerge nndescent.cu:1999-2087): the kNN graph of the union of
 * two point sets from the graphs of each.  X1 [n1, d], X2 [n2, d] float32;
 * G1 [n1, k], G2 [n2, k] NNDElement rows with ids local to their set (as
 * hdb_nndescent writes them; flags ignored) -> G [n1 + n2, k]: rows of set 1,
 * then set 2, ids of set 2 shifted by n1, sorted by ascending squared L2 with
 * flags as hdb_nndescent.  params: k of G1 and G2, sample_num =
 * MERGE_SAMPLE_NUM (reference 12), iterations = MERGE_ITERATION (reference
 * 11), precision HDB_PREC_FP32 (the merge join is the FP32 difference sum).
 * Each set needs more than k points.  A subgraph id outside its set, a self
 * id or a repeated id in a row gives HDB_ERR_ARG.  All pointers are device
 * memory (KNNMergeFromHost, knnmerge.cuh:14-18, is the caller's copies plus
 * this call). */
HDB_API hdb_status hdb_knn_merge(hdb_ctx *ctx, const float *X1, int64_t n1,
                                 const hdb_nnd_element *G1, const float *X2, int64_t n2,
                                 const hdb_nnd_element *G2, int32_t d,
                                 const hdb_knn_params *params, hdb_nnd_element *G);

/* The NNDElement -> (int ids, float distances) split of HDBSCAN/_new.cu:204-229. */
HDB_API hdb_status hdb_knn_split(hdb_ctx *ctx, const hdb_nnd_element *G, int64_t n, int32_t k,
                                 int32_t *ids, float *dist);

/* fix_distances, build_kNNG.cu:131-174 (calculate_euclidean_distance_fix :4-13):
 * dist[i, j] = sqrt-L2(X[i], X[ids[i, j]]) with the reference's rounding. */
HDB_API hdb_status hdb_fix_distances(hdb_ctx *ctx, const float *X, int64_t n, int32_t d,
                                     const int32_t *ids, int32_t k, float *dist);

/* buildEnhancedKNNG, HDBSCAN/graphs/graph.cuh:24 (graph.cu:108-176 and
 * buildECLgraph graph.cu:16-103): in-degrees, floor(sqrt(n)) antihubs, the
 * symmetric CSR with the antihub clique, core distances (distance to the k-th
 * neighbour) and mutual-reachability weights.  ids must be in [0, n), without
 * self ids or repeated ids in a row (HDB_ERR_ARG otherwise). */
HDB_API hdb_status hdb_enhanced_knng(hdb_ctx *ctx, const int32_t *ids, const float *dist,
                                     const float *X, int64_t n, int32_t d, int32_t k,
                                     hdb_graph *graph);

/* build_CoreSG / Union_kNNG_MST, HDBSCAN/core-sg/core-sg.cu:292-571 (the body
 * of the reference's built hdbscan_ entry, new.cu:92): the core-SG of a kNN
 * graph, i.e. its CSR (row i = its k kNN ids in list order, then every i'
 * with a non-mutual edge i'->i in ascending i') joined with the n-1 edges
 * of `mst`, the sorted MST of its enhanced kNN graph (hdb_mst's output):
 * each MST edge adds from_node to to_node's row and to_node to from_node's
 * row, in edge order, after the reverse entries.  eweight is the Euclidean
 * weight the reference leaves in place: dist[i][j] for kNN and reverse
 * entries (the distance as given, squared or not) and, for MST entries, the
 * float-accumulated pow / sqrtf distance of calculates.cu:275-283.  The
 * arrays are owned by the context (kept until the next hdb_core_sg call or
 * hdb_destroy); num_antihubs = 0.  ids, dist, X and mst are device memory;
 * ids are validated like hdb_enhanced_knng's, MST endpoints must lie in
 * [0, n), and n * k must stay below 2^32 (HDB_ERR_ARG otherwise). */
HDB_API hdb_status hdb_core_sg(hdb_ctx *ctx, const int32_t *ids, const float *dist, const float *X,
                               int64_t n, int32_t d, int32_t k, const hdb_mst_edge *mst,
                               hdb_graph *graph);

/* cpuMST + buildMST, HDBSCAN/mst/mst.cuh:64,91 (mst.cu:34-78, 291-336): the
 * minimum spanning tree under the order (weight, CSR edge index) of the
 * entries whose target exceeds their row, written as MSTedge[n-1] already
 * sorted the way sort_edges leaves it.  in_mst [edges] (optional, may be NULL)
 * receives the reference's bool-per-edge result.  HDB_ERR_DISCONNECTED if the
 * graph is not connected. */
HDB_API hdb_status hdb_mst(hdb_ctx *ctx, const hdb_graph *graph, uint8_t *in_mst,
                           hdb_mst_edge *mst, int32_t *rounds);

/* The mst_gpu = 1 MST of build_CoreSG (core-sg.cu:533-540): buildGPUgraph
 * (core-sg.cu:8-44) scales every weight to the int (int)(10^m * w), m =
 * ceil(-log10(min)) + 2 with `min` the smallest positive first-neighbour
 * distance as FileTool::GetMinDistanceFromKNNG takes it (row 0's distance
 * when positive, else 999, then any smaller positive one; dist[i * k] is row
 * i's first distance, device memory); gpuMST (mst.cu:210-288) spans the
 * graph under the order (int weight, CSR edge index); buildMST_gpu
 * (mst.cu:338-380) writes the tree with the weights (float)(q / 10^m), sorted
 * stably by weight.  A scaled weight beyond the int range becomes INT_MIN, as
 * the reference's conversion does on x86.  *multiplier (optional) receives m.
 * HDB_ERR_DISCONNECTED if the graph is not connected. */
HDB_API hdb_status hdb_mst_quantised(hdb_ctx *ctx, const hdb_graph *graph, const float *dist,
                                     int32_t k, uint8_t *in_mst, hdb_mst_edge *mst,
                                     int32_t *multiplier, int32_t *rounds);

/* hdb_mst under a chosen tie order.  HDB_ORDER_EDGE: the reference's
 * (weight, CSR edge index), the same result as hdb_mst.  HDB_ORDER_IDS:
 * (weight, min id, max id), ties of a repeated pair broken by edge index --
 * the tree and its listing both follow that order, so it depends only on the
 * weighted edge set, not on the order of the CSR rows' entries.  Both trees
 * have the same weight multiset (any two MSTs do); they differ only where
 * tied weights leave the choice open. */
HDB_API hdb_status hdb_mst_ordered(hdb_ctx *ctx, const hdb_graph *graph, int32_t order,
                                   uint8_t *in_mst, hdb_mst_edge *mst, int32_t *rounds);

/* sort_edges, HDBSCAN/merge_sort/merge_sort.cuh:30: stable ascending sort by
 * weight, in place. */
HDB_API hdb_status hdb_sort_edges(hdb_ctx *ctx, hdb_mst_edge *edges, int64_t m);

/* build_Linkage_tree, HDBSCAN/trees/tree.cuh:33 (tree.cu:171-202): the
 * single-linkage tree of n points from n-1 sorted MST edges. */
HDB_API hdb_status hdb_linkage_tree(hdb_ctx *ctx, const hdb_mst_edge *sorted, int64_t n,
                                    hdb_linkage_node *hierarchy);

/* build_Condensed_tree + compute_stability + get_clusters, tree.cuh:39-45
 * (tree.cu:255-746): labels [n] (-1 = noise, clusters 0.. in ascending
 * cluster id).  Optional outputs (NULL to skip): condensed [n + 2*(n/mpts) + 2]
 * rows sorted by (parent, child) with *condensed_size set; stability
 * [n/mpts*2 + 2] indexed by cluster id - n with *num_stability set. */
HDB_API hdb_status hdb_condense_select(hdb_ctx *ctx, const hdb_linkage_node *hierarchy,
                                       int64_t n, int32_t mpts, int32_t stability_mode,
                                       int32_t *labels, int32_t *num_clusters,
                                       hdb_condensed_node *condensed, int64_t *condensed_size,
                                       hdb_stability *stability, int64_t *num_stability);

/* The whole path in the HDBSCAN/_new.cu:149-358 order (hdbscan_ binary):
 * X [n, d] -> labels [n].  With params->host_io = 1 both are host pointers and
 * the copies run inside the call. */
HDB_API hdb_status hdb_run(hdb_ctx *ctx, const float *X, int64_t n, int32_t d,
                           const hdb_params *params, int32_t *labels, hdb_run_stats *stats);

/* hdb_run that also hands back the kNN graph it built, the in-memory form of
 * the .kgraph file the reference's hdbscan_ flow writes between its kNN
 * and HDBSCAN stages (build_kNNG.cu:131-174, read back at
 * HDBSCAN/_new.cu:199): G [n, params->knn.k] NNDElement rows as
 * hdb_nndescent writes them (squared distances, flags kept), the graph the
 * labels were computed from.  G may be NULL (then this is hdb_run); it is
 * device memory, or host memory with params->host_io = 1. */
HDB_API hdb_status hdb_run_with_graph(hdb_ctx *ctx, const float *X, int64_t n, int32_t d,
                                      const hdb_params *params, int32_t *labels,
                                      hdb_nnd_element *G, hdb_run_stats *stats);

/* The stages after the kNN graph in the HDBSCAN/_new.cu:196-347 order, which
 * reads a finished .kgraph (ReadBinaryVecs, _new.cu:199) instead of building
 * it: G [n, params->knn.k] NNDElement rows (flags allowed), X [n, d] ->
 * labels [n].  params->knn.sample_num / iterations / precision are ignored.
 * With params->host_io = 1, G, X and labels are host pointers. */
HDB_API hdb_status hdb_run_knn(hdb_ctx *ctx, const hdb_nnd_element *G, const float *X, int64_t n,
                               int32_t d, const hdb_params *params, int32_t *labels,
                               hdb_run_stats *stats);

/* One clustering instance of hdb_run_batched. */
typedef struct {
  const float *X;          /* [n, d] float32 row-major */
  int64_t n;               /* points; n > params->knn.k */
  int32_t d;
  int32_t num_clusters;    /* out: clusters found in this instance */
  int32_t *labels;         /* out: [n], -1 = noise, clusters 0.. per instance */
  hdb_nnd_element *G;      /* optional out (NULL to skip): [n, k] final kNN rows,
                              ids local to the instance, flags as hdb_nndescent
                              (the input graph for hdb_run_knn_batched) */
  int32_t status;          /* out: HDB_OK, or HDB_ERR_DISCONNECTED when the
                              instance's enhanced kNN graph is disconnected (its
                              labels are then all -1 and num_clusters 0) */
  int32_t reserved;
} hdb_instance;

/* hdb_run_batched -- many independent HDBSCAN runs (the hdbscan_ flow of
 * HDBSCAN/_new.cu on each instance) in shared kernel launches: consecutive
 * instances of equal d (up to 2^25 points at a time) are laid back to back
 * and every stage runs once over all of them,
 * each instance's kNN lists, antihubs, clique, MST tree, condensed tree and
 * cluster selection staying inside the instance.  Per instance the result is
 * what hdb_run computes on that instance alone from the same kNN graph (the
 * NN-Descent initial graph is the same too: ids are drawn with
 * instance-local positions).  insts is a HOST array of `count` descriptors;
 * X, labels and G are device pointers, or host pointers with
 * params->host_io = 1.  stats (optional) sums the stages over all instances.
 * Where hdb_run fails on a disconnected graph, only that instance fails here:
 * the call then returns HDB_ERR_DISCONNECTED with every other instance's
 * outputs complete (see hdb_instance.status). */
HDB_API hdb_status hdb_run_batched(hdb_ctx *ctx, hdb_instance *insts, int32_t count,
                                   const hdb_params *params, hdb_run_stats *stats);

/* hdb_run_knn_batched -- hdb_run_knn (the HDBSCAN/_new.cu flow from finished
 * .kgraph files) on many instances in shared launches: insts[i].G is the
 * INPUT kNN graph [n, params->knn.k] of instance i, ids local to the
 * instance (flags allowed); everything else as hdb_run_batched. */
HDB_API hdb_status hdb_run_knn_batched(hdb_ctx *ctx, hdb_instance *insts, int32_t count,
                                       const hdb_params *params, hdb_run_stats *stats);

/* hdb_bf16_distance_tiles -- a diagnostic with no counterpart in the
 * reference: the distances the BF16 tensor-core local join of hdb_nndescent
 * computes, for given slot lists instead of NN-Descent's samples.  Tile t
 * stages two row-joins j = 0, 1 of 64 slots each (ids[t*128 + 64*j + s]):
 * "new" slots s = 0..31, of which the first counts[t*4 + 2*j] are used, and
 * "old" slots s = 32..63, of which the first counts[t*4 + 2*j + 1] are used.
 * out[(t*128 + 64*j + r) * 64 + c] = |x_a|^2 + |x_b|^2 - 2 x_a.x_b for the
 * rows a, b in slots r and c of row-join j, with x rounded to BF16 and FP32
 * norms and accumulation (no clamp at 0); +inf where slot c is unused.  Rows
 * in unused slots r carry unspecified values.  X [n, d] (d <= 256), ids,
 * counts and out are device memory; counts must lie in [0, 32] and used ids
 * in [0, n) (both are checked, HDB_ERR_ARG). */
HDB_API hdb_status hdb_bf16_distance_tiles(hdb_ctx *ctx, const float *X, int64_t n, int32_t d,
                                           const int32_t *ids, const int32_t *counts,
                                           int64_t tiles, float *out);

/* hdb_sort_edges_noalloc -- no counterpart in the reference.  The same
 * stable ascending sort by weight as hdb_sort_edges, for callers that cannot
 * call cudaMalloc (a host framework that owns every device byte, or a device
 * that is already full): it allocates nothing and needs no context.  Its
 * working memory is a fixed ~7.3 MB static device array inside the library,
 * which every GPU that loads libhdb_b200.so keeps until the process exits, so
 * m may be at most 262144 edges (HDB_ERR_ARG above that).  `edges` is device
 * memory; work runs on `stream` (NULL = legacy default stream) of the current
 * device and the call returns when it is done.  The first call on each device
 * looks up the array's device address (cudaGetSymbolAddress); with CUDA's
 * lazy module loading that lookup is also what places the array on the
 * device, so it can fail (HDB_ERR_CUDA) on a device that is already full.
 * A failed lookup is retried by the next call.  Make one warm-up call on each
 * device before it fills and before any stream capture: m = 0 (edges may then
 * be NULL) places the array and sorts nothing; a call with m >= 2 also loads
 * the sort's kernels, which lazy loading otherwise places on the first real
 * sort.  All calls share the one
 * array: calls whose work overlaps on the GPU (for instance from different
 * streams or threads) race and corrupt each other's result. */
HDB_API hdb_status hdb_sort_edges_noalloc(hdb_mst_edge *edges, int64_t m, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HDB_HDB_H */
