/*
 * CPU oracle for the HDBSCAN hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C, the reference algorithm of
 * gorlando04/GPU_HDBSCAN for every stage of the path (kNN graph, enhanced kNN
 * graph, core distances / mutual reachability, Kruskal MST, stable edge sort,
 * single-linkage tree, condensed tree, stability, excess-of-mass selection and
 * labelling).  Each function cites the reference file:line it follows.
 *
 * Only the test-suite, the smoke check and the CPU-baseline leg of the
 * benchmark may load it, and only as the checker.  The product
 * (gpu_hdbscan_b200, libhdb_b200.so) never links or calls it.
 *
 * Tie-breaks the reference leaves unspecified (std::partial_sort on equal
 * degrees / equal scores, HDBSCAN/graphs/graph.cu:123 and
 * HDBSCAN/calculates/calculates.cu:513) are pinned here to "ascending vertex
 * index", the same rule the CUDA path uses.
 */
#ifndef HDB_ORACLE_H
#define HDB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layouts as HDBSCAN/structs/hdbscan_elements.cuh:40-83 */
typedef struct { int32_t from_node, to_node; float weight; } orc_mst_edge;
typedef struct { int32_t left_node, right_node; float weight; int32_t node_size; } orc_linkage_node;
typedef struct { int32_t parent, child; float lambda_val; int32_t child_size; } orc_condensed_node;
typedef struct { int32_t cluster_id; float lambda; } orc_stab;

enum { ORC_OK = 0, ORC_ERR_ARG = 1, ORC_ERR_ALLOC = 2, ORC_ERR_DISCONNECTED = 6 };

void orc_free(void *p);
int orc_num_threads(void);

/* ---- kNN graph (tools/nndescent_element.cuh, gpuknn/nndescent.cu) ---- */
uint64_t orc_xorshift64star(uint64_t x);
int orc_nndescent(const float *X, int64_t n, int32_t d, int32_t k, int32_t sample_num,
                  int32_t iterations, int32_t *ids_out, float *dist_out);
/* NN-Descent with the local join's candidate distances in a precision form,
 * exact initial distances and an exact FP32 re-rank at the end (the
 * evaluation of the BF16 / FP8 forms). */
enum { ORC_FORM_FP32 = 0, ORC_FORM_BF16 = 1, ORC_FORM_FP8 = 2, ORC_FORM_FP16 = 3 };
int orc_nndescent_form(const float *X, int64_t n, int32_t d, int32_t k, int32_t sample_num,
                       int32_t iterations, int32_t form, int32_t *ids_out, float *dist_out);
int orc_knn_merge(const float *X, int64_t n1, int64_t n2, int32_t d, const int32_t *ids1,
                  const int32_t *ids2, int32_t k, int32_t sample_num, int32_t iterations,
                  int32_t *ids_out, float *dist_out);
int orc_bruteforce_knn(const float *X, int64_t n, int32_t d, int32_t k,
                       const int64_t *queries, int64_t nq, int32_t *ids_out, double *dist_out);
double orc_recall(const int32_t *ids, int32_t k_ids, const int32_t *gt, int32_t k_gt,
                  int64_t rows, int32_t recall_at);
void orc_fix_distances(const float *X, int64_t n, int32_t d, const int32_t *ids, int32_t k,
                       float *dist_out);
float orc_euclid_ref(const float *a, const float *b, int32_t d);
float orc_diffsum(const float *a, const float *b, int32_t d);

/* ---- enhanced kNN graph (HDBSCAN/graphs/graph.cu:16-176) ---- */
int orc_validate_knn(const int32_t *ids, int64_t n, int32_t k);
void orc_degrees(const int32_t *ids, int64_t n, int32_t k, int32_t *deg_out);
int32_t orc_select_antihubs(const int32_t *ids, const int32_t *deg, int64_t n, int32_t k,
                            int32_t *antihubs_out);
int64_t orc_enhanced_knng(const int32_t *ids, const float *dist, const float *X, int64_t n,
                          int32_t d, int32_t k, int64_t **nindex_out, int32_t **nlist_out,
                          float **eweight_out, int32_t **antihubs_out, int32_t *num_antihubs_out);
/* Core-SG (kNN graph + MST), core-sg.cu; returns the edge count or -1. */
int64_t orc_core_sg(const int32_t *ids, const float *dist, const float *X, int64_t n, int32_t d,
                    int32_t k, const orc_mst_edge *mst, int64_t **nindex_out, int32_t **nlist_out,
                    float **eweight_out);

/* ---- MST (HDBSCAN/mst/mst.cu, HDBSCAN/merge_sort/merge_sort.cu) ---- */
int orc_kruskal(const int64_t *nindex, const int32_t *nlist, const float *eweight, int32_t nodes,
                int64_t edges, uint8_t *in_mst);
int orc_build_mst(const int64_t *nindex, const int32_t *nlist, const float *eweight,
                  int32_t nodes, int64_t edges, const uint8_t *in_mst, orc_mst_edge *out);
/* mst_gpu = 1 (core-sg.cu:8-44, mst.cu:210-288, 338-380): int-quantised MST,
 * dequantised weights, stably sorted.  first_dist[i]: row i's first kNN
 * distance as the .kgraph holds it. */
int orc_mst_quantised(const int64_t *nindex, const int32_t *nlist, const float *eweight,
                      int32_t nodes, int64_t edges, const float *first_dist, orc_mst_edge *out,
                      int32_t *mult_out);
void orc_sort_edges(orc_mst_edge *edges, int64_t m);
/* Tie orders of the float MST: cpuMST's (weight, CSR edge index) and
 * (weight, min id, max id, edge index). */
enum { ORC_ORDER_EDGE = 0, ORC_ORDER_IDS = 1 };
int orc_mst_ordered(const int64_t *nindex, const int32_t *nlist, const float *eweight,
                    int32_t nodes, int64_t edges, int32_t order, uint8_t *in_mst,
                    orc_mst_edge *out);

/* ---- trees (HDBSCAN/trees/tree.cu) ---- */
void orc_linkage_tree(const orc_mst_edge *sorted, int64_t num_points, orc_linkage_node *out);
int64_t orc_condensed_tree(const orc_linkage_node *hier, int64_t num_points, int32_t mpts,
                           orc_condensed_node **out);
int64_t orc_stability(const orc_condensed_node *tree, int64_t size, orc_stab **out,
                      double **out64);
int orc_get_clusters(const orc_condensed_node *tree, int64_t size, orc_stab *stab,
                     double *stab64, int64_t stab_size, int64_t num_points, int32_t *labels_out,
                     int32_t *num_clusters_out);

/* ---- end to end: kNN graph given -> labels ---- */
int orc_hdbscan_from_knn(const int32_t *ids, const float *dist, const float *X, int64_t n,
                         int32_t d, int32_t k, int32_t mpts, int32_t fp64_stability,
                         orc_mst_edge *mst_out, int32_t *labels_out, int32_t *num_clusters_out);
/* The same with the MST under a tie order (ORC_ORDER_EDGE is the above). */
int orc_hdbscan_from_knn_order(const int32_t *ids, const float *dist, const float *X, int64_t n,
                               int32_t d, int32_t k, int32_t mpts, int32_t fp64_stability,
                               int32_t order, orc_mst_edge *mst_out, int32_t *labels_out,
                               int32_t *num_clusters_out);

#ifdef __cplusplus
}
#endif
#endif
