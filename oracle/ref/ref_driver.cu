// Driver for the reference's own HDBSCAN code, compiled unmodified from the
// reference tree (see oracle/ref/Makefile).  TEST INFRASTRUCTURE ONLY: it
// produces golden outputs that pin the CPU oracle (oracle/hdb_oracle.c).
//
// The reference's multi-GPU plumbing (countDegrees, countThreshold_,
// calculateUntieScore, calculateMutualReachabilityDistance) loops over 3 GPUs;
// on a machine with one GPU those loops fail, so this driver calls the same reference
// kernels and host functions those wrappers call, on device 0, in the order of
// buildEnhancedKNNG / buildECLgraph (HDBSCAN/graphs/graph.cu:16-176).
// Everything after the graph -- cpuMST, buildMST (with sort_edges),
// build_Linkage_tree, build_Condensed_tree, compute_stability, get_clusters --
// is called directly.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <string>

#include "HDBSCAN/calculates/calculates.cuh"
#include "HDBSCAN/counts/count.cuh"
#include "HDBSCAN/getters/getters.cuh"
#include "HDBSCAN/initializer/initialize.cuh"
#include "HDBSCAN/mst/mst.cuh"
#include "HDBSCAN/structs/ECLgraph.h"
#include "HDBSCAN/structs/hdbscan_elements.cuh"
#include "HDBSCAN/trees/tree.cuh"
#include "HDBSCAN/graphs/graph.cuh"
#include "gpuknn/nndescent.cuh"
#include "tools/filetool.hpp"

// ---- stand-ins for the reference's fixed-path file helpers (build_kNNG.cu) ----
// The reference passes the kNN graph, the mutual flags, the vectors and the
// core-SG's Euclidean weights between its stages through files under fixed
// /nndescent/... paths.  Here each reader serves, and each writer keeps, the
// arrays of the current driver call.
static const float *g_vectors = nullptr;
static int g_dim = 0;
static const int *g_ids = nullptr;      // kNN ids [g_n, k] of the current call
static const float *g_dist = nullptr;   // their distances
static long g_n = 0;
static int *g_flags = nullptr;          // mutual flags kept by write_bool_dict
static float *g_euclid = nullptr;       // kept by write_euclidean_distance_vecs

// jesus (build_kNNG.cu:58-77) reads /nndescent/.../vectors.fvecs and gathers
// the antihub rows; here the rows come from the caller's array.
float *jesus(int *antihubs, int num_antihubs, int *paz) {
  float *out = new float[(size_t)g_dim * num_antihubs];
  for (long i = 0; i < num_antihubs; i++)
    for (long j = 0; j < g_dim; j++) out[i * g_dim + j] = g_vectors[(long)antihubs[i] * g_dim + j];
  *paz = g_dim;
  return out;
}
// write_bool_dict / read_bool_dict (build_kNNG.cu:79-87): the mutual flags of
// calculate_nindex, read back by Union_kNNG_MST (core-sg.cu:296).
void write_bool_dict(int *flags, long n, long kk) {
  free(g_flags);
  g_flags = (int *)malloc((size_t)n * kk * sizeof(int));
  memcpy(g_flags, flags, (size_t)n * kk * sizeof(int));
}
int *read_bool_dict() {
  int *out = (int *)malloc((size_t)g_n * k * sizeof(int));
  memcpy(out, g_flags, (size_t)g_n * k * sizeof(int));
  return out;
}
// ReadkNNGgraph: the .kgraph of the current call as NNDElement rows (the
// callers release it with delete, as they do the reader's array).
NNDElement *ReadkNNGgraph() {
  NNDElement *G = new NNDElement[(size_t)g_n * k];
  for (long i = 0; i < g_n * (long)k; i++) G[i] = NNDElement(g_dist[i], g_ids[i]);
  return G;
}
// ReadObjects: the vectors (core_sg_calculate_MRD_mst frees them with free()).
float *ReadObjects(long *pf) {
  float *out = (float *)malloc((size_t)g_n * g_dim * sizeof(float));
  memcpy(out, g_vectors, (size_t)g_n * g_dim * sizeof(float));
  *pf = g_dim;
  return out;
}
// The core-SG's Euclidean weights, written by Union_kNNG_MST (core-sg.cu:394)
// and read back by update_core_sg_weights (core-sg.cu:466).
void write_euclidean_distance_vecs(float *e, long edges) {
  free(g_euclid);
  g_euclid = (float *)malloc((size_t)edges * sizeof(float));
  memcpy(g_euclid, e, (size_t)edges * sizeof(float));
}
float *read_euclidean_distance_vecs() {
  float *out = g_euclid;  // ownership passes to the caller
  g_euclid = nullptr;
  return out;
}

// The helpers of HDBSCAN/core-sg/core-sg.cu that Union_kNNG_MST calls
// (defined there, not declared in its header).
void core_sg_calculate_nindex(long int nodes, int *flag_knn, int *kNN, ECLgraph *g,
                              MSTedge *mst_edges);
void core_sg_calculate_nlist(long int nodes, int *flag_knn, int *kNN, ECLgraph *g,
                             MSTedge *mst_edges, long int *auxiliar_edges, long int *offsets,
                             float *euclidean_distance, float *distance);
void core_sg_calculate_MRD_mst(ECLgraph *g, long int *auxiliar_edges, MSTedge *mst_edges,
                               long int nodes, float *euclidean_distance_);
void update_core_sg_weights(ECLgraph *g, int nodes, long int mpts);

static int check(const char *what) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    return 1;
  }
  return 0;
}

extern "C" {

// Enhanced kNN graph.  Outputs are malloc'd; free with ref_free.
long ref_enhanced_knng(const int *ids_in, const float *dist_in, const float *X, long n, int d,
                       int kk, long **nindex_out, int **nlist_out, float **ew_out,
                       int **antihubs_out, int *num_antihubs_out) {
  if (kk != k) {
    fprintf(stderr, "reference compiled with k = %d\n", k);
    return -1;
  }
  g_vectors = X;
  g_dim = d;
  long vectorSize = n * (long)k;
  int *kNN;
  float *distances;
  cudaMallocManaged(&kNN, vectorSize * sizeof(int));
  cudaMallocManaged(&distances, vectorSize * sizeof(float));
  memcpy(kNN, ids_in, vectorSize * sizeof(int));
  memcpy(distances, dist_in, vectorSize * sizeof(float));
  // calculate_degrees / countDegrees / countValues (calculates.cu:448, count.cu:10-110)
  int *finalCounts;
  cudaMallocManaged(&finalCounts, n * sizeof(int));
  cudaMemset(finalCounts, 0, n * sizeof(int));
  countValues<<<(unsigned)(vectorSize / blockSize + 1), blockSize>>>(kNN, finalCounts, vectorSize);
  if (check("countValues")) return -1;
  // buildEnhancedKNNG (graph.cu:108-151)
  Vertex *vertexes;
  cudaMallocManaged(&vertexes, n * sizeof(Vertex));
  initializeVertex<<<(unsigned)((n + blockSize - 1) / blockSize), blockSize>>>(vertexes, finalCounts, n);
  if (check("initializeVertex")) return -1;
  int pos_threshold = get_NumThreshold(n);
  std::partial_sort(vertexes, vertexes + pos_threshold, vertexes + n, compareVertexByDegree);
  int value_threshold = vertexes[pos_threshold - 1].grau;
  int countsTreshold = 0;  // countThreshold_ (count.cu:112-177)
  for (long i = 0; i < n; i++) countsTreshold += (vertexes[i].grau == value_threshold);
  int *antihubs = new int[pos_threshold];
  if (countsTreshold > 1) {
    // calculate_finalAntihubs (calculates.cu:491-523) with calculateUntieScore on one GPU
    int *treshold_idx;
    cudaMallocManaged(&treshold_idx, countsTreshold * sizeof(int));
    get_IndexThreshold(finalCounts, treshold_idx, value_threshold, n);
    Untie_hub *unties_dev;
    cudaMalloc(&unties_dev, countsTreshold * sizeof(Untie_hub));
    long numBlocks = countsTreshold / blockSize + 1;
    initializeUntieHubs<<<(unsigned)numBlocks, blockSize>>>(unties_dev, 0, countsTreshold);
    calculateScore<<<(unsigned)numBlocks, blockSize>>>(kNN, treshold_idx, unties_dev, finalCounts,
                                                       countsTreshold, k, 0);
    if (check("calculateScore")) return -1;
    Untie_hub *unties = new Untie_hub[countsTreshold];
    cudaMemcpy(unties, unties_dev, countsTreshold * sizeof(Untie_hub), cudaMemcpyDeviceToHost);
    cudaFree(unties_dev);
    int missing_ties = get_TiedVertexes(vertexes, pos_threshold, value_threshold);
    int not_ties = pos_threshold - missing_ties;
    std::partial_sort(unties, unties + missing_ties, unties + countsTreshold, compareVertexByScore);
    joinAntiHubs(antihubs, vertexes, not_ties, unties, missing_ties);
    delete[] unties;
    cudaFree(treshold_idx);
  } else {
    for (int i = 0; i < pos_threshold; i++) antihubs[i] = vertexes[i].index;
  }
  std::sort(antihubs, antihubs + pos_threshold);
  cudaFree(finalCounts);
  cudaFree(vertexes);
  // buildECLgraph (graph.cu:16-103)
  ECLgraph g;
  g.nodes = (int)n;
  cudaMallocManaged(&g.nindex, (n + 1) * sizeof(long));
  memset(g.nindex, 0, (n + 1) * sizeof(long));
  int *flag_knn = (int *)malloc(vectorSize * sizeof(int));
  calculate_nindex((int)n, kNN, flag_knn, &g, antihubs, pos_threshold);
  long *auxiliar_edges;
  cudaMallocManaged(&auxiliar_edges, n * sizeof(long));
  memset(auxiliar_edges, 0, n * sizeof(long));
  cudaMallocManaged(&g.nlist, g.nindex[n] * sizeof(int));
  g.edges = g.nindex[n];
  calculate_nlist((int)n, kNN, k, flag_knn, &g, antihubs, pos_threshold, auxiliar_edges);
  free(flag_knn);
  cudaMallocManaged(&g.eweight, g.edges * sizeof(float));
  int *aux_nodes;
  cudaMallocManaged(&aux_nodes, g.edges * sizeof(int));
  createNodeList(aux_nodes, &g);
  float *coreDistances;
  cudaMallocManaged(&coreDistances, n * sizeof(float));
  calculateCoreDistance(distances, coreDistances, n, k, k - 1);
  // calculateMutualReachabilityDistance (calculates.cu:199-273) on one GPU
  calculateMRD<<<(unsigned)(g.edges / blockSize + 1), blockSize>>>(g.eweight, aux_nodes, g.nlist,
                                                                   coreDistances, g.edges);
  if (check("calculateMRD")) return -1;
  calculate_coreDistance_antihubs(&g, auxiliar_edges, antihubs, pos_threshold);
  long E = g.edges;
  *nindex_out = (long *)malloc((n + 1) * sizeof(long));
  *nlist_out = (int *)malloc(E * sizeof(int));
  *ew_out = (float *)malloc(E * sizeof(float));
  *antihubs_out = (int *)malloc(pos_threshold * sizeof(int));
  memcpy(*nindex_out, g.nindex, (n + 1) * sizeof(long));
  memcpy(*nlist_out, g.nlist, E * sizeof(int));
  memcpy(*ew_out, g.eweight, E * sizeof(float));
  memcpy(*antihubs_out, antihubs, pos_threshold * sizeof(int));
  *num_antihubs_out = pos_threshold;
  delete[] antihubs;
  cudaFree(kNN);
  cudaFree(distances);
  cudaFree(aux_nodes);
  cudaFree(coreDistances);
  cudaFree(auxiliar_edges);
  cudaFree(g.nindex);
  cudaFree(g.nlist);
  cudaFree(g.eweight);
  return E;
}

// cpuMST + buildMST (sort_edges) + build_Linkage_tree + build_Condensed_tree
// + compute_stability + get_clusters (HDBSCAN/_new.cu:311-347).
int ref_mst_trees(const long *nindex, const int *nlist, const float *ew, long n, int mpts,
                  MSTedge *mst_out, SingleLinkageNode *hier_out, int *labels_out,
                  CondensedTreeNode **cond_out, long *cond_size, Stability **stab_out,
                  long *stab_size) {
  ECLgraph g;
  g.nodes = (int)n;
  g.edges = nindex[n];
  cudaMallocManaged(&g.nindex, (n + 1) * sizeof(long));
  cudaMallocManaged(&g.nlist, g.edges * sizeof(int));
  cudaMallocManaged(&g.eweight, g.edges * sizeof(float));
  memcpy(g.nindex, nindex, (n + 1) * sizeof(long));
  memcpy(g.nlist, nlist, g.edges * sizeof(int));
  memcpy(g.eweight, ew, g.edges * sizeof(float));
  bool *edges = cpuMST(g);
  MSTedge *mst = buildMST(g, edges);
  if (check("buildMST")) return 1;
  memcpy(mst_out, mst, (n - 1) * sizeof(MSTedge));
  SingleLinkageNode *h = build_Linkage_tree(mst, (int)n, (int)n);
  memcpy(hier_out, h, (n - 1) * sizeof(SingleLinkageNode));
  int csize = 0;
  CondensedTreeNode *ct = build_Condensed_tree(h, (int)n, (int)n - 1, mpts, &csize);
  int ssize = 0;
  Stability *st = compute_stability(ct, csize, &ssize);
  *stab_out = (Stability *)malloc(ssize * sizeof(Stability));
  memcpy(*stab_out, st, ssize * sizeof(Stability));  // before get_clusters updates it
  *stab_size = ssize;
  *cond_out = (CondensedTreeNode *)malloc(csize * sizeof(CondensedTreeNode));
  memcpy(*cond_out, ct, csize * sizeof(CondensedTreeNode));
  *cond_size = csize;
  int *labels = get_clusters(ct, csize, st, ssize, (int)n);
  memcpy(labels_out, labels, n * sizeof(int));
  cudaFree(g.nindex);
  cudaFree(g.nlist);
  cudaFree(g.eweight);
  return check("trees");
}

// gpuknn::NNDescent (gpuknn/nndescent.cu:2088-2199) as compiled: VEC_DIM = 12,
// NEIGHB_NUM_PER_LIST = 32, SAMPLE_NUM = 16.
int ref_nndescent(const float *X, long n, int d, int iterations, NNDElement *G_out) {
  if (d != VEC_DIM) return 1;
  float *Xd;
  cudaMalloc(&Xd, n * d * sizeof(float));
  cudaMemcpy(Xd, X, n * d * sizeof(float), cudaMemcpyHostToDevice);
  NNDElement *G = nullptr;
  gpuknn::NNDescent(&G, Xd, (int)n, d, iterations, false);
  if (check("NNDescent")) return 1;
  memcpy(G_out, G, n * NEIGHB_NUM_PER_LIST * sizeof(NNDElement));
  delete[] G;
  cudaFree(Xd);
  return 0;
}

// The mst_gpu = 1 branch of build_CoreSG (core-sg.cu:533-540): buildGPUgraph,
// gpuMST(g, INT_MAX), buildMST_gpu (dequantised weights, sort_edges).
// buildGPUgraph (core-sg.cu:8-44) itself is not called: it hands
// FileTool::GetMinDistanceFromKNNG an uninitialised `long` for the row width,
// of which the reader fills only 4 bytes (filetool.hpp:321), so it works only
// when that stack slot happens to be zero.  Here the same reader runs with the
// long zeroed, and buildGPUgraph's scaling (multiplier ceil(-log10|min|) + 2,
// weights (int)(10^m * w)) is repeated line for line; gpuMST and buildMST_gpu
// are the reference's.
int ref_mst_gpu(const long *nindex, const int *nlist, const float *ew, long n,
                const char *kgraph_path, MSTedge *mst_out, int *mult_out) {
  NNDElement *row = nullptr;
  long knng_num = 0, knng_dim = 0;
  double min_dist = FileTool::GetMinDistanceFromKNNG(std::string(kgraph_path), &row, &knng_num,
                                                     &knng_dim);
  delete[] row;
  int multiplica = ceil(-log10(fabs(min_dist))) + 2;
  GPUECLgraph gg;
  gg.nodes = (int)n;
  gg.edges = (int)nindex[n];
  gg.nindex = new int[n + 1];
  gg.nlist = new int[gg.edges];
  gg.eweight = new int[gg.edges];
  for (long i = 0; i <= n; i++) gg.nindex[i] = (int)nindex[i];
  for (long i = 0; i < gg.edges; i++) {
    gg.nlist[i] = nlist[i];
    gg.eweight[i] = (int)(pow(10.0, multiplica) * (double)ew[i] / 1);
  }
  bool *edges = gpuMST(gg, INT_MAX);
  MSTedge *mst = buildMST_gpu(gg, edges, multiplica);
  if (check("buildMST_gpu")) return 1;
  memcpy(mst_out, mst, (n - 1) * sizeof(MSTedge));
  *mult_out = multiplica;
  delete[] gg.nindex;
  delete[] gg.nlist;
  delete[] gg.eweight;
  gg.nindex = nullptr;
  gg.nlist = nullptr;
  gg.eweight = nullptr;
  return 0;
}

// build_CoreSG's graph (core-sg.cu:477-571 with mst_gpu = 0): Union_kNNG_MST
// (core-sg.cu:292-420) on the kNN graph and its sorted MST, then
// update_core_sg_weights (core-sg.cu:432-471), which leaves the Euclidean
// weights in eweight.  Union_kNNG_MST's body runs here step by step because
// its MRD pass (calculateMutualReachabilityDistance, calculates.cu:199-273)
// loops over three GPUs; the MRD kernel it launches (calculateMRD) runs once
// over all edges instead.  Its MRD weights are overwritten by
// update_core_sg_weights and are not part of the result.  The mutual flags
// come from calculate_nindex (calculates.cu:286-333), as buildEnhancedKNNG
// writes them.  Outputs are malloc'd; free with ref_free.
long ref_core_sg(const int *ids_in, const float *dist_in, const float *X, long n, int d,
                 int kk, const MSTedge *mst_in, long **nindex_out, int **nlist_out,
                 float **ew_out) {
  if (kk != k) {
    fprintf(stderr, "reference compiled with k = %d\n", k);
    return -1;
  }
  g_vectors = X;
  g_dim = d;
  g_ids = ids_in;
  g_dist = dist_in;
  g_n = n;
  long vectorSize = n * (long)k;
  int *kNN = new int[vectorSize];
  float *distances = new float[vectorSize];
  memcpy(kNN, ids_in, vectorSize * sizeof(int));
  memcpy(distances, dist_in, vectorSize * sizeof(float));
  // the mutual flags (write_bool_dict keeps them); no antihubs needed for them
  {
    ECLgraph t;
    t.nindex = (long *)calloc(n + 1, sizeof(long));
    int *flag_tmp = (int *)malloc(vectorSize * sizeof(int));
    int no_antihub = -1;
    calculate_nindex((int)n, kNN, flag_tmp, &t, &no_antihub, 0);
    free(flag_tmp);
    free(t.nindex);
  }
  int *flag_knn = read_bool_dict();
  MSTedge *mst_edges = (MSTedge *)malloc((n - 1) * sizeof(MSTedge));
  memcpy(mst_edges, mst_in, (n - 1) * sizeof(MSTedge));
  // Union_kNNG_MST (core-sg.cu:292-420)
  ECLgraph g;
  g.nodes = (int)n;
  cudaMallocManaged(&g.nindex, (n + 1) * sizeof(long));
  memset(g.nindex, 0, (n + 1) * sizeof(long));
  core_sg_calculate_nindex(n, flag_knn, kNN, &g, mst_edges);
  long *offsets, *auxiliar_edges;
  cudaMallocManaged(&offsets, n * sizeof(long));
  cudaMallocManaged(&auxiliar_edges, n * sizeof(long));
  memset(auxiliar_edges, 0, n * sizeof(long));
  cudaMallocManaged(&g.nlist, g.nindex[n] * sizeof(int));
  g.edges = g.nindex[n];
  float *euclidean_distance = new float[g.edges];
  core_sg_calculate_nlist(n, flag_knn, kNN, &g, mst_edges, auxiliar_edges, offsets,
                          euclidean_distance, distances);
  int *aux_nodes;
  cudaMallocManaged(&aux_nodes, g.edges * sizeof(int));
  createNodeList(aux_nodes, &g);
  if (check("createNodeList")) return -1;
  float *coreDistances;
  cudaMallocManaged(&coreDistances, n * sizeof(float));
  calculateCoreDistance(distances, coreDistances, n, k, mpts - 1);
  cudaMallocManaged(&g.eweight, g.edges * sizeof(float));
  calculateMRD<<<(unsigned)(g.edges / blockSize + 1), blockSize>>>(g.eweight, aux_nodes, g.nlist,
                                                                   coreDistances, g.edges);
  if (check("calculateMRD")) return -1;
  core_sg_calculate_MRD_mst(&g, offsets, mst_edges, n, euclidean_distance);
  write_euclidean_distance_vecs(euclidean_distance, g.edges);
  delete[] euclidean_distance;
  cudaFree(aux_nodes);
  cudaFree(coreDistances);
  cudaFree(offsets);
  cudaFree(auxiliar_edges);
  // update_core_sg_weights (core-sg.cu:432-471), unmodified: eweight becomes
  // the Euclidean weights kept above
  update_core_sg_weights(&g, (int)n, mpts);
  if (check("update_core_sg_weights")) return -1;
  long E = g.edges;
  *nindex_out = (long *)malloc((n + 1) * sizeof(long));
  *nlist_out = (int *)malloc(E * sizeof(int));
  *ew_out = (float *)malloc(E * sizeof(float));
  memcpy(*nindex_out, g.nindex, (n + 1) * sizeof(long));
  memcpy(*nlist_out, g.nlist, E * sizeof(int));
  memcpy(*ew_out, g.eweight, E * sizeof(float));
  free(g.eweight);  // the array read_euclidean_distance_vecs handed over
  cudaFree(g.nindex);
  cudaFree(g.nlist);
  free(mst_edges);
  free(flag_knn);
  delete[] kNN;
  delete[] distances;
  return E;
}

void ref_free(void *p) { free(p); }

}  // extern "C"
