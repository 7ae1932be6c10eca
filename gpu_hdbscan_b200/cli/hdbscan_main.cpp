// hdbscan_ -- command-line driver with the reference's argv
// (HDBSCAN/new.cu:18-45, HDBSCAN/_new.cu:149-347):
//
//   hdbscan_ NUM_VALUES mpts shards mst_gpu [options]
//
// Exactly four positional arguments, otherwise it prints "NUM_VALUES NOT
// SETTED" and exits 1; mpts must not exceed k (assert(k >= mpts)).  `shards`
// is accepted for compatibility (the path runs on one GPU); mst_gpu selects
// the MST as in the reference: 0 = the float MST of cpuMST, 1 = the
// int-quantised GPU MST of buildGPUgraph + gpuMST + buildMST_gpu (both run
// as GPU Boruvka here).  The stages run in the reference's order, one library
// call each:
// kNN graph (built, or read from a .kgraph), fix_distances, enhanced kNN
// graph, MST, linkage tree, condensed tree / stability / clusters.  Instead
// of the reference's hard-coded /nndescent/... paths the files are options:
//   --vectors PATH      .fvecs vectors (FileTool::ReadBinaryVecs layout)
//   --vectors-txt PATH  text vectors, "N d" then N*d values (ReadTxtVecs,
//                       written by the reference's data/artificial/create.py)
//   --write-fvecs PATH  write the vectors as .fvecs (PrepareVector)
//   --kgraph PATH       read this .kgraph (NNDElement rows) instead of building
//                       it (the reference's _new.cu reads NNDescent-KNNG.kgraph)
//   --save-kgraph PATH  write the kNN graph as NN-Descent leaves it (squared
//                       distances, old/new flags), as GenLargeKNNGraph does
//   --save-fixed-kgraph PATH  write it after fix_distances: sqrt-L2 distances
//                       with the reference's rounding, labels and flags
//                       untouched -- the file build_kNNG.cu:131-174 writes
//   --squared           skip fix_distances (keep the graph's distances)
//   --save-mst PATH     write the sorted MST as raw MSTedge[n-1] records
//                       (12 bytes: int32 from, int32 to, float32 weight)
//   --labels PATH       write one label per line (-1 = noise)
//   --fp64              FP64 stability sums (default: the reference's FP32)
//   --bf16              build the kNN graph with the BF16 tensor-core form
//   --fp16              build the kNN graph with the FP16 tensor-core form
//   --id-order          float MST (mst_gpu 0) under the tie order (weight,
//                       min id, max id) instead of (weight, CSR edge index)
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "hdb/hdb.h"

namespace {

// FileTool::ReadBinaryVecs / WriteBinaryVecs layout (tools/filetool.hpp:96-227):
// every row is an int32 dimension followed by that many elements.
template <typename T>
bool read_vecs(const std::string &path, std::vector<T> &out, long *num, long *dim) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) return false;
  int d = 0;
  if (fread(&d, 4, 1, f) != 1 || d <= 0) { fclose(f); return false; }
  fseek(f, 0, SEEK_END);
  long size = ftell(f);
  rewind(f);
  long rows = size / (4 + (long)d * (long)sizeof(T));
  out.resize((size_t)rows * d);
  for (long i = 0; i < rows; i++) {
    int dd = 0;
    if (fread(&dd, 4, 1, f) != 1 || dd != d ||
        fread(out.data() + (size_t)i * d, sizeof(T), d, f) != (size_t)d) {
      fclose(f);
      return false;
    }
  }
  fclose(f);
  *num = rows;
  *dim = d;
  return true;
}

template <typename T>
bool write_vecs(const std::string &path, const T *data, long num, int dim) {
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) return false;
  for (long i = 0; i < num; i++) {
    fwrite(&dim, 4, 1, f);
    fwrite(data + (size_t)i * dim, sizeof(T), dim, f);
  }
  return fclose(f) == 0;
}

// FileTool::ReadTxtVecs (tools/filetool.hpp:244-268): "num dim", then values.
bool read_txt_vecs(const std::string &path, std::vector<float> &out, long *num, long *dim) {
  std::ifstream in(path);
  if (!in.is_open()) return false;
  long n = 0, d = 0;
  if (!(in >> n >> d) || n <= 0 || d <= 0) return false;
  out.resize((size_t)n * d);
  for (size_t i = 0; i < out.size(); i++)
    if (!(in >> out[i])) return false;
  *num = n;
  *dim = d;
  return true;
}

int fail(const char *what) {
  fprintf(stderr, "%s: %s\n", what, hdb_last_error());
  return 1;
}

template <typename T>
T *to_device(const T *h, size_t count) {
  T *d = nullptr;
  if (cudaMalloc(&d, count * sizeof(T) + 16) != cudaSuccess) return nullptr;
  if (h) cudaMemcpy(d, h, count * sizeof(T), cudaMemcpyHostToDevice);
  return d;
}

double secs_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

}  // namespace

int main(int argc, char **argv) {
  std::vector<std::string> pos;
  std::string kgraph, vectors, vectors_txt, write_fvecs, labels_path, save_kgraph, save_fixed,
      save_mst;
  bool squared = false, fp64 = false, bf16 = false, fp16 = false, id_order = false;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto val = [&](std::string &dst) {
      if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); exit(1); }
      dst = argv[++i];
    };
    if (a == "--kgraph") val(kgraph);
    else if (a == "--vectors") val(vectors);
    else if (a == "--vectors-txt") val(vectors_txt);
    else if (a == "--write-fvecs") val(write_fvecs);
    else if (a == "--labels") val(labels_path);
    else if (a == "--save-kgraph") val(save_kgraph);
    else if (a == "--save-fixed-kgraph") val(save_fixed);
    else if (a == "--save-mst") val(save_mst);
    else if (a == "--squared") squared = true;
    else if (a == "--fp64") fp64 = true;
    else if (a == "--bf16") bf16 = true;
    else if (a == "--id-order") id_order = true;
    else if (a == "--fp16") fp16 = true;
    else pos.push_back(a);
  }
  if (pos.size() != 4) {
    printf("NUM_VALUES NOT SETTED\n");
    return 1;
  }
  long num_values = atol(pos[0].c_str());
  int mpts = atoi(pos[1].c_str());
  int shards = atoi(pos[2].c_str());
  int mst_gpu = atoi(pos[3].c_str());
  printf("NUM VALUES SET TO %ld.\nmpts SET TO %d.\nSHARDS SET TO %d.\nMST WILL BE CONSTRUCTED IN GPU: %d\n",
         num_values, mpts, shards, mst_gpu);
  const int k = 32;  // NEIGHB_NUM_PER_LIST
  if (!(k >= mpts)) {
    fprintf(stderr, "assertion k >= mpts failed\n");
    return 1;
  }
  std::vector<float> X;
  long n = 0, d = 0;
  if (!vectors.empty()) {
    if (!read_vecs(vectors, X, &n, &d)) {
      fprintf(stderr, "cannot read %s\n", vectors.c_str());
      return 1;
    }
  } else if (!vectors_txt.empty()) {
    if (!read_txt_vecs(vectors_txt, X, &n, &d)) {
      fprintf(stderr, "cannot read %s\n", vectors_txt.c_str());
      return 1;
    }
  } else {
    fprintf(stderr, "--vectors PATH (.fvecs) or --vectors-txt PATH is required\n");
    return 1;
  }
  if (!write_fvecs.empty() && !write_vecs(write_fvecs, X.data(), n, (int)d)) {
    fprintf(stderr, "cannot write %s\n", write_fvecs.c_str());
    return 1;
  }
  if (num_values > 0 && num_values < n) n = num_values;  // knng_num = numValues
  hdb_ctx *ctx = nullptr;
  if (hdb_create(&ctx, 0) != HDB_OK) return fail("hdb_create");
  hdb_knn_params kp{k, 16, 6, fp16 ? HDB_PREC_FP16 : bf16 ? HDB_PREC_BF16 : HDB_PREC_FP32};

  auto t_all = std::chrono::steady_clock::now();
  float *Xd = to_device(X.data(), (size_t)n * d);
  hdb_nnd_element *Gd = to_device<hdb_nnd_element>(nullptr, (size_t)n * k);
  int32_t *ids = to_device<int32_t>(nullptr, (size_t)n * k);
  float *dist = to_device<float>(nullptr, (size_t)n * k);
  hdb_mst_edge *mst = to_device<hdb_mst_edge>(nullptr, (size_t)n);
  hdb_linkage_node *hier = to_device<hdb_linkage_node>(nullptr, (size_t)n);
  int32_t *labels_d = to_device<int32_t>(nullptr, (size_t)n);
  if (!Xd || !Gd || !ids || !dist || !mst || !hier || !labels_d) {
    fprintf(stderr, "device allocation failed\n");
    return 1;
  }

  // kNN graph: read (the reference's _new.cu) or built by NN-Descent
  auto t = std::chrono::steady_clock::now();
  std::vector<hdb_nnd_element> G;
  if (!kgraph.empty()) {
    long gn = 0, gk = 0;
    if (!read_vecs(kgraph, G, &gn, &gk) || gk != k || gn < n) {
      fprintf(stderr, "cannot read a k=%d graph with %ld rows from %s\n", k, n, kgraph.c_str());
      return 1;
    }
    cudaMemcpy(Gd, G.data(), (size_t)n * k * sizeof(hdb_nnd_element), cudaMemcpyHostToDevice);
  } else {
    if (hdb_nndescent(ctx, Xd, n, (int)d, &kp, Gd) != HDB_OK) return fail("hdb_nndescent");
  }
  const double t_knn = secs_since(t);
  if (!save_kgraph.empty() || !save_fixed.empty()) {
    G.resize((size_t)n * k);
    cudaMemcpy(G.data(), Gd, G.size() * sizeof(hdb_nnd_element), cudaMemcpyDeviceToHost);
  }
  if (!save_kgraph.empty() && !write_vecs(save_kgraph, G.data(), n, k)) {
    fprintf(stderr, "cannot write %s\n", save_kgraph.c_str());
    return 1;
  }

  // fix_distances (build_kNNG.cu:131-174): sqrt-L2 with the reference's rounding
  t = std::chrono::steady_clock::now();
  if (hdb_knn_split(ctx, Gd, n, k, ids, dist) != HDB_OK) return fail("hdb_knn_split");
  if (!squared && hdb_fix_distances(ctx, Xd, n, (int)d, ids, k, dist) != HDB_OK)
    return fail("hdb_fix_distances");
  const double t_fix = secs_since(t);
  if (!save_fixed.empty()) {
    // SetDistance on every element: labels and their old/new flags stay as they are
    std::vector<float> hd((size_t)n * k);
    cudaMemcpy(hd.data(), dist, hd.size() * sizeof(float), cudaMemcpyDeviceToHost);
    for (size_t i = 0; i < hd.size(); i++) G[i].distance_ = hd[i];
    if (!write_vecs(save_fixed, G.data(), n, k)) {
      fprintf(stderr, "cannot write %s\n", save_fixed.c_str());
      return 1;
    }
  }

  // enhanced kNN graph, MST, trees
  t = std::chrono::steady_clock::now();
  hdb_graph g{};
  if (hdb_enhanced_knng(ctx, ids, dist, Xd, n, (int)d, k, &g) != HDB_OK)
    return fail("hdb_enhanced_knng");
  const double t_graph = secs_since(t);
  t = std::chrono::steady_clock::now();
  int32_t rounds = 0, mult = 0;
  if (mst_gpu) {
    if (hdb_mst_quantised(ctx, &g, dist, k, nullptr, mst, &mult, &rounds) != HDB_OK)
      return fail("hdb_mst_quantised");
    printf("MST WEIGHT MULTIPLIER: 10^%d\n", mult);
  } else if (hdb_mst_ordered(ctx, &g, id_order ? HDB_ORDER_IDS : HDB_ORDER_EDGE, nullptr, mst,
                             &rounds) != HDB_OK) {
    return fail("hdb_mst_ordered");
  }
  const double t_mst = secs_since(t);
  t = std::chrono::steady_clock::now();
  int32_t ncl = 0;
  if (hdb_linkage_tree(ctx, mst, n, hier) != HDB_OK) return fail("hdb_linkage_tree");
  if (hdb_condense_select(ctx, hier, n, mpts, fp64 ? HDB_STAB_FP64 : HDB_STAB_FP32, labels_d,
                          &ncl, nullptr, nullptr, nullptr, nullptr) != HDB_OK)
    return fail("hdb_condense_select");
  const double t_tree = secs_since(t);
  const double total = secs_since(t_all);

  printf("TEMPO KNNG: %lf\nTEMPO FIX DISTANCES: %lf\nTEMPO ENHANCED KNNG: %lf\nTEMPO MST: %lf\n"
         "TEMPO TREES: %lf\n",
         t_knn, t_fix, t_graph, t_mst, t_tree);
  printf("EDGES = %ld\nMST ROUNDS = %d\nCLUSTERS FIND = %d\nTOTAL: %lf s (%ld points, %.0f points/s)\n",
         (long)g.edges, rounds, ncl, total, n, n / total);
  if (!save_mst.empty()) {
    std::vector<hdb_mst_edge> hm((size_t)n - 1);
    cudaMemcpy(hm.data(), mst, hm.size() * sizeof(hdb_mst_edge), cudaMemcpyDeviceToHost);
    FILE *f = fopen(save_mst.c_str(), "wb");
    if (!f || fwrite(hm.data(), sizeof(hdb_mst_edge), hm.size(), f) != hm.size() || fclose(f)) {
      fprintf(stderr, "cannot write %s\n", save_mst.c_str());
      return 1;
    }
  }
  if (!labels_path.empty()) {
    std::vector<int32_t> labels((size_t)n);
    cudaMemcpy(labels.data(), labels_d, n * sizeof(int32_t), cudaMemcpyDeviceToHost);
    FILE *f = fopen(labels_path.c_str(), "w");
    if (!f) { fprintf(stderr, "cannot write %s\n", labels_path.c_str()); return 1; }
    for (long i = 0; i < n; i++) fprintf(f, "%d\n", labels[i]);
    fclose(f);
  }
  cudaFree(Xd);
  cudaFree(Gd);
  cudaFree(ids);
  cudaFree(dist);
  cudaFree(mst);
  cudaFree(hier);
  cudaFree(labels_d);
  hdb_destroy(ctx);
  return 0;
}
