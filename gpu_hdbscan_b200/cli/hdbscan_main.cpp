// hdbscan_ -- command-line driver with the reference's argv
// (HDBSCAN/new.cu:18-45, HDBSCAN/_new.cu:149-178):
//
//   hdbscan_ NUM_VALUES mpts shards mst_gpu [options]
//
// Exactly four positional arguments, otherwise it prints "NUM_VALUES NOT
// SETTED" and exits 1; mpts must not exceed k (assert(k >= mpts)).  `shards`
// and `mst_gpu` are accepted for compatibility: the path runs on one GPU and
// its MST is always the GPU Boruvka (bit-identical to the reference's
// cpuMST).  Instead of the reference's hard-coded /nndescent/... paths the
// files are options:
//   --kgraph PATH   read this .kgraph (NNDElement rows) instead of building it
//                   (the reference's _new.cu reads NNDescent-KNNG.kgraph)
//   --vectors PATH  .fvecs vectors (required)
//   --labels PATH   write one label per line (-1 = noise)
//   --save-kgraph PATH  write the kNN graph built from the vectors
//   --squared       keep NN-Descent's squared distances (default: the
//                   reference's fix_distances sqrt-L2)
//   --fp64          FP64 stability sums (default: the reference's FP32)
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
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

int fail(const char *what) {
  fprintf(stderr, "%s: %s\n", what, hdb_last_error());
  return 1;
}

}  // namespace

int main(int argc, char **argv) {
  std::vector<std::string> pos;
  std::string kgraph, vectors, labels_path, save_kgraph;
  bool squared = false, fp64 = false;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto val = [&](std::string &dst) {
      if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); exit(1); }
      dst = argv[++i];
    };
    if (a == "--kgraph") val(kgraph);
    else if (a == "--vectors") val(vectors);
    else if (a == "--labels") val(labels_path);
    else if (a == "--save-kgraph") val(save_kgraph);
    else if (a == "--squared") squared = true;
    else if (a == "--fp64") fp64 = true;
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
  if (vectors.empty()) {
    fprintf(stderr, "--vectors PATH (.fvecs) is required\n");
    return 1;
  }
  std::vector<float> X;
  long n = 0, d = 0;
  if (!read_vecs(vectors, X, &n, &d)) {
    fprintf(stderr, "cannot read %s\n", vectors.c_str());
    return 1;
  }
  if (num_values > 0 && num_values < n) n = num_values;  // knng_num = numValues
  hdb_ctx *ctx = nullptr;
  if (hdb_create(&ctx, 0) != HDB_OK) return fail("hdb_create");
  hdb_params p{};
  p.knn.k = k;
  p.knn.sample_num = 16;
  p.knn.iterations = 6;
  p.knn.precision = HDB_PREC_FP32;
  p.mpts = mpts;
  p.distance = squared ? HDB_DIST_SQUARED : HDB_DIST_SQRT;
  p.stability = fp64 ? HDB_STAB_FP64 : HDB_STAB_FP32;
  p.host_io = 1;
  std::vector<int32_t> labels(n);
  hdb_run_stats st{};
  auto t0 = std::chrono::steady_clock::now();
  std::vector<hdb_nnd_element> G;
  if (!kgraph.empty()) {
    long gn = 0, gk = 0;
    if (!read_vecs(kgraph, G, &gn, &gk) || gk != k || gn < n) {
      fprintf(stderr, "cannot read a k=%d graph with %ld rows from %s\n", k, n, kgraph.c_str());
      return 1;
    }
    if (hdb_run_knn(ctx, G.data(), X.data(), n, (int)d, &p, labels.data(), &st) != HDB_OK)
      return fail("hdb_run_knn");
  } else {
    if (hdb_run(ctx, X.data(), n, (int)d, &p, labels.data(), &st) != HDB_OK) return fail("hdb_run");
    if (!save_kgraph.empty()) {
      // rebuild on the device and save (the reference writes NNDescent-KNNG.kgraph)
      float *Xd = nullptr;
      hdb_nnd_element *Gd = nullptr;
      cudaMalloc(&Xd, (size_t)n * d * sizeof(float));
      cudaMalloc(&Gd, (size_t)n * k * sizeof(hdb_nnd_element));
      cudaMemcpy(Xd, X.data(), (size_t)n * d * sizeof(float), cudaMemcpyHostToDevice);
      if (hdb_nndescent(ctx, Xd, n, (int)d, &p.knn, Gd) != HDB_OK) return fail("hdb_nndescent");
      G.resize((size_t)n * k);
      cudaMemcpy(G.data(), Gd, G.size() * sizeof(hdb_nnd_element), cudaMemcpyDeviceToHost);
      cudaFree(Xd);
      cudaFree(Gd);
      if (!write_vecs(save_kgraph, G.data(), n, k)) fprintf(stderr, "cannot write %s\n", save_kgraph.c_str());
    }
  }
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  printf("TEMPO KNNG: %lf\nTEMPO ENHANCED KNNG: %lf\nTEMPO MST: %lf\nTEMPO TREES: %lf\n",
         st.ms_knn / 1e3, st.ms_graph / 1e3, st.ms_mst / 1e3, st.ms_tree / 1e3);
  printf("CLUSTERS FIND = %d\nTOTAL: %lf s (%ld points, %.0f points/s)\n", st.num_clusters, secs, n,
         n / secs);
  if (!labels_path.empty()) {
    FILE *f = fopen(labels_path.c_str(), "w");
    if (!f) { fprintf(stderr, "cannot write %s\n", labels_path.c_str()); return 1; }
    for (long i = 0; i < n; i++) fprintf(f, "%d\n", labels[i]);
    fclose(f);
  }
  hdb_destroy(ctx);
  return 0;
}
