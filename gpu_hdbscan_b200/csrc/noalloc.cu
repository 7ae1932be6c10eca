// hdb_sort_edges_noalloc: the MST edge sort for callers that cannot allocate.
//
// Some callers cannot call cudaMalloc: code that runs under a host framework
// which owns and accounts for every device byte (and forbids side
// allocations), or code that has to run while the device is already full.
// For them this entry point sorts MST edges without allocating anything --
// no cudaMalloc / cudaMallocAsync / cudaFree and no library allocator.  Its
// working memory is one file-scope __device__ array of kNoAllocScratchBytes
// that every GPU which loads libhdb_b200.so keeps until the process exits.
//
// Host code cannot use the array's name as a device address (in host code the
// symbol is a host-side stand-in); the device address is taken with
// cudaGetSymbolAddress on each device, with that device current, by the first
// call that succeeds there.  With lazy module loading (CUDA 12's default) that
// same lookup is what places the array and the sort kernels on the device, so
// it can fail with an out-of-memory error on a device that is already full; a
// failed lookup is not remembered, the next call tries again.  Callers who run
// on a full device make one warm-up call (m = 0 is enough) before it fills.
#include <mutex>

#include "hdb_internal.cuh"

namespace hdb {
namespace {

constexpr int64_t kNoAllocMaxEdges = int64_t(1) << 18;  // 262,144 edges
constexpr int64_t kTile = 2048;                           // radix sort tile
constexpr int64_t kNb = (kNoAllocMaxEdges + kTile - 1) / kTile;
constexpr int64_t kCounts = kNb * 256;
constexpr int64_t kScanSums = (kCounts + kTile - 1) / kTile;

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
// layout: keys | keys_tmp | idx | idx_tmp | edge copy | counts | offs | scan sums | scan offs
constexpr size_t kOffKeys = 0;
constexpr size_t kOffKeysTmp = kOffKeys + align256(kNoAllocMaxEdges * 4);
constexpr size_t kOffIdx = kOffKeysTmp + align256(kNoAllocMaxEdges * 4);
constexpr size_t kOffIdxTmp = kOffIdx + align256(kNoAllocMaxEdges * 4);
constexpr size_t kOffEdges = kOffIdxTmp + align256(kNoAllocMaxEdges * 4);
constexpr size_t kOffCounts = kOffEdges + align256(kNoAllocMaxEdges * sizeof(hdb_mst_edge));
constexpr size_t kOffOffs = kOffCounts + align256(kCounts * 4);
constexpr size_t kOffScanSums = kOffOffs + align256(kCounts * 4);
constexpr size_t kOffScanOffs = kOffScanSums + align256(kScanSums * 4);
constexpr size_t kNoAllocScratchBytes = kOffScanOffs + align256(kScanSums * 4);  // ~7.3 MB

// Shared by every call on a device; holds the last call's contents.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {};  // non-null once a lookup succeeded

// Device address of the scratch array on the current device.  Only a
// successful lookup is kept; a failed one (for instance out of memory while
// the module is placed) is reported and retried on the next call.
unsigned char *scratch_for_current_device() {
  int dev = -1;
  HDB_CUDA(cudaGetDevice(&dev));
  HDB_REQUIRE(dev >= 0 && dev < kMaxDevices, HDB_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_addr[dev] == nullptr) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();  // not sticky: leave no error behind for the caller
      throw_cuda(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
    }
    HDB_REQUIRE(p != nullptr, HDB_ERR_CUDA, "no device address for the scratch array");
    g_scratch_addr[dev] = p;
  }
  return static_cast<unsigned char *>(g_scratch_addr[dev]);
}

__global__ void k_na_keys(const hdb_mst_edge *__restrict__ e, int64_t m, uint32_t *__restrict__ keys,
                          uint32_t *__restrict__ idx, hdb_mst_edge *__restrict__ copy) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
       t += (int64_t)gridDim.x * blockDim.x) {
    hdb_mst_edge x = e[t];
    float w = x.weight == 0.0f ? 0.0f : x.weight;  // -0 and +0 are equal weights
    keys[t] = float_key(w);
    idx[t] = (uint32_t)t;
    copy[t] = x;
  }
}

__global__ void k_na_permute(const hdb_mst_edge *__restrict__ copy, const uint32_t *__restrict__ idx,
                             int64_t m, hdb_mst_edge *__restrict__ out) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
       t += (int64_t)gridDim.x * blockDim.x)
    out[t] = copy[idx[t]];
}

}  // namespace
}  // namespace hdb

using namespace hdb;

extern "C" HDB_API hdb_status hdb_sort_edges_noalloc(hdb_mst_edge *edges, int64_t m, void *stream) {
  return guard([&] {
    HDB_REQUIRE(m >= 0, HDB_ERR_ARG, "hdb_sort_edges_noalloc: negative edge count");
    HDB_REQUIRE(m <= kNoAllocMaxEdges, HDB_ERR_ARG,
                "hdb_sort_edges_noalloc: more than 262144 edges (the static scratch limit); "
                "use hdb_sort_edges");
    // placed and looked up before anything else, so that a call with m = 0
    // serves as the warm-up that places the array
    unsigned char *base = scratch_for_current_device();
    if (m <= 1) return;
    HDB_REQUIRE(edges != nullptr, HDB_ERR_ARG, "hdb_sort_edges_noalloc: NULL edges");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t *keys = reinterpret_cast<uint32_t *>(base + kOffKeys);
    uint32_t *keys_tmp = reinterpret_cast<uint32_t *>(base + kOffKeysTmp);
    uint32_t *idx = reinterpret_cast<uint32_t *>(base + kOffIdx);
    uint32_t *idx_tmp = reinterpret_cast<uint32_t *>(base + kOffIdxTmp);
    hdb_mst_edge *copy = reinterpret_cast<hdb_mst_edge *>(base + kOffEdges);
    uint32_t *counts = reinterpret_cast<uint32_t *>(base + kOffCounts);
    uint32_t *offs = reinterpret_cast<uint32_t *>(base + kOffOffs);
    uint32_t *ssum = reinterpret_cast<uint32_t *>(base + kOffScanSums);
    uint32_t *soff = reinterpret_cast<uint32_t *>(base + kOffScanOffs);
    const int grid = (int)((m + 255) / 256);
    // every scratch word read below is written first in this call (keys, idx
    // and the edge copy here; counts / offsets by the sort passes)
    k_na_keys<<<grid, 256, 0, st>>>(edges, m, keys, idx, copy);
    HDB_CHECK_LAUNCH();
    radix_sort_u32_buffers(st, keys, idx, keys_tmp, idx_tmp, counts, offs, ssum, soff, m, 0, 32);
    k_na_permute<<<grid, 256, 0, st>>>(copy, idx, m, edges);
    HDB_CHECK_LAUNCH();
    HDB_CUDA(cudaStreamSynchronize(st));
  });
}
