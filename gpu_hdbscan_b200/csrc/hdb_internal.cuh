// Internal declarations shared by the libhdb_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <map>
#include <stdexcept>
#include <string>

#include "hdb/hdb.h"

namespace hdb {

// ---------------------------------------------------------------------------
// Errors: internal code throws hdb::Error; every extern "C" entry point turns
// it into an hdb_status plus the thread-local message of hdb_last_error().
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
  hdb_status status;
  Error(hdb_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string &msg);

[[noreturn]] void throw_cuda(cudaError_t e, const char *what, const char *file, int line);

#define HDB_CUDA(call)                                                         \
  do {                                                                         \
    cudaError_t e__ = (call);                                                  \
    if (e__ != cudaSuccess) ::hdb::throw_cuda(e__, #call, __FILE__, __LINE__); \
  } while (0)

#define HDB_CHECK_LAUNCH() HDB_CUDA(cudaGetLastError())

#define HDB_REQUIRE(cond, status, msg)                     \
  do {                                                     \
    if (!(cond)) throw ::hdb::Error((status), (msg));      \
  } while (0)

template <typename F>
hdb_status guard(F &&f) {
  try {
    f();
    return HDB_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return HDB_ERR_ALLOC;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return HDB_ERR_INTERNAL;
  }
}

// Device-side error word bits (ctx->dev_err[0]); kernels atomicOr into it.
enum : uint32_t {
  DEVERR_ID_RANGE = 1u << 0,   // a kNN id outside [0, n)
  DEVERR_SELF_ID = 1u << 1,    // a row lists itself
  DEVERR_DUP_ID = 1u << 2,     // an id repeated within one row
  DEVERR_TIMEOUT = 1u << 3,    // a bounded wait gave up
  DEVERR_OVERFLOW = 1u << 4,   // an internal capacity was exceeded
};

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
struct Context;

// Scratch buffer from the context's block cache (Context::cache_take), given
// back to it when it goes out of scope.
class Scratch {
 public:
  Scratch() = default;
  Scratch(Context *ctx, size_t bytes);
  ~Scratch();
  Scratch(const Scratch &) = delete;
  Scratch &operator=(const Scratch &) = delete;
  Scratch(Scratch &&o) noexcept { *this = std::move(o); }
  Scratch &operator=(Scratch &&o) noexcept;
  void *get() const { return ptr_; }
  template <typename T>
  T *as() const { return static_cast<T *>(ptr_); }
  size_t bytes() const { return bytes_; }
  void reset(Context *ctx, size_t bytes);

 private:
  Context *ctx_ = nullptr;
  void *ptr_ = nullptr;
  size_t bytes_ = 0;
  size_t cls_ = 0;  // size class of the block
};

template <typename T>
struct Buf {
  Scratch s;
  Buf() = default;
  Buf(Context *ctx, size_t count) : s(ctx, count * sizeof(T) + 16) {}
  T *get() const { return s.as<T>(); }
  operator T *() const { return s.as<T>(); }
};

// Pinned host staging area: bytes [0, kPinnedErrOffset) are free for callers,
// the device error word is read back at kPinnedErrOffset.
constexpr size_t kPinnedBytes = 4096;
constexpr size_t kPinnedErrOffset = 3072;

struct Context {
  int device = 0;
  int num_sms = 148;
  int64_t l2_bytes = 126 << 20;
  // FP32 local join tile slots per lane: 0 = tuned per shape, 1 or 2 forced
  // (hdb_set_join_tiles)
  int join_tiles = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t *dev_err = nullptr;   // [4] device error words
  void *pinned = nullptr;        // small pinned host staging area
  // Persistent outputs of hdb_enhanced_knng (owned by the context).
  int64_t *g_nindex = nullptr;
  int32_t *g_nlist = nullptr;
  float *g_eweight = nullptr;
  int32_t *g_antihubs = nullptr;
  size_t g_nindex_cap = 0, g_nlist_cap = 0, g_eweight_cap = 0, g_antihubs_cap = 0;
  // Persistent outputs of hdb_core_sg.
  int64_t *sg_nindex = nullptr;
  int32_t *sg_nlist = nullptr;
  float *sg_eweight = nullptr;
  size_t sg_nindex_cap = 0, sg_nlist_cap = 0, sg_eweight_cap = 0;
  cudaEvent_t ev[8] = {};
  // Kernel launches issued by this context (all stages count them).
  int64_t launches = 0;
  // Live timing of the NN-Descent local join (hdb_run_stats.join_*).
  cudaEvent_t join_ev[2] = {};
  double join_ms = 0.0;
  int64_t join_launches = 0;

  // Scratch block cache: blocks are rounded up to a size class (four per
  // octave above 1 MB, powers of two below) and kept on a free list when
  // their Scratch goes away, so repeated calls reuse them instead of asking
  // the driver for multi-GB blocks every time.  All of a context's work is in
  // order on its stream, and every entry point ends with a stream sync, so a
  // block given back is free for the next taker.  Released by hdb_destroy,
  // or when the driver runs out of memory.
  std::multimap<size_t, void *> cache_free;
  size_t cache_bytes = 0;  // all blocks held (free or in use)
  void *cache_take(size_t bytes, size_t *cls);
  void cache_give(void *p, size_t cls);
  void cache_release();

  void sync();
  // Reads and clears the device error word.
  uint32_t take_dev_err();
};

void ensure_capacity(Context *ctx, void **ptr, size_t *cap, size_t bytes);

// ---------------------------------------------------------------------------
// Primitives (primitives.cu)
// ---------------------------------------------------------------------------
// Exclusive prefix sum; `total` (device, optional) receives the sum.
void scan_exclusive_i32_i64(Context *ctx, const int32_t *in, int64_t *out, int64_t n,
                            int64_t *total);
void scan_exclusive_i32_i32(Context *ctx, const int32_t *in, int32_t *out, int64_t n,
                            int32_t *total);
void scan_exclusive_u32_u32(Context *ctx, const uint32_t *in, uint32_t *out, int64_t n,
                            uint32_t *total);
// Stable LSD radix sort over bits [begin_bit, end_bit) of the keys; values
// (optional) are permuted along.  Results end in keys/values; tmp buffers are
// internal.  n < 2^32.
void radix_sort_u32(Context *ctx, uint32_t *keys, uint32_t *values, int64_t n, int begin_bit,
                    int end_bit);
void radix_sort_u64(Context *ctx, uint64_t *keys, uint32_t *values, int64_t n, int begin_bit,
                    int end_bit);
// The same with u64 values and digits of up to 9 bits (fewer passes for key
// ranges just above a multiple of 8 bits, e.g. 25-bit row ids: 3 passes).
void radix_sort_u32_u64(Context *ctx, uint32_t *keys, uint64_t *values, int64_t n, int begin_bit,
                        int end_bit);

void radix_sort_u32_buffers(cudaStream_t st, uint32_t *keys, uint32_t *vals, uint32_t *ktmp,
                            uint32_t *vtmp, uint32_t *counts, uint32_t *offs, uint32_t *scan_sums,
                            uint32_t *scan_offs, int64_t n, int begin_bit, int end_bit);

// Fixed-point grid sizing: a multiple of the SM count, capped by the work.
inline int grid_for(const Context *ctx, int64_t work, int per_block, int blocks_per_sm = 8) {
  int64_t need = (work + per_block - 1) / per_block;
  int64_t cap = (int64_t)ctx->num_sms * blocks_per_sm;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Independent clustering instances laid out back to back in one set of
// arrays (hdb_run_batched): points [off[t], off[t+1]) belong to instance t.
// count == 0 is the single-instance case (off unused).  Instance t holds at
// least two points; its MST edges, and so its linkage-tree ranks, occupy
// [off[t] - t, off[t+1] - t - 1) of the batch's sorted MST.
struct Segments {
  const int64_t *off = nullptr;       // device [count + 1]
  const int64_t *host_off = nullptr;  // the same offsets in host memory
  int32_t count = 0;
#ifdef __CUDACC__
  // Instance of point p: the largest t with off[t] <= p.
  __device__ __forceinline__ int32_t of_point(int64_t p) const {
    int32_t lo = 0, hi = count - 1;
    while (lo < hi) {
      const int32_t mid = (lo + hi + 1) >> 1;
      if (__ldg(off + mid) <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
  }
  // Instance of MST / linkage rank r: the largest t with off[t] - t <= r.
  __device__ __forceinline__ int32_t of_rank(int64_t r) const {
    int32_t lo = 0, hi = count - 1;
    while (lo < hi) {
      const int32_t mid = (lo + hi + 1) >> 1;
      if (__ldg(off + mid) - mid <= r) lo = mid; else hi = mid - 1;
    }
    return lo;
  }
#endif
};

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
#ifdef __CUDACC__
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Order-preserving map of a float to u32 (total order; -0 < +0).
__device__ __forceinline__ uint32_t float_key(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ __forceinline__ float key_float(uint32_t k) {
  uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}
#endif

}  // namespace hdb

struct hdb_ctx {
  hdb::Context c;
};
