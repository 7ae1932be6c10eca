// Context management, error reporting and stream-ordered scratch memory.
#include <cstdio>
#include <cstring>
#include <iterator>

#include "hdb_internal.cuh"

namespace hdb {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

void throw_cuda(cudaError_t e, const char *what, const char *file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error %d (%s) at %s:%d: %s", (int)e, cudaGetErrorString(e),
           file, line, what);
  hdb_status s = (e == cudaErrorMemoryAllocation) ? HDB_ERR_ALLOC : HDB_ERR_CUDA;
  throw Error(s, buf);
}

Scratch::Scratch(Context *ctx, size_t bytes) { reset(ctx, bytes); }

void Scratch::reset(Context *ctx, size_t bytes) {
  if (ptr_) ctx_->cache_give(ptr_, cls_);
  ptr_ = nullptr;
  ctx_ = ctx;
  bytes_ = bytes;
  ptr_ = ctx->cache_take(bytes == 0 ? 16 : bytes, &cls_);
}

Scratch &Scratch::operator=(Scratch &&o) noexcept {
  if (this != &o) {
    if (ptr_) ctx_->cache_give(ptr_, cls_);
    ctx_ = o.ctx_;
    ptr_ = o.ptr_;
    bytes_ = o.bytes_;
    cls_ = o.cls_;
    o.ptr_ = nullptr;
    o.bytes_ = 0;
  }
  return *this;
}

Scratch::~Scratch() {
  if (ptr_) ctx_->cache_give(ptr_, cls_);
}

static size_t size_class(size_t bytes) {
  size_t p = 512;
  while (p < bytes && p < (size_t(1) << 20)) p <<= 1;
  if (bytes <= p) return p;
  size_t top = size_t(1) << 20;
  while (top * 2 <= bytes) top <<= 1;  // largest power of two <= bytes
  const size_t step = top / 4;
  return (bytes + step - 1) / step * step;
}

void *Context::cache_take(size_t bytes, size_t *cls) {
  const size_t c = size_class(bytes);
  // the smallest idle block of this class or up to half again as large: a
  // call whose sizes differ a little from the last one's reuses its blocks
  // instead of asking the driver for new ones
  auto it = cache_free.lower_bound(c);
  if (it != cache_free.end() && it->first <= c + c / 2) {
    *cls = it->first;
    void *p = it->second;
    cache_free.erase(it);
    return p;
  }
  *cls = c;
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, c);
  if (e == cudaErrorMemoryAllocation && !cache_free.empty()) {
    // give idle blocks back, largest first, until the request fits (releasing
    // all of them would make the next caller allocate them all again)
    cudaGetLastError();
    cudaStreamSynchronize(stream);  // queued work may still use a free block
    while (e == cudaErrorMemoryAllocation && !cache_free.empty()) {
      auto last = std::prev(cache_free.end());
      cudaFree(last->second);
      cache_bytes -= last->first;
      cache_free.erase(last);
      cudaGetLastError();
      e = cudaMalloc(&p, c);
    }
  }
  HDB_CUDA(e);
  cache_bytes += c;
  return p;
}

void Context::cache_give(void *p, size_t cls) { cache_free.emplace(cls, p); }

void Context::cache_release() {
  cudaStreamSynchronize(stream);  // queued work may still use a free block
  for (auto &b : cache_free) {
    cudaFree(b.second);
    cache_bytes -= b.first;
  }
  cache_free.clear();
}

void Context::sync() { HDB_CUDA(cudaStreamSynchronize(stream)); }

uint32_t Context::take_dev_err() {
  // its own slot: callers keep other values staged at the start of `pinned`
  uint32_t *h = reinterpret_cast<uint32_t *>(static_cast<char *>(pinned) + kPinnedErrOffset);
  HDB_CUDA(cudaMemcpyAsync(h, dev_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
  HDB_CUDA(cudaMemsetAsync(dev_err, 0, sizeof(uint32_t), stream));
  sync();
  return h[0];
}

void ensure_capacity(Context *ctx, void **ptr, size_t *cap, size_t bytes) {
  if (bytes <= *cap && *ptr) return;
  if (*ptr) {
    HDB_CUDA(cudaStreamSynchronize(ctx->stream));
    HDB_CUDA(cudaFree(*ptr));
    *ptr = nullptr;
    *cap = 0;
  }
  // 25 % headroom: sizes that follow the kNN graph (edge counts) vary a little
  // from run to run, and a re-allocation of a multi-GB buffer costs far more
  // than the unused tail
  size_t want = bytes < 256 ? 256 : bytes + bytes / 4;
  HDB_CUDA(cudaMalloc(ptr, want));
  *cap = want;
}

}  // namespace hdb

using namespace hdb;

extern "C" {

HDB_API const char *hdb_version(void) { return "hdb_b200 0.1.0 (sm_100a)"; }

HDB_API const char *hdb_last_error(void) { return g_last_error.c_str(); }

HDB_API hdb_status hdb_create(hdb_ctx **out, int32_t device) {
  return guard([&] {
    HDB_REQUIRE(out != nullptr, HDB_ERR_ARG, "hdb_create: out is NULL");
    int count = 0;
    HDB_CUDA(cudaGetDeviceCount(&count));
    HDB_REQUIRE(device >= 0 && device < count, HDB_ERR_ARG, "hdb_create: no such device");
    HDB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    HDB_CUDA(cudaGetDeviceProperties(&prop, device));
    HDB_REQUIRE(prop.major == 10 && prop.minor == 0, HDB_ERR_ARG,
                "hdb_create: libhdb_b200 is built for sm_100a (B200) only");
    hdb_ctx *h = new hdb_ctx();
    Context &c = h->c;
    c.device = device;
    c.num_sms = prop.multiProcessorCount;
    c.l2_bytes = prop.l2CacheSize;
    try {
      HDB_CUDA(cudaStreamCreateWithFlags(&c.own_stream, cudaStreamNonBlocking));
      c.stream = c.own_stream;
      HDB_CUDA(cudaMalloc(&c.dev_err, 4 * sizeof(uint32_t)));
      HDB_CUDA(cudaMemset(c.dev_err, 0, 4 * sizeof(uint32_t)));
      HDB_CUDA(cudaMallocHost(&c.pinned, kPinnedBytes));
      for (auto &e : c.ev) HDB_CUDA(cudaEventCreate(&e));
    } catch (...) {
      hdb_destroy(h);
      throw;
    }
    *out = h;
  });
}

HDB_API hdb_status hdb_destroy(hdb_ctx *h) {
  if (!h) return HDB_OK;
  return guard([&] {
    Context &c = h->c;
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    cudaFree(c.g_nindex);
    cudaFree(c.g_nlist);
    cudaFree(c.g_eweight);
    cudaFree(c.g_antihubs);
    cudaFree(c.sg_nindex);
    cudaFree(c.sg_nlist);
    cudaFree(c.sg_eweight);
    cudaFree(c.dev_err);
    c.cache_release();
    if (c.pinned) cudaFreeHost(c.pinned);
    for (auto &e : c.ev)
      if (e) cudaEventDestroy(e);
    if (c.own_stream) cudaStreamDestroy(c.own_stream);
    delete h;
  });
}

HDB_API hdb_status hdb_set_stream(hdb_ctx *h, void *stream) {
  return guard([&] {
    HDB_REQUIRE(h != nullptr, HDB_ERR_ARG, "hdb_set_stream: NULL context");
    // cached scratch blocks were last used in the old stream's order
    if (h->c.stream) HDB_CUDA(cudaStreamSynchronize(h->c.stream));
    h->c.stream = stream ? static_cast<cudaStream_t>(stream) : h->c.own_stream;
  });
}

HDB_API hdb_status hdb_set_join_tiles(hdb_ctx *h, int32_t tiles) {
  return guard([&] {
    HDB_REQUIRE(h != nullptr, HDB_ERR_ARG, "hdb_set_join_tiles: NULL context");
    HDB_REQUIRE(tiles >= 0 && tiles <= 2, HDB_ERR_ARG, "hdb_set_join_tiles: tiles must be 0, 1 or 2");
    h->c.join_tiles = tiles;
  });
}

}  // extern "C"
