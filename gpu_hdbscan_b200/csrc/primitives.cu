// Device-wide primitives used by every stage: exclusive scans and a stable
// LSD radix sort.  Both are plain HBM-streaming kernels (tiles of 2048
// elements per 256-thread block); no library code.
#include "hdb_internal.cuh"

namespace hdb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
template <typename T>
__device__ T block_exclusive_scan(T v, T *total, T *warp_sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (int)(blockDim.x >> 5)) warp_sums[lane] = w;
  }
  __syncthreads();
  T warp_prefix = warp > 0 ? warp_sums[warp - 1] : T(0);
  *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

template <typename In, typename Out>
__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(const In *__restrict__ in,
                                                                Out *__restrict__ sums,
                                                                int64_t n) {
  __shared__ Out warp_sums[32];
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  Out s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    int64_t idx = base + (int64_t)i * kScanThreads + threadIdx.x;
    if (idx < n) s += (Out)in[idx];
  }
  Out total;
  block_exclusive_scan<Out>(s, &total, warp_sums);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename In, typename Out>
__global__ void __launch_bounds__(kScanThreads) scan_tile_apply(const In *__restrict__ in,
                                                                 Out *__restrict__ out,
                                                                 const Out *__restrict__ offsets,
                                                                 int64_t n, Out *total_out) {
  __shared__ Out tile[kScanTile];
  __shared__ Out warp_sums[32];
  int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    int idx = i * kScanThreads + threadIdx.x;
    int64_t g = base + idx;
    tile[idx] = g < n ? (Out)in[g] : Out(0);
  }
  __syncthreads();
  Out local[kScanItems];
  Out s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    local[i] = tile[threadIdx.x * kScanItems + i];
    s += local[i];
  }
  Out total;
  Out pre = block_exclusive_scan<Out>(s, &total, warp_sums);
  Out off = offsets ? offsets[blockIdx.x] : Out(0);
  Out run = off + pre;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    tile[threadIdx.x * kScanItems + i] = run;
    run += local[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    int idx = i * kScanThreads + threadIdx.x;
    int64_t g = base + idx;
    if (g < n) out[g] = tile[idx];
  }
  if (total_out && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total_out = off + total;
}

template <typename In, typename Out>
void scan_impl(Context *ctx, const In *in, Out *out, int64_t n, Out *total) {
  if (n <= 0) {
    if (total) HDB_CUDA(cudaMemsetAsync(total, 0, sizeof(Out), ctx->stream));
    return;
  }
  int64_t nb = ceil_div(n, kScanTile);
  if (nb == 1) {
    scan_tile_apply<In, Out><<<1, kScanThreads, 0, ctx->stream>>>(in, out, nullptr, n, total); ctx->launches++;
    HDB_CHECK_LAUNCH();
    return;
  }
  Buf<Out> sums(ctx, nb), offs(ctx, nb);
  scan_tile_sums<In, Out><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(in, sums, n); ctx->launches++;
  HDB_CHECK_LAUNCH();
  scan_impl<Out, Out>(ctx, sums, offs, nb, (Out *)nullptr);
  scan_tile_apply<In, Out><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(in, out, offs, n,
                                                                            total); ctx->launches++;
  HDB_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort, 8-bit digits, tiles of 2048 keys.
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kSortWarps = kSortThreads / 32;

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_hist(const K *__restrict__ keys,
                                                            uint32_t *__restrict__ counts,
                                                            int64_t n, int shift,
                                                            uint32_t nblocks) {
  __shared__ uint32_t hist[256];
  hist[threadIdx.x] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll
  for (int i = 0; i < kSortItems; i++) {
    int64_t idx = base + (int64_t)i * kSortThreads + threadIdx.x;
    if (idx < n) atomicAdd(&hist[(uint32_t)(keys[idx] >> shift) & 0xffu], 1u);
  }
  __syncthreads();
  counts[(int64_t)threadIdx.x * nblocks + blockIdx.x] = hist[threadIdx.x];
}

// Scatter of one 2048-key tile for one digit.  Keys are ranked per warp
// (match_any), the tile is laid out in digit order in shared memory (stable:
// input order within a digit), and each digit's run is then written by
// consecutive threads to consecutive addresses.
template <typename K, bool kVals>
__global__ void __launch_bounds__(kSortThreads) radix_scatter(
    const K *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, K *__restrict__ keys_out,
    uint32_t *__restrict__ vals_out, const uint32_t *__restrict__ offsets, int64_t n, int shift,
    uint32_t nblocks) {
  __shared__ uint32_t whist[kSortWarps][256];
  __shared__ uint32_t dstart[256];  // first tile position of each digit
  __shared__ uint32_t gofs[256];    // global position of the tile's first key of each digit
  __shared__ uint32_t wsum[kSortWarps];
  __shared__ K tk[kSortTile];
  __shared__ uint32_t tv[kVals ? kSortTile : 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&whist[0][0])[i] = 0;
  __syncthreads();
  const int64_t tile0 = (int64_t)blockIdx.x * kSortTile;
  const int64_t base = tile0 + (int64_t)warp * (32 * kSortItems);
  K k[kSortItems];
  uint32_t v[kSortItems];
  uint32_t local[kSortItems];
  uint32_t dig[kSortItems];
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    int64_t idx = base + j * 32 + lane;
    bool ok = idx < n;
    k[j] = ok ? keys_in[idx] : K(0);
    if (kVals) v[j] = ok ? vals_in[idx] : 0u;
    uint32_t d = ok ? ((uint32_t)(k[j] >> shift) & 0xffu) : (256u + lane);
    dig[j] = d;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t rank = __popc(peers & lanemask_lt());
    int leader = __ffs(peers) - 1;
    uint32_t b = 0;
    if (ok) b = whist[warp][d];
    __syncwarp();
    if (ok && lane == leader) whist[warp][d] = b + __popc(peers);
    __syncwarp();
    local[j] = b + rank;
  }
  __syncthreads();
  {
    // one digit per thread: warp prefixes, then the digit's count in the tile
    const uint32_t d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
      const uint32_t c = whist[w][d];
      whist[w][d] = run;
      run += c;
    }
    // exclusive scan of the 256 digit counts over the block
    uint32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    uint32_t wpre = 0;
    for (int w = 0; w < warp; w++) wpre += wsum[w];
    dstart[d] = wpre + x - run;
    gofs[d] = offsets[(int64_t)d * nblocks + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    if (dig[j] < 256u) {
      const uint32_t pos = dstart[dig[j]] + whist[warp][dig[j]] + local[j];
      tk[pos] = k[j];
      if (kVals) tv[pos] = v[j];
    }
  }
  __syncthreads();
  const int64_t valid = n - tile0 < kSortTile ? n - tile0 : kSortTile;
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    const int i = j * kSortThreads + threadIdx.x;
    if (i < valid) {
      const K key = tk[i];
      const uint32_t d = (uint32_t)(key >> shift) & 0xffu;
      const uint32_t pos = gofs[d] + (uint32_t)i - dstart[d];
      keys_out[pos] = key;
      if (kVals) vals_out[pos] = tv[i];
    }
  }
}

template <typename K>
void radix_sort_impl(Context *ctx, K *keys, uint32_t *vals, int64_t n, int begin_bit,
                     int end_bit) {
  if (n <= 1 || end_bit <= begin_bit) return;
  HDB_REQUIRE(n < (int64_t(1) << 32), HDB_ERR_ARG, "radix sort: more than 2^32 elements");
  uint32_t nb = (uint32_t)ceil_div(n, kSortTile);
  Buf<K> ktmp(ctx, n);
  Buf<uint32_t> vtmp;
  if (vals) vtmp = Buf<uint32_t>(ctx, n);
  Buf<uint32_t> counts(ctx, (size_t)nb * 256), offs(ctx, (size_t)nb * 256);
  K *kin = keys, *kout = ktmp;
  uint32_t *vin = vals, *vout = vals ? vtmp.get() : nullptr;
  int passes = 0;
  for (int shift = begin_bit; shift < end_bit; shift += 8, passes++) {
    radix_hist<K><<<nb, kSortThreads, 0, ctx->stream>>>(kin, counts, n, shift, nb); ctx->launches++;
    HDB_CHECK_LAUNCH();
    scan_exclusive_u32_u32(ctx, counts, offs, (int64_t)nb * 256, nullptr);
    if (vals)
      radix_scatter<K, true><<<nb, kSortThreads, 0, ctx->stream>>>(kin, vin, kout, vout, offs, n,
                                                                   shift, nb);
    else
      radix_scatter<K, false><<<nb, kSortThreads, 0, ctx->stream>>>(kin, nullptr, kout, nullptr,
                                                                    offs, n, shift, nb);
    ctx->launches++;
    HDB_CHECK_LAUNCH();
    K *t = kin; kin = kout; kout = t;
    uint32_t *tv = vin; vin = vout; vout = tv;
  }
  if (passes & 1) {
    HDB_CUDA(cudaMemcpyAsync(keys, kin, n * sizeof(K), cudaMemcpyDeviceToDevice, ctx->stream));
    if (vals)
      HDB_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                               ctx->stream));
  }
}

}  // namespace

void scan_exclusive_i32_i64(Context *ctx, const int32_t *in, int64_t *out, int64_t n,
                            int64_t *total) {
  scan_impl<int32_t, int64_t>(ctx, in, out, n, total);
}
void scan_exclusive_i32_i32(Context *ctx, const int32_t *in, int32_t *out, int64_t n,
                            int32_t *total) {
  scan_impl<int32_t, int32_t>(ctx, in, out, n, total);
}
void scan_exclusive_u32_u32(Context *ctx, const uint32_t *in, uint32_t *out, int64_t n,
                            uint32_t *total) {
  scan_impl<uint32_t, uint32_t>(ctx, in, out, n, total);
}
void radix_sort_u32(Context *ctx, uint32_t *keys, uint32_t *values, int64_t n, int begin_bit,
                    int end_bit) {
  radix_sort_impl<uint32_t>(ctx, keys, values, n, begin_bit, end_bit);
}
void radix_sort_u64(Context *ctx, uint64_t *keys, uint32_t *values, int64_t n, int begin_bit,
                    int end_bit) {
  radix_sort_impl<uint64_t>(ctx, keys, values, n, begin_bit, end_bit);
}

// Stable LSD radix sort of u32 keys with u32 values in caller-provided
// buffers (nothing is allocated): ktmp/vtmp hold n elements each, counts and
// offs hold ceil(n / 2048) * 256 entries, scan_sums and scan_offs hold
// ceil(counts / 2048) entries, and that count must itself fit one scan tile.
// The result ends in keys/vals.  Used by the allocation-free entry point.
void radix_sort_u32_buffers(cudaStream_t st, uint32_t *keys, uint32_t *vals, uint32_t *ktmp,
                            uint32_t *vtmp, uint32_t *counts, uint32_t *offs, uint32_t *scan_sums,
                            uint32_t *scan_offs, int64_t n, int begin_bit, int end_bit) {
  if (n <= 1 || end_bit <= begin_bit) return;
  const uint32_t nb = (uint32_t)ceil_div(n, kSortTile);
  const int64_t nc = (int64_t)nb * 256;
  const int64_t ns = ceil_div(nc, kScanTile);
  HDB_REQUIRE(ns <= kScanTile, HDB_ERR_ARG, "radix sort buffers: too many elements");
  uint32_t *kin = keys, *kout = ktmp, *vin = vals, *vout = vtmp;
  int passes = 0;
  for (int shift = begin_bit; shift < end_bit; shift += 8, passes++) {
    radix_hist<uint32_t><<<nb, kSortThreads, 0, st>>>(kin, counts, n, shift, nb);
    HDB_CHECK_LAUNCH();
    if (ns == 1) {
      scan_tile_apply<uint32_t, uint32_t><<<1, kScanThreads, 0, st>>>(counts, offs, nullptr, nc,
                                                                      nullptr);
    } else {
      scan_tile_sums<uint32_t, uint32_t><<<(unsigned)ns, kScanThreads, 0, st>>>(counts, scan_sums,
                                                                                nc);
      scan_tile_apply<uint32_t, uint32_t><<<1, kScanThreads, 0, st>>>(scan_sums, scan_offs, nullptr,
                                                                      ns, nullptr);
      scan_tile_apply<uint32_t, uint32_t><<<(unsigned)ns, kScanThreads, 0, st>>>(counts, offs,
                                                                                 scan_offs, nc,
                                                                                 nullptr);
    }
    HDB_CHECK_LAUNCH();
    radix_scatter<uint32_t, true><<<nb, kSortThreads, 0, st>>>(kin, vin, kout, vout, offs, n,
                                                               shift, nb);
    HDB_CHECK_LAUNCH();
    uint32_t *t = kin; kin = kout; kout = t;
    t = vin; vin = vout; vout = t;
  }
  if (passes & 1) {
    HDB_CUDA(cudaMemcpyAsync(keys, kin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    HDB_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  }
}

}  // namespace hdb
