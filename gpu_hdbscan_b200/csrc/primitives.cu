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
// Stable LSD radix sort.  One tile of kSortThreads * kItems keys per block;
// each pass sorts by (key >> shift) & mask, digits of up to 8 bits (256 bins)
// or 9 bits (512 bins).  The per-tile digit counts are laid out either
// digit-major ([digit][tile]: one flat exclusive scan gives every tile its
// output positions) or tile-major ([tile][digit]: every block reads and
// writes its own counts contiguously, and a column scan over chunks of
// tiles gives the positions).  The sorts of this file use tile-major counts
// and tiles of 4096 keys; the caller-buffer variant keeps the digit-major
// layout and 2048-key tiles its buffer sizes are stated in.
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;          // tile-major sorts: 4096-key tiles
constexpr int kSortItemsFlat = 8;       // digit-major (caller-buffer) sort: 2048-key tiles
constexpr int kColRows = 512;           // tiles per chunk of the column scan

// Dynamic shared memory of one scatter block: the tile's keys and values in
// digit order, the per-warp digit counts, each digit's first tile position
// and first output position, and the warp totals of the digit scan.
template <typename K, typename V, bool kVals, int kBins, int kItems>
struct SortSmem {
  static constexpr int kTile = kSortThreads * kItems;
  static constexpr size_t kValsAt = sizeof(K) * kTile;
  static constexpr size_t kHistAt = kValsAt + (kVals ? sizeof(V) * kTile : 0);
  static constexpr size_t kStartAt = kHistAt + sizeof(uint32_t) * kSortWarps * kBins;
  static constexpr size_t kGofsAt = kStartAt + sizeof(uint32_t) * kBins;
  static constexpr size_t kWsumAt = kGofsAt + sizeof(uint32_t) * kBins;
  static constexpr size_t kBytes = kWsumAt + sizeof(uint32_t) * kSortWarps;
};

template <bool kTileMajor>
__device__ __forceinline__ int64_t count_at(int d, uint32_t tile, uint32_t nblocks, int bins) {
  return kTileMajor ? (int64_t)tile * bins + d : (int64_t)d * nblocks + tile;
}

template <typename K, int kBins, int kItems, bool kTileMajor>
__global__ void __launch_bounds__(kSortThreads) radix_hist(const K *__restrict__ keys,
                                                            uint32_t *__restrict__ counts,
                                                            int64_t n, int shift, uint32_t mask,
                                                            uint32_t nblocks) {
  constexpr int kTile = kSortThreads * kItems;
  __shared__ uint32_t hist[kBins];
  for (int i = threadIdx.x; i < kBins; i += kSortThreads) hist[i] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kTile;
  K k[kItems];
#pragma unroll
  for (int i = 0; i < kItems; i++) {
    const int64_t idx = base + (int64_t)i * kSortThreads + threadIdx.x;
    k[i] = idx < n ? keys[idx] : K(0);
  }
#pragma unroll
  for (int i = 0; i < kItems; i++) {
    const int64_t idx = base + (int64_t)i * kSortThreads + threadIdx.x;
    if (idx < n) atomicAdd(&hist[(uint32_t)(k[i] >> shift) & mask], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kBins; i += kSortThreads)
    counts[count_at<kTileMajor>(i, blockIdx.x, nblocks, kBins)] = hist[i];
}

// Scatter of one tile for one digit.  Keys are ranked per warp (match_any),
// the tile is laid out in digit order in shared memory (stable: input order
// within a digit), and each digit's run is then written by consecutive
// threads to consecutive addresses.  Values of type V (u32 or u64) move with
// their keys when kVals.
template <typename K, typename V, bool kVals, int kBins, int kItems, bool kTileMajor>
__global__ void __launch_bounds__(kSortThreads, 3) radix_scatter(
    const K *__restrict__ keys_in, const V *__restrict__ vals_in, K *__restrict__ keys_out,
    V *__restrict__ vals_out, const uint32_t *__restrict__ offsets, int64_t n, int shift,
    uint32_t mask, uint32_t nblocks) {
  using L = SortSmem<K, V, kVals, kBins, kItems>;
  constexpr int kTile = L::kTile;
  constexpr int kPer = kBins / kSortThreads;  // digits owned by each thread in the scan
  extern __shared__ __align__(16) unsigned char sort_smem[];
  K *tk = reinterpret_cast<K *>(sort_smem);
  V *tv = reinterpret_cast<V *>(sort_smem + L::kValsAt);
  uint32_t(*whist)[kBins] = reinterpret_cast<uint32_t(*)[kBins]>(sort_smem + L::kHistAt);
  uint32_t *dstart = reinterpret_cast<uint32_t *>(sort_smem + L::kStartAt);
  uint32_t *gofs = reinterpret_cast<uint32_t *>(sort_smem + L::kGofsAt);
  uint32_t *wsum = reinterpret_cast<uint32_t *>(sort_smem + L::kWsumAt);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * kBins; i += kSortThreads) (&whist[0][0])[i] = 0;
  __syncthreads();
  const int64_t tile0 = (int64_t)blockIdx.x * kTile;
  const int64_t base = tile0 + (int64_t)warp * (32 * kItems);
  K k[kItems];
  V v[kItems];
  uint32_t dl[kItems];  // digit (low 16 bits) | rank among the warp's keys of that digit << 16
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const int64_t idx = base + j * 32 + lane;
    k[j] = idx < n ? keys_in[idx] : K(0);
    if (kVals) v[j] = idx < n ? vals_in[idx] : V(0);
  }
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const bool ok = base + j * 32 + lane < n;
    // past the end: a digit of its own per lane, outside [0, kBins)
    const uint32_t d = ok ? ((uint32_t)(k[j] >> shift) & mask) : ((uint32_t)kBins + lane);
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & lanemask_lt());
    const int leader = __ffs(peers) - 1;
    uint32_t b = 0;
    if (ok) b = whist[warp][d];
    __syncwarp();
    if (ok && lane == leader) whist[warp][d] = b + __popc(peers);
    __syncwarp();
    dl[j] = d | ((b + rank) << 16);
  }
  __syncthreads();
  {
    // kPer consecutive digits per thread: warp prefixes, then the digits'
    // counts in the tile, then an exclusive scan of the thread totals
    uint32_t run[kPer];
    uint32_t tsum = 0;
#pragma unroll
    for (int r = 0; r < kPer; r++) {
      const int d = threadIdx.x * kPer + r;
      uint32_t acc = 0;
#pragma unroll
      for (int w = 0; w < kSortWarps; w++) {
        const uint32_t c = whist[w][d];
        whist[w][d] = acc;
        acc += c;
      }
      run[r] = acc;
      tsum += acc;
    }
    uint32_t x = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    uint32_t excl = x - tsum;
    for (int w = 0; w < warp; w++) excl += wsum[w];
#pragma unroll
    for (int r = 0; r < kPer; r++) {
      const int d = threadIdx.x * kPer + r;
      dstart[d] = excl;
      excl += run[r];
      gofs[d] = offsets[count_at<kTileMajor>(d, blockIdx.x, nblocks, kBins)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const uint32_t d = dl[j] & 0xffffu;
    if (d < (uint32_t)kBins) {
      const uint32_t pos = dstart[d] + whist[warp][d] + (dl[j] >> 16);
      tk[pos] = k[j];
      if (kVals) tv[pos] = v[j];
    }
  }
  __syncthreads();
  const int64_t valid = n - tile0 < kTile ? n - tile0 : kTile;
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const int i = j * kSortThreads + threadIdx.x;
    if (i < valid) {
      const K key = tk[i];
      const uint32_t d = (uint32_t)(key >> shift) & mask;
      const uint32_t pos = gofs[d] + (uint32_t)i - dstart[d];
      keys_out[pos] = key;
      if (kVals) vals_out[pos] = tv[i];
    }
  }
}

// Column scan of tile-major counts [nblocks][kBins], one thread per digit.
// (1) per chunk of kColRows tiles, each digit's count in the chunk;
template <int kBins>
__global__ void __launch_bounds__(kBins) radix_col_sums(const uint32_t *__restrict__ counts,
                                                        uint32_t *__restrict__ csum,
                                                        uint32_t nblocks) {
  const int d = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * kColRows;
  const int64_t r1 = r0 + kColRows < (int64_t)nblocks ? r0 + kColRows : (int64_t)nblocks;
  uint32_t s = 0;
#pragma unroll 8
  for (int64_t r = r0; r < r1; r++) s += counts[r * kBins + d];
  csum[(int64_t)blockIdx.x * kBins + d] = s;
}

// (2) one block: each digit's exclusive prefix over the chunks (in place) and
// its first output position (base: exclusive scan of the digit totals);
template <int kBins>
__global__ void __launch_bounds__(kBins) radix_col_scan(uint32_t *__restrict__ csum,
                                                        uint32_t *__restrict__ base,
                                                        uint32_t nchunks) {
  __shared__ uint32_t warp_sums[32];
  const int d = threadIdx.x;
  uint32_t run = 0;
  for (uint32_t c0 = 0; c0 < nchunks; c0 += 8) {
    uint32_t v[8];
#pragma unroll
    for (int j = 0; j < 8; j++)
      v[j] = c0 + j < nchunks ? csum[(int64_t)(c0 + j) * kBins + d] : 0u;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if (c0 + j < nchunks) csum[(int64_t)(c0 + j) * kBins + d] = run;
      run += v[j];
    }
  }
  uint32_t total;
  base[d] = block_exclusive_scan<uint32_t>(run, &total, warp_sums);
}

// (3) every tile's output position of its first key of each digit.
template <int kBins>
__global__ void __launch_bounds__(kBins) radix_col_apply(const uint32_t *__restrict__ counts,
                                                         const uint32_t *__restrict__ csum,
                                                         const uint32_t *__restrict__ base,
                                                         uint32_t *__restrict__ offs,
                                                         uint32_t nblocks) {
  const int d = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * kColRows;
  const int64_t r1 = r0 + kColRows < (int64_t)nblocks ? r0 + kColRows : (int64_t)nblocks;
  uint32_t run = base[d] + csum[(int64_t)blockIdx.x * kBins + d];
#pragma unroll 8
  for (int64_t r = r0; r < r1; r++) {
    const uint32_t c = counts[r * kBins + d];
    offs[r * kBins + d] = run;
    run += c;
  }
}

template <typename K, typename V, bool kVals, int kBins, int kItems, bool kTileMajor>
void launch_scatter(cudaStream_t st, const K *kin, const V *vin, K *kout, V *vout,
                    const uint32_t *offs, int64_t n, int shift, uint32_t mask, uint32_t nb) {
  using L = SortSmem<K, V, kVals, kBins, kItems>;
  auto *fn = radix_scatter<K, V, kVals, kBins, kItems, kTileMajor>;
  if (L::kBytes > 48 * 1024)
    HDB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::kBytes));
  fn<<<nb, kSortThreads, L::kBytes, st>>>(kin, vin, kout, vout, offs, n, shift, mask, nb);
  HDB_CHECK_LAUNCH();
}

// Digit widths: the fewest passes of at most log2(kBins) bits over
// [begin_bit, end_bit), the bits spread evenly over them (25 bits with 512
// bins: 9 + 8 + 8).
template <typename K, typename V, int kBins>
void radix_sort_impl(Context *ctx, K *keys, V *vals, int64_t n, int begin_bit, int end_bit) {
  if (n <= 1 || end_bit <= begin_bit) return;
  HDB_REQUIRE(n < (int64_t(1) << 32), HDB_ERR_ARG, "radix sort: more than 2^32 elements");
  constexpr int kMaxBits = kBins == 512 ? 9 : 8;
  static_assert(kBins == 256 || kBins == 512, "radix sort: 256 or 512 bins");
  constexpr int kTile = kSortThreads * kSortItems;
  const cudaStream_t st = ctx->stream;
  const uint32_t nb = (uint32_t)ceil_div(n, kTile);
  const uint32_t nchunks = (uint32_t)ceil_div(nb, kColRows);
  Buf<K> ktmp(ctx, n);
  Buf<V> vtmp;
  if (vals) vtmp = Buf<V>(ctx, n);
  Buf<uint32_t> counts(ctx, (size_t)nb * kBins), offs(ctx, (size_t)nb * kBins),
      csum(ctx, (size_t)nchunks * kBins), base(ctx, kBins);
  K *kin = keys, *kout = ktmp;
  V *vin = vals, *vout = vals ? vtmp.get() : nullptr;
  int passes = 0;
  int left = end_bit - begin_bit;
  int npass = (left + kMaxBits - 1) / kMaxBits;
  for (int shift = begin_bit; left > 0; passes++, npass--) {
    const int bits = (left + npass - 1) / npass;
    const uint32_t mask = (1u << bits) - 1u;
    radix_hist<K, kBins, kSortItems, true><<<nb, kSortThreads, 0, st>>>(kin, counts, n, shift,
                                                                       mask, nb);
    HDB_CHECK_LAUNCH();
    radix_col_sums<kBins><<<nchunks, kBins, 0, st>>>(counts, csum, nb);
    HDB_CHECK_LAUNCH();
    radix_col_scan<kBins><<<1, kBins, 0, st>>>(csum, base, nchunks);
    HDB_CHECK_LAUNCH();
    radix_col_apply<kBins><<<nchunks, kBins, 0, st>>>(counts, csum, base, offs, nb);
    HDB_CHECK_LAUNCH();
    if (vals)
      launch_scatter<K, V, true, kBins, kSortItems, true>(st, kin, vin, kout, vout, offs, n, shift,
                                                          mask, nb);
    else
      launch_scatter<K, V, false, kBins, kSortItems, true>(st, kin, nullptr, kout, nullptr, offs,
                                                           n, shift, mask, nb);
    ctx->launches += 5;
    K *t = kin; kin = kout; kout = t;
    V *tv = vin; vin = vout; vout = tv;
    shift += bits;
    left -= bits;
  }
  if (passes & 1) {
    HDB_CUDA(cudaMemcpyAsync(keys, kin, n * sizeof(K), cudaMemcpyDeviceToDevice, st));
    if (vals)
      HDB_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(V), cudaMemcpyDeviceToDevice, st));
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
// 9-bit digits when they save a pass over 8-bit ones (e.g. 25-bit row ids).
static bool nine_bit_digits_help(int bits) { return (bits + 8) / 9 < (bits + 7) / 8; }

void radix_sort_u32(Context *ctx, uint32_t *keys, uint32_t *values, int64_t n, int begin_bit,
                    int end_bit) {
  if (nine_bit_digits_help(end_bit - begin_bit))
    radix_sort_impl<uint32_t, uint32_t, 512>(ctx, keys, values, n, begin_bit, end_bit);
  else
    radix_sort_impl<uint32_t, uint32_t, 256>(ctx, keys, values, n, begin_bit, end_bit);
}
void radix_sort_u64(Context *ctx, uint64_t *keys, uint32_t *values, int64_t n, int begin_bit,
                    int end_bit) {
  if (nine_bit_digits_help(end_bit - begin_bit))
    radix_sort_impl<uint64_t, uint32_t, 512>(ctx, keys, values, n, begin_bit, end_bit);
  else
    radix_sort_impl<uint64_t, uint32_t, 256>(ctx, keys, values, n, begin_bit, end_bit);
}
void radix_sort_u32_u64(Context *ctx, uint32_t *keys, uint64_t *values, int64_t n, int begin_bit,
                        int end_bit) {
  radix_sort_impl<uint32_t, uint64_t, 512>(ctx, keys, values, n, begin_bit, end_bit);
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
  const uint32_t nb = (uint32_t)ceil_div(n, kSortThreads * kSortItemsFlat);
  const int64_t nc = (int64_t)nb * 256;
  const int64_t ns = ceil_div(nc, kScanTile);
  HDB_REQUIRE(ns <= kScanTile, HDB_ERR_ARG, "radix sort buffers: too many elements");
  uint32_t *kin = keys, *kout = ktmp, *vin = vals, *vout = vtmp;
  int passes = 0;
  for (int shift = begin_bit; shift < end_bit; shift += 8, passes++) {
    radix_hist<uint32_t, 256, kSortItemsFlat, false><<<nb, kSortThreads, 0, st>>>(kin, counts, n,
                                                                                 shift, 0xffu, nb);
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
    launch_scatter<uint32_t, uint32_t, true, 256, kSortItemsFlat, false>(st, kin, vin, kout, vout,
                                                                         offs, n, shift, 0xffu, nb);
    uint32_t *t = kin; kin = kout; kout = t;
    t = vin; vin = vout; vout = t;
  }
  if (passes & 1) {
    HDB_CUDA(cudaMemcpyAsync(keys, kin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    HDB_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  }
}

}  // namespace hdb
