// NN-Descent kNN graph (gpuknn::NNDescent, gpuknn/nndescent.cu:2088-2199).
//
// Same algorithm as the reference -- hash-seeded random init, per iteration a
// sample of S new / S old neighbours plus reverse samples, a local join in
// which every new neighbour is offered its closest other new neighbour and
// its closest old neighbour and every old neighbour its closest new one --
// laid out for one B200:
//  * no per-row spin locks (InsertToGlobalGraph, nndescent.cu:969-1028): the
//    join appends candidates to a fixed per-row inbox (one atomicAdd each,
//    pre-filtered against the row's current k-th distance), and the next
//    pass merges each row's inbox in one warp (sort, de-duplicate, merge);
//  * the three sampling kernels, MarkAllToOld and the merge are one kernel
//    (k_sample), so an iteration is two launches;
//  * distances are the reference's sequential FP32 difference sum
//    (nndescent.cu:1086-1093, fmaf per element), so every pair has one exact
//    value wherever it is computed.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "hdb_internal.cuh"
#include "join_tc.cuh"
#include "knn.cuh"
#include "knn_common.cuh"

namespace hdb {

using namespace knn;

namespace {


__host__ __device__ __forceinline__ uint64_t xorshift64star(uint64_t x) {
  // gpuknn/knncuda_tools.cu:126-132
  x += 42;
  x ^= x >> 12;
  x ^= x << 25;
  x ^= x >> 27;
  return x * 0x2545F4914F6CDD1DULL;
}


// Ascending bitonic sort of one u64 per lane across the warp.
__device__ __forceinline__ uint64_t warp_sort32(uint64_t v) {
  const int lane = lane_id();
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      uint64_t o = __shfl_xor_sync(0xffffffffu, v, stride);
      bool up = ((lane & size) == 0);
      bool lower = (lane & stride) == 0;
      uint64_t mn = v < o ? v : o, mx = v < o ? o : v;
      v = (lower == up) ? mn : mx;
    }
  }
  return v;
}

// warp_sort32 with a 32-bit payload that moves with its key (keys distinct
// within the warp, or equal only where the payload does not matter).
__device__ __forceinline__ void warp_sort32_with(uint64_t &v, int32_t &pl) {
  const int lane = lane_id();
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const uint64_t o = __shfl_xor_sync(0xffffffffu, v, stride);
      const int32_t op = __shfl_xor_sync(0xffffffffu, pl, stride);
      const bool up = ((lane & size) == 0);
      const bool lower = (lane & stride) == 0;
      const bool take = (lower == up) ? o < v : v < o;  // the other lane's key is the min / max
      v = take ? o : v;
      pl = take ? op : pl;
    }
  }
}

// ---------------------------------------------------------------------------
// Exact sequential difference sums of one row against up to 32 other rows,
// one per lane.  The 32 rows are staged through shared memory 32 dimensions
// at a time, read as coalesced row segments (lanes on consecutive columns),
// and each lane then walks its own row's staged segment in dimension order:
// the reference's sequential FP32 difference sum (nndescent.cu:1086-1093),
// sum = fmaf(a_j - b_j, a_j - b_j, sum) for j = 0..d-1.
// Two FP32 differences b - a with one packed instruction: b + (-a), per
// component the same rounding as __fsub_rn(b, a) = -__fsub_rn(a, b), so its
// square is the square of the reference's a - b, bit for bit.
__device__ __forceinline__ float2 neg_diff2(float2 b, float2 a) {
  return __fadd2_rn(b, make_float2(-a.x, -a.y));
}

constexpr int kStageCols = 32;
constexpr int kStageLd = kStageCols + 1;                    // conflict-free column walk
constexpr int kRingSlot = kStageCols + 32 * kStageCols;     // 16-byte form: own + 32 rows
constexpr int kStageFloats = 2 * kRingSlot;                 // >= kStageCols + 32 * kStageLd

// 16-byte form for d % 4 == 0 (rows 16-byte aligned): a two-slot ring of
// chunks filled by cp.async, so the next chunk of the 33 rows is in flight
// while this one is summed.  Per chunk, lane i copies piece q = i & 7 of rows
// i >> 3, + 4, ... (eight 16-byte copies per lane) into rows of 32 floats
// whose pieces are permuted by the row (piece q of row r at q ^ (r & 7)), so
// the lanes' walks of their own rows read distinct bank groups.  Same sums as
// below, element by element.
__device__ __forceinline__ float diffsum_staged_v4(const float *__restrict__ X, int d, int64_t row,
                                                   int32_t id, bool active, float *__restrict__ sm) {
  const int lane = lane_id();
  const uint32_t act = __ballot_sync(0xffffffffu, active);
  const int q = lane & 7, rb = lane >> 3;
  int32_t rid[8];
#pragma unroll
  for (int t = 0; t < 8; t++) rid[t] = __shfl_sync(0xffffffffu, id, rb + 4 * t);
  const int nchunks = (d + kStageCols - 1) / kStageCols;
  // chunk c into ring slot c & 1: the own row's segment and the rows' pieces
  auto issue = [&](int c) {
    const int c0 = c * kStageCols;
    const int nq = min(kStageCols, d - c0) >> 2;
    float *own = sm + (c & 1) * kRingSlot;
    float *nb = own + kStageCols;
    if (lane < nq) {
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(own + 4 * lane);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(dst),
                   "l"(X + row * d + c0 + 4 * lane)
                   : "memory");
    }
    if (q < nq) {
#pragma unroll
      for (int t = 0; t < 8; t++) {
        const int r = rb + 4 * t;
        if ((act >> r) & 1u) {
          const uint32_t dst =
              (uint32_t)__cvta_generic_to_shared(nb + r * kStageCols + 4 * (q ^ (r & 7)));
          asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(dst),
                       "l"(X + (int64_t)rid[t] * d + c0 + 4 * q)
                       : "memory");
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  __syncwarp();  // the ring's previous contents are no longer read
  issue(0);
  float s = 0.0f;
  for (int c = 0; c < nchunks; c++) {
    if (c + 1 < nchunks) {
      __syncwarp();  // slot (c + 1) & 1 held chunk c - 1, summed by every lane
      issue(c + 1);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncwarp();  // every lane's copies of chunk c have landed
    if (active) {
      const int nq = min(kStageCols, d - c * kStageCols) >> 2;
      const float *own = sm + (c & 1) * kRingSlot;
      const float *mine = own + kStageCols + lane * kStageCols;
      for (int p = 0; p < nq; p++) {
        const float4 b = *reinterpret_cast<const float4 *>(mine + 4 * (p ^ (lane & 7)));
        const float4 a = *reinterpret_cast<const float4 *>(own + 4 * p);
        const float2 d01 = neg_diff2(make_float2(b.x, b.y), make_float2(a.x, a.y));
        const float2 d23 = neg_diff2(make_float2(b.z, b.w), make_float2(a.z, a.w));
        s = __fmaf_rn(d01.x, d01.x, s);
        s = __fmaf_rn(d01.y, d01.y, s);
        s = __fmaf_rn(d23.x, d23.x, s);
        s = __fmaf_rn(d23.y, d23.y, s);
      }
    }
  }
  __syncwarp();
  return s;
}

__device__ __forceinline__ float diffsum_staged(const float *__restrict__ X, int d, int64_t row,
                                                int32_t id, bool active, float *__restrict__ sm) {
  const int lane = lane_id();
  if ((d & 3) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0)
    return diffsum_staged_v4(X, d, row, id, active, sm);
  float *own = sm;
  float *nb = sm + kStageCols;
  const uint32_t act = __ballot_sync(0xffffffffu, active);
  float s = 0.0f;
  for (int c0 = 0; c0 < d; c0 += kStageCols) {
    const int w = min(kStageCols, d - c0);
    __syncwarp();
    if (lane < w) own[lane] = X[row * d + c0 + lane];
    if (w == kStageCols) {
      // full chunk: row i's segment is one coalesced load (lane = column), and
      // all 32 are issued before any is stored, so they are in flight together
      float t[kStageCols];
#pragma unroll
      for (int i = 0; i < kStageCols; i++) {
        const int32_t rid = __shfl_sync(0xffffffffu, id, i);
        t[i] = ((act >> i) & 1u) ? __ldg(X + (int64_t)rid * d + c0 + lane) : 0.0f;
      }
#pragma unroll
      for (int i = 0; i < kStageCols; i++) nb[i * kStageLd + lane] = t[i];
    } else {
      // ragged chunk: 32 rows x w columns, flattened: element e -> row e / w, column e % w
#pragma unroll 8
      for (int i = 0; i < w; i++) {
        const int e = i * 32 + lane;
        const int r = e / w, c = e - r * w;
        const int32_t rid = __shfl_sync(0xffffffffu, id, r);
        if ((act >> r) & 1u) nb[r * kStageLd + c] = __ldg(X + (int64_t)rid * d + c0 + c);
      }
    }
    __syncwarp();
    if (active) {
      const float *mine = nb + lane * kStageLd;
      for (int j = 0; j < w; j++) {
        float df = __fsub_rn(own[j], mine[j]);
        s = __fmaf_rn(df, df, s);
      }
    }
  }
  return s;
}

// With instances (seg.count > 0) every row draws from its own instance with
// the instance-local position and size, so an instance starts from the graph
// a run on that instance alone starts from.  With a renumbering (order: new
// row -> caller's row, inv: caller's row -> new row; X in the new numbering)
// the ids are drawn for the caller's row from the caller's numbering and then
// mapped, so the lists are exactly the caller-numbered initial graph
// renumbered (instances keep their ranges under the renumbering).
__global__ void __launch_bounds__(256, 3) k_init(const float *__restrict__ X, int64_t n, int d, int k, Segments seg,
                       const uint32_t *__restrict__ order, const int32_t *__restrict__ inv,
                       int32_t *__restrict__ gid, float *__restrict__ gdist,
                       float *__restrict__ worst) {
  extern __shared__ float smem_stage[];
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  float *sm = smem_stage + (threadIdx.x >> 5) * kStageFloats;
  for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < n;
       row += (int64_t)gridDim.x * wpb) {
    int64_t base = 0, cnt = n;
    if (seg.count > 0) {
      const int32_t t = seg.of_point(row);
      base = seg.off[t];
      cnt = seg.off[t + 1] - base;
    }
    const int64_t lrow = (order ? (int64_t)order[row] : row) - base;
    // InitKNNGraphIndexKernel (nndescent.cu:1673-1692): xorshift64star(pos) % n,
    // advanced past the row itself -- and here also past ids already taken:
    // slot t takes the first of its draw, draw + 1, ... (mod n) that is
    // neither the row nor taken by a slot before it.  All slots advance
    // together, each while it equals the row or an earlier slot's current id
    // (one match_any per round); a slot never steps over its final id that
    // way (the ids it steps over are the row or earlier slots' final ids), so
    // the fixed point is that sequential result.  A slot steps at most k
    // times, so k * (k + 1) / 2 rounds bound the loop.
    const int32_t lrow32 = (int32_t)lrow, cnt32 = (int32_t)cnt;
    int32_t label = (int32_t)(xorshift64star((uint64_t)(lrow * k + lane)) % (uint64_t)cnt);
    const uint32_t below = lanemask_lt();
    for (int round = 0; round <= kMaxK * (kMaxK + 1) / 2; round++) {
      // lanes past k carry values no id takes
      const uint32_t same = __match_any_sync(0xffffffffu, lane < k ? label : (int32_t)(0x80000000u | lane));
      const bool step = lane < k && (label == lrow32 || (same & below) != 0);
      if (__ballot_sync(0xffffffffu, step) == 0) break;
      if (step) label = label + 1 == cnt32 ? 0 : label + 1;
    }
    int64_t lab64 = (int64_t)label + base;
    if (order && lane < k) lab64 = inv[lab64];
    const float ds = diffsum_staged(X, d, row, (int32_t)lab64, lane < k, sm);
    uint64_t key = ~0ull;
    if (lane < k) key = pack(ds, (int32_t)lab64);
    key = warp_sort32(key);
    if (lane < k) {
      gid[row * k + lane] = pk_id(key);  // all "new"
      gdist[row * k + lane] = pk_dist(key);
    }
    float w = __shfl_sync(0xffffffffu, pk_dist(key), k - 1);
    if (lane == 0) worst[row] = w;
  }
}

// Initial graph of the merge of two point sets A = [0, n1) and B = [n1, n)
// (InitRandomBlockedKNNGraph, knnmerge.cu:80-185, then the distance pass and
// per-row sort of InitRandomKNNGraph nndescent.cu:1800-1871 that
// NNDescentForMerge :2013 runs on it), one warp per row: the first k - k/2
// entries of the row's own subgraph row (ids shifted into the merged
// numbering, flagged old as after MarkAllToOld), then k/2 ids of the other
// set drawn as xorshift64star(local row * (k/2) + t) % |other set|, flagged
// new.  An id drawn twice is advanced to the next free one (the reference
// keeps repeats), and every distance is the sequential FP32 difference sum of
// the join (the reference's distance pass sums over a warp tree).  The rows
// are sorted by (distance, id); an entry's flag follows from its set: ids of
// the other set are the new ones.  Own-subgraph ids outside their set, self
// ids and repeats set DEVERR_ID_RANGE / SELF / DUP and are replaced by a
// valid id of the set so that no gather leaves X.
__global__ void __launch_bounds__(256, 3) k_merge_init(const float *__restrict__ X, int64_t n, int d, int k, int64_t n1,
                             const hdb_nnd_element *__restrict__ G1,
                             const hdb_nnd_element *__restrict__ G2, int32_t *__restrict__ gid,
                             float *__restrict__ gdist, float *__restrict__ worst,
                             uint32_t *__restrict__ err) {
  extern __shared__ float smem_stage[];
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  float *sm = smem_stage + (threadIdx.x >> 5) * kStageFloats;
  const int h = k - k / 2, r = k / 2;
  for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < n;
       row += (int64_t)gridDim.x * wpb) {
    const bool inb = row >= n1;
    const int64_t local = inb ? row - n1 : row;
    const int64_t own_n = inb ? n - n1 : n1, own_off = inb ? n1 : 0;
    const int64_t oth_n = inb ? n1 : n - n1, oth_off = inb ? 0 : n1;
    const hdb_nnd_element *own = inb ? G2 : G1;
    int64_t label = 0;
    uint32_t bad = 0;
    if (lane < h) {
      label = decode(own[local * k + lane].label_);
      if (label < 0 || label >= own_n) {
        bad |= DEVERR_ID_RANGE;
        label = (local + 1 + lane) % own_n;
      } else if (label == local) {
        bad |= DEVERR_SELF_ID;
        label = (local + 1 + lane) % own_n;
      }
    } else if (lane < k) {
      label = (int64_t)(xorshift64star((uint64_t)(local * r + (lane - h))) % (uint64_t)oth_n);
    }
    // repeats among the own entries (input error) and among the drawn ones
    const uint32_t same = __match_any_sync(0xffffffffu, lane < h ? label : -1 - (int64_t)lane);
    if (lane < h && (__ffs(same) - 1) != lane) bad |= DEVERR_DUP_ID;
    for (int t = 0; t < r; t++) {
      while (true) {
        const int64_t c = __shfl_sync(0xffffffffu, label, h + t);
        const bool dup = lane >= h && lane < h + t && label == c;
        if (__ballot_sync(0xffffffffu, dup) == 0) break;
        if (lane == h + t) label = (label + 1) % oth_n;
      }
    }
    const uint32_t anybad = __reduce_or_sync(0xffffffffu, bad);
    if (anybad && lane == 0) atomicOr(err, anybad);
    if (anybad & DEVERR_DUP_ID) {
      // keep the rows valid: the own half becomes the next h ids of its set
      if (lane < h) label = (local + 1 + lane) % own_n;
    }
    label += lane < h ? own_off : oth_off;
    const float ds = diffsum_staged(X, d, row, (int32_t)label, lane < k, sm);
    uint64_t key = ~0ull;
    if (lane < k) key = pack(ds, (int32_t)label);
    key = warp_sort32(key);
    if (lane < k) {
      const int32_t id = pk_id(key);
      const bool isnew = (id >= n1) != inb;
      gid[row * k + lane] = isnew ? id : -id - 1;
      gdist[row * k + lane] = pk_dist(key);
    }
    const float w = __shfl_sync(0xffffffffu, pk_dist(key), k - 1);
    if (lane == 0) worst[row] = w;
  }
}

// Offers a chunk of up to 32 candidates (one per lane, ~0 for none) to the
// row held one sorted entry per lane (lane < k; key = (distance, id)).  Only
// candidates below the row's current k-th key can enter, and the k-th key
// never grows, so those are found with one ballot; each is then placed by
// rank (ballot of the keys below it) unless its id is already listed, the
// entries above it moving up one lane and the last one dropping out.  The
// result is the first k distinct ids of the union in key order, whatever the
// order of the candidates.  Inserted entries carry the "new" flag.
template <bool kCheckIds = true>
__device__ __forceinline__ void insert_chunk(int k, uint64_t &rkey, int32_t &lab, uint64_t cand) {
  const int lane = lane_id();
  const bool have = lane < k;
  const uint64_t kth = __shfl_sync(0xffffffffu, rkey, k - 1);
  uint32_t todo = __ballot_sync(0xffffffffu, cand < kth);
  while (todo) {
    const int t = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint64_t c = __shfl_sync(0xffffffffu, cand, t);
    const int pos = __popc(__ballot_sync(0xffffffffu, have && rkey < c));
    if (pos >= k) continue;
    const int32_t cid = pk_id(c);
    if (kCheckIds && __any_sync(0xffffffffu, have && pk_id(rkey) == cid)) continue;
    const uint64_t up = __shfl_up_sync(0xffffffffu, rkey, 1);
    const int32_t uplab = __shfl_up_sync(0xffffffffu, lab, 1);
    if (lane == pos) {
      rkey = c;
      lab = cid;
    } else if (have && lane > pos) {
      rkey = up;
      lab = uplab;
    }
  }
}

// Rank of x among the sorted keys held by lanes 0..m-1 (number of keys
// below x), by binary search over shuffled lanes; every lane its own x.
__device__ __forceinline__ int rank_in_lanes(uint64_t sorted, int m, uint64_t x) {
  int lo = 0, hi = m;
#pragma unroll
  for (int it = 0; it < 6; it++) {  // 2^6 > 33 possible answers
    const int mid = (lo + hi) >> 1;
    const uint64_t v = __shfl_sync(0xffffffffu, sorted, mid & 31);
    if (lo < hi) {
      if (v < x) lo = mid + 1; else hi = mid;
    }
  }
  return lo;
}

// Per-warp shared memory of the merge: an open-addressing table of the ids
// seen (128 slots, -1 empty), the compacted survivors of a batch, and the
// merged row.
constexpr int kMergeTable = 128;
struct MergeSmem {
  int32_t tbl[kMergeTable];
  uint64_t stage[64];
  uint64_t sk[32];
  int32_t sl[32];
};

// Inserts id into the table; true if it was not there yet.  A batch puts at
// most 32 + 64 ids into the 128 slots, so a free slot is always found.
__device__ __forceinline__ bool table_insert(int32_t *tbl, int32_t id) {
  uint32_t h = ((uint32_t)id * 0x9E3779B1u) >> 25;
  for (int probe = 0; probe < kMergeTable; probe++) {
    const int32_t prev = atomicCAS(&tbl[h], -1, id);
    if (prev == -1) return true;
    if (prev == id) return false;
    h = (h + 1) & (kMergeTable - 1);
  }
  return false;
}

// Offers up to 64 candidates (c0, c1 per lane; ~0 for none) to the row held
// one sorted entry per lane (lane < k; key = (distance, id)), with the same
// result as insert_chunk on each of them.  Candidates at or above the row's
// k-th key cannot enter (the k-th key never grows).  The others go through a
// per-warp hash table holding the row's ids first, so a candidate whose id
// is listed or was already offered in the batch drops out (a pair's repeats
// carry equal keys, so which one stays does not matter); the survivors are
// compacted and either inserted one at a time (few) or sorted across the
// lanes and merged by rank -- each side finds its rank in the other by binary
// search -- with the first k entries placed through shared memory.
__device__ __forceinline__ void merge_batch(int k, uint64_t &rkey, int32_t &lab, uint64_t c0,
                                            uint64_t c1, MergeSmem &ms) {
  const int lane = lane_id();
  const bool have = lane < k;
  const uint64_t kth = __shfl_sync(0xffffffffu, rkey, k - 1);
  bool ok0 = c0 < kth, ok1 = c1 < kth;
  if (!__any_sync(0xffffffffu, ok0 || ok1)) return;
#pragma unroll
  for (int j = 0; j < kMergeTable / 32; j++) ms.tbl[lane + 32 * j] = -1;
  __syncwarp();
  if (have) table_insert(ms.tbl, pk_id(rkey));
  __syncwarp();
  if (ok0) ok0 = table_insert(ms.tbl, pk_id(c0));
  if (ok1) ok1 = table_insert(ms.tbl, pk_id(c1));
  const uint32_t b0 = __ballot_sync(0xffffffffu, ok0), b1 = __ballot_sync(0xffffffffu, ok1);
  const int nsurv = __popc(b0) + __popc(b1);
  if (nsurv == 0) return;
  const uint32_t lt = lanemask_lt();
  if (ok0) ms.stage[__popc(b0 & lt)] = c0;
  if (ok1) ms.stage[__popc(b0) + __popc(b1 & lt)] = c1;
  __syncwarp();
  for (int base = 0; base < nsurv; base += 32) {
    const int nc = min(32, nsurv - base);
    const uint64_t cand = lane < nc ? ms.stage[base + lane] : ~0ull;
    if (nc <= 12) {
      insert_chunk<false>(k, rkey, lab, cand);
      continue;
    }
    const uint64_t c = warp_sort32(cand);                // survivors in lanes 0..nc-1
    const int pos_r = lane + rank_in_lanes(c, nc, rkey);  // row entry: its merged rank
    const int pos_c = lane + rank_in_lanes(rkey, k, c);   // candidate: its merged rank
    __syncwarp();
    if (have && pos_r < k) {
      ms.sk[pos_r] = rkey;
      ms.sl[pos_r] = lab;
    }
    if (lane < nc && pos_c < k) {
      ms.sk[pos_c] = c;
      ms.sl[pos_c] = pk_id(c);  // inserted as "new"
    }
    __syncwarp();
    if (have) {
      rkey = ms.sk[lane];
      lab = ms.sl[lane];
    }
  }
}

// Merge of everything offered to a row (inbox, best dropped, the row's
// segment of the sorted candidate list) into its sorted list (one warp), in
// batches of 64.  On return, lane j (< k) holds the j-th entry of the merged
// row.  The list forms keep no inboxes (ib.inboxes = 0).
__device__ __forceinline__ void merge_row(int64_t row, int k, int32_t &lab, float &dist,
                                          const Inbox &ib, MergeSmem &ms) {
  const int lane = lane_id();
  int cnt = ib.inboxes ? ib.cnt[row] : 0;
  const uint64_t ov = ib.best[row];  // the best candidate that found no room (normally none)
  const uint32_t o0 = ib.ostart[row], o1 = ib.oend[row];
  if (cnt == 0 && ov == ~0ull && o0 == o1) return;
  __syncwarp();
  if (lane == 0) {
    if (cnt != 0) ib.cnt[row] = 0;
    if (ov != ~0ull) ib.best[row] = ~0ull;
    if (o0 != o1) { ib.ostart[row] = 0; ib.oend[row] = 0; }
  }
  if (cnt > kInboxCap) cnt = kInboxCap;
  const bool have = lane < k;
  uint64_t rkey = have ? pack(dist, decode(lab)) : ~0ull;
  // candidate i of the row: inbox slots, then the best dropped, then the
  // segment of the sorted list
  const uint64_t *inbox = ib.slots + row * kInboxCap;
  const int64_t nov = ov != ~0ull ? 1 : 0;
  const int64_t m = (int64_t)cnt + nov + (int64_t)(o1 - o0);
  auto at = [&](int64_t i) -> uint64_t {
    if (i < cnt) return inbox[i];
    if (i < cnt + nov) return ov;
    return ib.ovf_key[o0 + (i - cnt - nov)];
  };
  for (int64_t base = 0; base < m; base += 64) {
    const uint64_t c0 = base + lane < m ? at(base + lane) : ~0ull;
    const uint64_t c1 = base + 32 + lane < m ? at(base + 32 + lane) : ~0ull;
    merge_batch(k, rkey, lab, c0, c1, ms);
  }
  if (have) dist = pk_dist(rkey);
}

// Merge (iterations >= 1), sample (PrepareGraph :44-98 and reverse samples
// PrepareReverseGraph :293-346) and MarkAllToOld (:1398), one warp per row.
// split > 0 is the merge of two point sets [0, split) and [split, n)
// (PrepareGraphForMerge :100-166): old entries are sampled only from the
// row's own set; new entries and reverse samples are not filtered.
__global__ void k_sample(int64_t n, int k, int S, int do_merge, int32_t *__restrict__ gid,
                         float *__restrict__ gdist, float *__restrict__ worst, Inbox ib,
                         int32_t *__restrict__ newS,
                         int32_t *__restrict__ oldS, int8_t *__restrict__ nf, int8_t *__restrict__ of,
                         int32_t *__restrict__ nrev, int32_t *__restrict__ orev, int64_t split) {
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  __shared__ MergeSmem merge_smem[8];  // per-warp merge scratch (8 warps per block)
  MergeSmem &ms = merge_smem[threadIdx.x >> 5];
  for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < n;
       row += (int64_t)gridDim.x * wpb) {
    const bool have = lane < k;
    int32_t lab = have ? gid[row * k + lane] : 0;
    float dist = have ? gdist[row * k + lane] : 0.0f;
    if (do_merge) merge_row(row, k, lab, dist, ib, ms);
    const int32_t id = decode(lab);
    const bool isnew = have && lab >= 0;
    const bool isold = have && lab < 0 && (split <= 0 || ((row < split) == (id < split)));
    uint32_t nm = __ballot_sync(0xffffffffu, isnew), om = __ballot_sync(0xffffffffu, isold);
    int rn = __popc(nm & lanemask_lt()), ro = __popc(om & lanemask_lt());
    const int64_t sb = row * (2 * S);
    if (isnew && rn < S) {
      newS[sb + rn] = id;
      int p = atomicAdd(&nrev[id], 1);
      if (p < S) newS[(int64_t)id * (2 * S) + S + p] = (int32_t)row;
    }
    if (isold && ro < S) {
      oldS[sb + ro] = id;
      int p = atomicAdd(&orev[id], 1);
      if (p < S) oldS[(int64_t)id * (2 * S) + S + p] = (int32_t)row;
    }
    if (lane == 0) {
      nf[row] = (int8_t)min(__popc(nm), S);
      of[row] = (int8_t)min(__popc(om), S);
    }
    if (have) {
      gid[row * k + lane] = isnew ? -id - 1 : lab;  // MarkAllToOld
      gdist[row * k + lane] = dist;
    }
    float w = __shfl_sync(0xffffffffu, dist, k - 1);
    if (lane == 0) worst[row] = w;
  }
}

// Final merge after the last join; writes NNDElement rows with their flags.
__global__ void k_finalize(int64_t n, int k, const int32_t *__restrict__ gid,
                           const float *__restrict__ gdist, Inbox ib,
                           hdb_nnd_element *__restrict__ out) {
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  __shared__ MergeSmem merge_smem[8];  // per-warp merge scratch (8 warps per block)
  MergeSmem &ms = merge_smem[threadIdx.x >> 5];
  for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < n;
       row += (int64_t)gridDim.x * wpb) {
    const bool have = lane < k;
    int32_t lab = have ? gid[row * k + lane] : 0;
    float dist = have ? gdist[row * k + lane] : 0.0f;
    merge_row(row, k, lab, dist, ib, ms);
    if (have) {
      hdb_nnd_element e;
      e.distance_ = dist;
      e.label_ = lab;
      out[row * k + lane] = e;
    }
  }
}

// ---- FP32 local join -----------------------------------------------------
// Shared memory of one warp: best candidates (u64: best other-new and best old
// per new row; best new per old row) | slot ids | one chunk of kJc dimensions
// of every staged row.  Rows are staged a chunk at a time, so a warp needs
// ~9 KB whatever d is and an SM keeps 16 warps of joins in flight.
constexpr int kJc = 32;              // dimensions per staged chunk
constexpr int kJoinWarps = 8;
struct JoinSmem {
  static constexpr int kBest = 96;   // u64 entries
  static constexpr int kIds = 64;
  static constexpr size_t kBytes = kBest * 8 + kIds * 4 + (size_t)64 * kJc * 4;
};

// Float offset of 16-byte piece q of staged row r: the pieces of a row are
// permuted by the row's group of four, so the rows one warp-wide 16-byte load
// reads (one per tile group) fall into different bank groups.
__device__ __forceinline__ int stage_off(int r, int q) { return r * kJc + ((q ^ ((r >> 2) & 7)) << 2); }

// Stages dimensions [c0, c0 + 4 * nq) of the nn new rows (slots 0..) and the
// no old rows (slots 32..): 16-byte cp.async copies when every row piece is
// 16-byte aligned (d % 4 == 0), else scalar loads, zero padded to a multiple
// of four (adding fmaf(0, 0, s) = s leaves every sum unchanged).
__device__ __forceinline__ void stage_chunk(const float *__restrict__ X, int d, int c0, int nq,
                                            const int32_t *ids, int nn, int no, float *Xs,
                                            bool vec) {
  const int lane = lane_id();
  const int items = (nn + no) * nq;
  if (vec && nq == kJc / 4) {  // full chunk: eight pieces per row, no division
    for (int it = lane; it < items; it += 32) {
      const int r = it >> 3, q = it & 7;
      const int slot = r < nn ? r : 32 + (r - nn);
      const float *src = X + (int64_t)ids[slot] * d + c0 + 4 * q;
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(Xs + stage_off(slot, q));
      asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
  } else if (vec) {
    for (int it = lane; it < items; it += 32) {
      const int r = it / nq, q = it - r * nq;
      const int slot = r < nn ? r : 32 + (r - nn);
      const float *src = X + (int64_t)ids[slot] * d + c0 + 4 * q;
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(Xs + stage_off(slot, q));
      asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
  } else {
    for (int it = lane; it < items; it += 32) {
      const int r = it / nq, q = it - r * nq;
      const int slot = r < nn ? r : 32 + (r - nn);
      const float *src = X + (int64_t)ids[slot] * d;
      float4 v;
      const int c = c0 + 4 * q;
      v.x = c < d ? __ldg(src + c) : 0.0f;
      v.y = c + 1 < d ? __ldg(src + c + 1) : 0.0f;
      v.z = c + 2 < d ? __ldg(src + c + 2) : 0.0f;
      v.w = c + 3 < d ? __ldg(src + c + 3) : 0.0f;
      *reinterpret_cast<float4 *>(Xs + stage_off(slot, q)) = v;
    }
  }
  __syncwarp();
}

// Tile t of a row-join with rg row groups (new rows), cgn new and cgo old
// column groups: the new x new tiles are the upper triangle i <= j (a pair of
// different groups is computed once and offered to both rows), then the new x
// old tiles.  Returns the first slot of its rows (r0) and of its columns (c0)
// and its kind: 1 diagonal, 2 above the diagonal, 3 old columns.
__device__ __forceinline__ int tile_of(int t, int rg, int cgn, int cgo, int &r0, int &c0) {
  const int tri = cgn > 0 ? rg * (rg + 1) / 2 : 0;
  if (t < tri) {
    int i = 0;
    while (t >= rg - i) { t -= rg - i; i++; }
    r0 = 4 * i;
    c0 = 4 * (i + t);
    return t == 0 ? 1 : 2;
  }
  t -= tri;
  const int i = t / cgo;
  r0 = 4 * i;
  c0 = 32 + 4 * (t - i * cgo);
  return 3;
}

// Local join, one warp per row (UpdateGraph, nndescent.cu:1487-1580).  The
// distance matrix new x (new U old) is cut into 4 x 4 tiles, up to
// kJoinTiles per lane; a lane keeps its tiles' sums in registers while the
// rows pass through shared memory a chunk of kJc dimensions at a time, so
// every pair is the reference's sequential FP32 difference sum over
// j = 0..d-1.  Tile row/column minima go to the per-row best candidates with
// one 64-bit shared-memory atomicMin each: every new neighbour gets its closest
// other new one and its closest old one, every old neighbour its closest new
// one.  cross_only (the merge join, TiledNewOldNeighborsCompareKernelForMerge
// :1328-1383 launched without the new x new kernel, UpdateGraphForMerge
// :1582-1640) leaves out the new x new tiles: new neighbours get their closest
// old one only.
// kTiles: 4 x 4 register tiles per lane and pass (32 * kTiles per pass over
// the staged rows); one tile needs 80 registers and fits three blocks per SM,
// two need 122 and fit two -- the FP32 join tuner picks per (d, k, S).
template <int kTiles>
__global__ void __launch_bounds__(32 * kJoinWarps, kTiles == 1 ? 3 : 2)
    k_join(const float *__restrict__ X, int64_t n, int d, int S, const int32_t *__restrict__ newS,
           const int32_t *__restrict__ oldS, const int8_t *__restrict__ nf,
           const int8_t *__restrict__ of, int32_t *__restrict__ nrev, int32_t *__restrict__ orev,
           const float *__restrict__ worst, Inbox ib, int cross_only) {
  extern __shared__ __align__(16) unsigned char smem_join[];
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  unsigned char *base = smem_join + (threadIdx.x >> 5) * JoinSmem::kBytes;
  unsigned long long *best = reinterpret_cast<unsigned long long *>(base);
  unsigned long long *best1 = best, *best2 = best + 32, *best3 = best + 64;
  int32_t *ids = reinterpret_cast<int32_t *>(base + JoinSmem::kBest * 8);
  float *Xs = reinterpret_cast<float *>(base + JoinSmem::kBest * 8 + JoinSmem::kIds * 4);
  const bool vec = (d & 3) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0;
  unsigned long long w_rows = 0, w_cands = 0, w_pairs = 0;
  ListCursor cur;  // this warp's space in the candidate list
  const int64_t stride = (int64_t)gridDim.x * wpb;
  // a row's counts and both sample lists in one memory round trip, loaded one
  // row ahead so that they are in flight while the previous row is joined
  int32_t q_nraw = 0, q_oraw = 0;
  int q_cnf = 0, q_cof = 0, q_cnr = 0, q_cor = 0;
  auto load_lists = [&](int64_t r) {
    if (r >= n) return;
    const int64_t sb = r * (2 * S);
    q_nraw = lane < 2 * S ? newS[sb + lane] : 0;
    q_oraw = lane < 2 * S ? oldS[sb + lane] : 0;
    q_cnf = nf[r];
    q_cof = of[r];
    q_cnr = nrev[r];
    q_cor = orev[r];
  };
  int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5);
  load_lists(row);
  for (; row < n; row += stride) {
    const int32_t nraw = q_nraw, oraw = q_oraw;
    const int cnf = q_cnf, cof = q_cof;
    const int cnr = min(q_cnr, S), cor = min(q_cor, S);
    load_lists(row + stride);
    __syncwarp();
    if (lane == 0) { nrev[row] = 0; orev[row] = 0; }
    // slot t < S: forward sample t; slot S + t: reverse sample t
    bool vn = (lane < S) ? (lane < cnf) : (lane < 2 * S && lane - S < cnr);
    bool vo = (lane < S) ? (lane < cof) : (lane < 2 * S && lane - S < cor);
    const int32_t nid = vn ? nraw : -1 - lane;
    const int32_t oid = vo ? oraw : -100 - lane;
    // de-duplicate (ShrinkGraph RemoveDuplicates, :285-291)
    const uint32_t pn = __match_any_sync(0xffffffffu, nid);
    vn = vn && (__ffs(pn) - 1 == lane);
    const uint32_t po = __match_any_sync(0xffffffffu, oid);
    vo = vo && (__ffs(po) - 1 == lane);
    const uint32_t bo = __ballot_sync(0xffffffffu, vo);
    const int no = __popc(bo);
    if (vo) ids[32 + __popc(bo & lanemask_lt())] = oid;
    __syncwarp();
    // new \ old (:468-486)
    {
      bool in_old = false;  // independent reads, not a chain
#pragma unroll 8
      for (int t = 0; t < no; t++) in_old |= ids[32 + t] == nid;
      vn = vn && !in_old;
    }
    const uint32_t bn = __ballot_sync(0xffffffffu, vn);
    const int nn = __popc(bn);
    if (vn) ids[__popc(bn & lanemask_lt())] = nid;
    best1[lane] = ~0ull;
    best2[lane] = ~0ull;
    best3[lane] = ~0ull;
    __syncwarp();
    if (nn == 0 || nn + no < 2 || (cross_only && no == 0)) continue;
    w_rows += nn + no;
    w_pairs += (cross_only ? 0 : nn * (nn - 1) / 2) + nn * no;  // the reference's pairs
    const int rg = (nn + 3) >> 2;                              // row groups (new rows)
    const int cgn = cross_only ? 0 : rg, cgo = (no + 3) >> 2;  // column groups: new, old
    const int tiles = (cgn > 0 ? rg * (rg + 1) / 2 : 0) + rg * cgo;
    // up to 32 * kTiles tiles per pass through the rows (rows with more
    // samples take further passes; at most 100 tiles)
    for (int t0 = 0; t0 < tiles; t0 += 32 * kTiles) {
      int r0[kTiles], c0[kTiles], kind[kTiles];
      float acc[kTiles][4][4];
#pragma unroll
      for (int u = 0; u < kTiles; u++) {
        const int t = t0 + lane + 32 * u;
        kind[u] = t < tiles ? tile_of(t, rg, cgn, cgo, r0[u], c0[u]) : 0;
        if (kind[u] == 0) { r0[u] = 0; c0[u] = 0; }
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[u][i][j] = 0.0f;
      }
      for (int cd = 0; cd < d; cd += kJc) {
        const int nq = (min(kJc, d - cd) + 3) >> 2;
        __syncwarp();  // the previous chunk is no longer read
        stage_chunk(X, d, cd, nq, ids, nn, no, Xs, vec);
#pragma unroll
        for (int u = 0; u < kTiles; u++) {
          if (kind[u] == 0) continue;
          // the four rows of a tile side share one piece permutation
          const int ka = (r0[u] >> 2) & 7, kc = (c0[u] >> 2) & 7;
          for (int q = 0; q < nq; q++) {
            const float *pa = Xs + r0[u] * kJc + ((q ^ ka) << 2);
            const float *pc = Xs + c0[u] * kJc + ((q ^ kc) << 2);
            float4 xc[4];
#pragma unroll
            for (int j = 0; j < 4; j++) xc[j] = *reinterpret_cast<const float4 *>(pc + j * kJc);
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const float4 xa = *reinterpret_cast<const float4 *>(pa + i * kJc);
#pragma unroll
              for (int j = 0; j < 4; j++) {
                const float2 d01 = neg_diff2(make_float2(xc[j].x, xc[j].y), make_float2(xa.x, xa.y));
                const float2 d23 = neg_diff2(make_float2(xc[j].z, xc[j].w), make_float2(xa.z, xa.w));
                float s_ = __fmaf_rn(d01.x, d01.x, acc[u][i][j]);
                s_ = __fmaf_rn(d01.y, d01.y, s_);
                s_ = __fmaf_rn(d23.x, d23.x, s_);
                acc[u][i][j] = __fmaf_rn(d23.y, d23.y, s_);
              }
            }
          }
        }
      }
      // tile minima -> per-row best candidates
#pragma unroll
      for (int u = 0; u < kTiles; u++) {
        if (kind[u] == 0) continue;
        const bool oldcols = kind[u] == 3;
        const int ncol = oldcols ? no : nn;
        const int cb = oldcols ? c0[u] - 32 : c0[u];  // first column within its block
        uint64_t colmin[4] = {~0ull, ~0ull, ~0ull, ~0ull};
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int a = r0[u] + i;
          if (a >= nn) continue;
          uint64_t rmin = ~0ull;
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const int c = cb + j;
            if (c >= ncol || (kind[u] == 1 && c == a)) continue;
            const uint64_t kr = pack(acc[u][i][j], ids[c0[u] + j]);
            rmin = kr < rmin ? kr : rmin;
            if (kind[u] != 1) {
              const uint64_t kc = pack(acc[u][i][j], ids[a]);
              colmin[j] = kc < colmin[j] ? kc : colmin[j];
            }
          }
          if (rmin != ~0ull) atomicMin(oldcols ? &best2[a] : &best1[a], (unsigned long long)rmin);
        }
        if (kind[u] != 1) {
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (colmin[j] != ~0ull)
              atomicMin(oldcols ? &best3[cb + j] : &best1[cb + j], (unsigned long long)colmin[j]);
        }
      }
    }  // passes
    __syncwarp();
    // the candidates that can enter their target's list go to the candidate
    // list, which is sorted by target before the merge (space reserved 1024
    // slots at a time per warp; no returning atomic per candidate)
    const int32_t x = lane < nn ? ids[lane] : 0;
    const uint64_t b1 = lane < nn ? best1[lane] : ~0ull, b2 = lane < nn ? best2[lane] : ~0ull;
    const float wx = lane < nn ? worst[x] : 0.0f;
    const int32_t x3 = lane < no ? ids[32 + lane] : 0;
    const uint64_t b3 = lane < no ? best3[lane] : ~0ull;
    const float wx3 = lane < no ? worst[x3] : 0.0f;
    const bool v1 = b1 != ~0ull && pk_dist(b1) < wx, v2 = b2 != ~0ull && pk_dist(b2) < wx;
    const bool v3 = b3 != ~0ull && pk_dist(b3) < wx3;
    w_cands += append_candidates(ib, cur, (uint32_t)n, v1, x, b1, v2, x, b2);
    w_cands += append_candidates(ib, cur, (uint32_t)n, v3, x3, b3, false, 0, 0ull);
    __syncwarp();
  }
  list_fill(ib, cur.pos, cur.end, (uint32_t)n);  // the rest of the last chunk
  // per-warp totals, one atomic each (no block-wide barrier)
#pragma unroll
  for (int o = 16; o; o >>= 1) w_cands += __shfl_xor_sync(0xffffffffu, w_cands, o);
  if (lane == 0) {
    if (w_rows) atomicAdd(&ib.counters[1], w_rows);
    if (w_cands) atomicAdd(&ib.counters[2], w_cands);
    if (w_pairs) atomicAdd(&ib.counters[4], w_pairs);
  }
}
// ---------------------------------------------------------------------------
// BF16 tensor-core form of the local join.
//
// Candidate distances come from ||x||^2 + ||y||^2 - 2 x.y with x, y rounded to
// BF16 (norms of the rounded rows, FP32), the dot products on the tensor cores
// with FP32 accumulation (mma.sync m16n8k16, operands staged with cp.async
// and ldmatrix).  One pair always gets one value, whichever row joins it.
// After the last iteration every kept neighbour is re-ranked with the exact
// FP32 difference sum (k_rerank), so the graph handed on carries the
// reference's distances.
// ---------------------------------------------------------------------------
struct JoinSmemBf16 {
  // per warp: best[96] u64 | ids[64] | norms[64] | rows [64][dpad + 8] bf16
  __host__ __device__ static size_t bytes(int dpad) {
    return 96 * 8 + 64 * 4 + 64 * 4 + (size_t)64 * (dpad + 8) * 2;
  }
};

// Column sums of X (FP64, one thread per column, rows split over blocks):
// the BF16 copy is taken of the centred rows.
__global__ void k_col_sums(const float *__restrict__ X, int64_t n, int d, double *__restrict__ sums) {
  for (int j = threadIdx.x; j < d; j += blockDim.x) {
    double s = 0.0;
#pragma unroll 8
    for (int64_t row = blockIdx.x; row < n; row += gridDim.x) s += (double)X[row * d + j];
    atomicAdd(&sums[j], s);
  }
}

__global__ void k_col_mean(const double *__restrict__ sums, int d, int64_t n, float *__restrict__ mean) {
  for (int j = threadIdx.x; j < d; j += blockDim.x) mean[j] = (float)(sums[j] / (double)n);
}

// Largest |x - mean| over X (float bits: non-negative floats order as
// unsigned integers), for the FP16 form's power-of-two scale.
__global__ void k_abs_max(const float *__restrict__ X, int64_t n, int d,
                          const float *__restrict__ mean, uint32_t *__restrict__ out) {
  uint32_t m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * d;
       i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, __float_as_uint(fabsf(__fsub_rn(X[i], mean[i % d]))));
#pragma unroll
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane_id() == 0 && m) atomicMax(out, m);
}

// 16-bit operand formats of the tensor-core forms.
struct Bf16Op {
  using T = __nv_bfloat16;
  static __device__ __forceinline__ T from(float x) { return __float2bfloat16_rn(x); }
  static __device__ __forceinline__ float to(T x) { return __bfloat162float(x); }
};
struct Fp16Op {
  using T = __half;
  static __device__ __forceinline__ T from(float x) { return __float2half_rn(x); }
  static __device__ __forceinline__ float to(T x) { return __half2float(x); }
};

// 16-bit copy of (X - mean) / scale (mean may be null: no centring; scale a
// power of two, 1 for BF16), zero padded to dpad columns, and the FP32
// squared norm of every rounded row taken back to the original scale.
// Distances do not change under a common shift, and centring keeps the
// coordinates small, which is where the rounding is finest.
template <typename Op>
__global__ void k_half_prepare(const float *__restrict__ X, int64_t n, int d, int dpad,
                               const float *__restrict__ mean, float inv_scale, float scale,
                               typename Op::T *__restrict__ Xh, float *__restrict__ nrm) {
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < n;
       row += (int64_t)gridDim.x * wpb) {
    float part = 0.0f;
    for (int j = lane; j < dpad; j += 32) {
      const float x = j < d ? __fsub_rn(X[row * d + j], mean ? mean[j] : 0.0f) : 0.0f;
      const typename Op::T h = Op::from(__fmul_rn(x, inv_scale));
      Xh[row * dpad + j] = h;
      const float v = __fmul_rn(Op::to(h), scale);
      part = __fmaf_rn(v, v, part);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) part = __fadd_rn(part, __shfl_xor_sync(0xffffffffu, part, o));
    if (lane == 0) nrm[row] = part;
  }
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::);
}
__device__ __forceinline__ void ldsm_x4(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3,
                                        const void *smem) {
  uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(s));
}
template <bool kFp16>
__device__ __forceinline__ void mma_16(float *c, const uint32_t *a, uint32_t b0, uint32_t b1) {
  if (kFp16)
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
  else
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// kFp16: FP16 operands (scaled rows; dscale = -2 scale^2), else BF16
// (dscale = -2).  Xb holds the 16-bit rows.
template <bool kFp16>
__global__ void __launch_bounds__(128) k_join_bf16(const uint16_t *__restrict__ Xb,
                                                   const float *__restrict__ nrm, int64_t n,
                                                   int dpad, int S, float dscale,
                                                   const int32_t *__restrict__ newS,
                                                   const int32_t *__restrict__ oldS,
                                                   const int8_t *__restrict__ nf,
                                                   const int8_t *__restrict__ of,
                                                   int32_t *__restrict__ nrev,
                                                   int32_t *__restrict__ orev,
                                                   const float *__restrict__ worst, Inbox ib) {
  extern __shared__ __align__(16) unsigned char smem_bf[];
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  unsigned char *base = smem_bf + (threadIdx.x >> 5) * JoinSmemBf16::bytes(dpad);
  unsigned long long *best = reinterpret_cast<unsigned long long *>(base);
  unsigned long long *best1 = best, *best2 = best + 32, *best3 = best + 64;
  int32_t *ids = reinterpret_cast<int32_t *>(base + 96 * 8);
  float *nr = reinterpret_cast<float *>(base + 96 * 8 + 256);
  uint16_t *Bs = reinterpret_cast<uint16_t *>(base + 96 * 8 + 512);
  const int ld = dpad + 8;  // row stride in elements (16-byte aligned, ldmatrix conflict free)
  const int chunks = dpad >> 3;  // 16-byte chunks per row
  unsigned long long w_rows = 0, w_cands = 0;
  for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < n;
       row += (int64_t)gridDim.x * wpb) {
    const int cnf = nf[row], cof = of[row];
    const int cnr = min(nrev[row], S), cor = min(orev[row], S);
    __syncwarp();
    if (lane == 0) { nrev[row] = 0; orev[row] = 0; }
    const int64_t sb = row * (2 * S);
    bool vn = (lane < S) ? (lane < cnf) : (lane < 2 * S && lane - S < cnr);
    bool vo = (lane < S) ? (lane < cof) : (lane < 2 * S && lane - S < cor);
    int32_t nid = vn ? newS[sb + lane] : -1 - lane;
    int32_t oid = vo ? oldS[sb + lane] : -100 - lane;
    uint32_t pn = __match_any_sync(0xffffffffu, nid);
    vn = vn && (__ffs(pn) - 1 == lane);
    uint32_t po = __match_any_sync(0xffffffffu, oid);
    vo = vo && (__ffs(po) - 1 == lane);
    uint32_t bo = __ballot_sync(0xffffffffu, vo);
    const int no = __popc(bo);
    if (vo) ids[32 + __popc(bo & lanemask_lt())] = oid;
    __syncwarp();
    {
      bool in_old = false;  // independent reads, not a chain
#pragma unroll 8
      for (int t = 0; t < no; t++) in_old |= ids[32 + t] == nid;
      vn = vn && !in_old;
    }
    uint32_t bn = __ballot_sync(0xffffffffu, vn);
    const int nn = __popc(bn);
    if (vn) ids[__popc(bn & lanemask_lt())] = nid;
    best1[lane] = ~0ull;
    best2[lane] = ~0ull;
    best3[lane] = ~0ull;
    __syncwarp();
    if (nn == 0 || nn + no < 2) continue;
    w_rows += nn + no;
    // stage rows: new at slots 0..nn-1, old at 32..32+no-1 (cp.async, 16 B)
    const int T = nn + no;
    for (int idx = lane; idx < T * chunks; idx += 32) {
      int r = idx / chunks, c = idx - r * chunks;
      int slot = r < nn ? r : 32 + (r - nn);
      cp_async16(Bs + slot * ld + c * 8, Xb + (int64_t)ids[slot] * dpad + c * 8);
    }
    if (lane < nn) nr[lane] = nrm[ids[lane]];
    if (lane < no) nr[32 + lane] = nrm[ids[32 + lane]];
    cp_async_wait_all();
    __syncwarp();
    // G = B_new (32 x dpad) * B_all (64 x dpad)^T
    float acc[2][8][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 8; j++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[i][j][e] = 0.0f;
    const int mts = nn > 16 ? 2 : 1;
    const bool any_old = no > 0;
    for (int kt = 0; kt < dpad; kt += 16) {
      uint32_t a[2][4];
#pragma unroll
      for (int mt = 0; mt < 2; mt++)
        if (mt < mts)
          ldsm_x4(a[mt][0], a[mt][1], a[mt][2], a[mt][3],
                  Bs + (16 * mt + (lane & 15)) * ld + kt + ((lane >> 4) << 3));
#pragma unroll
      for (int pr = 0; pr < 4; pr++) {
        if (pr >= 2 && !any_old) continue;
        uint32_t b0, b1, b2, b3;
        const int prow = 16 * pr + ((lane >> 4) << 3) + (lane & 7);
        ldsm_x4(b0, b1, b2, b3, Bs + prow * ld + kt + (((lane >> 3) & 1) << 3));
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
          if (mt >= mts) continue;
          mma_16<kFp16>(acc[mt][2 * pr], a[mt], b0, b1);
          mma_16<kFp16>(acc[mt][2 * pr + 1], a[mt], b2, b3);
        }
      }
    }
    // epilogue: distances, row minima (best1 / best2) and old-column minima (best3)
    uint64_t cmin[4][2];  // old n-tiles 4..7, two columns each
#pragma unroll
    for (int q = 0; q < 4; q++) cmin[q][0] = cmin[q][1] = ~0ull;
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int a = 16 * mt + (lane >> 2) + 8 * h;
        const bool arow = mt < mts && a < nn;
        const float na = arow ? nr[a] : 0.0f;
        uint64_t rn = ~0ull, ro = ~0ull;
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int c = 8 * nt + 2 * (lane & 3) + e;
            const bool oldc = c >= 32;
            const bool ok = arow && (oldc ? (c - 32 < no) : (c < nn && c != a));
            if (!ok) continue;
            float dd = __fmaf_rn(dscale, acc[mt][nt][2 * h + e], __fadd_rn(na, nr[c]));
            dd = dd > 0.0f ? dd : 0.0f;
            const uint64_t kr = pack(dd, ids[c]);
            if (oldc) {
              ro = kr < ro ? kr : ro;
              const uint64_t kc = pack(dd, ids[a]);
              uint64_t &m = cmin[nt - 4][e];
              m = kc < m ? kc : m;
            } else {
              rn = kr < rn ? kr : rn;
            }
          }
        }
        // the four lanes of a row
#pragma unroll
        for (int o = 1; o <= 2; o <<= 1) {
          uint64_t x = __shfl_xor_sync(0xffffffffu, rn, o);
          rn = x < rn ? x : rn;
          x = __shfl_xor_sync(0xffffffffu, ro, o);
          ro = x < ro ? x : ro;
        }
        if (arow && (lane & 3) == 0) {
          best1[a] = rn;
          best2[a] = ro;
        }
      }
    }
    // the eight row-lanes of a column
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int e = 0; e < 2; e++) {
        uint64_t m = cmin[q][e];
#pragma unroll
        for (int o = 4; o <= 16; o <<= 1) {
          uint64_t x = __shfl_xor_sync(0xffffffffu, m, o);
          m = x < m ? x : m;
        }
        const int c = 8 * q + 2 * (lane & 3) + e;  // old column index
        if (lane < 4 && c < no) best3[c] = m;
      }
    __syncwarp();
    int pushed = 0;
    if (lane < nn) {
      const int32_t x = ids[lane];
      const uint64_t b1 = best1[lane], b2 = best2[lane];
      if (b1 != ~0ull) pushed += push_candidate(x, pk_id(b1), pk_dist(b1), worst, ib);
      if (b2 != ~0ull) pushed += push_candidate(x, pk_id(b2), pk_dist(b2), worst, ib);
    }
    if (lane < no) {
      const uint64_t b3 = best3[lane];
      if (b3 != ~0ull) pushed += push_candidate(ids[32 + lane], pk_id(b3), pk_dist(b3), worst, ib);
    }
    w_cands += pushed;
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) w_cands += __shfl_xor_sync(0xffffffffu, w_cands, o);
  if (lane == 0) {
    if (w_rows) atomicAdd(&ib.counters[1], w_rows);
    if (w_cands) atomicAdd(&ib.counters[2], w_cands);
  }
}

// FP32 re-rank of every kept neighbour (one warp per row): the reference's
// difference sum for each (row, neighbour) pair, rows re-sorted by (distance,
// id); old/new flags travel with their ids.
__global__ void __launch_bounds__(256, 3) k_rerank(const float *__restrict__ X, int64_t n, int d, int k,
                         hdb_nnd_element *__restrict__ G) {
  extern __shared__ float smem_stage[];
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  float *sm = smem_stage + (threadIdx.x >> 5) * kStageFloats;
  for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < n;
       row += (int64_t)gridDim.x * wpb) {
    int32_t lab = 0;
    if (lane < k) lab = G[row * k + lane].label_;
    const int32_t id = decode(lab);
    const float ds = diffsum_staged(X, d, row, id, lane < k, sm);
    uint64_t key = lane < k ? pack(ds, id) : ~0ull;
    int32_t slab = lab;  // the entry (with its old/new flag) moves with its key
    warp_sort32_with(key, slab);
    if (lane < k) {
      hdb_nnd_element e;
      e.distance_ = pk_dist(key);
      e.label_ = slab;
      G[row * k + lane] = e;
    }
  }
}

__global__ void k_split(const hdb_nnd_element *__restrict__ G, int64_t total, int32_t *__restrict__ ids,
                        float *__restrict__ dist) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    hdb_nnd_element e = G[i];
    if (ids) ids[i] = decode(e.label_);
    if (dist) dist[i] = e.distance_;
  }
}

__device__ __forceinline__ float euclid_ref(const float *__restrict__ a, const float *__restrict__ b,
                                           int d) {
  float soma = 0.0f;
  for (int i = 0; i < d; i++) {
    float diff = __fsub_rn(a[i], b[i]);
    double sq = __dmul_rn((double)diff, (double)diff);
    soma = __double2float_rn(__dadd_rn((double)soma, sq));
  }
  return __fsqrt_rn(soma);
}

__global__ void k_fix_distances(const float *__restrict__ X, int64_t n, int d,
                                const int32_t *__restrict__ ids, int k, float *__restrict__ dist) {
  const int64_t total = n * k;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t row = i / k;
    dist[i] = euclid_ref(X + row * d, X + (int64_t)ids[i] * d, d);
  }
}

// Segment [ostart, oend) of every target row in the target-sorted overflow
// list; sentinel entries (target n, the unused tail of a chunk) sort last and
// are skipped.
__global__ void k_ovf_bounds(const uint32_t *__restrict__ tgt, int64_t cnt, int64_t n,
                             uint32_t *__restrict__ ostart, uint32_t *__restrict__ oend) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t t = tgt[i];
    if (t >= n) continue;
    if (i == 0 || tgt[i - 1] != t) ostart[t] = (uint32_t)i;
    if (i == cnt - 1 || tgt[i + 1] != t) oend[t] = (uint32_t)(i + 1);
  }
}

// ---- locality order ---------------------------------------------------------
// The local join gathers the rows of every row's samples, i.e. of its current
// neighbours.  With ids in arbitrary order those rows lie anywhere in X, and
// the ~2,000 consecutive rows the join works on at any moment fetch them all
// from HBM.  After the initial graph the points are renumbered so that near
// points get near ids: by instance, then by the Morton code of three
// projections on fixed +-1 vectors (10 bits each over the projection's range).
// The rows in flight then gather from a few MB of X, which L2 holds.  The final
// graph is mapped back to the original ids and every row re-sorted by
// (distance, id), so the order is the caller's.
constexpr int kLocProj = 3;

__device__ __forceinline__ float loc_sign(int p, int j) {
  return (xorshift64star(((uint64_t)(p + 1) << 32) | (uint32_t)j) >> 63) ? -1.0f : 1.0f;
}

// One warp per row: the three projections; per block the range of each.
__global__ void k_loc_project(const float *__restrict__ X, int64_t n, int d,
                              float *__restrict__ proj, uint32_t *__restrict__ range) {
  __shared__ uint32_t blk[2 * kLocProj];
  if (threadIdx.x < 2 * kLocProj) blk[threadIdx.x] = (threadIdx.x & 1) ? 0u : 0xffffffffu;
  __syncthreads();
  const int lane = lane_id(), wpb = blockDim.x >> 5;
  uint32_t lo[kLocProj], hi[kLocProj];
#pragma unroll
  for (int p = 0; p < kLocProj; p++) { lo[p] = 0xffffffffu; hi[p] = 0u; }
  for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < n;
       row += (int64_t)gridDim.x * wpb) {
    float acc[kLocProj] = {0.0f, 0.0f, 0.0f};
    for (int j = lane; j < d; j += 32) {
      const float x = X[row * d + j];
#pragma unroll
      for (int p = 0; p < kLocProj; p++) acc[p] += loc_sign(p, j) * x;
    }
#pragma unroll
    for (int p = 0; p < kLocProj; p++) {
#pragma unroll
      for (int o = 16; o; o >>= 1) acc[p] += __shfl_xor_sync(0xffffffffu, acc[p], o);
      const uint32_t key = float_key(acc[p]);
      lo[p] = min(lo[p], key);
      hi[p] = max(hi[p], key);
      if (lane == p) proj[row * kLocProj + p] = acc[p];
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int p = 0; p < kLocProj; p++) {
      atomicMin(&blk[2 * p], lo[p]);
      atomicMax(&blk[2 * p + 1], hi[p]);
    }
  }
  __syncthreads();
  if (threadIdx.x < kLocProj) {
    atomicMin(&range[2 * threadIdx.x], blk[2 * threadIdx.x]);
    atomicMax(&range[2 * threadIdx.x + 1], blk[2 * threadIdx.x + 1]);
  }
}

__device__ __forceinline__ uint32_t spread3(uint32_t x) {  // 10 bits -> every third bit
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__global__ void k_loc_keys(const float *__restrict__ proj, int64_t n, Segments seg,
                           const uint32_t *__restrict__ range, uint64_t *__restrict__ keys,
                           uint32_t *__restrict__ vals) {
  float lo[kLocProj], scale[kLocProj];
#pragma unroll
  for (int p = 0; p < kLocProj; p++) {
    lo[p] = key_float(range[2 * p]);
    const float w = key_float(range[2 * p + 1]) - lo[p];
    scale[p] = w > 0.0f ? 1024.0f / w : 0.0f;
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t m = 0;
#pragma unroll
    for (int p = 0; p < kLocProj; p++) {
      const float q = (proj[i * kLocProj + p] - lo[p]) * scale[p];
      const uint32_t c = q <= 0.0f ? 0u : (q >= 1023.0f ? 1023u : (uint32_t)q);
      m |= spread3(c) << p;
    }
    const uint64_t inst = seg.count > 0 ? (uint64_t)seg.of_point(i) : 0;
    keys[i] = (inst << 32) | m;
    vals[i] = (uint32_t)i;
  }
}

__global__ void k_loc_inverse(const uint32_t *__restrict__ order, int64_t n, int32_t *__restrict__ inv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    inv[order[i]] = (int32_t)i;
}

__global__ void k_loc_rows(const float *__restrict__ X, const uint32_t *__restrict__ order, int64_t n,
                           int d, float *__restrict__ Xp) {
  const int lane = lane_id(), wpb = blockDim.x >> 5;
  for (int64_t r = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); r < n;
       r += (int64_t)gridDim.x * wpb) {
    const int64_t o = order[r];
    for (int j = lane; j < d; j += 32) Xp[r * d + j] = X[o * d + j];
  }
}

// A row with every id mapped through idmap, re-sorted by (distance, mapped
// id); each entry keeps its old/new flag.  One warp per row.
__device__ __forceinline__ void remap_row(int k, int32_t in_lab, float in_dist,
                                          const int32_t *__restrict__ idmap, int32_t &out_lab,
                                          float &out_dist) {
  const int lane = lane_id();
  const bool have = lane < k;
  const int32_t id = have ? idmap[decode(in_lab)] : 0;
  uint64_t key = have ? pack(in_dist, id) : ~0ull;
  int32_t flag = have && in_lab < 0;  // moves with its key (ids are distinct within a row)
  warp_sort32_with(key, flag);
  const int32_t mine = pk_id(key);
  out_dist = pk_dist(key);
  out_lab = flag ? -mine - 1 : mine;
}

__global__ void k_loc_restore(const hdb_nnd_element *__restrict__ Gp, const uint32_t *__restrict__ order,
                              int64_t n, int k, hdb_nnd_element *__restrict__ G) {
  const int lane = lane_id(), wpb = blockDim.x >> 5;
  for (int64_t r = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); r < n;
       r += (int64_t)gridDim.x * wpb) {
    hdb_nnd_element e = lane < k ? Gp[r * k + lane] : hdb_nnd_element{0.0f, 0};
    int32_t ol;
    float od;
    remap_row(k, e.label_, e.distance_, reinterpret_cast<const int32_t *>(order), ol, od);
    if (lane < k) G[(int64_t)order[r] * k + lane] = hdb_nnd_element{od, ol};
  }
}

int bits_for_rows(int64_t n) {
  int b = 1;
  while (b < 40 && (int64_t(1) << b) < n) b++;
  return b;
}

}  // namespace

// Sorts the join's overflow list by target row and records each row's
// segment for the next merge; resets the list.
static void sort_overflow(Context *ctx, const Inbox &ib, int64_t n) {
  cudaStream_t st = ctx->stream;
  unsigned long long *h = reinterpret_cast<unsigned long long *>(ctx->pinned);
  HDB_CUDA(cudaMemcpyAsync(h, ib.counters + 3, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  ctx->sync();
  int64_t c = (int64_t)h[0];
  if (c == 0) return;
  if (c > ib.ovf_cap) c = ib.ovf_cap;
  // the packed candidates move with their targets, so the merge reads each
  // row's segment contiguously
  // n + 1 values: the rows and the sentinel n of unused chunk slots
  radix_sort_u32_u64(ctx, ib.ovf_tgt, ib.ovf_key, c, 0, bits_for_rows(n + 1));
  k_ovf_bounds<<<grid_for(ctx, c, 256), 256, 0, st>>>(ib.ovf_tgt, c, n, ib.ostart, ib.oend); ctx->launches++;
  HDB_CHECK_LAUNCH();
  HDB_CUDA(cudaMemsetAsync(ib.counters + 3, 0, sizeof(unsigned long long), st));
}

namespace {

// Dynamic shared memory of the kernels that stage rows for difference sums
// (two ring slots of 33 rows x 32 dimensions per warp: 66 KB for 8 warps).
void stage_smem_attrs(size_t bytes) {
  HDB_CUDA(cudaFuncSetAttribute(k_init, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  HDB_CUDA(cudaFuncSetAttribute(k_merge_init, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  HDB_CUDA(cudaFuncSetAttribute(k_rerank, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// Device state of one NN-Descent run over n rows: the graph lists, the
// samples of an iteration and the join's inboxes and candidate list.
// list_only: the tensor-core join, which keeps no inboxes and appends a whole
// iteration's candidates to the list.
struct NndState {
  Buf<int32_t> gid, newS, oldS, nrev, orev, inbox_cnt;
  Buf<float> gdist, worst;
  Buf<int8_t> nf, of;
  Buf<uint64_t> inbox, ovf_key;
  Buf<unsigned long long> ovf, dropped;
  Buf<uint32_t> ovf_tgt, ostart, oend;
  Inbox ib;

  NndState(Context *ctx, int64_t n, int k, int S, bool list_only) {
    cudaStream_t st = ctx->stream;
    gid = Buf<int32_t>(ctx, n * k);
    gdist = Buf<float>(ctx, n * k);
    worst = Buf<float>(ctx, n);
    newS = Buf<int32_t>(ctx, n * 2 * S);
    oldS = Buf<int32_t>(ctx, n * 2 * S);
    nrev = Buf<int32_t>(ctx, n);
    orev = Buf<int32_t>(ctx, n);
    inbox_cnt = Buf<int32_t>(ctx, n);
    nf = Buf<int8_t>(ctx, n);
    of = Buf<int8_t>(ctx, n);
    inbox = Buf<uint64_t>(ctx, list_only ? 1 : (size_t)n * kInboxCap);
    ovf = Buf<unsigned long long>(ctx, n);
    dropped = Buf<unsigned long long>(ctx, 5);
    // room for a pass's candidates; the joins' warps also leave the unused
    // tail of their last list chunk (at most one chunk per warp: 8 epilogue
    // warps per SM in the tensor-core join, up to 24 in the FP32 join)
    const int64_t rows = list_only ? 64 : 16;
    const int64_t cap = (n * rows > (1 << 22) ? n * rows : (1 << 22)) +
                        (list_only ? (int64_t)24 * ctx->num_sms * kListChunk : 0);
    ovf_tgt = Buf<uint32_t>(ctx, cap);
    ovf_key = Buf<uint64_t>(ctx, cap);
    ostart = Buf<uint32_t>(ctx, n);
    oend = Buf<uint32_t>(ctx, n);
    HDB_CUDA(cudaMemsetAsync(ostart, 0, n * 4, st));
    HDB_CUDA(cudaMemsetAsync(oend, 0, n * 4, st));
    ib = Inbox{inbox_cnt, inbox, ovf, ovf_tgt, ovf_key, ostart, oend, dropped, cap, list_only ? 0 : 1};
    HDB_CUDA(cudaMemsetAsync(nrev, 0, n * 4, st));
    HDB_CUDA(cudaMemsetAsync(orev, 0, n * 4, st));
    clear_inboxes(ctx, n);
  }
  // the inbox state a join starts an iteration from: empty inboxes, no
  // candidates in the list, nothing dropped
  void clear_inboxes(Context *ctx, int64_t n) {
    cudaStream_t st = ctx->stream;
    HDB_CUDA(cudaMemsetAsync(inbox_cnt, 0, n * 4, st));
    HDB_CUDA(cudaMemsetAsync(ovf, 0xff, n * 8, st));
    HDB_CUDA(cudaMemsetAsync(dropped, 0, 5 * sizeof(unsigned long long), st));
  }
};

// One FP32 local join over s's samples with `tiles` 4 x 4 tiles per lane.
void fp32_join(Context *ctx, int tiles, const float *X, int64_t n, int d, int S, const NndState &s,
               int cross_only) {
  const int jw = kJoinWarps;
  const size_t smem = JoinSmem::kBytes * jw;
  // the blocks that fit on the GPU at once (a grid-stride loop over the rows):
  // each warp holds one chunk of list space, so their number bounds what the
  // list loses to unused chunk tails
  const int grid = grid_for(ctx, n, jw, tiles == 1 ? 3 : 2);
  cudaStream_t st = ctx->stream;
  if (tiles == 1) {
    HDB_CUDA(cudaFuncSetAttribute(k_join<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_join<1><<<grid, 32 * jw, smem, st>>>(X, n, d, S, s.newS, s.oldS, s.nf, s.of, s.nrev, s.orev,
                                           s.worst, s.ib, cross_only);
  } else {
    HDB_CUDA(cudaFuncSetAttribute(k_join<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_join<2><<<grid, 32 * jw, smem, st>>>(X, n, d, S, s.newS, s.oldS, s.nf, s.of, s.nrev, s.orev,
                                           s.worst, s.ib, cross_only);
  }
  ctx->launches++;
}

struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  EventPair() {
    HDB_CUDA(cudaEventCreate(&a));
    HDB_CUDA(cudaEventCreate(&b));
  }
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

std::mutex g_tune_mutex;
// (device, d, k, S, whether the rows fit in L2) -> tile slots
std::map<std::array<int, 5>, int> g_join_tiles;

}  // namespace

// Tile slots per lane of the FP32 local join: the one forced on the context,
// else the one tuned for this shape.  An untuned shape is timed on the first
// m rows of Xw (the caller's rows in locality order; m = 64K..1M, enough to
// leave L2 at d >= 64): the initial graph of those rows, one iteration
// (sample, join, merge) so that the rows hold old and new entries as in the
// later iterations, the second sample, then both forms -- k_join<1> (80
// registers, three blocks per SM) and k_join<2> (122 registers, two blocks
// per SM) -- three times each, alternating, from the same sample and inbox
// state, the first round untimed.  The faster form is kept for the process.
// Without Xw (the merge) an untuned shape takes two.  The trial's launches
// count in ctx->launches.
int fp32_join_tiles(Context *ctx, int d, int k, int S, bool resident, const float *Xw, int64_t n) {
  if (ctx->join_tiles) return ctx->join_tiles;
  const std::array<int, 5> key{ctx->device, d, k, S, resident ? 1 : 0};
  {
    std::lock_guard<std::mutex> g(g_tune_mutex);
    auto it = g_join_tiles.find(key);
    if (it != g_join_tiles.end()) return it->second;
  }
  if (!Xw) return 2;
  cudaStream_t st = ctx->stream;
  const int64_t want = (int64_t(256) << 20) / (4 * (int64_t)d);
  const int64_t m = std::min<int64_t>(
      n, std::max<int64_t>(65536, std::min<int64_t>(int64_t(1) << 20, want)));
  NndState t(ctx, m, k, S, true);
  Buf<int32_t> nrev0(ctx, m), orev0(ctx, m);
  const int wpb = 8;
  const int grid_rows = grid_for(ctx, m, wpb, 16);
  const size_t smem_stage = (size_t)wpb * kStageFloats * sizeof(float);
  stage_smem_attrs(smem_stage);
  k_init<<<grid_rows, 32 * wpb, smem_stage, st>>>(Xw, m, d, k, Segments{}, nullptr, nullptr, t.gid,
                                                  t.gdist, t.worst);
  ctx->launches++;
  HDB_CHECK_LAUNCH();
  for (int it = 0; it < 2; it++) {
    if (it == 1) {
      fp32_join(ctx, 2, Xw, m, d, S, t, 0);
      HDB_CHECK_LAUNCH();
      sort_overflow(ctx, t.ib, m);
    }
    k_sample<<<grid_rows, 32 * wpb, 0, st>>>(m, k, S, it, t.gid, t.gdist, t.worst, t.ib, t.newS,
                                             t.oldS, t.nf, t.of, t.nrev, t.orev, 0);
    ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  // the join clears the reverse-sample counts it reads: each trial starts
  // from a copy
  HDB_CUDA(cudaMemcpyAsync(nrev0, t.nrev, m * 4, cudaMemcpyDeviceToDevice, st));
  HDB_CUDA(cudaMemcpyAsync(orev0, t.orev, m * 4, cudaMemcpyDeviceToDevice, st));
  EventPair ev;
  double ms[3] = {0.0, 0.0, 0.0};
  for (int rep = 0; rep < 3; rep++) {
    for (int tiles = 1; tiles <= 2; tiles++) {
      HDB_CUDA(cudaMemcpyAsync(t.nrev, nrev0, m * 4, cudaMemcpyDeviceToDevice, st));
      HDB_CUDA(cudaMemcpyAsync(t.orev, orev0, m * 4, cudaMemcpyDeviceToDevice, st));
      t.clear_inboxes(ctx, m);
      HDB_CUDA(cudaEventRecord(ev.a, st));
      fp32_join(ctx, tiles, Xw, m, d, S, t, 0);
      HDB_CUDA(cudaEventRecord(ev.b, st));
      HDB_CHECK_LAUNCH();
      HDB_CUDA(cudaEventSynchronize(ev.b));
      float e = 0.0f;
      HDB_CUDA(cudaEventElapsedTime(&e, ev.a, ev.b));
      if (rep > 0) ms[tiles] += e;
    }
  }
  const int pick = ms[1] < ms[2] ? 1 : 2;
  std::lock_guard<std::mutex> g(g_tune_mutex);
  g_join_tiles[key] = pick;
  return pick;
}

int64_t nndescent_bytes_per_point(int32_t d, const hdb_knn_params &p) {
  const int64_t k = p.k, S = p.sample_num;
  const bool half = p.precision == HDB_PREC_BF16 || p.precision == HDB_PREC_FP16;
  const bool tc = half && tc_dpad(d) <= kTcMaxDpad;
  const bool list = tc || !half;                 // the tensor-core and FP32 joins
  const int64_t dpad = tc ? tc_dpad(d) : (d + 15) & ~15;
  int64_t b = 4 * (int64_t)d;                    // X in locality order
  if (half) b += 2 * dpad + 4;                   // 16-bit rows + norms
  b += 8 * k + 4 + 16 * S + 30;                  // lists, worst, samples, counters
  if (!list) b += 8 * kInboxCap;                 // per-row inboxes
  b += 2 * 12 * (list ? 64 : 16);                // candidate list + sort buffers
  b += 8 * k;                                    // graph in locality order
  return b;
}

void nndescent(Context *ctx, const float *X, int64_t n, int32_t d, const hdb_knn_params &p,
               hdb_nnd_element *G, int64_t *dropped_out, JoinStats *js, const Segments &seg) {
  const int k = p.k, S = p.sample_num;
  HDB_REQUIRE(k >= 1 && k <= kMaxK, HDB_ERR_ARG, "NN-Descent: k must be in [1, 32]");
  HDB_REQUIRE(S >= 1 && 2 * S <= k, HDB_ERR_ARG,
              "NN-Descent: SAMPLE_NUM must satisfy 1 <= SAMPLE_NUM and 2*SAMPLE_NUM <= k");
  HDB_REQUIRE(n > k && n < (int64_t(1) << 31) - 1, HDB_ERR_ARG, "NN-Descent: need k < n < 2^31");
  HDB_REQUIRE(d >= 1 && d <= 4096, HDB_ERR_ARG, "NN-Descent: d must be in [1, 4096]");
  HDB_REQUIRE(p.iterations >= 0, HDB_ERR_ARG, "NN-Descent: negative iteration count");
  HDB_REQUIRE(p.precision == HDB_PREC_FP32 || p.precision == HDB_PREC_BF16 ||
                  p.precision == HDB_PREC_FP16,
              HDB_ERR_ARG, "NN-Descent: unknown precision");
  cudaStream_t st = ctx->stream;
  // The tensor-core join and the FP32 join append every candidate to the
  // list that sort_overflow groups by target for the merge (a returning inbox
  // atomic per candidate cost them more than the sort), so they need no
  // inboxes and a list for a whole iteration's candidates.  The mma.sync join
  // (16-bit forms past 256 dimensions) keeps the per-row inboxes.
  const bool tc_form = (p.precision == HDB_PREC_BF16 || p.precision == HDB_PREC_FP16) &&
                       tc_dpad(d) <= kTcMaxDpad;
  const bool list_form = tc_form || p.precision == HDB_PREC_FP32;
  NndState s(ctx, n, k, S, list_form);
  int32_t *gid = s.gid, *newS = s.newS, *oldS = s.oldS, *nrev = s.nrev, *orev = s.orev;
  float *gdist = s.gdist, *worst = s.worst;
  int8_t *nf = s.nf, *of = s.of;
  const Inbox &ib = s.ib;
  unsigned long long *dropped = s.dropped;
  std::vector<cudaEvent_t> jev;
  if (js) {
    jev.resize(2 * (size_t)p.iterations);
    for (auto &e : jev) HDB_CUDA(cudaEventCreate(&e));
  }

  const int wpb = 8;
  const int grid_rows = grid_for(ctx, n, wpb, 16);
  const size_t smem_stage = (size_t)wpb * kStageFloats * sizeof(float);
  stage_smem_attrs(smem_stage);
  // renumber the points in locality order (k_loc_project); X stays the
  // caller's, the iterations work on Xw and the renumbered lists, and the
  // initial graph is drawn straight into the new numbering
  Buf<uint32_t> order(ctx, n);
  Buf<float> Xp(ctx, (size_t)n * d);
  {
    Buf<float> proj(ctx, (size_t)n * kLocProj);
    Buf<uint32_t> range(ctx, 2 * kLocProj);
    const uint32_t range0[2 * kLocProj] = {0xffffffffu, 0u, 0xffffffffu, 0u, 0xffffffffu, 0u};
    HDB_CUDA(cudaMemcpyAsync(range, range0, sizeof(range0), cudaMemcpyHostToDevice, st));
    k_loc_project<<<grid_rows, 32 * wpb, 0, st>>>(X, n, d, proj, range); ctx->launches++;
    Buf<uint64_t> keys(ctx, n);
    k_loc_keys<<<grid_for(ctx, n, 256), 256, 0, st>>>(proj, n, seg, range, keys, order); ctx->launches++;
    HDB_CHECK_LAUNCH();
    int ibits = 0;
    while (seg.count > 0 && (int64_t(1) << ibits) < seg.count) ibits++;
    radix_sort_u64(ctx, keys, order, n, 0, 30 + (seg.count > 0 ? 2 + ibits : 0));
    Buf<int32_t> inv(ctx, n);
    k_loc_inverse<<<grid_for(ctx, n, 256), 256, 0, st>>>(order, n, inv); ctx->launches++;
    k_loc_rows<<<grid_rows, 32 * wpb, 0, st>>>(X, order, n, d, Xp); ctx->launches++;
    HDB_CHECK_LAUNCH();
    k_init<<<grid_rows, 32 * wpb, smem_stage, st>>>(Xp, n, d, k, seg, order, inv, gid, gdist, worst);
    ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  const float *Xw = Xp;
  Buf<hdb_nnd_element> Gp(ctx, (size_t)n * k);
  // 16-bit forms: BF16, or FP16 of the rows scaled by one power of two; the
  // tensor-core tile pipeline (tcgen05) up to 256 padded dimensions, the
  // mma.sync join beyond
  const bool fp16 = p.precision == HDB_PREC_FP16;
  const bool bf16 = p.precision == HDB_PREC_BF16 || fp16;
  const bool use_tc = bf16 && tc_dpad(d) <= kTcMaxDpad;
  const int dpad = use_tc ? tc_dpad(d) : (d + 15) & ~15;
  Buf<uint16_t> Xb;
  Buf<float> nrm;
  int jw16 = 4;
  size_t smem_bf = 0;
  int grid_bf = 0;
  float dscale = -2.0f;
  TcJoin tj;
  if (bf16) {
    Xb = Buf<uint16_t>(ctx, (size_t)n * dpad);
    nrm = Buf<float>(ctx, n);
    Buf<double> csum(ctx, d);
    Buf<float> cmean(ctx, d);
    HDB_CUDA(cudaMemsetAsync(csum, 0, d * sizeof(double), st));
    k_col_sums<<<16 * ctx->num_sms, 256, 0, st>>>(Xw, n, d, csum); ctx->launches++;
    k_col_mean<<<1, 256, 0, st>>>(csum, d, n, cmean); ctx->launches++;
    HDB_CHECK_LAUNCH();
    if (fp16) {
      // one power-of-two scale s with max |x - mean| / s in [2^14, 2^15): far
      // from the FP16 overflow and subnormal ranges, exact to apply
      Buf<uint32_t> amax(ctx, 1);
      HDB_CUDA(cudaMemsetAsync(amax, 0, sizeof(uint32_t), st));
      k_abs_max<<<grid_for(ctx, n * d, 256), 256, 0, st>>>(Xw, n, d, cmean, amax); ctx->launches++;
      HDB_CHECK_LAUNCH();
      HDB_CUDA(cudaMemcpyAsync(ctx->pinned, amax, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      ctx->sync();
      float gmax;
      memcpy(&gmax, ctx->pinned, sizeof(float));
      int e = 0;
      if (gmax > 0.0f && std::isfinite(gmax)) std::frexp(gmax, &e);
      const float sc = std::ldexp(1.0f, e - 15);
      dscale = -2.0f * sc * sc;
      k_half_prepare<Fp16Op><<<grid_rows, 32 * wpb, 0, st>>>(
          Xw, n, d, dpad, cmean, 1.0f / sc, sc, reinterpret_cast<__half *>(Xb.get()), nrm);
    } else {
      k_half_prepare<Bf16Op><<<grid_rows, 32 * wpb, 0, st>>>(
          Xw, n, d, dpad, cmean, 1.0f, 1.0f, reinterpret_cast<__nv_bfloat16 *>(Xb.get()), nrm);
    }
    ctx->launches++;
    HDB_CHECK_LAUNCH();
    if (use_tc) {
      tc_join_prepare(ctx, Xb, n, dpad, fp16, dscale, &tj);
    } else {
      smem_bf = JoinSmemBf16::bytes(dpad) * jw16;
      HDB_REQUIRE(smem_bf <= 227 * 1024, HDB_ERR_ARG, "NN-Descent 16-bit form: d too large for the join tile");
      HDB_CUDA(cudaFuncSetAttribute(fp16 ? k_join_bf16<true> : k_join_bf16<false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bf));
      grid_bf = grid_for(ctx, n, jw16, 64);
    }
  }
  // FP32 form: the join's tile slots per lane, tuned per shape
  const int tiles =
      bf16 ? 0 : fp32_join_tiles(ctx, d, k, S, n * d * 4 <= ctx->l2_bytes, Xw, n);
  if (js) js->config = tiles;
  for (int it = 0; it < p.iterations; it++) {
    k_sample<<<grid_rows, 32 * wpb, 0, st>>>(n, k, S, it > 0, gid, gdist, worst, ib,
                                                       newS, oldS, nf, of, nrev, orev, 0); ctx->launches++;
    HDB_CHECK_LAUNCH();
    if (js) HDB_CUDA(cudaEventRecord(jev[2 * it], st));
    if (use_tc) {
      tc_join_launch(ctx, tj, S, nrm, newS, oldS, nf, of, nrev, orev, worst, ib);
    } else {
      if (fp16)
        k_join_bf16<true><<<grid_bf, 32 * jw16, smem_bf, st>>>(Xb, nrm, n, dpad, S, dscale, newS,
                                                               oldS, nf, of, nrev, orev, worst, ib);
      else if (bf16)
        k_join_bf16<false><<<grid_bf, 32 * jw16, smem_bf, st>>>(Xb, nrm, n, dpad, S, dscale, newS,
                                                                oldS, nf, of, nrev, orev, worst, ib);
      else
        fp32_join(ctx, tiles, Xw, n, d, S, s, 0);
      if (bf16) ctx->launches++;
    }
    if (js) HDB_CUDA(cudaEventRecord(jev[2 * it + 1], st));
    HDB_CHECK_LAUNCH();
    sort_overflow(ctx, ib, n);
    HDB_CHECK_LAUNCH();
  }
  k_finalize<<<grid_rows, 32 * wpb, 0, st>>>(n, k, gid, gdist, ib, Gp); ctx->launches++;
  HDB_CHECK_LAUNCH();
  if (bf16) {
    k_rerank<<<grid_rows, 32 * wpb, smem_stage, st>>>(Xw, n, d, k, Gp); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  k_loc_restore<<<grid_rows, 32 * wpb, 0, st>>>(Gp, order, n, k, G); ctx->launches++;
  HDB_CHECK_LAUNCH();
  HDB_CUDA(cudaMemcpyAsync(ctx->pinned, dropped, 5 * sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, st));
  ctx->sync();
  if (use_tc)
    HDB_REQUIRE(!(ctx->take_dev_err() & DEVERR_TIMEOUT), HDB_ERR_TIMEOUT,
                "NN-Descent: a wait of the tensor-core join pipeline gave up");
  const int64_t *hs = static_cast<const int64_t *>(ctx->pinned);
  if (dropped_out) *dropped_out = hs[0];
  if (js) {
    js->rows_gathered = hs[1];
    js->candidates = hs[2];
    js->pairs = hs[4];
    js->launches = p.iterations;
    js->ms = 0.0;
    for (int it = 0; it < p.iterations; it++) {
      float ms = 0.0f;
      HDB_CUDA(cudaEventElapsedTime(&ms, jev[2 * it], jev[2 * it + 1]));
      js->ms += ms;
    }
    for (auto &e : jev) cudaEventDestroy(e);
  }
}

void knn_merge(Context *ctx, const float *X1, int64_t n1, const hdb_nnd_element *G1,
               const float *X2, int64_t n2, const hdb_nnd_element *G2, int32_t d,
               const hdb_knn_params &p, hdb_nnd_element *G, int64_t *dropped_out) {
  const int k = p.k, S = p.sample_num;
  HDB_REQUIRE(k >= 1 && k <= kMaxK, HDB_ERR_ARG, "KNNMerge: k must be in [1, 32]");
  HDB_REQUIRE(S >= 1 && 2 * S <= k, HDB_ERR_ARG,
              "KNNMerge: MERGE_SAMPLE_NUM must satisfy 1 <= SAMPLE_NUM and 2*SAMPLE_NUM <= k");
  HDB_REQUIRE(n1 > k && n2 > k, HDB_ERR_ARG, "KNNMerge: each point set needs more than k points");
  const int64_t n = n1 + n2;
  HDB_REQUIRE(n < (int64_t(1) << 31) - 1, HDB_ERR_ARG, "KNNMerge: need n1 + n2 < 2^31");
  HDB_REQUIRE(d >= 1 && d <= 4096, HDB_ERR_ARG, "KNNMerge: d must be in [1, 4096]");
  HDB_REQUIRE(p.iterations >= 0, HDB_ERR_ARG, "KNNMerge: negative iteration count");
  HDB_REQUIRE(p.precision == HDB_PREC_FP32, HDB_ERR_ARG,
              "KNNMerge: the merge join is the FP32 difference sum (precision must be FP32)");
  cudaStream_t st = ctx->stream;
  (void)ctx->take_dev_err();
  // MergeVectors (knnmerge.cu:358-399): the two sets back to back
  Buf<float> X(ctx, (size_t)n * d);
  HDB_CUDA(cudaMemcpyAsync(X.get(), X1, (size_t)n1 * d * sizeof(float), cudaMemcpyDeviceToDevice, st));
  HDB_CUDA(cudaMemcpyAsync(X.get() + (size_t)n1 * d, X2, (size_t)n2 * d * sizeof(float),
                           cudaMemcpyDeviceToDevice, st));
  NndState s(ctx, n, k, S, true);
  int32_t *gid = s.gid;
  float *gdist = s.gdist, *worst = s.worst;
  const Inbox &ib = s.ib;
  unsigned long long *dropped = s.dropped;

  const int wpb = 8;
  const int grid_rows = grid_for(ctx, n, wpb, 16);
  const size_t smem_stage = (size_t)wpb * kStageFloats * sizeof(float);
  stage_smem_attrs(smem_stage);
  k_merge_init<<<grid_rows, 32 * wpb, smem_stage, st>>>(X, n, d, k, n1, G1, G2, gid, gdist, worst,
                                                        ctx->dev_err);
  ctx->launches++;
  HDB_CHECK_LAUNCH();
  ctx->sync();
  const uint32_t e = ctx->take_dev_err();
  HDB_REQUIRE(!(e & DEVERR_ID_RANGE), HDB_ERR_ARG, "KNNMerge: a subgraph id lies outside its set");
  HDB_REQUIRE(!(e & DEVERR_SELF_ID), HDB_ERR_ARG, "KNNMerge: a subgraph row lists itself");
  HDB_REQUIRE(!(e & DEVERR_DUP_ID), HDB_ERR_ARG, "KNNMerge: a subgraph row repeats an id");

  // the merge takes the forced tile slots, else the ones tuned for this
  // shape by an earlier nndescent call, else two
  const int tiles = fp32_join_tiles(ctx, d, k, S, n * d * 4 <= ctx->l2_bytes, nullptr, 0);
  // NNDescentForMerge (nndescent.cu:1999-2087): PrepareForUpdateForMerge +
  // UpdateGraphForMerge per iteration
  for (int it = 0; it < p.iterations; it++) {
    k_sample<<<grid_rows, 32 * wpb, 0, st>>>(n, k, S, it > 0, gid, gdist, worst, ib, s.newS,
                                             s.oldS, s.nf, s.of, s.nrev, s.orev, n1);
    ctx->launches++;
    HDB_CHECK_LAUNCH();
    fp32_join(ctx, tiles, X, n, d, S, s, 1);
    HDB_CHECK_LAUNCH();
    sort_overflow(ctx, ib, n);
    HDB_CHECK_LAUNCH();
  }
  k_finalize<<<grid_rows, 32 * wpb, 0, st>>>(n, k, gid, gdist, ib, G); ctx->launches++;
  HDB_CHECK_LAUNCH();
  HDB_CUDA(cudaMemcpyAsync(ctx->pinned, dropped, sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, st));
  ctx->sync();
  if (dropped_out) *dropped_out = *static_cast<const int64_t *>(ctx->pinned);
}

void bf16_distance_tiles(Context *ctx, const float *X, int64_t n, int32_t d, const int32_t *ids,
                         const int32_t *counts, int64_t tiles, float *out) {
  HDB_REQUIRE(n >= 1 && n < (int64_t(1) << 31) && d >= 1 && tc_dpad(d) <= kTcMaxDpad, HDB_ERR_ARG,
              "BF16 distance tiles: need 1 <= n < 2^31 and 1 <= d <= 256");
  HDB_REQUIRE(tiles >= 0, HDB_ERR_ARG, "BF16 distance tiles: negative tile count");
  if (tiles == 0) return;
  const int dpad = tc_dpad(d);
  Buf<uint16_t> Xb(ctx, (size_t)n * dpad);
  Buf<float> nrm(ctx, n);
  k_half_prepare<Bf16Op><<<grid_for(ctx, n, 8, 16), 256, 0, ctx->stream>>>(
      X, n, d, dpad, nullptr, 1.0f, 1.0f, reinterpret_cast<__nv_bfloat16 *>(Xb.get()), nrm);
  ctx->launches++;
  HDB_CHECK_LAUNCH();
  tc_gram_probe(ctx, Xb, nrm, n, dpad, ids, counts, tiles, out);
  ctx->sync();
  HDB_REQUIRE(!(ctx->take_dev_err() & DEVERR_TIMEOUT), HDB_ERR_TIMEOUT,
              "BF16 distance tiles: a pipeline wait gave up");
}

void knn_split(Context *ctx, const hdb_nnd_element *G, int64_t n, int32_t k, int32_t *ids,
               float *dist) {
  k_split<<<grid_for(ctx, n * k, 256), 256, 0, ctx->stream>>>(G, n * k, ids, dist); ctx->launches++;
  HDB_CHECK_LAUNCH();
}

void fix_distances(Context *ctx, const float *X, int64_t n, int32_t d, const int32_t *ids,
                   int32_t k, float *dist) {
  k_fix_distances<<<grid_for(ctx, n * k, 256), 256, 0, ctx->stream>>>(X, n, d, ids, k, dist); ctx->launches++;
  HDB_CHECK_LAUNCH();
}

}  // namespace hdb
