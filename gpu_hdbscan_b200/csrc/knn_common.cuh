// Shared pieces of the NN-Descent kernels (knn.cu, join_tc.cu): packed
// (distance, id) keys, the per-row candidate inbox and the push of one
// candidate into it.
#pragma once
#include "hdb_internal.cuh"

namespace hdb {
namespace knn {

constexpr int kMaxK = 32;
constexpr int kInboxCap = 127;  // + 1 overflow slot = 128 sorted candidates per merge

// Key of a candidate: distance bits (non-negative floats order as unsigned)
// above the id, so an unsigned compare orders by (distance, id).
__device__ __forceinline__ uint64_t pack(float d, int32_t id) {
  return ((uint64_t)__float_as_uint(d) << 32) | (uint32_t)id;
}
__device__ __forceinline__ float pk_dist(uint64_t k) { return __uint_as_float((uint32_t)(k >> 32)); }
__device__ __forceinline__ int32_t pk_id(uint64_t k) { return (int32_t)(uint32_t)k; }

// NNDElement::label(): "old" entries are stored as -id-1.
__device__ __forceinline__ int32_t decode(int32_t label) { return label >= 0 ? label : -label - 1; }

// Where the join leaves its candidates: a fixed inbox per row, then a global
// overflow list (radix-sorted by target row between the join and the merge).
// Only when the overflow list is full is a candidate dropped; the best
// dropped one per row is still kept in `best`.
struct Inbox {
  int32_t *cnt;                  // [n] candidates offered this iteration
  uint64_t *slots;               // [n * kInboxCap] packed (distance, id)
  unsigned long long *best;      // [n]
  uint32_t *ovf_tgt;             // [ovf_cap] overflow: target row (sorted in place)
  uint64_t *ovf_key;             // [ovf_cap] overflow: packed candidate (sorted along)
  uint32_t *ostart, *oend;       // [n] segment of each row in the sorted overflow list
  unsigned long long *counters;  // [0] dropped [1] rows gathered [2] candidates [3] overflow
                                 // [4] distance pairs computed (FP32 join)
  int64_t ovf_cap;
  int32_t inboxes;               // 0: no per-row inboxes (the tensor-core join's list only)
};

// Space of the candidate list a warp writes into: [pos, end), taken from the
// list in chunks of kListChunk slots with one atomic on the list's counter,
// so that the warps of a join do not all queue on that one counter.
constexpr uint32_t kListChunk = 1024;
struct ListCursor {
  unsigned long long pos = 0, end = 0;
};

// Writes the sentinel entry (target row `n`, sorted after every row and
// skipped by the segment bounds; key ~0) at list positions [from, to).
__device__ __forceinline__ void list_fill(const Inbox &ib, unsigned long long from,
                                          unsigned long long to, uint32_t n) {
  for (unsigned long long p = from + (threadIdx.x & 31); p < to; p += 32)
    if ((int64_t)p < ib.ovf_cap) {
      ib.ovf_tgt[p] = n;
      ib.ovf_key[p] = ~0ull;
    }
}

// Appends this lane's candidates (up to two: target row, packed key; the
// caller has checked each against its target's worst[]) to the list that is
// sorted by target before the next merge.  The warp writes them at its
// cursor; when they do not fit in the cursor's chunk, the rest of that chunk
// becomes sentinel entries and one lane takes a new chunk.  Past the list's
// capacity only the best dropped candidate of each target is kept.  Returns
// the lane's count.  Called by all 32 lanes of a warp; n is the row count.
__device__ __forceinline__ int append_candidates(const Inbox &ib, ListCursor &cur, uint32_t n,
                                                 bool v0, int32_t t0, uint64_t k0, bool v1,
                                                 int32_t t1, uint64_t k1) {
  const int lane = threadIdx.x & 31;
  uint32_t lt;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
  const uint32_t b0 = __ballot_sync(0xffffffffu, v0), b1 = __ballot_sync(0xffffffffu, v1);
  const uint32_t tot = __popc(b0) + __popc(b1);
  if (tot == 0) return 0;
  if (cur.pos + tot > cur.end) {
    list_fill(ib, cur.pos, cur.end, n);
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&ib.counters[3], (unsigned long long)kListChunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    cur.pos = base;
    cur.end = base + kListChunk;
  }
  const unsigned long long p0 = cur.pos + __popc(b0 & lt);
  const unsigned long long p1 = cur.pos + __popc(b0) + __popc(b1 & lt);
  cur.pos += tot;
  const int32_t tt[2] = {t0, t1};
  const uint64_t kk[2] = {k0, k1};
  const unsigned long long pp[2] = {p0, p1};
  const bool vv[2] = {v0, v1};
#pragma unroll
  for (int q = 0; q < 2; q++) {
    if (!vv[q]) continue;
    if ((int64_t)pp[q] < ib.ovf_cap) {
      ib.ovf_tgt[pp[q]] = (uint32_t)tt[q];
      ib.ovf_key[pp[q]] = kk[q];
    } else {
      atomicMin(&ib.best[tt[q]], (unsigned long long)kk[q]);
      atomicAdd(&ib.counters[0], 1ull);
    }
  }
  return (v0 ? 1 : 0) + (v1 ? 1 : 0);
}

__device__ __forceinline__ int push_candidate(int32_t target, int32_t id, float d,
                                              const float *__restrict__ worst, const Inbox &ib) {
  if (!(d < worst[target])) return 0;  // cannot enter the target's list
  int slot = atomicAdd(&ib.cnt[target], 1);
  uint64_t key = pack(d, id);
  if (slot < kInboxCap) {
    ib.slots[(int64_t)target * kInboxCap + slot] = key;
  } else {
    unsigned long long pos = atomicAdd(&ib.counters[3], 1ull);
    if ((int64_t)pos < ib.ovf_cap) {
      ib.ovf_tgt[pos] = (uint32_t)target;
      ib.ovf_key[pos] = key;
    } else {
      atomicMin(&ib.best[target], (unsigned long long)key);
      atomicAdd(&ib.counters[0], 1ull);
    }
  }
  return 1;
}

}  // namespace knn
}  // namespace hdb
