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
  uint64_t *ovf_key;             // [ovf_cap] overflow: packed candidate
  uint32_t *ovf_idx;             // [ovf_cap] overflow: permutation from the sort
  uint32_t *ostart, *oend;       // [n] segment of each row in the sorted overflow list
  unsigned long long *counters;  // [0] dropped [1] rows gathered [2] candidates [3] overflow
  int64_t ovf_cap;
};

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
