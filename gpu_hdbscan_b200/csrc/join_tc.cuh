// BF16 local join of NN-Descent on the sm_100a tensor cores (join_tc.cu).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>

#include "hdb_internal.cuh"
#include "knn_common.cuh"

namespace hdb {

// Rows of one tensor-core tile: two row-joins of 64 sample slots each.
constexpr int kTcTileRows = 128;
// The staged rows are BF16 with this many elements per 128-byte swizzle row;
// the row length (dpad) is a multiple of it.
constexpr int kTcKBlock = 64;
// Largest padded dimension the tile pipeline stages (three stages fit in
// shared memory up to this size).
constexpr int kTcMaxDpad = 256;

inline int tc_dpad(int d) { return (d + kTcKBlock - 1) / kTcKBlock * kTcKBlock; }

// Per-call state of the tensor-core join: the TMA descriptor of the BF16
// rows and the launch shape.
struct TcJoin {
  CUtensorMap xmap;
  int64_t n = 0;
  int dpad = 0;
  size_t smem = 0;
  int grid = 0;
  uint32_t idesc = 0;    // tcgen05 instruction descriptor (operand format)
  float dscale = -2.0f;  // distance = |a|^2 + |c|^2 + dscale * (a.c of the stored rows)
};

// Builds the TMA descriptor over the 16-bit rows Xh [n, dpad] (dpad =
// tc_dpad(d) <= kTcMaxDpad): BF16, or FP16 (fp16 = true) of rows stored
// divided by a power-of-two scale s, with dscale = -2 s^2 (-2 for BF16).
void tc_join_prepare(Context *ctx, const uint16_t *Xh, int64_t n, int dpad, bool fp16,
                     float dscale, TcJoin *tj);

// One local-join pass over all rows: the sample lists of k_sample in, the
// candidates out through the inbox's overflow list only (ib.ovf_cap must hold
// a pass's candidates; sort_overflow groups them by target for the merge).
void tc_join_launch(Context *ctx, const TcJoin &tj, int S, const float *nrm, const int32_t *newS,
                    const int32_t *oldS, const int8_t *nf, const int8_t *of, int32_t *nrev,
                    int32_t *orev, const float *worst, const knn::Inbox &ib);

// Distance tiles for explicit slot lists (testing the gather / MMA / TMEM
// path): ids [tiles * 128], counts [tiles * 4] = (new0, old0, new1, old1),
// out [tiles * 128 * 64] = the BF16 distance of every staged row against the
// 64 slots of its own row-join (+inf for empty columns).
void tc_gram_probe(Context *ctx, const uint16_t *Xb, const float *nrm, int64_t n, int dpad,
                   const int32_t *ids, const int32_t *counts, int64_t tiles, float *out);

}  // namespace hdb
