// Minimum spanning tree of the enhanced kNN graph and the MST edge sort.
//
// Reference: cpuMST (HDBSCAN/mst/mst.cu:34-78) runs Kruskal over the entries
// (weight, CSR edge index, row, target) whose target exceeds their row, and
// buildMST (mst.cu:291-336) + sort_edges (merge_sort/merge_sort.cu:226-279)
// list the chosen edges stably sorted by weight -- i.e. in (weight, edge
// index) order.  Under that strict total order the MST is unique, so a
// Boruvka MST that compares packed 64-bit keys (order-preserving weight bits
// << 32 | edge index) selects exactly Kruskal's edge set.  Each round:
// atomicMin of the key at both component representatives, hooking of every
// component to its chosen neighbour (a mutual pair keeps the smaller id as
// root), pointer jumping, and compaction of the edges that still cross
// components.  The chosen keys, radix-sorted, give the reference's sorted
// MSTedge list directly.
//
// The (weight, min id, max id) tie order replaces the edge index in the key's
// low half by the edge's rank under (row, target, edge index) -- row and
// target are the min and max id of a canonical entry -- so the same packed
// comparison spans the graph under that order; the rank is mapped back to the
// edge index once the tree is sorted.
#include <cmath>
#include <cstring>
#include <vector>

#include "hdb_internal.cuh"
#include "mst.cuh"

namespace hdb {

namespace {

constexpr int kWarps = 8;

struct alignas(16) CEdge {
  int32_t a, b;  // current component representatives of the endpoints
  uint64_t key;  // float_key(weight) << 32 | CSR edge index
};

__device__ __forceinline__ uint32_t weight_key(float w) {
  // -0.0 and +0.0 compare equal in the reference (std::sort / merge on <)
  return float_key(w == 0.0f ? 0.0f : w);
}

// ---- the reference's mst_gpu = 1 mode (int-quantised weights) ------------
// buildGPUgraph (core-sg.cu:33-36): (int)(10^m * w); a product outside the
// int range takes INT_MIN, the value x86's truncating conversion gives it.
__device__ __forceinline__ int32_t quantise(float w, double p10) {
  const double v = __dmul_rn(p10, (double)w);
  return (v < 2147483648.0 && v > -2147483649.0) ? (int32_t)v : INT32_MIN;
}
// buildMST_gpu (mst.cu:360): (1.0 * q) / 10^m, stored as float.
__device__ __forceinline__ float dequantise(int32_t q, double p10) {
  return __double2float_rn(__ddiv_rn((double)q, p10));
}
// gpuMST's key (mst.cu:163): the int weight's bits above the edge index, so
// an INT_MIN weight sorts after every other one.
__device__ __forceinline__ uint64_t quant_key(int32_t q, int64_t j) {
  return ((uint64_t)(uint32_t)q << 32) | (uint64_t)(uint32_t)j;
}

// Smallest positive first-neighbour distance of every instance's rows after
// its first (GetMinDistanceFromKNNG, tools/filetool.hpp:330-336); the first
// row's own rule is applied on the host.  Positive floats order as their bits.
__global__ void k_first_min(const float *__restrict__ first, int64_t stride, int64_t n, Segments seg,
                            uint32_t *__restrict__ minbits) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = seg.count > 0 ? seg.of_point(i) : 0;
    if (i == (seg.count > 0 ? seg.off[t] : 0)) continue;
    const float d = first[i * stride];
    if (d > 0.0f) atomicMin(&minbits[t], __float_as_uint(d));
  }
}

__global__ void k_first_rows(const float *__restrict__ first, int64_t stride, Segments seg,
                             float *__restrict__ out) {
  const int32_t T = seg.count > 0 ? seg.count : 1;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < T;
       t += (int64_t)gridDim.x * blockDim.x)
    out[t] = first[(seg.count > 0 ? seg.off[t] : 0) * stride];
}

__global__ void k_count_canon(const int64_t *__restrict__ nindex, const int32_t *__restrict__ nlist,
                              int64_t n, int32_t *__restrict__ cnt, uint32_t *err) {
  const int lane = lane_id();
  int64_t row = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  for (; row < n; row += (int64_t)gridDim.x * kWarps) {
    int64_t b = nindex[row], e = nindex[row + 1];
    int c = 0;
    for (int64_t j = b + lane; j < e; j += 32) {
      int32_t v = nlist[j];
      if (v < 0 || v >= n) { atomicOr(err, DEVERR_ID_RANGE); continue; }
      c += v > row;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[row] = c;
  }
}

// quant (optional): per-instance 10^m of the mst_gpu = 1 mode; keys then
// order by (int weight, edge index) as gpuMST's do.
__global__ void k_emit_canon(const int64_t *__restrict__ nindex, const int32_t *__restrict__ nlist,
                             const float *__restrict__ ew, const int64_t *__restrict__ off,
                             int64_t n, const double *__restrict__ quant, Segments seg,
                             CEdge *__restrict__ el) {
  const int lane = lane_id();
  int64_t row = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  for (; row < n; row += (int64_t)gridDim.x * kWarps) {
    int64_t b = nindex[row], e = nindex[row + 1];
    int64_t p = off[row];
    const double p10 = quant ? quant[seg.count > 0 ? seg.of_point(row) : 0] : 0.0;
    for (int64_t j0 = b; j0 < e; j0 += 32) {
      int64_t j = j0 + lane;
      bool take = j < e && nlist[j] > row;
      uint32_t m = __ballot_sync(0xffffffffu, take);
      if (take) {
        CEdge c;
        c.a = (int32_t)row;
        c.b = nlist[j];
        c.key = quant ? quant_key(quantise(ew[j], p10), j)
                      : ((uint64_t)weight_key(ew[j]) << 32) | (uint64_t)(uint32_t)j;
        el[p + __popc(m & lanemask_lt())] = c;
      }
      p += __popc(m);
    }
  }
}

// (weight, min id, max id) order, step 1: every canonical entry's
// (row << bits | target) and edge index, in CSR order (a stable sort of the
// pairs then breaks a repeated pair's tie by edge index).
__global__ void k_emit_pairs(const int64_t *__restrict__ nindex, const int32_t *__restrict__ nlist,
                             const int64_t *__restrict__ off, int64_t n, int bits,
                             uint64_t *__restrict__ pair, uint32_t *__restrict__ eidx) {
  const int lane = lane_id();
  int64_t row = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  for (; row < n; row += (int64_t)gridDim.x * kWarps) {
    int64_t b = nindex[row], e = nindex[row + 1];
    int64_t p = off[row];
    for (int64_t j0 = b; j0 < e; j0 += 32) {
      int64_t j = j0 + lane;
      const int32_t t = j < e ? nlist[j] : -1;
      bool take = t > row;
      uint32_t m = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int64_t q = p + __popc(m & lanemask_lt());
        pair[q] = ((uint64_t)row << bits) | (uint64_t)t;
        eidx[q] = (uint32_t)j;
      }
      p += __popc(m);
    }
  }
}

// Step 2: the edges with their rank r under (min id, max id, edge index) in
// the key's low half.
__global__ void k_emit_ranked(const uint64_t *__restrict__ pair, const uint32_t *__restrict__ eidx,
                              const float *__restrict__ ew, int64_t m, int bits,
                              CEdge *__restrict__ el) {
  const uint64_t mask = (uint64_t(1) << bits) - 1;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t pk = pair[r];
    CEdge c;
    c.a = (int32_t)(pk >> bits);
    c.b = (int32_t)(pk & mask);
    c.key = ((uint64_t)weight_key(ew[eidx[r]]) << 32) | (uint64_t)r;
    el[r] = c;
  }
}

// Step 3 (after the chosen keys are sorted): the rank back to the edge index.
__global__ void k_rank_to_edge(uint64_t *__restrict__ keys, int64_t m,
                               const uint32_t *__restrict__ eidx) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
       t += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[t];
    keys[t] = (k & 0xffffffff00000000ull) | (uint64_t)eidx[(uint32_t)k];
  }
}

__global__ void k_iota(int32_t *__restrict__ v, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (int32_t)i;
}

// Minimum incident edge of every representative.  The edge list is written
// row by row and compaction keeps each warp's order, so lanes that name the
// same `a` endpoint sit in runs of consecutive lanes: each run reduces its keys
// with redux.sync (the high halves, then the low halves of the lanes holding
// the least high half) and one lane of the run updates minkey.  The `b`
// endpoints of a run are distinct targets; each updates its own entry behind
// a read of the current minimum.
__global__ void k_min_edge(const CEdge *__restrict__ el, int64_t m,
                           unsigned long long *__restrict__ minkey) {
  const int lane = lane_id();
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < m; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    const bool valid = i < m;
    CEdge c;
    c.a = -1;  // an invalid lane is a run of its own that nobody reduces
    c.b = -1;
    c.key = ~0ull;
    if (valid) c = el[i];
    const int32_t aprev = __shfl_up_sync(0xffffffffu, c.a, 1);
    const uint32_t heads = __ballot_sync(0xffffffffu, lane == 0 || aprev != c.a);
    if (!valid) continue;
    const uint32_t le = heads & (0xffffffffu >> (31 - lane));  // heads at or below this lane
    const uint32_t gt = heads & ~(0xffffffffu >> (31 - lane));  // heads above it
    const int first = 31 - __clz(le);
    const int end = gt ? __ffs(gt) - 1 : 32;
    const uint32_t run = (end == 32 ? 0xffffffffu : ((1u << end) - 1)) & ~((1u << first) - 1);
    const uint32_t hi = (uint32_t)(c.key >> 32), lo = (uint32_t)c.key;
    const uint32_t mh = __reduce_min_sync(run, hi);
    const uint32_t low = run & __ballot_sync(run, hi == mh);
    if (hi == mh) {
      const uint32_t ml = __reduce_min_sync(low, lo);
      if (lane == __ffs(low) - 1) {
        const unsigned long long k = ((unsigned long long)mh << 32) | ml;
        if (k < minkey[c.a]) atomicMin(&minkey[c.a], k);
      }
    }
    if (c.key < minkey[c.b]) atomicMin(&minkey[c.b], c.key);
  }
}

__global__ void k_winner(const CEdge *__restrict__ el, int64_t m,
                         const unsigned long long *__restrict__ minkey, int32_t *__restrict__ other) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    CEdge c = el[i];
    if (minkey[c.a] == c.key) other[c.a] = c.b;
    if (minkey[c.b] == c.key) other[c.b] = c.a;
  }
}

// Hook every representative to the component across its minimum edge.  The
// chosen keys are appended with one atomicAdd per warp.
__global__ void k_hook(const int32_t *__restrict__ reps, int64_t nr,
                       unsigned long long *__restrict__ minkey, const int32_t *__restrict__ other,
                       int32_t *__restrict__ parent, uint64_t *__restrict__ mst_keys,
                       unsigned long long *__restrict__ mst_count, int64_t cap) {
  const int lane = lane_id();
  for (int64_t t0 = (int64_t)blockIdx.x * blockDim.x; t0 < nr; t0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = t0 + threadIdx.x;
    bool emit = false;
    unsigned long long mk = ~0ull;
    if (t < nr) {
      const int32_t v = reps[t];
      mk = minkey[v];
      if (mk != ~0ull) {
        const int32_t o = other[v];
        const bool mutual = other[o] == v;
        parent[v] = (mutual && v < o) ? v : o;
        emit = !(mutual && v > o);
      }
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, emit);
    unsigned long long base = 0;
    if (lane == 0 && bal) base = atomicAdd(mst_count, (unsigned long long)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (emit) {
      const unsigned long long idx = base + __popc(bal & lanemask_lt());
      if ((int64_t)idx < cap) mst_keys[idx] = mk;
    }
  }
}

__global__ void k_reset_minkey(const int32_t *__restrict__ reps, int64_t nr,
                               unsigned long long *__restrict__ minkey) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nr;
       t += (int64_t)gridDim.x * blockDim.x)
    minkey[reps[t]] = ~0ull;
}

// Pointer jumping to the roots (concurrent halving: every write moves a
// pointer up its own tree, so each thread's walk ends at its root).
__global__ void k_jump(const int32_t *__restrict__ reps, int64_t nr, int32_t *parent,
                       uint32_t *err) {
  volatile int32_t *vp = parent;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nr;
       t += (int64_t)gridDim.x * blockDim.x) {
    int32_t v = reps[t];
    int32_t p = vp[v];
    int64_t steps = 0;
    while (true) {
      int32_t gp = vp[p];
      if (gp == p) break;
      vp[v] = gp;
      p = gp;
      if (++steps > nr) {  // a forest path is shorter than the node count
        atomicOr(err, DEVERR_TIMEOUT);
        break;
      }
    }
  }
}

// Relabel both endpoints to their new roots and keep the edges that still
// join two components (order does not matter).  Each thread takes kRfItems
// edges per tile, so their parent gathers are in flight together, and the
// block reserves its output with one atomicAdd per tile: the count is a single
// address, and one atomic per warp serialised on it at the first rounds' edge
// counts.
constexpr int kRfItems = 4, kRfThreads = 256;
__global__ void __launch_bounds__(kRfThreads)
    k_relabel_filter(const CEdge *__restrict__ el, int64_t m, const int32_t *__restrict__ parent,
                     CEdge *__restrict__ out, unsigned long long *__restrict__ out_count) {
  __shared__ uint32_t wofs[kRfThreads / 32];
  __shared__ unsigned long long bbase;
  const int lane = lane_id(), w = threadIdx.x >> 5;
  const int64_t tile = (int64_t)kRfThreads * kRfItems;
  for (int64_t t0 = (int64_t)blockIdx.x * tile; t0 < m; t0 += (int64_t)gridDim.x * tile) {
    CEdge c[kRfItems];
    bool keep[kRfItems];
#pragma unroll
    for (int j = 0; j < kRfItems; j++) {
      const int64_t i = t0 + (int64_t)j * kRfThreads + threadIdx.x;
      keep[j] = i < m;
      if (keep[j]) c[j] = el[i];
    }
#pragma unroll
    for (int j = 0; j < kRfItems; j++) {
      if (keep[j]) {
        c[j].a = parent[c[j].a];
        c[j].b = parent[c[j].b];
        keep[j] = c[j].a != c[j].b;
      }
    }
    uint32_t bal[kRfItems];
    uint32_t cnt = 0;
#pragma unroll
    for (int j = 0; j < kRfItems; j++) {
      bal[j] = __ballot_sync(0xffffffffu, keep[j]);
      cnt += __popc(bal[j]);
    }
    if (lane == 0) wofs[w] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t tot = 0;
      for (int k = 0; k < kRfThreads / 32; k++) {
        const uint32_t v = wofs[k];
        wofs[k] = tot;
        tot += v;
      }
      bbase = tot ? atomicAdd(out_count, (unsigned long long)tot) : 0ull;
    }
    __syncthreads();
    unsigned long long p = bbase + wofs[w];
#pragma unroll
    for (int j = 0; j < kRfItems; j++) {
      if (keep[j]) out[p + __popc(bal[j] & lanemask_lt())] = c[j];
      p += __popc(bal[j]);
    }
    __syncthreads();  // wofs and bbase are rewritten by the next tile
  }
}

__global__ void k_roots(const int32_t *__restrict__ reps, int64_t nr,
                        const int32_t *__restrict__ parent, int32_t *__restrict__ out,
                        unsigned long long *__restrict__ count) {
  const int lane = lane_id();
  for (int64_t t0 = (int64_t)blockIdx.x * blockDim.x; t0 < nr; t0 += (int64_t)gridDim.x * blockDim.x) {
    int64_t t = t0 + threadIdx.x;
    int32_t v = 0;
    bool keep = false;
    if (t < nr) {
      v = reps[t];
      keep = parent[v] == v;
    }
    uint32_t bal = __ballot_sync(0xffffffffu, keep);
    unsigned long long base = 0;
    if (lane == 0 && bal) base = atomicAdd(count, (unsigned long long)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (keep) out[base + __popc(bal & lanemask_lt())] = v;
  }
}

__device__ __forceinline__ int32_t row_of(const int64_t *__restrict__ nindex, int64_t n, int64_t j) {
  int64_t lo = 0, hi = n - 1;  // largest r with nindex[r] <= j
  while (lo < hi) {
    int64_t mid = (lo + hi + 1) >> 1;
    if (nindex[mid] <= j) lo = mid; else hi = mid - 1;
  }
  return (int32_t)lo;
}

// quant (optional): write the dequantised weight (buildMST_gpu).
__global__ void k_gather_mst(const uint64_t *__restrict__ keys, int64_t m,
                             const int64_t *__restrict__ nindex, const int32_t *__restrict__ nlist,
                             const float *__restrict__ ew, int64_t n, const double *__restrict__ quant,
                             Segments seg, hdb_mst_edge *__restrict__ out,
                             uint8_t *__restrict__ in_mst) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = (uint32_t)keys[t];
    hdb_mst_edge e;
    e.from_node = row_of(nindex, n, j);
    e.to_node = nlist[j];
    if (quant) {
      const double p10 = quant[seg.count > 0 ? seg.of_point(e.from_node) : 0];
      e.weight = dequantise(quantise(ew[j], p10), p10);
    } else {
      e.weight = ew[j];
    }
    out[t] = e;
    if (in_mst) in_mst[j] = 1;
  }
}

// mst_gpu = 1 output order: buildMST_gpu lists the tree in CSR order and
// sort_edges sorts it stably by the dequantised weight, i.e. by (weight, edge
// index).  Re-key the chosen edges that way.
__global__ void k_quant_rekey(uint64_t *__restrict__ keys, int64_t m,
                              const int64_t *__restrict__ nindex, const float *__restrict__ ew,
                              int64_t n, const double *__restrict__ quant, Segments seg) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = (uint32_t)keys[t];
    const double p10 = quant[seg.count > 0 ? seg.of_point(row_of(nindex, n, j)) : 0];
    keys[t] = ((uint64_t)weight_key(dequantise(quantise(ew[j], p10), p10)) << 32) | (uint64_t)j;
  }
}

__global__ void k_edge_keys(const hdb_mst_edge *__restrict__ e, int64_t m, uint32_t *__restrict__ keys,
                            uint32_t *__restrict__ vals) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
       t += (int64_t)gridDim.x * blockDim.x) {
    keys[t] = weight_key(e[t].weight);
    vals[t] = (uint32_t)t;
  }
}

__global__ void k_edge_instance(const hdb_mst_edge *__restrict__ e, int64_t m, Segments seg,
                                uint32_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
       t += (int64_t)gridDim.x * blockDim.x) {
    keys[t] = (uint32_t)seg.of_point(e[t].from_node);
    vals[t] = (uint32_t)t;
  }
}

// Chosen MST edges per instance (the key's low half is the CSR edge index).
__global__ void k_count_inst_edges(const uint64_t *__restrict__ keys, int64_t m,
                                   const int64_t *__restrict__ nindex, int64_t n, Segments seg,
                                   int32_t *__restrict__ cnt) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
       t += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&cnt[seg.of_point(row_of(nindex, n, (uint32_t)keys[t]))], 1);
}

__global__ void k_permute_edges(const hdb_mst_edge *__restrict__ in, const uint32_t *__restrict__ idx,
                                int64_t m, hdb_mst_edge *__restrict__ out) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
       t += (int64_t)gridDim.x * blockDim.x)
    out[t] = in[idx[t]];
}

}  // namespace

void quant_scales(Context *ctx, const float *first, int64_t stride, int64_t n, const Segments &seg,
                  double *p10_dev, int32_t *mult_out) {
  cudaStream_t st = ctx->stream;
  const int32_t T = seg.count > 0 ? seg.count : 1;
  Buf<uint32_t> minbits(ctx, T);
  Buf<float> row0(ctx, T);
  std::vector<uint32_t> hb((size_t)T, 0x7f800000u);  // +inf: no positive distance
  HDB_CUDA(cudaMemcpyAsync(minbits, hb.data(), T * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  k_first_min<<<grid_for(ctx, n, 256), 256, 0, st>>>(first, stride, n, seg, minbits); ctx->launches++;
  k_first_rows<<<grid_for(ctx, T, 256), 256, 0, st>>>(first, stride, seg, row0); ctx->launches++;
  HDB_CHECK_LAUNCH();
  std::vector<float> h0((size_t)T);
  HDB_CUDA(cudaMemcpyAsync(hb.data(), minbits, T * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  HDB_CUDA(cudaMemcpyAsync(h0.data(), row0, T * sizeof(float), cudaMemcpyDeviceToHost, st));
  ctx->sync();
  std::vector<double> p10((size_t)T);
  for (int32_t t = 0; t < T; t++) {
    // GetMinDistanceFromKNNG (filetool.hpp:318-336): start at 999, the first
    // row's distance replaces it when positive, later ones when smaller
    double m = h0[t] > 0.0f ? (double)h0[t] : 999.0;
    float later;
    memcpy(&later, &hb[t], sizeof(float));
    if ((double)later < m) m = (double)later;
    // buildGPUgraph (core-sg.cu:13, 35): m = ceil(-log10|min|) + 2, 10^m
    const int32_t mult = (int32_t)(std::ceil(-std::log10(std::fabs(m))) + 2);
    p10[t] = std::pow(10.0, mult);
    if (mult_out) mult_out[t] = mult;
  }
  HDB_CUDA(cudaMemcpyAsync(p10_dev, p10.data(), T * sizeof(double), cudaMemcpyHostToDevice, st));
  ctx->sync();
}

int64_t boruvka_mst(Context *ctx, const hdb_graph *g, uint8_t *in_mst, hdb_mst_edge *mst,
                    int32_t *rounds_out, const Segments &seg, int32_t *inst_edges,
                    const double *quant, bool id_order) {
  const int64_t n = g->nodes;
  HDB_REQUIRE(n >= 2, HDB_ERR_ARG, "MST: need at least 2 nodes");
  HDB_REQUIRE(!(id_order && quant), HDB_ERR_ARG,
              "MST: the (weight, min id, max id) order is a float-weight mode");
  // one tree per instance: n - (number of instances) edges
  const int64_t me = n - (seg.count > 0 ? seg.count : 1);
  HDB_REQUIRE(g->edges < (int64_t(1) << 32), HDB_ERR_ARG, "MST: 2^32 or more edges");
  cudaStream_t st = ctx->stream;
  const int gw = grid_for(ctx, n, kWarps);
  Buf<int32_t> cnt(ctx, n);
  Buf<int64_t> off(ctx, n + 1);
  k_count_canon<<<gw, 32 * kWarps, 0, st>>>(g->nindex, g->nlist, n, cnt, ctx->dev_err); ctx->launches++;
  HDB_CHECK_LAUNCH();
  HDB_REQUIRE(!(ctx->take_dev_err() & DEVERR_ID_RANGE), HDB_ERR_ARG,
              "MST: graph has a neighbour id outside [0, nodes)");
  scan_exclusive_i32_i64(ctx, cnt, off, n, off.get() + n);
  int64_t *h = static_cast<int64_t *>(ctx->pinned);
  HDB_CUDA(cudaMemcpyAsync(h, off.get() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  ctx->sync();
  int64_t m = h[0];
  Buf<CEdge> el(ctx, m > 0 ? m : 1), el2(ctx, m > 0 ? m : 1);
  Buf<uint32_t> eidx;  // id order: the edge index of every rank
  if (id_order) {
    int bits = 1;
    while (bits < 31 && (int64_t(1) << bits) < n) bits++;
    eidx = Buf<uint32_t>(ctx, m > 0 ? m : 1);
    Buf<uint64_t> pair(ctx, m > 0 ? m : 1);
    k_emit_pairs<<<gw, 32 * kWarps, 0, st>>>(g->nindex, g->nlist, off, n, bits, pair, eidx); ctx->launches++;
    HDB_CHECK_LAUNCH();
    radix_sort_u64(ctx, pair, eidx, m, 0, 2 * bits);
    k_emit_ranked<<<grid_for(ctx, m > 0 ? m : 1, 256), 256, 0, st>>>(pair, eidx, g->eweight, m, bits,
                                                                     el); ctx->launches++;
  } else {
    k_emit_canon<<<gw, 32 * kWarps, 0, st>>>(g->nindex, g->nlist, g->eweight, off, n, quant, seg, el); ctx->launches++;
  }
  HDB_CHECK_LAUNCH();

  Buf<unsigned long long> minkey(ctx, n);
  Buf<int32_t> other(ctx, n), parent(ctx, n), reps(ctx, n), reps2(ctx, n);
  Buf<uint64_t> keys(ctx, n);
  Buf<unsigned long long> counters(ctx, 4);  // [0] mst edges, [1] live edges, [2] reps
  HDB_CUDA(cudaMemsetAsync(minkey, 0xff, n * sizeof(unsigned long long), st));
  HDB_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), st));
  const int gn = grid_for(ctx, n, 256);
  k_iota<<<gn, 256, 0, st>>>(parent, n); ctx->launches++;
  k_iota<<<gn, 256, 0, st>>>(reps, n); ctx->launches++;
  HDB_CHECK_LAUNCH();
  int64_t nr = n;
  int rounds = 0;
  int32_t *rp = reps, *rp2 = reps2;
  CEdge *ep = el, *ep2 = el2;
  while (m > 0) {
    HDB_REQUIRE(rounds < 64, HDB_ERR_INTERNAL, "MST: Boruvka did not converge");
    rounds++;
    const int ge = grid_for(ctx, m, 256);
    const int gr = grid_for(ctx, nr, 256);
    k_min_edge<<<ge, 256, 0, st>>>(ep, m, minkey); ctx->launches++;
    k_winner<<<ge, 256, 0, st>>>(ep, m, minkey, other); ctx->launches++;
    k_hook<<<gr, 256, 0, st>>>(rp, nr, minkey, other, parent, keys, counters, me); ctx->launches++;
    k_reset_minkey<<<gr, 256, 0, st>>>(rp, nr, minkey); ctx->launches++;
    k_jump<<<gr, 256, 0, st>>>(rp, nr, parent, ctx->dev_err); ctx->launches++;
    HDB_CUDA(cudaMemsetAsync(counters.get() + 1, 0, 2 * sizeof(unsigned long long), st));
    k_relabel_filter<<<grid_for(ctx, (m + kRfItems - 1) / kRfItems, kRfThreads), kRfThreads, 0, st>>>(
        ep, m, parent, ep2, counters.get() + 1); ctx->launches++;
    k_roots<<<gr, 256, 0, st>>>(rp, nr, parent, rp2, counters.get() + 2); ctx->launches++;
    HDB_CHECK_LAUNCH();
    HDB_CUDA(cudaMemcpyAsync(h, counters, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    ctx->sync();
    m = h[1];
    nr = h[2];
    HDB_REQUIRE(!(ctx->take_dev_err() & DEVERR_TIMEOUT), HDB_ERR_INTERNAL,
                "MST: pointer jumping exceeded its bound");
    std::swap(ep, ep2);
    std::swap(rp, rp2);
  }
  if (rounds == 0) {
    HDB_CUDA(cudaMemcpyAsync(h, counters, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    ctx->sync();
  }
  const int64_t chosen = h[0];
  if (id_order && chosen > 0 && chosen <= me) {
    // sorted by (weight, rank) now; the low halves become edge indices after
    radix_sort_u64(ctx, keys, nullptr, chosen, 0, 64);
    k_rank_to_edge<<<grid_for(ctx, chosen, 256), 256, 0, st>>>(keys, chosen, eidx); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  if (inst_edges && seg.count > 0) {
    // a forest that may miss edges: report each instance's count instead
    HDB_REQUIRE(chosen <= me, HDB_ERR_INTERNAL, "MST: more edges than points");
    Buf<int32_t> cnt(ctx, seg.count);
    HDB_CUDA(cudaMemsetAsync(cnt, 0, seg.count * sizeof(int32_t), st));
    if (chosen > 0) {
      k_count_inst_edges<<<grid_for(ctx, chosen, 256), 256, 0, st>>>(keys, chosen, g->nindex, n,
                                                                      seg, cnt); ctx->launches++;
      HDB_CHECK_LAUNCH();
    }
    HDB_CUDA(cudaMemcpyAsync(inst_edges, cnt, seg.count * sizeof(int32_t), cudaMemcpyDeviceToHost,
                             st));
    ctx->sync();
  } else {
    HDB_REQUIRE(chosen == me, HDB_ERR_DISCONNECTED,
                seg.count > 0
                    ? "MST forest does not have n - instances edges: an instance's enhanced kNN "
                      "graph is disconnected"
                    : "MST does not have n-1 edges: the enhanced kNN graph is disconnected");
  }
  if (in_mst) HDB_CUDA(cudaMemsetAsync(in_mst, 0, g->edges, st));
  if (chosen == 0) {
    if (rounds_out) *rounds_out = rounds;
    return 0;
  }
  const int gm = grid_for(ctx, chosen, 256);
  if (quant) {
    k_quant_rekey<<<gm, 256, 0, st>>>(keys, chosen, g->nindex, g->eweight, n, quant, seg); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  if (!id_order) radix_sort_u64(ctx, keys, nullptr, chosen, 0, 64);
  if (seg.count > 1) {
    // each instance's edges together, in (weight, edge index) order inside it
    Buf<hdb_mst_edge> tmp(ctx, chosen);
    k_gather_mst<<<gm, 256, 0, st>>>(keys, chosen, g->nindex, g->nlist, g->eweight, n, quant, seg,
                                     tmp, in_mst); ctx->launches++;
    Buf<uint32_t> ikeys(ctx, chosen), idx(ctx, chosen);
    k_edge_instance<<<gm, 256, 0, st>>>(tmp, chosen, seg, ikeys, idx); ctx->launches++;
    HDB_CHECK_LAUNCH();
    int bits = 1;
    while (bits < 31 && (int64_t(1) << bits) < seg.count) bits++;
    radix_sort_u32(ctx, ikeys, idx, chosen, 0, bits);
    k_permute_edges<<<gm, 256, 0, st>>>(tmp, idx, chosen, mst); ctx->launches++;
  } else {
    k_gather_mst<<<gm, 256, 0, st>>>(keys, chosen, g->nindex, g->nlist, g->eweight, n, quant, seg,
                                     mst, in_mst); ctx->launches++;
  }
  HDB_CHECK_LAUNCH();
  ctx->sync();
  if (rounds_out) *rounds_out = rounds;
  return chosen;
}

void sort_mst_edges(Context *ctx, hdb_mst_edge *edges, int64_t m) {
  if (m <= 1) return;
  cudaStream_t st = ctx->stream;
  Buf<uint32_t> keys(ctx, m), idx(ctx, m);
  Buf<hdb_mst_edge> tmp(ctx, m);
  const int g = grid_for(ctx, m, 256);
  k_edge_keys<<<g, 256, 0, st>>>(edges, m, keys, idx); ctx->launches++;
  HDB_CHECK_LAUNCH();
  radix_sort_u32(ctx, keys, idx, m, 0, 32);
  HDB_CUDA(cudaMemcpyAsync(tmp, edges, m * sizeof(hdb_mst_edge), cudaMemcpyDeviceToDevice, st));
  k_permute_edges<<<g, 256, 0, st>>>(tmp, idx, m, edges); ctx->launches++;
  HDB_CHECK_LAUNCH();
  ctx->sync();
}

}  // namespace hdb
