// Enhanced kNN graph: in-degrees, antihub selection, the symmetric CSR with
// the antihub clique, core distances and mutual-reachability weights.
//
// Reference: buildEnhancedKNNG / buildECLgraph (HDBSCAN/graphs/graph.cu:16-176)
// with calculate_degrees (calculates.cu:448-473, counts/count.cu:10-110),
// calculate_nindex / calculate_nlist (calculates.cu:286-410),
// calculateCoreDistance (calculates.cu:185-197), calculateMRD (:61-82) and
// calculate_coreDistance_antihubs (:412-446).  The reference does these as
// serial host loops plus sharded 3-GPU kernels; here every step is a
// single-device pass over HBM-resident arrays.
#include <vector>

#include "hdb_internal.cuh"
#include "graph.cuh"

namespace hdb {

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kDegHistBins = 65536;

// Squared-free sqrt-L2 with the reference's rounding (build_kNNG.cu:4-13,
// calculates.cu:275-283): float accumulator, each term pow(float diff, 2)
// evaluated in double, sqrt of the float sum.
__device__ __forceinline__ float euclid_ref(const float *__restrict__ a,
                                           const float *__restrict__ b, int d) {
  float soma = 0.0f;
  for (int i = 0; i < d; i++) {
    float diff = __fsub_rn(a[i], b[i]);
    double sq = __dmul_rn((double)diff, (double)diff);
    soma = __double2float_rn(__dadd_rn((double)soma, sq));
  }
  return __fsqrt_rn(soma);
}

// One warp per row: validate the row (range, self, duplicates) and count
// in-degrees (countValues, count.cu:10-19).
// With instances, ids must stay inside the row's instance.
__global__ void k_degrees(const int32_t *__restrict__ ids, int64_t n, int k, Segments seg,
                          int32_t *__restrict__ deg, uint32_t *err) {
  const int lane = lane_id();
  int64_t row = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int64_t stride = (int64_t)gridDim.x * kWarpsPerBlock;
  for (; row < n; row += stride) {
    int32_t v = lane < k ? ids[row * k + lane] : -1 - lane;
    int64_t lo = 0, hi = n;
    if (seg.count > 0) {
      const int32_t t = seg.of_point(row);
      lo = seg.off[t];
      hi = seg.off[t + 1];
    }
    uint32_t bad = 0;
    if (lane < k) {
      if (v < lo || v >= hi) bad |= DEVERR_ID_RANGE;
      else if (v == row) bad |= DEVERR_SELF_ID;
    }
    uint32_t peers = __match_any_sync(0xffffffffu, v);
    if (lane < k && __popc(peers) > 1) bad |= DEVERR_DUP_ID;
    if (bad) atomicOr(err, bad);
    else if (lane < k) atomicAdd(&deg[v], 1);
  }
}

// Histogram of degrees (clamped to the last bin), warp-aggregated.
__global__ void k_degree_hist(const int32_t *__restrict__ deg, int64_t n,
                              uint32_t *__restrict__ hist) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i - threadIdx.x < n; i += stride) {
    bool ok = i < n;
    int v = ok ? min(deg[i], kDegHistBins - 1) : -1;
    uint32_t peers = __match_any_sync(0xffffffffu, v);
    if (ok && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[v], __popc(peers));
  }
}

// Finds the threshold degree T = the P-th smallest degree.  out[0] = T,
// out[1] = #{deg < T}, out[2] = #{deg == T}.  One block of 1024 threads, each
// owning a chunk of 64 bins.
__global__ void k_find_threshold(const uint32_t *__restrict__ hist, int64_t P, int64_t *out) {
  __shared__ int64_t chunk_sum[1024];
  const int per = kDegHistBins / 1024;
  int64_t s = 0;
  for (int b = 0; b < per; b++) s += hist[threadIdx.x * per + b];
  chunk_sum[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t cum = 0;
    int c = 0;
    while (c < 1024 && cum + chunk_sum[c] < P) cum += chunk_sum[c++];
    int64_t T = -1, below = 0, at = 0;
    if (c < 1024) {
      for (int b = c * per; b < (c + 1) * per; b++) {
        if (cum + (int64_t)hist[b] >= P) {
          T = b;
          below = cum;
          at = hist[b];
          break;
        }
        cum += hist[b];
      }
    }
    out[0] = T;
    out[1] = below;
    out[2] = at;
  }
}

__global__ void k_flag_eq(const int32_t *__restrict__ deg, int64_t n, int32_t T,
                          int32_t *__restrict__ flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = deg[i] == T;
}

// Tied vertices (deg == T) in index order with calculateScore's tie score
// (calculates.cu:21-36): sum of the neighbours' degrees.
__global__ void k_tie_keys(const int32_t *__restrict__ deg, const int32_t *__restrict__ flag,
                           const int64_t *__restrict__ pos, const int32_t *__restrict__ ids,
                           int64_t n, int k, uint64_t *__restrict__ keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    int32_t score = 0;
    for (int j = 0; j < k; j++) score += deg[ids[i * k + j]];
    keys[pos[i]] = ((uint64_t)(uint32_t)score << 32) | (uint64_t)(uint32_t)i;
  }
}

__global__ void k_mark_selected_ties(const uint64_t *__restrict__ keys, int64_t missing,
                                     int32_t *__restrict__ is_ah) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < missing;
       t += (int64_t)gridDim.x * blockDim.x)
    is_ah[(uint32_t)keys[t]] = 1;
}

__global__ void k_flag_below(const int32_t *__restrict__ deg, int64_t n, int32_t T,
                             int32_t *__restrict__ is_ah, int all_ties) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    is_ah[i] = deg[i] < T || (all_ties && deg[i] == T);
}

__global__ void k_compact_flags(const int32_t *__restrict__ flag, const int64_t *__restrict__ pos,
                                int64_t n, int32_t *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (flag[i]) out[pos[i]] = (int32_t)i;
}

// ---- antihubs of independent instances -----------------------------------
// Every instance takes its own floor(sqrt(n_t)) lowest in-degrees, ties at the
// threshold by (score, index) -- the set the single-instance selection picks
// on that instance alone, since that order is (degree, score, index).
// Sort key: instance << 32 | degree, value: point.  The stable sort keeps
// equal keys in index order.
__global__ void k_seg_deg_keys(const int32_t *__restrict__ deg, int64_t n, Segments seg,
                               uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    keys[i] = ((uint64_t)seg.of_point(i) << 32) | (uint32_t)deg[i];
    vals[i] = (uint32_t)i;
  }
}

struct AhRun {
  int64_t lb, ub;   // sorted positions of the instance's threshold-degree run
  int64_t missing;  // how many of the run are antihubs
  int32_t ties;     // 1: the run is longer than that -> (score, index) tie-break
  int32_t pad;
};

// One thread per instance t: P_t = ah_off[t+1] - ah_off[t] antihubs; the P_t-th
// smallest key of the instance's sorted range [off[t], off[t+1]) fixes the
// threshold degree and its run [lb, ub).
__global__ void k_seg_threshold(const uint64_t *__restrict__ keys, Segments seg,
                                const int64_t *__restrict__ ah_off, AhRun *__restrict__ run) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < seg.count;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = seg.off[t], b = seg.off[t + 1];
    const int64_t P = ah_off[t + 1] - ah_off[t];
    const uint64_t kT = keys[a + P - 1];
    int64_t lo = a, hi = a + P - 1;  // first position with key == kT
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < kT) lo = mid + 1; else hi = mid;
    }
    const int64_t lb = lo;
    lo = a + P - 1;
    hi = b;  // first position with key > kT
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (keys[mid] <= kT) lo = mid + 1; else hi = mid;
    }
    AhRun r;
    r.lb = lb;
    r.ub = lo;
    r.missing = P - (lb - a);
    r.ties = (lo - lb) > r.missing ? 1 : 0;
    r.pad = 0;
    run[t] = r;
  }
}

// Per sorted position: below the run -> antihub; in a run that fits -> antihub;
// in a run that does not -> a tie, decided by (score, index).
__global__ void k_seg_mark(const uint64_t *__restrict__ keys, const uint32_t *__restrict__ vals,
                           int64_t n, const AhRun *__restrict__ run, int32_t *__restrict__ is_ah,
                           int32_t *__restrict__ tie) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const AhRun r = run[keys[p] >> 32];
    const bool in_run = p >= r.lb && p < r.ub;
    is_ah[vals[p]] = (p < r.lb || (in_run && !r.ties)) ? 1 : 0;
    tie[p] = in_run && r.ties;
  }
}

// Tied points in sorted-position order with calculateScore's tie score
// (calculates.cu:21-36), as k_tie_keys computes it.
__global__ void k_seg_tie_keys(const uint32_t *__restrict__ vals, const int32_t *__restrict__ tie,
                               const int64_t *__restrict__ tpos, int64_t n,
                               const int32_t *__restrict__ deg, const int32_t *__restrict__ ids,
                               int k, uint64_t *__restrict__ tkeys, uint32_t *__restrict__ tvals) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    if (!tie[p]) continue;
    const uint32_t i = vals[p];
    int32_t score = 0;
    for (int j = 0; j < k; j++) score += deg[ids[(int64_t)i * k + j]];
    tkeys[tpos[p]] = ((uint64_t)(uint32_t)score << 32) | (uint64_t)i;
    tvals[tpos[p]] = i;
  }
}

__global__ void k_seg_tie_inst(const uint32_t *__restrict__ tvals, int64_t cnt, Segments seg,
                               uint32_t *__restrict__ tinst) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < cnt;
       q += (int64_t)gridDim.x * blockDim.x)
    tinst[q] = (uint32_t)seg.of_point(tvals[q]);
}

// Ties sorted by (instance, score, index): the first `missing` of each
// instance's run are antihubs.  The run of instance t starts where its first
// tie sits in the position-ordered tie list.
__global__ void k_seg_tie_select(const uint32_t *__restrict__ tinst, const uint32_t *__restrict__ tvals,
                                 int64_t cnt, const AhRun *__restrict__ run,
                                 const int64_t *__restrict__ tpos, int32_t *__restrict__ is_ah) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < cnt;
       q += (int64_t)gridDim.x * blockDim.x) {
    const AhRun r = run[tinst[q]];
    if (q - tpos[r.lb] < r.missing) is_ah[tvals[q]] = 1;
  }
}

// One warp per row i: which of i's neighbours list i back (findKNNlist,
// getters.cu:41-49).  Non-mutual edges i->v become reverse entries of v.
__global__ void k_mutual(const int32_t *__restrict__ ids, int64_t n, int k,
                         uint32_t *__restrict__ mutual, int32_t *__restrict__ revcnt,
                         int32_t *__restrict__ nonmutual) {
  // One warp per row: neighbour t's list is read as one coalesced segment
  // (lane = position), eight lists in flight at a time, and a vote tells
  // whether the row is in it.
  const int lane = lane_id();
  int64_t row = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int64_t stride = (int64_t)gridDim.x * kWarpsPerBlock;
  for (; row < n; row += stride) {
    const int32_t v = lane < k ? ids[row * k + lane] : 0;
    uint32_t m = 0;
    for (int t0 = 0; t0 < k; t0 += 8) {
      int32_t x[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int t = t0 + u;
        const int32_t vt = __shfl_sync(0xffffffffu, v, t & 31);
        x[u] = (t < k && lane < k) ? __ldg(ids + (int64_t)vt * k + lane) : -1;
      }
#pragma unroll
      for (int u = 0; u < 8; u++)
        if (__any_sync(0xffffffffu, x[u] == (int32_t)row)) m |= 1u << (t0 + u);
    }
    if (k < 32) m &= (1u << k) - 1u;
    if (lane < k && !((m >> lane) & 1u)) atomicAdd(&revcnt[v], 1);
    if (lane == 0) {
      mutual[row] = m;
      nonmutual[row] = k - __popc(m);
    }
  }
}

// Row length: k own ids, the reverse entries, and for an antihub the other
// antihubs of its instance.
__global__ void k_row_sizes(const int32_t *__restrict__ revcnt, const int32_t *__restrict__ is_ah,
                            int64_t n, int k, int32_t P, Segments seg,
                            const int64_t *__restrict__ ah_off, int32_t *__restrict__ sizes) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int32_t clique = 0;
    if (is_ah[i]) {
      if (seg.count > 0) {
        const int32_t t = seg.of_point(i);
        clique = (int32_t)(ah_off[t + 1] - ah_off[t]) - 1;
      } else {
        clique = P - 1;
      }
    }
    sizes[i] = k + revcnt[i] + clique;
  }
}

// Emits (v, i) for every non-mutual edge i->v in (i, j) order.
__global__ void k_emit_reverse(const int32_t *__restrict__ ids, const uint32_t *__restrict__ mutual,
                               const int64_t *__restrict__ off, int64_t n, int k,
                               uint32_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  const int lane = lane_id();
  int64_t row = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int64_t stride = (int64_t)gridDim.x * kWarpsPerBlock;
  const uint32_t valid = k >= 32 ? 0xffffffffu : ((1u << k) - 1u);
  for (; row < n; row += stride) {
    uint32_t nm = ~mutual[row] & valid;
    if (lane < k && ((nm >> lane) & 1u)) {
      int64_t p = off[row] + __popc(nm & lanemask_lt());
      keys[p] = (uint32_t)ids[row * k + lane];
      vals[p] = (uint32_t)row;
    }
  }
}

__global__ void k_core_from_dist(const float *__restrict__ dist, int64_t n, int k, int col,
                                 float *__restrict__ core) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    core[i] = dist[i * k + col];
}

// Core distance as the reference's fix_distances would give it for the k-th
// neighbour (only that entry of each row reaches the MRD weights).
// Core distance with the reference's rounding (euclid_ref) against the k-th
// neighbour: one warp per 32 rows (lane = row).  Each 32-column chunk of the
// 32 own rows and of their 32 neighbour rows is staged in shared memory by
// coalesced row-segment loads; every lane then walks its pair of rows in
// dimension order, so the sum is the same sequence as euclid_ref's.
constexpr int kCoreCols = 32, kCoreLd = kCoreCols + 1, kCoreWarps = 4;
__global__ void __launch_bounds__(32 * kCoreWarps)
    k_core_sqrt(const float *__restrict__ X, const int32_t *__restrict__ ids, int64_t n, int d, int k,
                int col, float *__restrict__ core) {
  __shared__ float stage[kCoreWarps][2][32 * kCoreLd];
  const int lane = lane_id(), w = threadIdx.x >> 5;
  float *own = stage[w][0], *nb = stage[w][1];
  for (int64_t r0 = ((int64_t)blockIdx.x * kCoreWarps + w) * 32; r0 < n;
       r0 += (int64_t)gridDim.x * kCoreWarps * 32) {
    const int64_t row = r0 + lane;
    const bool active = row < n;
    const uint32_t act = __ballot_sync(0xffffffffu, active);
    const int32_t v = active ? ids[row * k + col] : 0;
    float soma = 0.0f;
    for (int c0 = 0; c0 < d; c0 += kCoreCols) {
      const int wd = min(kCoreCols, d - c0);
      __syncwarp();
      // eight rows' segments (own and neighbour) loaded before any is stored,
      // so sixteen loads of the warp are in flight at a time
      for (int i0 = 0; i0 < 32; i0 += 8) {
        float xo[8], xn[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int i = i0 + u;
          const int32_t vi = __shfl_sync(0xffffffffu, v, i);
          const bool ok = ((act >> i) & 1u) && lane < wd;
          xo[u] = ok ? X[(r0 + i) * d + c0 + lane] : 0.0f;
          xn[u] = ok ? X[(int64_t)vi * d + c0 + lane] : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          own[(i0 + u) * kCoreLd + lane] = xo[u];
          nb[(i0 + u) * kCoreLd + lane] = xn[u];
        }
      }
      __syncwarp();
      if (active) {
        const float *a = own + lane * kCoreLd, *b = nb + lane * kCoreLd;
        for (int j = 0; j < wd; j++) {
          const float diff = __fsub_rn(a[j], b[j]);
          const double sq = __dmul_rn((double)diff, (double)diff);
          soma = __double2float_rn(__dadd_rn((double)soma, sq));
        }
      }
    }
    if (active) core[row] = __fsqrt_rn(soma);
  }
}

__device__ __forceinline__ float mrd(float a, float b) { return a > b ? a : b; }

// One warp per row: own kNN ids, then the sorted reverse entries, with MRD
// weights (calculate_nlist calculates.cu:340-390, calculateMRD :61-82).
__global__ void k_fill(const int32_t *__restrict__ ids, const float *__restrict__ core,
                       const int64_t *__restrict__ nindex, const int32_t *__restrict__ revcnt,
                       const int64_t *__restrict__ rev_off, const uint32_t *__restrict__ rev_src,
                       int64_t n, int k, int32_t *__restrict__ nlist,
                       float *__restrict__ eweight) {
  const int lane = lane_id();
  int64_t row = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int64_t stride = (int64_t)gridDim.x * kWarpsPerBlock;
  for (; row < n; row += stride) {
    const int64_t base = nindex[row];
    const float cr = core[row];
    if (lane < k) {
      int32_t u = ids[row * k + lane];
      nlist[base + lane] = u;
      eweight[base + lane] = mrd(cr, core[u]);
    }
    const int32_t rc = revcnt[row];
    const int64_t ro = rev_off[row];
    for (int t = lane; t < rc; t += 32) {
      int32_t s = (int32_t)rev_src[ro + t];
      nlist[base + k + t] = s;
      eweight[base + k + t] = mrd(cr, core[s]);
    }
  }
}

__global__ void k_gather_rows(const float *__restrict__ X, const int32_t *__restrict__ rows,
                              int64_t m, int d, float *__restrict__ out) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m * d;
       t += (int64_t)gridDim.x * blockDim.x)
    out[t] = X[(int64_t)rows[t / d] * d + (t % d)];
}

// One block per antihub row: the other antihubs (of its instance) in
// ascending order with max(MRD, sqrt-L2) weights (calculate_nlist :392-407
// and calculate_coreDistance_antihubs :412-446).
__global__ void k_clique(const int32_t *__restrict__ ah, int32_t P, Segments seg,
                         const int64_t *__restrict__ ah_off, const float *__restrict__ Xah,
                         int d, const float *__restrict__ core, const int64_t *__restrict__ nindex,
                         const int32_t *__restrict__ revcnt, int k, int32_t *__restrict__ nlist,
                         float *__restrict__ eweight) {
  extern __shared__ float xa[];
  const int64_t r = blockIdx.x;
  const int32_t a = ah[r];
  int64_t lo = 0, cnt = P;
  if (seg.count > 0) {
    const int32_t t = seg.of_point(a);
    lo = ah_off[t];
    cnt = ah_off[t + 1] - lo;
  }
  const int64_t rr = r - lo;
  for (int t = threadIdx.x; t < d; t += blockDim.x) xa[t] = Xah[r * d + t];
  __syncthreads();
  const int64_t base = nindex[a] + k + revcnt[a];
  const float ca = core[a];
  for (int64_t t = threadIdx.x; t < cnt - 1; t += blockDim.x) {
    const int64_t o = lo + (t < rr ? t : t + 1);
    int32_t b = ah[o];
    float w = mrd(ca, core[b]);
    float eu = euclid_ref(xa, Xah + (int64_t)o * d, d);
    if (w < eu) w = eu;
    nlist[base + t] = b;
    eweight[base + t] = w;
  }
}

// ---- Core-SG (HDBSCAN/core-sg/core-sg.cu) -------------------------------------
// Euclidean distance (euclid_ref rounding) of m pairs (from[e], to[e]) of MST
// edges: one warp per 32 edges, rows staged like k_core_sqrt.
__global__ void __launch_bounds__(32 * kCoreWarps)
    k_edge_euclid(const float *__restrict__ X, int d, const hdb_mst_edge *__restrict__ mst, int64_t m,
                  float *__restrict__ out) {
  __shared__ float stage[kCoreWarps][2][32 * kCoreLd];
  const int lane = lane_id(), w = threadIdx.x >> 5;
  float *sa = stage[w][0], *sb = stage[w][1];
  for (int64_t e0 = ((int64_t)blockIdx.x * kCoreWarps + w) * 32; e0 < m;
       e0 += (int64_t)gridDim.x * kCoreWarps * 32) {
    const int64_t e = e0 + lane;
    const bool active = e < m;
    const uint32_t act = __ballot_sync(0xffffffffu, active);
    const int32_t a = active ? mst[e].from_node : 0, b = active ? mst[e].to_node : 0;
    float soma = 0.0f;
    for (int c0 = 0; c0 < d; c0 += kCoreCols) {
      const int wd = min(kCoreCols, d - c0);
      __syncwarp();
      for (int i = 0; i < 32; i++) {
        if (!((act >> i) & 1u)) continue;
        const int32_t ai = __shfl_sync(0xffffffffu, a, i), bi = __shfl_sync(0xffffffffu, b, i);
        if (lane < wd) {
          sa[i * kCoreLd + lane] = X[(int64_t)ai * d + c0 + lane];
          sb[i * kCoreLd + lane] = X[(int64_t)bi * d + c0 + lane];
        }
      }
      __syncwarp();
      if (active) {
        const float *x = sa + lane * kCoreLd, *y = sb + lane * kCoreLd;
        for (int j = 0; j < wd; j++) {
          const float diff = __fsub_rn(x[j], y[j]);
          const double sq = __dmul_rn((double)diff, (double)diff);
          soma = __double2float_rn(__dadd_rn((double)soma, sq));
        }
      }
    }
    if (active) out[e] = __fsqrt_rn(soma);
  }
}

// Endpoints in [0, n); incident-edge counts; the two row entries of every
// edge (to_node's first: key = row, value = 2e or 2e + 1).
__global__ void k_mst_entries(const hdb_mst_edge *__restrict__ mst, int64_t m, int64_t n,
                              int32_t *__restrict__ mdeg, uint32_t *__restrict__ keys,
                              uint32_t *__restrict__ vals, uint32_t *err) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = mst[e].from_node, b = mst[e].to_node;
    if (a < 0 || a >= n || b < 0 || b >= n) {
      atomicOr(err, DEVERR_ID_RANGE);
      keys[2 * e] = 0; vals[2 * e] = 0xffffffffu;
      keys[2 * e + 1] = 0; vals[2 * e + 1] = 0xffffffffu;
      continue;
    }
    atomicAdd(&mdeg[b], 1);
    atomicAdd(&mdeg[a], 1);
    keys[2 * e] = (uint32_t)b;
    vals[2 * e] = (uint32_t)(2 * e);
    keys[2 * e + 1] = (uint32_t)a;
    vals[2 * e + 1] = (uint32_t)(2 * e + 1);
  }
}

// Reverse entries for Core-SG: key = target row, value = the source's flat
// list index (source * k + slot), so the entry can carry dist[source][slot].
__global__ void k_emit_reverse_flat(const int32_t *__restrict__ ids, const uint32_t *__restrict__ mutual,
                                    const int64_t *__restrict__ off, int64_t n, int k,
                                    uint32_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  const int lane = lane_id();
  int64_t row = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int64_t stride = (int64_t)gridDim.x * kWarpsPerBlock;
  const uint32_t valid = k >= 32 ? 0xffffffffu : ((1u << k) - 1u);
  for (; row < n; row += stride) {
    uint32_t nm = ~mutual[row] & valid;
    if (lane < k && ((nm >> lane) & 1u)) {
      int64_t p = off[row] + __popc(nm & lanemask_lt());
      keys[p] = (uint32_t)ids[row * k + lane];
      vals[p] = (uint32_t)(row * k + lane);
    }
  }
}

__global__ void k_row_sizes_sg(const int32_t *__restrict__ revcnt, const int32_t *__restrict__ mdeg,
                               int64_t n, int k, int32_t *__restrict__ sizes) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    sizes[i] = k + revcnt[i] + mdeg[i];
}

// One warp per row: kNN ids with their distances, the non-mutual sources in
// ascending order with the source's distance, then the MST neighbours in
// edge order with the edge's Euclidean distance.
__global__ void k_fill_sg(const int32_t *__restrict__ ids, const float *__restrict__ dist,
                          const int64_t *__restrict__ nindex, const int32_t *__restrict__ revcnt,
                          const int64_t *__restrict__ rev_off, const uint32_t *__restrict__ rev_flat,
                          const int32_t *__restrict__ mdeg, const int64_t *__restrict__ m_off,
                          const uint32_t *__restrict__ m_vals, const hdb_mst_edge *__restrict__ mst,
                          const float *__restrict__ eu, int64_t n, int k,
                          int32_t *__restrict__ nlist, float *__restrict__ eweight) {
  const int lane = lane_id();
  int64_t row = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int64_t stride = (int64_t)gridDim.x * kWarpsPerBlock;
  for (; row < n; row += stride) {
    const int64_t base = nindex[row];
    if (lane < k) {
      nlist[base + lane] = ids[row * k + lane];
      eweight[base + lane] = dist[row * k + lane];
    }
    const int32_t rc = revcnt[row];
    const int64_t ro = rev_off[row];
    for (int t = lane; t < rc; t += 32) {
      const uint32_t f = rev_flat[ro + t];
      nlist[base + k + t] = (int32_t)(f / (uint32_t)k);
      eweight[base + k + t] = dist[f];
    }
    const int32_t mc = mdeg[row];
    const int64_t mo = m_off[row];
    for (int t = lane; t < mc; t += 32) {
      const uint32_t v = m_vals[mo + t];
      const int64_t e = v >> 1;
      nlist[base + k + rc + t] = (v & 1u) ? mst[e].to_node : mst[e].from_node;
      eweight[base + k + rc + t] = eu[e];
    }
  }
}

int bits_for(int64_t n) {
  int b = 0;
  while (b < 63 && (int64_t(1) << b) < n) b++;
  return b < 1 ? 1 : b;
}

}  // namespace

void core_distances(Context *ctx, const float *dist, const float *X, const int32_t *ids,
                    int64_t n, int32_t d, int32_t k, int32_t mode, float *core, int32_t col) {
  int g = grid_for(ctx, n, 256);
  if (col < 0) col = k - 1;
  HDB_REQUIRE(col < k, HDB_ERR_ARG, "core distances: column outside the kNN rows");
  if (mode == HDB_DIST_SQRT)
    k_core_sqrt<<<grid_for(ctx, (n + 31) / 32, kCoreWarps, 8), 32 * kCoreWarps, 0, ctx->stream>>>(
        X, ids, n, d, k, col, core);
  else
    k_core_from_dist<<<g, 256, 0, ctx->stream>>>(dist, n, k, col, core);
  ctx->launches++;
  HDB_CHECK_LAUNCH();
}

// Antihubs of every instance (is_ah[i] = 1 for the chosen points); see
// k_seg_deg_keys.  ah_off: device prefix sums of the per-instance counts.
static void select_antihubs_segmented(Context *ctx, const int32_t *deg, const int32_t *ids,
                                      int64_t n, int32_t k, const Segments &seg,
                                      const int64_t *ah_off, int32_t *is_ah) {
  cudaStream_t st = ctx->stream;
  const int ge = grid_for(ctx, n, 256);
  Buf<uint64_t> keys(ctx, n);
  Buf<uint32_t> vals(ctx, n);
  k_seg_deg_keys<<<ge, 256, 0, st>>>(deg, n, seg, keys, vals); ctx->launches++;
  HDB_CHECK_LAUNCH();
  radix_sort_u64(ctx, keys, vals, n, 0, 32 + bits_for(seg.count));
  Buf<AhRun> run(ctx, seg.count);
  k_seg_threshold<<<grid_for(ctx, seg.count, 128), 128, 0, st>>>(keys, seg, ah_off, run); ctx->launches++;
  Buf<int32_t> tie(ctx, n);
  k_seg_mark<<<ge, 256, 0, st>>>(keys, vals, n, run, is_ah, tie); ctx->launches++;
  HDB_CHECK_LAUNCH();
  Buf<int64_t> tpos(ctx, n + 1);
  scan_exclusive_i32_i64(ctx, tie, tpos, n, tpos.get() + n);
  int64_t *h = static_cast<int64_t *>(ctx->pinned);
  HDB_CUDA(cudaMemcpyAsync(h, tpos.get() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  ctx->sync();
  const int64_t nt = h[0];
  if (nt == 0) return;
  Buf<uint64_t> tkeys(ctx, nt);
  Buf<uint32_t> tvals(ctx, nt), tinst(ctx, nt);
  k_seg_tie_keys<<<ge, 256, 0, st>>>(vals, tie, tpos, n, deg, ids, k, tkeys, tvals); ctx->launches++;
  HDB_CHECK_LAUNCH();
  radix_sort_u64(ctx, tkeys, tvals, nt, 0, 64);
  const int gt = grid_for(ctx, nt, 256);
  k_seg_tie_inst<<<gt, 256, 0, st>>>(tvals, nt, seg, tinst); ctx->launches++;
  HDB_CHECK_LAUNCH();
  radix_sort_u32(ctx, tinst, tvals, nt, 0, bits_for(seg.count));
  k_seg_tie_select<<<gt, 256, 0, st>>>(tinst, tvals, nt, run, tpos, is_ah); ctx->launches++;
  HDB_CHECK_LAUNCH();
}

void build_enhanced_knng(Context *ctx, const int32_t *ids, const float *core, const float *X,
                         int64_t n, int32_t d, int32_t k, hdb_graph *out, GraphTimes *times,
                         const Segments &seg) {
  HDB_REQUIRE(n >= 2 && n < (int64_t(1) << 31) - 1, HDB_ERR_ARG, "enhanced kNN graph: bad n");
  HDB_REQUIRE(k >= 1 && k <= 32 && k < n, HDB_ERR_ARG, "enhanced kNN graph: k must be in [1, 32]");
  HDB_REQUIRE(d >= 1, HDB_ERR_ARG, "enhanced kNN graph: bad d");
  cudaStream_t st = ctx->stream;
  const int gw = grid_for(ctx, n, kWarpsPerBlock);
  const int ge = grid_for(ctx, n, 256);

  // 1. in-degrees + validation
  Buf<int32_t> deg(ctx, n);
  HDB_CUDA(cudaMemsetAsync(deg, 0, n * sizeof(int32_t), st));
  k_degrees<<<gw, 32 * kWarpsPerBlock, 0, st>>>(ids, n, k, seg, deg, ctx->dev_err); ctx->launches++;
  HDB_CHECK_LAUNCH();
  uint32_t err = ctx->take_dev_err();
  HDB_REQUIRE(!(err & DEVERR_ID_RANGE), HDB_ERR_ARG,
              seg.count > 0 ? "kNN graph: neighbour id outside its instance"
                            : "kNN graph: neighbour id outside [0, n)");
  HDB_REQUIRE(!(err & DEVERR_SELF_ID), HDB_ERR_ARG, "kNN graph: a row lists its own id");
  HDB_REQUIRE(!(err & DEVERR_DUP_ID), HDB_ERR_ARG, "kNN graph: an id repeats within a row");

  // 2. antihubs: the P = (int)sqrt(n) lowest degrees (get_NumThreshold,
  //    getters.cu:6-9); ties at the threshold by (score, index).  With
  //    instances, floor(sqrt(n_t)) of each.
  int64_t *h = static_cast<int64_t *>(ctx->pinned);
  int32_t P = (int32_t)sqrt((double)n);
  Buf<int32_t> is_ah(ctx, n);
  Buf<int64_t> pos(ctx, n + 1);
  Buf<int64_t> ah_off;
  int64_t P_total = P;
  if (seg.count > 0) {
    std::vector<int64_t> ho((size_t)seg.count + 1, 0);
    for (int32_t t = 0; t < seg.count; t++) {
      const int64_t nt = seg.host_off[t + 1] - seg.host_off[t];
      HDB_REQUIRE(nt > k, HDB_ERR_ARG, "enhanced kNN graph: every instance needs more than k points");
      ho[t + 1] = ho[t] + (int64_t)sqrt((double)nt);
    }
    P_total = ho[seg.count];
    ah_off = Buf<int64_t>(ctx, seg.count + 1);
    HDB_CUDA(cudaMemcpyAsync(ah_off, ho.data(), ho.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                             st));
    select_antihubs_segmented(ctx, deg, ids, n, k, seg, ah_off, is_ah);
    P = 0;  // per instance from ah_off
  } else {
    Buf<uint32_t> hist(ctx, kDegHistBins);
    Buf<int64_t> thr(ctx, 4);
    HDB_CUDA(cudaMemsetAsync(hist, 0, kDegHistBins * sizeof(uint32_t), st));
    k_degree_hist<<<ge, 256, 0, st>>>(deg, n, hist); ctx->launches++;
    HDB_CHECK_LAUNCH();
    k_find_threshold<<<1, 1024, 0, st>>>(hist, P, thr); ctx->launches++;
    HDB_CHECK_LAUNCH();
    HDB_CUDA(cudaMemcpyAsync(h, thr, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    ctx->sync();
    const int64_t T = h[0], below = h[1], at = h[2];
    HDB_REQUIRE(T >= 0 && T < kDegHistBins - 1, HDB_ERR_INTERNAL,
                "antihub threshold degree out of histogram range");
    const int64_t missing = P - below;
    Buf<int32_t> flag(ctx, n);
    k_flag_below<<<ge, 256, 0, st>>>(deg, n, (int32_t)T, is_ah, at == missing ? 1 : 0); ctx->launches++;
    HDB_CHECK_LAUNCH();
    if (at > missing) {
      k_flag_eq<<<ge, 256, 0, st>>>(deg, n, (int32_t)T, flag); ctx->launches++;
      HDB_CHECK_LAUNCH();
      scan_exclusive_i32_i64(ctx, flag, pos, n, nullptr);
      Buf<uint64_t> keys(ctx, at);
      k_tie_keys<<<ge, 256, 0, st>>>(deg, flag, pos, ids, n, k, keys); ctx->launches++;
      HDB_CHECK_LAUNCH();
      radix_sort_u64(ctx, keys, nullptr, at, 0, 64);
      k_mark_selected_ties<<<grid_for(ctx, missing, 256), 256, 0, st>>>(keys, missing, is_ah); ctx->launches++;
      HDB_CHECK_LAUNCH();
    }
  }
  ensure_capacity(ctx, (void **)&ctx->g_antihubs, &ctx->g_antihubs_cap,
                  (size_t)(P_total > 0 ? P_total : 1) * sizeof(int32_t));
  scan_exclusive_i32_i64(ctx, is_ah, pos, n, pos.get() + n);
  k_compact_flags<<<ge, 256, 0, st>>>(is_ah, pos, n, ctx->g_antihubs); ctx->launches++;
  HDB_CHECK_LAUNCH();
  if (seg.count > 0) {
    HDB_CUDA(cudaMemcpyAsync(h, pos.get() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    ctx->sync();
    HDB_REQUIRE(h[0] == P_total, HDB_ERR_INTERNAL, "antihub selection: wrong count");
  }
  if (times) HDB_CUDA(cudaEventRecord(times->after_antihubs, st));

  // 3. mutual flags and reverse counts
  Buf<uint32_t> mutual(ctx, n);
  Buf<int32_t> revcnt(ctx, n), nonmutual(ctx, n);
  HDB_CUDA(cudaMemsetAsync(revcnt, 0, n * sizeof(int32_t), st));
  k_mutual<<<gw, 32 * kWarpsPerBlock, 0, st>>>(ids, n, k, mutual, revcnt, nonmutual); ctx->launches++;
  HDB_CHECK_LAUNCH();

  // 4. row sizes -> nindex
  ensure_capacity(ctx, (void **)&ctx->g_nindex, &ctx->g_nindex_cap, (n + 1) * sizeof(int64_t));
  {
    Buf<int32_t> sizes(ctx, n);
    k_row_sizes<<<ge, 256, 0, st>>>(revcnt, is_ah, n, k, P, seg, ah_off.get(), sizes); ctx->launches++;
    HDB_CHECK_LAUNCH();
    scan_exclusive_i32_i64(ctx, sizes, ctx->g_nindex, n, ctx->g_nindex + n);
  }
  // 5. reverse entries (v, i) in i order, stable-sorted by v
  Buf<int64_t> roff(ctx, n + 1);
  scan_exclusive_i32_i64(ctx, nonmutual, roff, n, roff.get() + n);
  int64_t hv[2];
  HDB_CUDA(cudaMemcpyAsync(h, roff.get() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  HDB_CUDA(cudaMemcpyAsync(h + 1, ctx->g_nindex + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  ctx->sync();
  hv[0] = h[0];
  hv[1] = h[1];
  const int64_t R = hv[0], E = hv[1];
  HDB_REQUIRE(E < (int64_t(1) << 32), HDB_ERR_ARG,
              "enhanced kNN graph has 2^32 or more edges (edge indices are 32-bit)");
  Buf<uint32_t> rkeys(ctx, R), rvals(ctx, R);
  k_emit_reverse<<<gw, 32 * kWarpsPerBlock, 0, st>>>(ids, mutual, roff, n, k, rkeys, rvals); ctx->launches++;
  HDB_CHECK_LAUNCH();
  radix_sort_u32(ctx, rkeys, rvals, R, 0, bits_for(n));
  Buf<int64_t> rev_off(ctx, n + 1);
  scan_exclusive_i32_i64(ctx, revcnt, rev_off, n, nullptr);

  // 6. fill rows + MRD weights
  ensure_capacity(ctx, (void **)&ctx->g_nlist, &ctx->g_nlist_cap, (size_t)E * sizeof(int32_t));
  ensure_capacity(ctx, (void **)&ctx->g_eweight, &ctx->g_eweight_cap, (size_t)E * sizeof(float));
  k_fill<<<gw, 32 * kWarpsPerBlock, 0, st>>>(ids, core, ctx->g_nindex, revcnt, rev_off, rvals, n,
                                             k, ctx->g_nlist, ctx->g_eweight); ctx->launches++;
  HDB_CHECK_LAUNCH();
  if (P_total > (seg.count > 0 ? seg.count : 1)) {  // some clique has two or more members
    Buf<float> Xah(ctx, (size_t)P_total * d);
    k_gather_rows<<<grid_for(ctx, P_total * d, 256), 256, 0, st>>>(X, ctx->g_antihubs, P_total, d,
                                                                     Xah); ctx->launches++;
    HDB_CHECK_LAUNCH();
    k_clique<<<(unsigned)P_total, 256, d * sizeof(float), st>>>(
        ctx->g_antihubs, P, seg, ah_off.get(), Xah, d, core, ctx->g_nindex, revcnt, k,
        ctx->g_nlist, ctx->g_eweight); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  ctx->sync();
  out->nodes = (int32_t)n;
  out->edges = E;
  out->nindex = ctx->g_nindex;
  out->nlist = ctx->g_nlist;
  out->eweight = ctx->g_eweight;
  out->num_antihubs = (int32_t)P_total;
  out->antihubs = ctx->g_antihubs;
}


void build_core_sg(Context *ctx, const int32_t *ids, const float *dist, const float *X, int64_t n,
                   int32_t d, int32_t k, const hdb_mst_edge *mst, hdb_graph *out) {
  HDB_REQUIRE(n >= 2 && n < (int64_t(1) << 31) - 1, HDB_ERR_ARG, "core-SG: bad n");
  HDB_REQUIRE(k >= 1 && k <= 32 && k < n, HDB_ERR_ARG, "core-SG: k must be in [1, 32]");
  HDB_REQUIRE(d >= 1, HDB_ERR_ARG, "core-SG: bad d");
  HDB_REQUIRE(n * k < (int64_t(1) << 32) && 2 * (n - 1) < (int64_t(1) << 32), HDB_ERR_ARG,
              "core-SG: n * k must stay below 2^32");
  cudaStream_t st = ctx->stream;
  const int gw = grid_for(ctx, n, kWarpsPerBlock);
  const int ge = grid_for(ctx, n, 256);
  const int64_t m = n - 1;

  Buf<int32_t> deg(ctx, n);
  HDB_CUDA(cudaMemsetAsync(deg, 0, n * sizeof(int32_t), st));
  k_degrees<<<gw, 32 * kWarpsPerBlock, 0, st>>>(ids, n, k, Segments{}, deg, ctx->dev_err); ctx->launches++;
  HDB_CHECK_LAUNCH();
  // MST entries (validated with the ids)
  Buf<int32_t> mdeg(ctx, n);
  Buf<uint32_t> mkeys(ctx, 2 * m), mvals(ctx, 2 * m);
  HDB_CUDA(cudaMemsetAsync(mdeg, 0, n * sizeof(int32_t), st));
  k_mst_entries<<<grid_for(ctx, m, 256), 256, 0, st>>>(mst, m, n, mdeg, mkeys, mvals, ctx->dev_err);
  ctx->launches++;
  HDB_CHECK_LAUNCH();
  uint32_t err = ctx->take_dev_err();
  HDB_REQUIRE(!(err & DEVERR_ID_RANGE), HDB_ERR_ARG,
              "core-SG: a kNN id or an MST endpoint lies outside [0, n)");
  HDB_REQUIRE(!(err & DEVERR_SELF_ID), HDB_ERR_ARG, "kNN graph: a row lists its own id");
  HDB_REQUIRE(!(err & DEVERR_DUP_ID), HDB_ERR_ARG, "kNN graph: an id repeats within a row");
  radix_sort_u32(ctx, mkeys, mvals, 2 * m, 0, bits_for(n));  // stable: edge order within a row
  Buf<int64_t> m_off(ctx, n + 1);
  scan_exclusive_i32_i64(ctx, mdeg, m_off, n, m_off.get() + n);
  Buf<float> eu(ctx, m);
  k_edge_euclid<<<grid_for(ctx, (m + 31) / 32, kCoreWarps, 8), 32 * kCoreWarps, 0, st>>>(X, d, mst, m,
                                                                                            eu);
  ctx->launches++;
  HDB_CHECK_LAUNCH();

  // mutual flags, reverse entries sorted by target (stable: ascending source)
  Buf<uint32_t> mutual(ctx, n);
  Buf<int32_t> revcnt(ctx, n), nonmutual(ctx, n);
  HDB_CUDA(cudaMemsetAsync(revcnt, 0, n * sizeof(int32_t), st));
  k_mutual<<<gw, 32 * kWarpsPerBlock, 0, st>>>(ids, n, k, mutual, revcnt, nonmutual); ctx->launches++;
  HDB_CHECK_LAUNCH();
  Buf<int64_t> roff(ctx, n + 1);
  scan_exclusive_i32_i64(ctx, nonmutual, roff, n, roff.get() + n);
  ensure_capacity(ctx, (void **)&ctx->sg_nindex, &ctx->sg_nindex_cap, (n + 1) * sizeof(int64_t));
  {
    Buf<int32_t> sizes(ctx, n);
    k_row_sizes_sg<<<ge, 256, 0, st>>>(revcnt, mdeg, n, k, sizes); ctx->launches++;
    HDB_CHECK_LAUNCH();
    scan_exclusive_i32_i64(ctx, sizes, ctx->sg_nindex, n, ctx->sg_nindex + n);
  }
  int64_t *h = static_cast<int64_t *>(ctx->pinned);
  HDB_CUDA(cudaMemcpyAsync(h, roff.get() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  HDB_CUDA(cudaMemcpyAsync(h + 1, ctx->sg_nindex + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  ctx->sync();
  const int64_t R = h[0], E = h[1];
  Buf<uint32_t> rkeys(ctx, R), rvals(ctx, R);
  k_emit_reverse_flat<<<gw, 32 * kWarpsPerBlock, 0, st>>>(ids, mutual, roff, n, k, rkeys, rvals);
  ctx->launches++;
  HDB_CHECK_LAUNCH();
  radix_sort_u32(ctx, rkeys, rvals, R, 0, bits_for(n));
  Buf<int64_t> rev_off(ctx, n + 1);
  scan_exclusive_i32_i64(ctx, revcnt, rev_off, n, nullptr);

  ensure_capacity(ctx, (void **)&ctx->sg_nlist, &ctx->sg_nlist_cap, (size_t)E * sizeof(int32_t));
  ensure_capacity(ctx, (void **)&ctx->sg_eweight, &ctx->sg_eweight_cap, (size_t)E * sizeof(float));
  k_fill_sg<<<gw, 32 * kWarpsPerBlock, 0, st>>>(ids, dist, ctx->sg_nindex, revcnt, rev_off, rvals, mdeg,
                                                m_off, mvals, mst, eu, n, k, ctx->sg_nlist,
                                                ctx->sg_eweight);
  ctx->launches++;
  HDB_CHECK_LAUNCH();
  ctx->sync();
  out->nodes = (int32_t)n;
  out->edges = E;
  out->nindex = ctx->sg_nindex;
  out->nlist = ctx->sg_nlist;
  out->eweight = ctx->sg_eweight;
  out->num_antihubs = 0;
  out->antihubs = nullptr;
}

}  // namespace hdb
