// Single-linkage tree, condensed tree, stability, excess-of-mass selection
// and labels -- all on the device.
//
// Reference: build_Linkage_tree, build_Condensed_tree, compute_stability,
// get_clusters and do_labelling (HDBSCAN/trees/tree.cu:171-746), which run as
// serial host loops (union-find replay, BFS, per-cluster scans).
//
// Linkage tree.  Node N+r merges the two components joined by sorted MST edge
// r; its children are the components' current roots, i.e. the largest edge
// rank inside each endpoint's component among edges < r (or the vertex itself).
// Edge ranks are processed as a binary divide and conquer: at every level each
// block of ranks [s, s+S) unions its lower half with a lock-free union-find,
// tags each component with its largest rank, and relabels the endpoints of its
// upper half by those tags.  Endpoint labels seen by different blocks of one
// level are disjoint, so all blocks share one union-find array.  After log2(N)
// levels every edge's endpoint labels are exactly its two children.
//
// Condensed tree.  A node is visited by the reference's BFS iff it is the root
// or holds >= mpts points.  Chains of "one big child" nodes share a cluster; a
// node whose children are both big starts two clusters, numbered in BFS order
// (depth, then left-to-right = preorder).  Depth, preorder and chain heads come
// from pointer jumping; each point falls out at the lowest visited ancestor.
// Stability is summed per cluster in the reference's row order (chain nodes
// top-down, identical terms for the points of each small side), in FP32 with
// separate multiply/add roundings, or in FP64 when asked.
#include "hdb_internal.cuh"
#include "trees.cuh"

namespace hdb {

namespace {

// ---------------------------------------------------------------------------
// Linkage tree
// ---------------------------------------------------------------------------
// Union-find over labels [0, 2n-1); hooks always point to a larger label, so
// every path ends at a root.  Hooking the smaller root keeps the hot labels
// -- a big component's internal label n + rank, which many edges of a level
// name -- as parents: the vertices joining it each hook their own record
// instead of contending for the hot one.  The step bounds only guard against corrupted
// state and report through the device error word.  A label's state at one
// level -- parent, the largest rank tagged to it (as a root), whether it was
// counted, the points its root accumulated -- is one 16-byte record, so the
// reset of a label is one store and a root's fields share a sector.
constexpr int64_t kUfBound = int64_t(1) << 31;

struct __align__(16) UfNode {
  int32_t p, maxr, seen, acc;
};

__device__ __forceinline__ int32_t uf_find(UfNode *u, int32_t x) {
  for (int64_t s = 0; s < kUfBound; s++) {
    const int32_t px = *reinterpret_cast<volatile int32_t *>(&u[x].p);
    if (px == x) return x;
    const int32_t ppx = *reinterpret_cast<volatile int32_t *>(&u[px].p);
    if (ppx != px) *reinterpret_cast<volatile int32_t *>(&u[x].p) = ppx;
    x = px;
  }
  return x;
}

__device__ __forceinline__ void uf_union(UfNode *u, int32_t a, int32_t b, uint32_t *err) {
  for (int64_t s = 0; s < kUfBound; s++) {
    a = uf_find(u, a);
    b = uf_find(u, b);
    if (a == b) return;
    if (a < b) { int32_t t = a; a = b; b = t; }
    if (atomicCAS(&u[b].p, b, a) == b) return;
  }
  atomicOr(err, DEVERR_TIMEOUT);
}

// Lower-half edge of a block that has an upper half at block size S.
__device__ __forceinline__ bool active_lower(int64_t r, int64_t S, int64_t m) {
  int64_t pos = r & (S - 1);
  int64_t half = S >> 1;
  return pos < half && (r - pos) + half < m;
}

__global__ void k_link_init(const hdb_mst_edge *__restrict__ mst, int64_t m,
                            int32_t *__restrict__ la, int32_t *__restrict__ lb) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    la[r] = mst[r].from_node;
    lb[r] = mst[r].to_node;
  }
}

__global__ void k_uf_init(int64_t total, int64_t n, UfNode *__restrict__ u,
                          int32_t *__restrict__ size) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    u[i] = UfNode{(int32_t)i, -1, 0, 0};
    size[i] = i < n ? 1 : 0;
  }
}

__global__ void k_level_union(const int32_t *__restrict__ la, const int32_t *__restrict__ lb,
                              int64_t m, int64_t S, UfNode *u, uint32_t *err) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x)
    if (active_lower(r, S, m)) uf_union(u, la[r], lb[r], err);
}

// MST input check: endpoints in [0, n).
__global__ void k_validate_mst(const hdb_mst_edge *__restrict__ mst, int64_t m, int64_t n,
                               uint32_t *err) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    hdb_mst_edge e = mst[r];
    if (e.from_node < 0 || e.from_node >= n || e.to_node < 0 || e.to_node >= n)
      atomicOr(err, DEVERR_ID_RANGE);
  }
}

// Tags every component with its largest rank and counts its points.  At the
// upper levels most active edges of a block share one root, so the lanes that
// share the first active lane's root combine their rank maximum and point
// count with redux.sync and one of them updates the root; the other lanes
// update their own roots.
__global__ void k_level_tag(const int32_t *__restrict__ la, const int32_t *__restrict__ lb,
                            int64_t m, int64_t S, int64_t n, UfNode *u,
                            const int32_t *__restrict__ size) {
  const int lane = lane_id();
  for (int64_t r0 = (int64_t)blockIdx.x * blockDim.x; r0 < m; r0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = r0 + threadIdx.x;
    const bool act = r < m && active_lower(r, S, m);
    int32_t root = -1, add = 0;
    if (act) {
      const int32_t a = la[r], b = lb[r];
      root = uf_find(u, a);
      if (atomicExch(&u[a].seen, 1) == 0) add += a < n ? 1 : size[a];
      if (atomicExch(&u[b].seen, 1) == 0) add += b < n ? 1 : size[b];
    }
    const uint32_t am = __ballot_sync(0xffffffffu, act);
    if (!act) continue;
    const int32_t lead = __shfl_sync(am, root, __ffs(am) - 1);
    const uint32_t same = __ballot_sync(am, root == lead);
    if (root == lead) {
      const int32_t mr = __reduce_max_sync(same, (int32_t)r);
      const int32_t sum = __reduce_add_sync(same, add);
      if (lane == __ffs(same) - 1) {
        atomicMax(&u[root].maxr, mr);
        if (sum != 0) atomicAdd(&u[root].acc, sum);
      }
    } else {
      atomicMax(&u[root].maxr, (int32_t)r);
      if (add != 0) atomicAdd(&u[root].acc, add);
    }
  }
}

__global__ void k_level_produce(const int32_t *__restrict__ la, int64_t m, int64_t S, int64_t n,
                                UfNode *u, int32_t *__restrict__ size) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (!active_lower(r, S, m)) continue;
    const int32_t root = uf_find(u, la[r]);
    if (u[root].maxr == (int32_t)r) size[n + r] = u[root].acc;
  }
}

__global__ void k_level_relabel(int32_t *__restrict__ la, int32_t *__restrict__ lb, int64_t m,
                                int64_t S, int64_t n, UfNode *u) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    if ((r & (S - 1)) < (S >> 1)) continue;
    int32_t a = la[r], b = lb[r];
    int32_t ra = uf_find(u, a), rb = uf_find(u, b);
    int32_t ma = u[ra].maxr, mb = u[rb].maxr;
    if (ma >= 0) la[r] = (int32_t)(n + ma);
    if (mb >= 0) lb[r] = (int32_t)(n + mb);
  }
}

__global__ void k_level_reset(const int32_t *__restrict__ la, const int32_t *__restrict__ lb,
                              int64_t m, int64_t S, UfNode *__restrict__ u) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (!active_lower(r, S, m)) continue;
    const int32_t a = la[r], b = lb[r];
    u[a] = UfNode{a, -1, 0, 0};
    u[b] = UfNode{b, -1, 0, 0};
  }
}

__global__ void k_link_out(const hdb_mst_edge *__restrict__ mst, const int32_t *__restrict__ la,
                           const int32_t *__restrict__ lb, const int32_t *__restrict__ size,
                           int64_t m, int64_t n, hdb_linkage_node *__restrict__ out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    int32_t a = la[r], b = lb[r];
    hdb_linkage_node o;
    o.left_node = a;
    o.right_node = b;
    o.weight = mst[r].weight;
    o.node_size = (a < n ? 1 : size[a]) + (b < n ? 1 : size[b]);
    out[r] = o;
  }
}

// ---------------------------------------------------------------------------
// Condensed tree, stability, EOM, labels
// ---------------------------------------------------------------------------
enum : int8_t { KIND_SPLIT = 0, KIND_BOTHSMALL = 1, KIND_LEFTBIG = 2, KIND_RIGHTBIG = 3 };

// A single-linkage tree, or a forest with one tree per instance (seg):
// internal node n + r for rank r < m, where m = n - (number of trees).
struct TreeView {
  const hdb_linkage_node *h;
  int64_t n;  // points
  int64_t m;  // internal nodes
  int32_t mpts;
  Segments seg;
  __device__ __forceinline__ int32_t sz(int64_t x) const {
    return x < n ? 1 : h[x - n].node_size;
  }
  // Root of its tree: the last rank of the tree's instance.
  __device__ __forceinline__ bool is_root(int64_t r) const {
    if (seg.count == 0) return r == m - 1;
    const int32_t t = seg.of_rank(r);
    return r == seg.off[t + 1] - t - 2;
  }
};

__device__ __forceinline__ float lambda_of(float w) {
  // tree.cu:308-313: INFINITE = INT_MAX, else 1.0 / weight in double
  return w > 0.0f ? __double2float_rn(__drcp_rn((double)w)) : 2147483648.0f;
}

// Hierarchy input check: children are earlier nodes and sizes add up, so
// parent pointers always go to larger ids (every upward walk ends at the root).
__global__ void k_validate_hier(TreeView t, uint32_t *err) {
  const int64_t m = t.m;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    hdb_linkage_node h = t.h[r];
    int64_t lim = t.n + r;
    bool ok = h.left_node >= 0 && h.left_node < lim && h.right_node >= 0 &&
              h.right_node < lim && h.left_node != h.right_node;
    if (ok) ok = (int64_t)t.sz(h.left_node) + t.sz(h.right_node) == h.node_size;
    if (!ok) atomicOr(err, DEVERR_ID_RANGE);
  }
}

// Per internal node: parent pointers, side, kind, visited flag, lambda.
__global__ void k_nodes(TreeView t, int32_t *__restrict__ par, int8_t *__restrict__ side,
                        int8_t *__restrict__ kind, int8_t *__restrict__ visited,
                        float *__restrict__ lam) {
  const int64_t m = t.m;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    hdb_linkage_node h = t.h[r];
    int64_t x = t.n + r;
    par[h.left_node] = (int32_t)x;
    par[h.right_node] = (int32_t)x;
    side[h.left_node] = 0;
    side[h.right_node] = 1;
    bool lb = t.sz(h.left_node) >= t.mpts, rb = t.sz(h.right_node) >= t.mpts;
    kind[r] = (lb && rb) ? KIND_SPLIT : (!lb && !rb) ? KIND_BOTHSMALL : lb ? KIND_LEFTBIG : KIND_RIGHTBIG;
    visited[r] = t.is_root(r) || h.node_size >= t.mpts;
    lam[r] = lambda_of(h.weight);
  }
}

// Doubling state for visited nodes: jump pointer, depth and preorder sums,
// and the chain-head pointer.
__global__ void k_path_init(TreeView t, const int32_t *__restrict__ par, const int8_t *__restrict__ side,
                            const int8_t *__restrict__ kind, const int8_t *__restrict__ visited,
                            int32_t *__restrict__ jmp, int64_t *__restrict__ dep,
                            int64_t *__restrict__ pre, int32_t *__restrict__ head) {
  const int64_t m = t.m;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (!visited[r]) { jmp[r] = -1; head[r] = -1; continue; }
    int64_t x = t.n + r;
    if (t.is_root(r)) {
      jmp[r] = -1; dep[r] = 0; pre[r] = 0; head[r] = (int32_t)r;
      continue;
    }
    int32_t p = par[x];
    int64_t pr = p - t.n;
    jmp[r] = (int32_t)pr;
    dep[r] = 1;
    int64_t d = 1;
    if (side[x] == 1) {
      int32_t sib = t.h[pr].left_node;
      d += 2 * (int64_t)t.sz(sib) - 1;
    }
    pre[r] = d;
    int8_t pk = kind[pr];
    bool inherit = (pk == KIND_LEFTBIG && side[x] == 0) || (pk == KIND_RIGHTBIG && side[x] == 1);
    head[r] = inherit ? (int32_t)pr : (int32_t)r;
  }
}

__global__ void k_path_jump(int64_t m, const int32_t *__restrict__ jmp, const int64_t *__restrict__ dep,
                            const int64_t *__restrict__ pre, int32_t *__restrict__ jmp2,
                            int64_t *__restrict__ dep2, int64_t *__restrict__ pre2,
                            int32_t *changed) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    int32_t j = jmp[r];
    if (j < 0) { jmp2[r] = j; dep2[r] = dep[r]; pre2[r] = pre[r]; continue; }
    dep2[r] = dep[r] + dep[j];
    pre2[r] = pre[r] + pre[j];
    jmp2[r] = jmp[j];
    *changed = 1;
  }
}

__global__ void k_head_jump(int64_t m, int32_t *head, int32_t *changed) {
  volatile int32_t *vh = head;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    int32_t h = vh[r];
    if (h < 0) continue;
    int32_t hh = vh[h];
    if (hh != h) {
      vh[r] = hh;
      *changed = 1;
    }
  }
}

__global__ void k_split_keys(int64_t m, const int8_t *__restrict__ kind,
                             const int8_t *__restrict__ visited, const int64_t *__restrict__ dep,
                             const int64_t *__restrict__ pre, int32_t *__restrict__ flag) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x)
    flag[r] = visited[r] && kind[r] == KIND_SPLIT;
}

__global__ void k_split_emit(int64_t m, const int32_t *__restrict__ flag, const int64_t *__restrict__ pos,
                             const int64_t *__restrict__ dep, const int64_t *__restrict__ pre,
                             uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[r]) continue;
    keys[pos[r]] = ((uint64_t)dep[r] << 32) | (uint64_t)pre[r];
    vals[pos[r]] = (uint32_t)r;
  }
}

// Cluster ids: root = n; the t-th split node in BFS order gives n+1+2t (left)
// and n+2+2t (right).  cid is indexed by internal-node rank r (-1 otherwise).
// A forest numbers its clusters tree after tree: the splits are sorted by
// (instance, BFS order), split q of instance s gives indices s+1+2q and
// s+2+2q, and instance s's root the index just before its first split's.
__global__ void k_assign_cids(TreeView t, const uint32_t *__restrict__ split_nodes, int64_t ns,
                              const uint32_t *__restrict__ split_inst, int32_t *__restrict__ cid,
                              int32_t *__restrict__ split_rank) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < ns;
       q += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = split_nodes[q];
    const int64_t base = split_inst ? split_inst[q] : 0;
    hdb_linkage_node h = t.h[r];
    cid[h.left_node - t.n] = (int32_t)(t.n + base + 1 + 2 * q);
    cid[h.right_node - t.n] = (int32_t)(t.n + base + 2 + 2 * q);
    split_rank[r] = (int32_t)q;
  }
}

__global__ void k_split_inst(const uint32_t *__restrict__ split_nodes, int64_t ns, Segments seg,
                             uint32_t *__restrict__ inst) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < ns;
       q += (int64_t)gridDim.x * blockDim.x)
    inst[q] = (uint32_t)seg.of_rank(split_nodes[q]);
}

// One thread per instance s: its root's cluster index croot[s] = s + 2 *
// (splits of earlier instances), the root node's cid, and cseg of the root.
__global__ void k_forest_roots(TreeView t, const uint32_t *__restrict__ split_inst, int64_t ns,
                               int32_t *__restrict__ cid, int32_t *__restrict__ croot,
                               int32_t *__restrict__ cseg, int64_t C) {
  const int32_t T = t.seg.count;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s <= T;
       s += (int64_t)gridDim.x * blockDim.x) {
    if (s == T) { croot[T] = (int32_t)C; continue; }
    int64_t lo = 0, hi = ns;  // first split of an instance >= s
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((int64_t)split_inst[mid] < s) lo = mid + 1; else hi = mid;
    }
    const int64_t c = s + 2 * lo;
    croot[s] = (int32_t)c;
    cseg[c] = (int32_t)s;
    cid[t.seg.off[s + 1] - s - 2] = (int32_t)(t.n + c);
  }
}

// Cluster of every visited node; per-cluster info (index c - n).
__global__ void k_node_cluster(int64_t m, int64_t n, const int8_t *__restrict__ visited,
                               const int32_t *__restrict__ head, const int32_t *__restrict__ cid,
                               int32_t *__restrict__ ncl) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x)
    ncl[r] = visited[r] ? cid[head[r]] : -1;
}

__global__ void k_cluster_info(TreeView t, const uint32_t *__restrict__ split_nodes, int64_t ns,
                               const uint32_t *__restrict__ split_inst,
                               const int32_t *__restrict__ ncl, const float *__restrict__ lam,
                               float *__restrict__ birth, int32_t *__restrict__ cparent,
                               int32_t *__restrict__ ckid0, int32_t *__restrict__ cseg) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < ns;
       q += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = split_nodes[q];
    int32_t pc = ncl[r];  // cluster whose chain ends at this split
    const int32_t base = split_inst ? (int32_t)split_inst[q] : 0;
    int32_t c0 = (int32_t)(base + 1 + 2 * q), c1 = c0 + 1;
    if (cseg) cseg[c0] = cseg[c1] = base;
    birth[c0] = lam[r];
    birth[c1] = lam[r];
    cparent[c0] = pc - (int32_t)t.n;
    cparent[c1] = pc - (int32_t)t.n;
    ckid0[pc - t.n] = c0;
  }
}

// Chain nodes grouped by cluster, top-down: key (cluster index << 32) | depth.
__global__ void k_chain_keys(int64_t m, int64_t n, const int32_t *__restrict__ ncl,
                             const int64_t *__restrict__ dep, const int64_t *__restrict__ pos,
                             uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (ncl[r] < 0) continue;
    keys[pos[r]] = ((uint64_t)(ncl[r] - n) << 32) | (uint64_t)dep[r];
    vals[pos[r]] = (uint32_t)r;
  }
}

// Chain node data laid out in chain order, so the per-cluster sums stream
// contiguous memory: lambda, and either (count of points falling out, 0) or,
// for the split that ends the chain, (-size(left), size(right)).
struct ChainItem {
  float lam;
  int32_t a, b;
  int32_t pad;
};

__global__ void k_chain_items(TreeView t, const uint32_t *__restrict__ chain, int64_t cnt,
                              const int8_t *__restrict__ kind, const float *__restrict__ lam,
                              ChainItem *__restrict__ items) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t r = chain[i];
    const hdb_linkage_node h = t.h[r];
    const int8_t kd = kind[r];
    ChainItem it;
    it.lam = lam[r];
    it.pad = 0;
    if (kd == KIND_SPLIT) {
      it.a = -t.sz(h.left_node);
      it.b = t.sz(h.right_node);
    } else {
      it.a = kd == KIND_LEFTBIG ? t.sz(h.right_node)
             : kd == KIND_RIGHTBIG ? t.sz(h.left_node)
                                   : t.sz(h.left_node) + t.sz(h.right_node);
      it.b = 0;
    }
    items[i] = it;
  }
}

template <typename T> struct FpBits;
template <> struct FpBits<float> {
  static constexpr int kMant = 23;
  __device__ static int exp_field(float x) { return (__float_as_uint(x) >> 23) & 0xff; }
  __device__ static float pow2(int e) { return __uint_as_float((uint32_t)(e + 127) << 23); }
  __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
  __device__ static float sub(float a, float b) { return __fsub_rn(a, b); }
  __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
  static constexpr int kBias = 127;
};
template <> struct FpBits<double> {
  static constexpr int kMant = 52;
  __device__ static int exp_field(double x) {
    return (int)((__double_as_longlong(x) >> 52) & 0x7ff);
  }
  __device__ static double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }
  __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
  __device__ static double sub(double a, double b) { return __dsub_rn(a, b); }
  __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
  static constexpr int kBias = 1023;
};

// s after `cnt` sequential round-to-nearest-even additions of v >= 0 --
// exactly what one row per point gives (compute_stability, tree.cu:504-512).
// Inside one binade of s the additions advance s by a fixed multiple of its
// ulp; with v an odd multiple of half an ulp (a tie) the first step may differ
// and every later one is equal.  So: take single steps until two consecutive
// increments inside one binade agree (and v < s, which keeps s1 - s exact),
// then jump to the last step that stays in the binade.
template <typename T>
__device__ T add_repeated(T s, T v, int64_t cnt) {
  using B = FpBits<T>;
  if (!(v > T(0))) {
    for (; cnt > 0; cnt--) s = B::add(s, v);
    return s;
  }
  T last_inc = T(-1);
  int last_exp = -1;
  while (cnt > 0) {
    const T s1 = B::add(s, v);
    cnt--;
    const int e0 = B::exp_field(s), e1 = B::exp_field(s1);
    if (!(v < s) || e0 == 0 || e0 != e1) {  // large step, subnormal, or binade change
      s = s1;
      last_inc = T(-1);
      continue;
    }
    const T inc = B::sub(s1, s);  // exact: s <= s1 <= 2s
    s = s1;
    if (inc == T(0)) return s;  // v under half an ulp: s stays put from now on
    if (inc == last_inc && e1 == last_exp && cnt > 0) {
      // steady: s advances by inc = dq ulps per step while it stays in binade e1
      const T u = B::pow2(e1 - B::kBias - B::kMant);
      const int64_t q = (int64_t)B::mul(s, B::pow2(B::kMant - (e1 - B::kBias)));  // s / u
      const int64_t dq = (int64_t)B::mul(inc, B::pow2(B::kMant - (e1 - B::kBias)));
      const int64_t qmax = (int64_t(1) << (B::kMant + 1)) - 1;
      int64_t t = (qmax - q) / dq;
      if (t > cnt) t = cnt;
      if (t > 0) {
        s = B::mul((T)(q + t * dq), u);  // exact: integer significand times a power of two
        cnt -= t;
      }
      last_inc = T(-1);
      continue;
    }
    last_inc = inc;
    last_exp = e1;
  }
  return s;
}

// One warp per cluster: stability in the reference's row order.  The warp
// loads 32 chain items at a time (coalesced) and every lane replays the same
// sequential sum from registers, so the serial chain walk never waits on a
// dependent global load; lane 0 stores the result.
// Stability of each cluster: its chain items summed in FP32 in the
// reference's row order (and in FP64 alongside when kBoth).  One warp per
// cluster, 32 items per load; each lane forms its item's addends first, so the
// serial part is just the chain of adds, unrolled over the 32 items.  Items
// that stand for many rows with one addend go through add_repeated.
template <bool kBoth>
__global__ void k_stability(int64_t C, const int64_t *__restrict__ seg_start,
                            const int64_t *__restrict__ seg_end, const ChainItem *__restrict__ items,
                            const float *__restrict__ birth, float *__restrict__ stab,
                            double *__restrict__ stab64) {
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  for (int64_t c = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); c < C;
       c += (int64_t)gridDim.x * wpb) {
    const float b = birth[c];
    float s = 0.0f;
    double s64 = 0.0;
    const int64_t e = seg_end[c];
    for (int64_t base = seg_start[c]; base < e; base += 32) {
      ChainItem mine = {0.0f, 1, 0, 0};
      const bool valid = base + lane < e;
      if (valid) mine = items[base + lane];
      const int m = (int)min((int64_t)32, e - base);
      const float v = __fsub_rn(mine.lam, b);
      // split rows: (lambda - birth) * child_size, left then right; one row: v
      const bool split = mine.a < 0;
      const float x0 = split ? __fmul_rn(v, (float)(-mine.a)) : v;
      const float x1 = split ? __fmul_rn(v, (float)mine.b) : 0.0f;
      const uint32_t split_mask = __ballot_sync(0xffffffffu, valid && split);
      const uint32_t rep_mask = __ballot_sync(0xffffffffu, valid && mine.a > 1);
      if (!kBoth && rep_mask == 0) {
#pragma unroll
        for (int t = 0; t < 32; t++) {
          const float y0 = __shfl_sync(0xffffffffu, x0, t);
          const float y1 = __shfl_sync(0xffffffffu, x1, t);
          if (t < m) {
            s = __fadd_rn(s, y0);
            if ((split_mask >> t) & 1u) s = __fadd_rn(s, y1);
          }
        }
        continue;
      }
      for (int t = 0; t < m; t++) {
        const float lam = __shfl_sync(0xffffffffu, mine.lam, t);
        const int32_t ia = __shfl_sync(0xffffffffu, mine.a, t);
        const int32_t ib = __shfl_sync(0xffffffffu, mine.b, t);
        const float vt = __fsub_rn(lam, b);
        const double v64 = __dsub_rn((double)lam, (double)b);
        if (ia < 0) {
          s = __fadd_rn(s, __fmul_rn(vt, (float)(-ia)));
          s = __fadd_rn(s, __fmul_rn(vt, (float)ib));
          if (kBoth) {
            s64 = __dadd_rn(s64, __dmul_rn(v64, (double)(-ia)));
            s64 = __dadd_rn(s64, __dmul_rn(v64, (double)ib));
          }
        } else if (ia == 1) {  // one row
          s = __fadd_rn(s, vt);
          if (kBoth) s64 = __dadd_rn(s64, v64);
        } else {  // one row per point falling out here
          s = add_repeated<float>(s, vt, ia);
          if (kBoth) s64 = add_repeated<double>(s64, v64, ia);
        }
      }
    }
    if (lane == 0) {
      stab[c] = s;
      stab64[c] = kBoth ? s64 : (double)s;
    }
  }
}

// Excess of mass, bottom-up: the last of two siblings to finish continues
// with their parent (get_clusters, tree.cu:692-725).  Roots (the clusters
// without a parent: index 0, or one per tree of a forest) are never
// evaluated, as in the reference.
__global__ void k_eom(int64_t C, const int32_t *__restrict__ ckid0, const int32_t *__restrict__ cparent,
                      const float *__restrict__ stab, const double *__restrict__ stab64, int fp64,
                      float *sub, double *sub64, int8_t *self_sel, int32_t *arrive) {
  for (int64_t c0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c0 < C;
       c0 += (int64_t)gridDim.x * blockDim.x) {
    if (cparent[c0] < 0 || ckid0[c0] >= 0) continue;  // start from leaf clusters
    int64_t c = c0;
    // leaf: no children -> subtree stability 0, never above its own
    volatile float *vsub = sub;
    volatile double *vsub64 = sub64;
    vsub[c] = stab[c];
    vsub64[c] = stab64[c];
    self_sel[c] = 1;
    for (int64_t guard = 0; guard < C; guard++) {
      int64_t p = cparent[c];
      if (p < 0 || cparent[p] < 0) break;  // parent is a root
      __threadfence();
      if (atomicAdd(&arrive[p], 1) == 0) break;  // sibling not done yet
      __threadfence();
      int32_t k0 = ckid0[p];
      bool over;
      if (fp64) {
        double ssum = vsub64[k0] + vsub64[k0 + 1];
        over = ssum > stab64[p];
        vsub64[p] = over ? ssum : stab64[p];
        vsub[p] = over ? (float)ssum : stab[p];
      } else {
        float ssum = __fadd_rn(__fadd_rn(0.0f, vsub[k0]), vsub[k0 + 1]);
        over = ssum > stab[p];
        vsub[p] = over ? ssum : stab[p];
        vsub64[p] = vsub[p];
      }
      self_sel[p] = over ? 0 : 1;
      c = p;
    }
  }
}

// Nearest self-selected proper ancestor (roots excluded) by doubling.
__global__ void k_sel_init(int64_t C, const int32_t *__restrict__ cparent, const int8_t *__restrict__ self_sel,
                           int32_t *__restrict__ jmp, int8_t *__restrict__ anc) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < C;
       c += (int64_t)gridDim.x * blockDim.x) {
    int32_t p = cparent[c];
    if (p < 0 || cparent[p] < 0) { jmp[c] = -1; anc[c] = 0; }
    else { jmp[c] = p; anc[c] = self_sel[p]; }
  }
}

__global__ void k_sel_jump(int64_t C, const int32_t *__restrict__ jmp, const int8_t *__restrict__ anc,
                           int32_t *__restrict__ jmp2, int8_t *__restrict__ anc2, int32_t *changed) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < C;
       c += (int64_t)gridDim.x * blockDim.x) {
    int32_t j = jmp[c];
    if (j < 0) { jmp2[c] = -1; anc2[c] = anc[c]; continue; }
    anc2[c] = anc[c] | anc[j];
    jmp2[c] = jmp[j];
    *changed = 1;
  }
}

__global__ void k_selected(int64_t C, const int32_t *__restrict__ cparent,
                           const int8_t *__restrict__ self_sel, const int8_t *__restrict__ anc,
                           int32_t *__restrict__ sel) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < C;
       c += (int64_t)gridDim.x * blockDim.x)
    sel[c] = (cparent[c] >= 0 && self_sel[c] && !anc[c]) ? 1 : 0;
}

// Selected cluster covering each cluster (itself or nearest selected ancestor).
__global__ void k_cover_init(int64_t C, const int32_t *__restrict__ cparent, const int32_t *__restrict__ sel,
                             int32_t *__restrict__ jmp, int32_t *__restrict__ cover) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < C;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (sel[c]) { cover[c] = (int32_t)c; jmp[c] = -1; continue; }
    cover[c] = -1;
    int32_t p = cparent[c];
    jmp[c] = (p >= 0 && cparent[p] >= 0) ? p : -1;
  }
}

__global__ void k_cover_jump(int64_t C, const int32_t *__restrict__ jmp, const int32_t *__restrict__ cover,
                             int32_t *__restrict__ jmp2, int32_t *__restrict__ cover2, int32_t *changed) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < C;
       c += (int64_t)gridDim.x * blockDim.x) {
    int32_t j = jmp[c];
    if (cover[c] >= 0 || j < 0) { cover2[c] = cover[c]; jmp2[c] = -1; continue; }
    cover2[c] = cover[j];
    jmp2[c] = cover[j] >= 0 ? -1 : jmp[j];
    *changed = 1;
  }
}

// Points: fall-out node = parent of the highest ancestor holding < mpts points.
__global__ void k_points(TreeView t, const int32_t *__restrict__ par, const int32_t *__restrict__ ncl,
                         const float *__restrict__ lam, const int32_t *__restrict__ cover,
                         const float *__restrict__ birth, const int32_t *__restrict__ label_of,
                         int32_t *__restrict__ labels, int32_t *__restrict__ pcl,
                         float *__restrict__ plam) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < t.n;
       p += (int64_t)gridDim.x * blockDim.x) {
    int64_t a = p;
    while (true) {
      int32_t up = par[a];
      if (up < 0 || t.sz(up) >= t.mpts) break;
      a = up;
    }
    int64_t f = par[a] < 0 ? a : par[a];  // a is the root only if n < mpts
    int64_t fr = f - t.n;
    int32_t c = ncl[fr];
    float lp = lam[fr];
    int32_t s = cover[c - t.n];
    int32_t lab = -1;
    if (s >= 0 && lp > birth[s]) lab = label_of[s];
    labels[p] = lab;
    if (pcl) { pcl[p] = c; plam[p] = lp; }
  }
}

// Label of a selected cluster: its rank among the selected clusters of its
// tree (a forest restarts the count at each instance's root).
__global__ void k_label_map(int64_t C, const int32_t *__restrict__ sel, const int32_t *__restrict__ pos,
                            const int32_t *__restrict__ cseg, const int32_t *__restrict__ croot,
                            int32_t *__restrict__ label_of) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < C;
       c += (int64_t)gridDim.x * blockDim.x)
    label_of[c] = sel[c] ? pos[c] - (cseg ? pos[croot[cseg[c]]] : 0) : -1;
}

__global__ void k_inst_clusters(int32_t T, const int32_t *__restrict__ pos,
                                const int32_t *__restrict__ croot, int32_t *__restrict__ out) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < T;
       s += (int64_t)gridDim.x * blockDim.x)
    out[s] = pos[croot[s + 1]] - pos[croot[s]];
}

__global__ void k_condensed_rows(TreeView t, const uint32_t *__restrict__ split_nodes, int64_t ns,
                                 const int32_t *__restrict__ ncl, const float *__restrict__ lam,
                                 const int32_t *__restrict__ pcl, const float *__restrict__ plam,
                                 hdb_condensed_node *__restrict__ rows, uint64_t *__restrict__ keys,
                                 uint32_t *__restrict__ vals) {
  const int64_t total = t.n + 2 * ns;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    hdb_condensed_node row;
    if (i < t.n) {
      row.parent = pcl[i];
      row.child = (int32_t)i;
      row.lambda_val = plam[i];
      row.child_size = 1;
    } else {
      int64_t q = (i - t.n) >> 1;
      int side = (int)((i - t.n) & 1);
      int64_t r = split_nodes[q];
      hdb_linkage_node h = t.h[r];
      row.parent = ncl[r];
      row.child = (int32_t)(t.n + 1 + 2 * q + side);
      row.lambda_val = lam[r];
      row.child_size = t.sz(side ? h.right_node : h.left_node);
    }
    rows[i] = row;
    keys[i] = ((uint64_t)(uint32_t)row.parent << 32) | (uint32_t)row.child;
    vals[i] = (uint32_t)i;
  }
}

__global__ void k_permute_rows(const hdb_condensed_node *__restrict__ in, const uint32_t *__restrict__ idx,
                               int64_t cnt, hdb_condensed_node *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[idx[i]];
}

__global__ void k_stab_out(int64_t C, int64_t n, const float *__restrict__ stab,
                           hdb_stability *__restrict__ out) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < C;
       c += (int64_t)gridDim.x * blockDim.x) {
    hdb_stability s;
    s.cluster_id = (int32_t)(n + c);
    s.lambda = stab[c];
    out[c] = s;
  }
}

__global__ void k_seg_bounds(const uint64_t *__restrict__ keys, int64_t cnt, int64_t *__restrict__ s0,
                             int64_t *__restrict__ s1) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t c = (uint32_t)(keys[i] >> 32);
    if (i == 0 || (uint32_t)(keys[i - 1] >> 32) != c) s0[c] = i;
    if (i == cnt - 1 || (uint32_t)(keys[i + 1] >> 32) != c) s1[c] = i + 1;
  }
}

__global__ void k_flag_nonneg(const int32_t *__restrict__ v, int64_t m, int32_t *__restrict__ flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = v[i] >= 0;
}

int bits_for(int64_t v) {
  int b = 0;
  while (b < 63 && (int64_t(1) << b) <= v) b++;
  return b < 1 ? 1 : b;
}

}  // namespace

void linkage_tree(Context *ctx, const hdb_mst_edge *mst, int64_t n, hdb_linkage_node *out,
                  const Segments &seg) {
  HDB_REQUIRE(n >= 2 && n < (int64_t(1) << 30), HDB_ERR_ARG, "linkage tree: bad n");
  cudaStream_t st = ctx->stream;
  const int64_t m = n - (seg.count > 0 ? seg.count : 1), total = n + m;
  Buf<int32_t> la(ctx, m), lb(ctx, m), size(ctx, total);
  Buf<UfNode> u(ctx, total);
  const int gm = grid_for(ctx, m, 256), gt = grid_for(ctx, total, 256);
  k_validate_mst<<<gm, 256, 0, st>>>(mst, m, n, ctx->dev_err); ctx->launches++;
  HDB_CHECK_LAUNCH();
  HDB_REQUIRE(!(ctx->take_dev_err() & DEVERR_ID_RANGE), HDB_ERR_ARG,
              "linkage tree: MST edge endpoint outside [0, n)");
  k_link_init<<<gm, 256, 0, st>>>(mst, m, la, lb); ctx->launches++;
  k_uf_init<<<gt, 256, 0, st>>>(total, n, u, size); ctx->launches++;
  HDB_CHECK_LAUNCH();
  int64_t S = 1;
  while (S < m) S <<= 1;
  for (; S >= 2; S >>= 1) {
    k_level_union<<<gm, 256, 0, st>>>(la, lb, m, S, u, ctx->dev_err); ctx->launches++;
    k_level_tag<<<gm, 256, 0, st>>>(la, lb, m, S, n, u, size); ctx->launches++;
    k_level_produce<<<gm, 256, 0, st>>>(la, m, S, n, u, size); ctx->launches++;
    k_level_relabel<<<gm, 256, 0, st>>>(la, lb, m, S, n, u); ctx->launches++;
    k_level_reset<<<gm, 256, 0, st>>>(la, lb, m, S, u); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  k_link_out<<<gm, 256, 0, st>>>(mst, la, lb, size, m, n, out); ctx->launches++;
  HDB_CHECK_LAUNCH();
  HDB_REQUIRE(!(ctx->take_dev_err() & DEVERR_TIMEOUT), HDB_ERR_INTERNAL,
              "linkage tree: union-find exceeded its step bound");
}

void condense_select(Context *ctx, const hdb_linkage_node *h, int64_t n, int32_t mpts,
                     int32_t stab_mode, int32_t *labels, int32_t *num_clusters,
                     hdb_condensed_node *condensed, int64_t *condensed_size,
                     hdb_stability *stability, int64_t *num_stability, const Segments &seg,
                     int32_t *inst_clusters) {
  HDB_REQUIRE(n >= 2 && n < (int64_t(1) << 30), HDB_ERR_ARG, "condensed tree: bad n");
  HDB_REQUIRE(mpts >= 2, HDB_ERR_ARG, "condensed tree: mpts (min cluster size) must be >= 2");
  const bool forest = seg.count > 0;
  HDB_REQUIRE(!forest || (!condensed && !stability), HDB_ERR_ARG,
              "condensed tree: condensed rows and stabilities are per single tree");
  cudaStream_t st = ctx->stream;
  const int64_t trees = forest ? seg.count : 1;
  const int64_t m = n - trees, total = n + m;
  TreeView t{h, n, m, mpts, seg};
  const int gm = grid_for(ctx, m, 256), gn = grid_for(ctx, n, 256);
  int64_t *hp = static_cast<int64_t *>(ctx->pinned);
  int32_t *hflag = reinterpret_cast<int32_t *>(hp + 8);

  Buf<int32_t> par(ctx, total);
  Buf<int8_t> side(ctx, total), kind(ctx, m), visited(ctx, m);
  Buf<float> lam(ctx, m);
  HDB_CUDA(cudaMemsetAsync(par, 0xff, total * sizeof(int32_t), st));
  k_validate_hier<<<gm, 256, 0, st>>>(t, ctx->dev_err); ctx->launches++;
  HDB_CHECK_LAUNCH();
  HDB_REQUIRE(!(ctx->take_dev_err() & DEVERR_ID_RANGE), HDB_ERR_ARG,
              "condensed tree: hierarchy is not a valid single-linkage tree");
  k_nodes<<<gm, 256, 0, st>>>(t, par, side, kind, visited, lam); ctx->launches++;
  HDB_CHECK_LAUNCH();

  // depth / preorder / chain heads by pointer jumping
  Buf<int32_t> jmp(ctx, m), jmp2(ctx, m), head(ctx, m);
  Buf<int64_t> dep(ctx, m), dep2(ctx, m), pre(ctx, m), pre2(ctx, m);
  Buf<int32_t> changed(ctx, 2);
  k_path_init<<<gm, 256, 0, st>>>(t, par, side, kind, visited, jmp, dep, pre, head); ctx->launches++;
  HDB_CHECK_LAUNCH();
  int32_t *j0 = jmp, *j1 = jmp2;
  int64_t *d0 = dep, *d1 = dep2, *p0 = pre, *p1 = pre2;
  for (int it = 0; it < 64; it++) {
    HDB_CUDA(cudaMemsetAsync(changed, 0, 2 * sizeof(int32_t), st));
    k_path_jump<<<gm, 256, 0, st>>>(m, j0, d0, p0, j1, d1, p1, changed); ctx->launches++;
    k_head_jump<<<gm, 256, 0, st>>>(m, head, changed.get() + 1); ctx->launches++;
    HDB_CHECK_LAUNCH();
    HDB_CUDA(cudaMemcpyAsync(hflag, changed, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    ctx->sync();
    std::swap(j0, j1);
    std::swap(d0, d1);
    std::swap(p0, p1);
    if (!hflag[0] && !hflag[1]) break;
    HDB_REQUIRE(it < 63, HDB_ERR_INTERNAL, "condensed tree: pointer jumping did not converge");
  }
  // head pointers may need extra rounds beyond the path sums
  for (int it = 0; it < 64; it++) {
    HDB_CUDA(cudaMemsetAsync(changed, 0, sizeof(int32_t), st));
    k_head_jump<<<gm, 256, 0, st>>>(m, head, changed); ctx->launches++;
    HDB_CHECK_LAUNCH();
    HDB_CUDA(cudaMemcpyAsync(hflag, changed, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    ctx->sync();
    if (!hflag[0]) break;
  }

  // split nodes in BFS order -> cluster ids
  Buf<int32_t> flag(ctx, m);
  Buf<int64_t> pos(ctx, m + 1);
  k_split_keys<<<gm, 256, 0, st>>>(m, kind, visited, d0, p0, flag); ctx->launches++;
  HDB_CHECK_LAUNCH();
  scan_exclusive_i32_i64(ctx, flag, pos, m, pos.get() + m);
  HDB_CUDA(cudaMemcpyAsync(hp, pos.get() + m, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  ctx->sync();
  const int64_t ns = hp[0];
  const int64_t C = trees + 2 * ns;
  Buf<uint64_t> skeys(ctx, ns > 0 ? ns : 1);
  Buf<uint32_t> snodes(ctx, ns > 0 ? ns : 1), sinst;
  Buf<int32_t> cid(ctx, m), split_rank(ctx, m), cseg, croot;
  HDB_CUDA(cudaMemsetAsync(cid, 0xff, m * sizeof(int32_t), st));
  if (forest) {
    sinst = Buf<uint32_t>(ctx, ns > 0 ? ns : 1);
    cseg = Buf<int32_t>(ctx, C);
    croot = Buf<int32_t>(ctx, trees + 1);
  }
  if (ns > 0) {
    k_split_emit<<<gm, 256, 0, st>>>(m, flag, pos, d0, p0, skeys, snodes); ctx->launches++;
    HDB_CHECK_LAUNCH();
    radix_sort_u64(ctx, skeys, snodes, ns, 0, 64);
    if (forest) {  // (instance, BFS order)
      k_split_inst<<<grid_for(ctx, ns, 256), 256, 0, st>>>(snodes, ns, seg, sinst); ctx->launches++;
      HDB_CHECK_LAUNCH();
      radix_sort_u32(ctx, sinst, snodes, ns, 0, bits_for(seg.count));
    }
    k_assign_cids<<<grid_for(ctx, ns, 256), 256, 0, st>>>(t, snodes, ns, sinst.get(), cid,
                                                           split_rank); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  // root cluster ids
  if (forest) {
    k_forest_roots<<<grid_for(ctx, trees + 1, 256), 256, 0, st>>>(t, sinst, ns, cid, croot, cseg,
                                                                   C); ctx->launches++;
    HDB_CHECK_LAUNCH();
  } else {
    int32_t root_cid = (int32_t)n;
    HDB_CUDA(cudaMemcpyAsync(cid.get() + (m - 1), &root_cid, sizeof(int32_t),
                             cudaMemcpyHostToDevice, st));
    ctx->sync();
  }
  Buf<int32_t> ncl(ctx, m);
  k_node_cluster<<<gm, 256, 0, st>>>(m, n, visited, head, cid, ncl); ctx->launches++;
  HDB_CHECK_LAUNCH();

  // per-cluster info
  Buf<float> birth(ctx, C), stab(ctx, C), sub(ctx, C);
  Buf<double> stab64(ctx, C), sub64(ctx, C);
  Buf<int32_t> cparent(ctx, C), ckid0(ctx, C), arrive(ctx, C);
  Buf<int8_t> self_sel(ctx, C);
  HDB_CUDA(cudaMemsetAsync(birth, 0, C * sizeof(float), st));
  HDB_CUDA(cudaMemsetAsync(cparent, 0xff, C * sizeof(int32_t), st));
  HDB_CUDA(cudaMemsetAsync(ckid0, 0xff, C * sizeof(int32_t), st));
  HDB_CUDA(cudaMemsetAsync(arrive, 0, C * sizeof(int32_t), st));
  HDB_CUDA(cudaMemsetAsync(self_sel, 0, C, st));
  if (ns > 0) {
    k_cluster_info<<<grid_for(ctx, ns, 256), 256, 0, st>>>(t, snodes, ns, sinst.get(), ncl, lam,
                                                            birth, cparent, ckid0, cseg.get()); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }

  // chain segments (cluster, depth), then stability per cluster
  Buf<int64_t> s0(ctx, C), s1(ctx, C);
  HDB_CUDA(cudaMemsetAsync(s0, 0, C * sizeof(int64_t), st));
  HDB_CUDA(cudaMemsetAsync(s1, 0, C * sizeof(int64_t), st));
  Buf<uint32_t> chain(ctx, m);
  int64_t nv_total = 0;
  {
    k_flag_nonneg<<<gm, 256, 0, st>>>(ncl, m, flag); ctx->launches++;
    HDB_CHECK_LAUNCH();
    scan_exclusive_i32_i64(ctx, flag, pos, m, pos.get() + m);
    HDB_CUDA(cudaMemcpyAsync(hp, pos.get() + m, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    ctx->sync();
    const int64_t nv = hp[0];
    nv_total = nv;
    Buf<uint64_t> ckeys(ctx, nv);
    k_chain_keys<<<gm, 256, 0, st>>>(m, n, ncl, d0, pos, ckeys, chain); ctx->launches++;
    HDB_CHECK_LAUNCH();
    radix_sort_u64(ctx, ckeys, chain, nv, 0, 32 + bits_for(C));
    k_seg_bounds<<<grid_for(ctx, nv, 256), 256, 0, st>>>(ckeys, nv, s0, s1); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  const int gc = grid_for(ctx, C, 128);
  {
    Buf<ChainItem> items(ctx, nv_total);
    k_chain_items<<<grid_for(ctx, nv_total, 256), 256, 0, st>>>(t, chain, nv_total, kind, lam,
                                                                items); ctx->launches++;
    if (stab_mode == HDB_STAB_FP64)
      k_stability<true><<<grid_for(ctx, C, 4), 128, 0, st>>>(C, s0, s1, items, birth, stab, stab64);
    else
      k_stability<false><<<grid_for(ctx, C, 4), 128, 0, st>>>(C, s0, s1, items, birth, stab, stab64);
    ctx->launches++;
    HDB_CHECK_LAUNCH();
  }

  // excess of mass
  const int fp64 = stab_mode == HDB_STAB_FP64;
  k_eom<<<gc, 128, 0, st>>>(C, ckid0, cparent, stab, stab64, fp64, sub, sub64, self_sel, arrive); ctx->launches++;
  HDB_CHECK_LAUNCH();
  Buf<int32_t> cj(ctx, C), cj2(ctx, C), sel(ctx, C), cover(ctx, C), cover2(ctx, C);
  Buf<int8_t> anc(ctx, C), anc2(ctx, C);
  k_sel_init<<<gc, 128, 0, st>>>(C, cparent, self_sel, cj, anc); ctx->launches++;
  HDB_CHECK_LAUNCH();
  {
    int32_t *ja = cj, *jb = cj2;
    int8_t *aa = anc, *ab = anc2;
    for (int it = 0; it < 64; it++) {
      HDB_CUDA(cudaMemsetAsync(changed, 0, sizeof(int32_t), st));
      k_sel_jump<<<gc, 128, 0, st>>>(C, ja, aa, jb, ab, changed); ctx->launches++;
      HDB_CHECK_LAUNCH();
      HDB_CUDA(cudaMemcpyAsync(hflag, changed, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      ctx->sync();
      std::swap(ja, jb);
      std::swap(aa, ab);
      if (!hflag[0]) break;
    }
    k_selected<<<gc, 128, 0, st>>>(C, cparent, self_sel, aa, sel); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  Buf<int32_t> selpos(ctx, C + 1), label_of(ctx, C);
  scan_exclusive_i32_i32(ctx, sel, selpos, C, selpos.get() + C);
  k_label_map<<<gc, 128, 0, st>>>(C, sel, selpos, cseg.get(), croot.get(), label_of); ctx->launches++;
  k_cover_init<<<gc, 128, 0, st>>>(C, cparent, sel, cj, cover); ctx->launches++;
  HDB_CHECK_LAUNCH();
  int32_t *cov_final = cover;
  {
    int32_t *ja = cj, *jb = cj2, *ca = cover, *cb = cover2;
    for (int it = 0; it < 64; it++) {
      HDB_CUDA(cudaMemsetAsync(changed, 0, sizeof(int32_t), st));
      k_cover_jump<<<gc, 128, 0, st>>>(C, ja, ca, jb, cb, changed); ctx->launches++;
      HDB_CHECK_LAUNCH();
      HDB_CUDA(cudaMemcpyAsync(hflag, changed, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      ctx->sync();
      std::swap(ja, jb);
      std::swap(ca, cb);
      if (!hflag[0]) break;
    }
    cov_final = ca;
  }

  // labels (and the per-point condensed rows when asked)
  Buf<int32_t> pcl;
  Buf<float> plam;
  if (condensed) {
    pcl = Buf<int32_t>(ctx, n);
    plam = Buf<float>(ctx, n);
  }
  k_points<<<gn, 256, 0, st>>>(t, par, ncl, lam, cov_final, birth, label_of, labels,
                               condensed ? pcl.get() : nullptr, condensed ? plam.get() : nullptr); ctx->launches++;
  HDB_CHECK_LAUNCH();
  HDB_CUDA(cudaMemcpyAsync(hflag, selpos.get() + C, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  Buf<int32_t> icl;
  if (forest && inst_clusters) {
    icl = Buf<int32_t>(ctx, trees);
    k_inst_clusters<<<grid_for(ctx, trees, 256), 256, 0, st>>>(seg.count, selpos, croot, icl); ctx->launches++;
    HDB_CHECK_LAUNCH();
    HDB_CUDA(cudaMemcpyAsync(inst_clusters, icl, trees * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  }
  if (condensed) {
    const int64_t rows = n + 2 * ns;
    Buf<hdb_condensed_node> tmp(ctx, rows);
    Buf<uint64_t> rkeys(ctx, rows);
    Buf<uint32_t> ridx(ctx, rows);
    k_condensed_rows<<<grid_for(ctx, rows, 256), 256, 0, st>>>(t, snodes, ns, ncl, lam, pcl, plam,
                                                                tmp, rkeys, ridx); ctx->launches++;
    HDB_CHECK_LAUNCH();
    radix_sort_u64(ctx, rkeys, ridx, rows, 0, 64);
    k_permute_rows<<<grid_for(ctx, rows, 256), 256, 0, st>>>(tmp, ridx, rows, condensed); ctx->launches++;
    HDB_CHECK_LAUNCH();
    if (condensed_size) *condensed_size = rows;
  }
  if (stability) {
    k_stab_out<<<gc, 128, 0, st>>>(C, n, stab, stability); ctx->launches++;
    HDB_CHECK_LAUNCH();
  }
  if (num_stability) *num_stability = C;
  ctx->sync();
  if (num_clusters) *num_clusters = hflag[0];
}

}  // namespace hdb
