// BF16 local join of NN-Descent (UpdateGraph, nndescent.cu:1487-1580) on the
// 5th-generation tensor cores.
//
// One tile holds two row-joins: for each of two consecutive rows of the graph,
// its new sample at slots 0..31 and its old sample at slots 32..63, as
// compacted beforehand by k_join_lists (the reference's de-duplication,
// ShrinkGraph :285-291, and new \ old, :468-486).  The staged BF16 rows are
// gathered by TMA (tile::gather4, four rows per instruction, 128-byte
// swizzle) straight into the K-major operand layout of tcgen05.mma, and one
// M = N = 128 MMA chain per tile computes their Gram matrix G = R R^T into
// tensor memory (FP32).  Only the two 64 x 64 diagonal blocks are read back:
// distance = ||a||^2 + ||c||^2 - 2 a.c with the norms of the rounded rows, as
// in the SIMT BF16 join.
//
// Warp roles (256 threads, a persistent loop over tiles):
//   warps 4-6   producers (take tiles in turn): slot lists into the tile's
//               metadata slot (ids, nn / no, cp.async of the rows' norms and
//               worst[]), then TMA gathers of the rows, one 64-element K block
//               of the tile per operand stage; a TMA gather occupies its
//               issuing warp for a while, so two warps keep more gathers in
//               flight;
//   warp 7      one thread issues the MMAs, K block by K block, and commits
//               each operand stage back to its producer as soon as the MMAs
//               reading it are done, and the finished tile to the epilogue;
//   warps 0..3  epilogue: tcgen05.ld of the accumulator (warp w reads TMEM
//               lanes 32w..32w+31 = tile rows), row minima against the
//               metadata slot, and the candidates appended to the
//               target-sorted list of the merge (one reservation per warp and
//               tile; the per-row inboxes of the SIMT joins would cost a
//               returning atomic per candidate).
// Three rings, each with full / empty mbarriers: operand stages (one K block
// of a tile each, held only from the gather to the end of its MMAs), metadata
// slots (held until the epilogue is done with the tile) and two
// accumulators.  A stage is therefore not held while the epilogue works,
// which keeps more gathers in flight per SM.  Every wait is bounded in time:
// a wait that gives up sets DEVERR_TIMEOUT and makes every role of the CTA
// stop, after which the CTA still waits (bounded) for its own copies and MMAs
// before it frees its tensor memory and exits.  tcgen05.ld / alloc are
// .sync.aligned: the warp is reconverged with __syncwarp() right before each,
// because the code ahead of them branches per lane.
//
// Row minima: each distance is clamped at 0 and its float bits (order-preserving
// for non-negative floats) have their low 6 bits replaced by the column, so one
// unsigned min picks the closest column; the pushed distance is that value with
// the column bits cleared.  The candidate therefore carries its distance to
// within 2^-17 relative, and every (row, column) pair maps to one value.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "join_tc.cuh"

namespace hdb {

using namespace knn;

namespace {

constexpr int kStages = 6;    // operand stages (one 64-element K block of a tile each)
constexpr int kMetaSlots = 8; // tile metadata slots
constexpr int kKBlockBytes = kTcTileRows * 128;  // one 64-element K block of a tile
constexpr int kAccCols = 128;                     // FP32 accumulator columns (N)
constexpr uint32_t kTmemCols = 2 * kAccCols;
constexpr int kEpiWarps = 4;
constexpr int kProducers = 3;  // producer warps, alternating tiles
constexpr int kProducerWarp0 = kEpiWarps;
constexpr int kMmaWarp = kProducerWarp0 + kProducers;
constexpr int kThreads = 32 * (kMmaWarp + 1);
constexpr uint32_t kMetaArrivals = 1 + 32;          // producer + one cp.async arrival per lane
constexpr uint64_t kWaitNs = 2000000000ull;         // 2 s
constexpr uint32_t kNoKey = 0x7F800000u;            // keys at or above: no candidate
// Shared memory is padded to at least this size so that no more than two
// CTAs (2 x 256 tensor-memory columns = all 512) are resident on one SM.
constexpr size_t kMinSmem = 80 * 1024;

// M = N = 128, 16-bit x 16-bit -> FP32, both operands K-major; A and B
// always have the same format (BF16 or FP16: both come from one tile).
constexpr uint32_t idesc_for(bool fp16) {
  return (1u << 4)                                   // D format F32
         | (fp16 ? 0u : (1u << 7) | (1u << 10))      // A, B format: F16 (0) or BF16 (1)
         | ((uint32_t)(128 >> 3) << 17)              // N / 8
         | ((uint32_t)(128 >> 4) << 24);             // M / 16
}

struct StageMeta {
  int32_t ids[kTcTileRows];
  float nrm[kTcTileRows];  // squared norm of the staged row; +inf marks an empty column
  float wst[kTcTileRows];  // worst[] of the slot's row: the push threshold
  int32_t nn[2], no[2];    // per row-join: new and old rows staged
};

struct Shared {
  StageMeta meta[kMetaSlots];
  unsigned long long full[kStages], empty[kStages];        // operand stages
  unsigned long long mfull[kMetaSlots], mempty[kMetaSlots];  // metadata slots
  unsigned long long acc_full[2], acc_empty[2];
  uint32_t armed[kStages];       // uses of each operand stage armed so far (for the drain)
  uint32_t marmed[kMetaSlots];   // uses of each metadata slot armed so far
  uint32_t tmem_base;
  int abort;
};

struct JoinArgs {
  const float *nrm;
  const int32_t *newS, *oldS;
  const int8_t *nf, *of;
  int32_t *nrev, *orev;
  const float *worst;
  Inbox ib;
  // probe mode
  const int32_t *probe_ids, *probe_counts;
  float *probe_out;
  uint32_t *err;
  uint32_t idesc;  // instruction descriptor of the operand format
  float dscale;    // distance = |a|^2 + |c|^2 + dscale * accumulator
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// ---- mbarriers --------------------------------------------------------------
__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase of `bar` with the given parity.  Gives up after kWaitNs,
// or (when `abort` is non-null) as soon as another role of the CTA gave up.
// A waiting warp backs off with __nanosleep after its first polls, so that
// it does not take issue slots from the warps of its SM sub-partition that
// have work (the epilogue's minima, the producers' gathers).
__device__ __noinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity,
                                       volatile int *abort) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; it++) {
    if (mbar_try(bar, parity)) return true;
    if (it > 8) __nanosleep(it > 64 ? 256 : 32);
    if ((it & 15) == 0) {
      if (abort && *abort) return false;
      if (globaltimer() - t0 > kWaitNs) return false;
    }
  }
}

// Waits until *cnt (how many uses of a ring entry have been armed) reaches
// `need`.  A parity wait can tell only the barrier's current phase from the
// one before, so a waiter must never be two phases ahead: a producer first
// waits here for the entry's previous use to be armed -- by whichever
// producer had it -- and only then for that use's release.  Bounded like
// mbar_wait.
__device__ __noinline__ bool wait_armed(const uint32_t *cnt, uint32_t need, volatile int *abort) {
  const volatile uint32_t *c = cnt;
  if (*c >= need) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; it++) {
    if (*c >= need) return true;
    if (it > 8) __nanosleep(32);
    if ((it & 15) == 0) {
      if (abort && *abort) return false;
      if (globaltimer() - t0 > kWaitNs) return false;
    }
  }
}

__device__ __forceinline__ void give_up(Shared &sh, uint32_t *err) {
  *reinterpret_cast<volatile int *>(&sh.abort) = 1;
  atomicOr(err, DEVERR_TIMEOUT);
}

// ---- copies -----------------------------------------------------------------
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_arrive_noinc(unsigned long long *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Four rows (r0..r3) x 64 BF16 columns starting at column x, written as four
// consecutive 128-byte rows at dst (128-byte swizzle); completes on bar.
__device__ __forceinline__ void tma_gather4(void *dst, const CUtensorMap *map, int32_t x,
                                            int32_t r0, int32_t r1, int32_t r2, int32_t r3,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(r0), "r"(r1), "r"(r2), "r"(r3),
      "r"(smem_u32(bar))
      : "memory");
}

// ---- tensor memory and MMA ---------------------------------------------------
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Shared-memory operand descriptor: K-major rows of 128 bytes, 128-byte
// swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)1 << 16;                            // leading byte offset (unused here)
  d |= (uint64_t)(1024 >> 4) << 32;                  // stride byte offset
  d |= (uint64_t)1 << 46;                            // descriptor version
  d |= (uint64_t)2 << 61;                            // 128-byte swizzle
  return d;
}
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z)
      : "memory");
}
__device__ __forceinline__ void tc_commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
// 32 consecutive accumulator columns of TMEM lane (warp's lane base + lane).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  __syncwarp();  // .sync.aligned: the whole warp issues it together
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
        "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
        "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}
// Waits for this thread's tensor-memory loads; the registers are tied to the
// wait so that no use of them is scheduled before it.
__device__ __forceinline__ void tmem_wait_ld2(uint32_t (&v)[32], uint32_t (&w)[32]) {
  asm volatile(
      "tcgen05.wait::ld.sync.aligned;"
      : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]),
        "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]),
        "+r"(v[14]), "+r"(v[15]), "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]),
        "+r"(v[20]), "+r"(v[21]), "+r"(v[22]), "+r"(v[23]), "+r"(v[24]), "+r"(v[25]),
        "+r"(v[26]), "+r"(v[27]), "+r"(v[28]), "+r"(v[29]), "+r"(v[30]), "+r"(v[31]),
        "+r"(w[0]), "+r"(w[1]), "+r"(w[2]), "+r"(w[3]), "+r"(w[4]), "+r"(w[5]), "+r"(w[6]),
        "+r"(w[7]), "+r"(w[8]), "+r"(w[9]), "+r"(w[10]), "+r"(w[11]), "+r"(w[12]), "+r"(w[13]),
        "+r"(w[14]), "+r"(w[15]), "+r"(w[16]), "+r"(w[17]), "+r"(w[18]), "+r"(w[19]),
        "+r"(w[20]), "+r"(w[21]), "+r"(w[22]), "+r"(w[23]), "+r"(w[24]), "+r"(w[25]),
        "+r"(w[26]), "+r"(w[27]), "+r"(w[28]), "+r"(w[29]), "+r"(w[30]), "+r"(w[31])
      :
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.wait::ld.sync.aligned;"
      : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]),
        "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]),
        "+r"(v[14]), "+r"(v[15]), "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]),
        "+r"(v[20]), "+r"(v[21]), "+r"(v[22]), "+r"(v[23]), "+r"(v[24]), "+r"(v[25]),
        "+r"(v[26]), "+r"(v[27]), "+r"(v[28]), "+r"(v[29]), "+r"(v[30]), "+r"(v[31])
      :
      : "memory");
}

// ---- slot lists ------------------------------------------------------------------
// One warp per row, before the join: the row's new and old samples (forward
// slots 0..S-1, reverse slots S..2S-1) de-duplicated (ShrinkGraph
// RemoveDuplicates :285-291), new minus old (:468-486), written back in place
// as compact lists with every partly used group of four padded with the
// group's first id; nf / of become the list lengths (both 0 when the row has
// nothing to compare).  The reverse counters are reset for the next iteration.
__global__ void k_join_lists(int64_t n, int S, int32_t *__restrict__ newS, int32_t *__restrict__ oldS,
                             int8_t *__restrict__ nf, int8_t *__restrict__ of,
                             int32_t *__restrict__ nrev, int32_t *__restrict__ orev) {
  __shared__ int32_t news_smem[8][32], olds_smem[8][32];  // launched with 8 warps
  const int lane = lane_id();
  const int wpb = blockDim.x >> 5;
  int32_t *news = news_smem[threadIdx.x >> 5];
  int32_t *olds = olds_smem[threadIdx.x >> 5];
  for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < n;
       row += (int64_t)gridDim.x * wpb) {
    // the row's counts and both lists are loaded together (the lists do not
    // wait for the counts: one memory round trip per row)
    const int64_t sb = row * (2 * S);
    const int32_t nraw = lane < 2 * S ? newS[sb + lane] : 0;
    const int32_t oraw = lane < 2 * S ? oldS[sb + lane] : 0;
    const int cnf = nf[row], cof = of[row];
    const int cnr = min(nrev[row], S), cor = min(orev[row], S);
    bool vn = (lane < S) ? (lane < cnf) : (lane < 2 * S && lane - S < cnr);
    bool vo = (lane < S) ? (lane < cof) : (lane < 2 * S && lane - S < cor);
    const int32_t nid = vn ? nraw : -1 - lane;
    const int32_t oid = vo ? oraw : -100 - lane;
    const uint32_t pn = __match_any_sync(0xffffffffu, nid);
    vn = vn && (__ffs(pn) - 1 == lane);
    const uint32_t po = __match_any_sync(0xffffffffu, oid);
    vo = vo && (__ffs(po) - 1 == lane);
    const uint32_t bo = __ballot_sync(0xffffffffu, vo);
    int no = __popc(bo);
    if (vo) olds[__popc(bo & lanemask_lt())] = oid;
    __syncwarp();
    {
      bool in_old = false;  // independent reads, not a chain
#pragma unroll 8
      for (int t = 0; t < no; t++) in_old |= olds[t] == nid;
      vn = vn && !in_old;
    }
    const uint32_t bn = __ballot_sync(0xffffffffu, vn);
    int nn = __popc(bn);
    if (vn) news[__popc(bn & lanemask_lt())] = nid;
    if (nn == 0 || nn + no < 2) nn = no = 0;  // nothing to compare
    __syncwarp();
    // compact lists; the last group of four padded with its first id
    int32_t outn = lane < nn ? news[lane] : 0;
    int32_t outo = lane < no ? olds[lane] : 0;
    const int32_t firstn = __shfl_sync(0xffffffffu, outn, lane & ~3);
    const int32_t firsto = __shfl_sync(0xffffffffu, outo, lane & ~3);
    if (lane >= nn) outn = firstn;
    if (lane >= no) outo = firsto;
    __syncwarp();
    if (lane < 2 * S) {
      newS[sb + lane] = outn;
      oldS[sb + lane] = outo;
    }
    if (lane == 0) {
      nf[row] = (int8_t)nn;
      of[row] = (int8_t)no;
      nrev[row] = 0;
      orev[row] = 0;
    }
  }
}

// ---- producer ------------------------------------------------------------------
// The compact slot lists of one row (k_join_lists), one slot per lane.
struct RowLoad {
  int32_t nid, oid;
  int8_t nn, no;
};

__device__ __forceinline__ RowLoad load_row(const JoinArgs &a, int64_t row, int64_t n, int S) {
  const int lane = lane_id();
  RowLoad r{0, 0, 0, 0};
  if (row >= n) return r;
  r.nn = a.nf[row];
  r.no = a.of[row];
  if (lane < 2 * S) {
    r.nid = a.newS[row * (2 * S) + lane];
    r.oid = a.oldS[row * (2 * S) + lane];
  }
  return r;
}

// Fills row-join j of stage m from its compact lists: ids (padded groups of
// four), nn / no, norms (+inf for every slot that is not a staged row) and
// worst[] by cp.async.  Returns the number of four-row groups to gather.
__device__ __forceinline__ int stage_join(const JoinArgs &a, const RowLoad &r, int j, StageMeta &m,
                                          int &nn_out, int &no_out) {
  const int lane = lane_id();
  const int base = 64 * j;
  const int nn = r.nn, no = r.no;
  const int gnn = (nn + 3) & ~3, gno = (no + 3) & ~3;
  if (lane < gnn) m.ids[base + lane] = r.nid;
  if (lane < gno) m.ids[base + 32 + lane] = r.oid;
  const float inf = __int_as_float(0x7f800000);
  if (lane < nn) {
    cp_async4(&m.nrm[base + lane], a.nrm + r.nid);
    cp_async4(&m.wst[base + lane], a.worst + r.nid);
  } else {
    m.nrm[base + lane] = inf;
  }
  if (lane < no) {
    cp_async4(&m.nrm[base + 32 + lane], a.nrm + r.oid);
    cp_async4(&m.wst[base + 32 + lane], a.worst + r.oid);
  } else {
    m.nrm[base + 32 + lane] = inf;
  }
  if (lane == 0) {
    m.nn[j] = nn;
    m.no[j] = no;
  }
  nn_out = nn;
  no_out = no;
  return (gnn + gno) >> 2;
}

// Probe form of stage_join: the slot lists are given.
__device__ __forceinline__ int stage_probe(const JoinArgs &a, int64_t t, int j, StageMeta &m,
                                           int &nn_out, int &no_out) {
  const int lane = lane_id();
  const int base = 64 * j;
  const int nn = a.probe_counts[t * 4 + 2 * j], no = a.probe_counts[t * 4 + 2 * j + 1];
  const int32_t *src = a.probe_ids + t * kTcTileRows + base;
  const int gnn = (nn + 3) & ~3, gno = (no + 3) & ~3;
  const float inf = __int_as_float(0x7f800000);
  int32_t idn = src[lane < nn ? lane : (lane & ~3)];
  int32_t ido = src[32 + (lane < no ? lane : (lane & ~3))];
  if (lane < gnn) m.ids[base + lane] = idn;
  if (lane < gno) m.ids[base + 32 + lane] = ido;
  if (lane < nn) cp_async4(&m.nrm[base + lane], a.nrm + idn); else m.nrm[base + lane] = inf;
  if (lane < no) cp_async4(&m.nrm[base + 32 + lane], a.nrm + ido); else m.nrm[base + 32 + lane] = inf;
  m.wst[base + lane] = inf;
  m.wst[base + 32 + lane] = inf;
  if (lane == 0) {
    m.nn[j] = nn;
    m.no[j] = no;
  }
  nn_out = nn;
  no_out = no;
  return (gnn + gno) >> 2;
}

// Producer p of the CTA stages the CTA's tiles i = p, p + kProducers, ...
// (tile index blockIdx.x + i * gridDim.x): the tile's metadata into slot
// i % kMetaSlots, then its rows, one K block per operand stage; stage
// positions are i * kbc + kb around the ring, the order in which the MMA
// thread consumes them.  TMA gathers are issued lane by lane and occupy the
// issuing warp, so several producer warps keep more of them in flight.
template <bool kProbe>
__device__ void producer(int p, const CUtensorMap *xmap, const JoinArgs &a, Shared &sh,
                         unsigned char *tiles, int64_t n, int64_t ntiles, int kbc, int S,
                         unsigned long long &rows_staged) {
  const int lane = lane_id();
  const int64_t step = (int64_t)kProducers * gridDim.x;
  int64_t t = blockIdx.x + (int64_t)p * gridDim.x;
  RowLoad cur[2], nxt[2];
  if (!kProbe && t < ntiles) {
    cur[0] = load_row(a, 2 * t, n, S);
    cur[1] = load_row(a, 2 * t + 1, n, S);
  }
  for (uint32_t i = p; t < ntiles; t += step, i += kProducers) {
    const int m = i % kMetaSlots;
    const uint32_t muse = i / kMetaSlots;
    if (!__all_sync(0xffffffffu, wait_armed(&sh.marmed[m], muse, &sh.abort) &&
                                     mbar_wait(&sh.mempty[m], (muse & 1) ^ 1, &sh.abort))) {
      give_up(sh, a.err);
      break;
    }
    StageMeta &M = sh.meta[m];
    int nn[2], no[2], groups;
    if (kProbe) {
      groups = stage_probe(a, t, 0, M, nn[0], no[0]);
      groups += stage_probe(a, t, 1, M, nn[1], no[1]);
    } else {
      groups = stage_join(a, cur[0], 0, M, nn[0], no[0]);
      groups += stage_join(a, cur[1], 1, M, nn[1], no[1]);
      // this warp's next tile: its lists are in flight while this one is gathered
      const int64_t tn = t + step;
      if (tn < ntiles) {
        nxt[0] = load_row(a, 2 * tn, n, S);
        nxt[1] = load_row(a, 2 * tn + 1, n, S);
      }
    }
    rows_staged += nn[0] + no[0] + nn[1] + no[1];
    __syncwarp();  // the slot's ids / counts are written (and read below by every lane)
    cp_async_arrive_noinc(&sh.mfull[m]);
    if (lane == 0) {
      mbar_arrive(&sh.mfull[m]);
      atomicAdd(&sh.marmed[m], 1u);
    }
    // lane g: four-row group g & 15 of row-join g >> 4 (new groups 0..7,
    // old groups 8..15)
    const int j = lane >> 4, q = lane & 15;
    const bool oldg = q >= 8;
    const int slot = oldg ? 32 + 4 * (q - 8) : 4 * q;
    const bool mine = 4 * (q & 7) < (oldg ? no[j] : nn[j]);
    const int32_t *gi = M.ids + 64 * j + slot;
    bool ok = true;
    for (int kb = 0; kb < kbc; kb++) {
      const uint32_t g = i * (uint32_t)kbc + kb;
      const int s = g % kStages;
      const uint32_t use = g / kStages;
      if (!__all_sync(0xffffffffu, wait_armed(&sh.armed[s], use, &sh.abort) &&
                                       mbar_wait(&sh.empty[s], (use & 1) ^ 1, &sh.abort))) {
        ok = false;
        break;
      }
      if (lane == 0) {
        mbar_arrive_tx(&sh.full[s], (uint32_t)groups * 512u);
        atomicAdd(&sh.armed[s], 1u);
      }
      __syncwarp();
      if (mine) {
        unsigned char *dst = tiles + (size_t)s * kKBlockBytes + (64 * j + slot) * 128;
        tma_gather4(dst, xmap, kb * kTcKBlock, gi[0], gi[1], gi[2], gi[3], &sh.full[s]);
      }
    }
    if (!ok) {
      give_up(sh, a.err);
      break;
    }
    if (!kProbe) {
      cur[0] = nxt[0];
      cur[1] = nxt[1];
    }
  }
}

__device__ void mma_issuer(Shared &sh, unsigned char *tiles, uint32_t tmem, int64_t ntiles,
                           int kbc, uint32_t idesc, uint32_t *err) {
  int64_t t = blockIdx.x;
  int last_b = -1;
  uint32_t last_parity = 0;
  for (uint32_t i = 0; t < ntiles; t += gridDim.x, i++) {
    const int b = i & 1;
    const uint32_t ub = i >> 1;
    if (!mbar_wait(&sh.acc_empty[b], (ub & 1) ^ 1, &sh.abort)) {
      give_up(sh, err);
      break;
    }
    tc_fence_after();
    const uint32_t d = tmem + (uint32_t)(b * kAccCols);
    int issued = 0;
    for (int kb = 0; kb < kbc; kb++) {
      const uint32_t g = i * (uint32_t)kbc + kb;
      const int s = g % kStages;
      if (!mbar_wait(&sh.full[s], (g / kStages) & 1, &sh.abort)) break;
      issued++;
      tc_fence_after();
      const uint32_t base = smem_u32(tiles + (size_t)s * kKBlockBytes);
#pragma unroll
      for (int kk = 0; kk < kTcKBlock / 16; kk++) {
        const uint64_t desc = sw128_desc(base + 32u * kk);
        tc_mma(d, desc, desc, idesc, (kb | kk) != 0 ? 1u : 0u);
      }
      tc_commit(&sh.empty[s]);  // the stage goes back once these MMAs are done
    }
    if (issued > 0) {  // also after a give-up mid-tile: the drain below then covers it
      tc_commit(&sh.acc_full[b]);
      last_b = b;
      last_parity = ub & 1;
    }
    if (issued < kbc) {
      give_up(sh, err);
      break;
    }
  }
  // drain: the last MMA chain has completed before tensor memory is freed
  if (last_b >= 0 && !mbar_wait(&sh.acc_full[last_b], last_parity, nullptr))
    atomicOr(err, DEVERR_TIMEOUT);
}

// Row minimum over 32 columns: key = clamped distance bits with the column in
// the low 6 bits (skip_col: the row's own column, or -1).
template <bool kSkip>
__device__ __forceinline__ uint32_t row_min32(const uint32_t (&v)[32], const float *cn, float na,
                                              float dscale, int skip_col) {
  uint32_t best[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};  // four chains
#pragma unroll
  for (int c4 = 0; c4 < 8; c4++) {
    const float4 nc = reinterpret_cast<const float4 *>(cn)[c4];
    const float ncs[4] = {nc.x, nc.y, nc.z, nc.w};
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int c = 4 * c4 + e;
      const float dd = fmaxf(__fmaf_rn(dscale, __uint_as_float(v[c]), __fadd_rn(na, ncs[e])), 0.0f);
      uint32_t key = (__float_as_uint(dd) & ~63u) | (uint32_t)c;
      if (kSkip) key = c == skip_col ? 0xffffffffu : key;
      best[e] = min(best[e], key);
    }
  }
  return min(min(best[0], best[1]), min(best[2], best[3]));
}

// row_min32 of this lane's row (keys carry the column) and, from the same
// distances, the minimum of every column over the warp's 32 rows: on return
// lane l holds column l's minimum, keyed by the row's lane.  The column minima
// take 31 shuffles: at each step a lane keeps half of its live columns and
// takes the other lane's values for them (recursive halving).
__device__ __forceinline__ uint32_t row_col_min32(uint32_t (&v)[32], const float *cn, float na,
                                                  float dscale, int lane, uint32_t &colmin) {
  uint32_t best[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
#pragma unroll
  for (int c4 = 0; c4 < 8; c4++) {
    const float4 nc = reinterpret_cast<const float4 *>(cn)[c4];
    const float ncs[4] = {nc.x, nc.y, nc.z, nc.w};
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int c = 4 * c4 + e;
      const float dd = fmaxf(__fmaf_rn(dscale, __uint_as_float(v[c]), __fadd_rn(na, ncs[e])), 0.0f);
      const uint32_t db = __float_as_uint(dd) & ~63u;
      best[e] = min(best[e], db | (uint32_t)c);
      v[c] = db | (uint32_t)lane;
    }
  }
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const bool up = (lane & s) != 0;
#pragma unroll
    for (int i = 0; i < s; i++) {
      const uint32_t send = up ? v[i] : v[i + s];
      const uint32_t keep = up ? v[i + s] : v[i];
      v[i] = min(keep, __shfl_xor_sync(0xffffffffu, send, s));
    }
  }
  colmin = v[0];
  return min(min(best[0], best[1]), min(best[2], best[3]));
}

template <bool kProbe>
__device__ void epilogue(const JoinArgs &a, Shared &sh, uint32_t tmem, int64_t n, int64_t ntiles,
                         unsigned long long &cands) {
  ListCursor cur;
  const int w = threadIdx.x >> 5, lane = lane_id();
  const int j = w >> 1;                 // row-join of this warp's 32 rows
  const bool isnew = (w & 1) == 0;      // new rows (slots 0..31) or old rows (32..63)
  const int slot = (isnew ? 0 : 32) + lane;
  int64_t t = blockIdx.x;
  for (uint32_t i = 0; t < ntiles; t += gridDim.x, i++) {
    const int m = i % kMetaSlots;
    const uint32_t muse = i / kMetaSlots;
    const int b = i & 1;
    const uint32_t ub = i >> 1;
    if (!__all_sync(0xffffffffu, mbar_wait(&sh.mfull[m], muse & 1, &sh.abort))) {
      give_up(sh, a.err);
      break;
    }
    const StageMeta &M = sh.meta[m];
    const int nn = M.nn[j], no = M.no[j];
    const bool vrow = isnew ? lane < nn : lane < no;
    const int32_t myid = M.ids[64 * j + slot];
    const float na = M.nrm[64 * j + slot];
    const float wst = M.wst[64 * j + slot];
    if (!__all_sync(0xffffffffu, mbar_wait(&sh.acc_full[b], ub & 1, &sh.abort))) {
      give_up(sh, a.err);
      break;
    }
    tc_fence_after();
    uint32_t v0[32], v1[32];
    const uint32_t taddr = tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)(b * kAccCols + 64 * j);
    tmem_ld32(taddr, v0);
    if (kProbe) {  // both loads in flight, one wait
      tmem_ld32(taddr + 32, v1);
      tmem_wait_ld2(v0, v1);
    } else {
      tmem_wait_ld(v0);  // the new columns: the old ones come from the old rows' warp
    }
    tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(&sh.acc_empty[b]);
    const float *cn = M.nrm + 64 * j;
    if (kProbe) {
      float *o = a.probe_out + ((size_t)t * kTcTileRows + 64 * j + slot) * 64;
#pragma unroll
      for (int c = 0; c < 32; c++) {
        o[c] = __fmaf_rn(a.dscale, __uint_as_float(v0[c]), __fadd_rn(na, cn[c]));
        o[32 + c] = __fmaf_rn(a.dscale, __uint_as_float(v1[c]), __fadd_rn(na, cn[32 + c]));
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.mempty[m]);
      continue;
    }
    // new rows: their closest other new row.  Old rows: their closest new
    // row, and -- the new x old block being the transpose of the old x new
    // one -- the closest old row of every new row, as column minima over the
    // old rows; lane l then speaks for new row l.
    uint32_t k1, k2 = 0xffffffffu;
    int32_t id1 = -1, id2 = -1, tgt2 = -1;
    float wst2 = 0.0f;
    if (isnew) {
      k1 = row_min32<true>(v0, cn, na, a.dscale, lane);
    } else {
      k1 = row_col_min32(v0, cn, na, a.dscale, lane, k2);
      if (k2 < kNoKey) id2 = M.ids[64 * j + 32 + (k2 & 63u)];
      tgt2 = M.ids[64 * j + lane];
      wst2 = M.wst[64 * j + lane];
    }
    if (k1 < kNoKey) id1 = M.ids[64 * j + (k1 & 63u)];
    __syncwarp();
    if (lane == 0) mbar_arrive(&sh.mempty[m]);
    // candidates that can enter their target's list, appended to the list
    // that is sorted by target before the next merge: one reservation per
    // warp instead of a returning inbox atomic per candidate
    const float d1 = __uint_as_float(k1 & ~63u), d2 = __uint_as_float(k2 & ~63u);
    const bool c1 = vrow && id1 >= 0 && d1 < wst;
    const bool c2 = !isnew && lane < nn && id2 >= 0 && d2 < wst2;
    cands += append_candidates(a.ib, cur, (uint32_t)n, c1, myid, pack(d1, id1), c2, tgt2,
                               pack(d2, id2));
  }
  if (!kProbe) list_fill(a.ib, cur.pos, cur.end, (uint32_t)n);  // the rest of the last chunk
}

template <bool kProbe>
__global__ void __launch_bounds__(kThreads, 1)
    k_join_tc(const __grid_constant__ CUtensorMap xmap, int64_t n, int64_t ntiles, int kbc, int S,
              JoinArgs a) {
  extern __shared__ unsigned char smem_raw[];
  // the swizzled operand tiles start on a 1024-byte boundary of shared memory
  unsigned char *tiles = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  Shared &sh = *reinterpret_cast<Shared *>(tiles + (size_t)kStages * kKBlockBytes);
  const int warp = threadIdx.x >> 5;
  // stale columns of a stage must hold finite values: start from zeros
  {
    uint4 *z = reinterpret_cast<uint4 *>(tiles);
    const int nz = kStages * kKBlockBytes / 16;
    for (int i = threadIdx.x; i < nz; i += kThreads) z[i] = make_uint4(0, 0, 0, 0);
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&sh.full[s], 1);   // the producer's expect_tx; the gathers complete it
      mbar_init(&sh.empty[s], 1);  // the MMA thread's commit
      sh.armed[s] = 0;
    }
    for (int m = 0; m < kMetaSlots; m++) {
      mbar_init(&sh.mfull[m], kMetaArrivals);
      mbar_init(&sh.mempty[m], kEpiWarps);
      sh.marmed[m] = 0;
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&sh.acc_full[b], 1);
      mbar_init(&sh.acc_empty[b], kEpiWarps);
    }
    sh.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == kMmaWarp) {
    __syncwarp();  // .sync.aligned: after the per-thread zeroing loop, reconverge first
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&sh.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh.tmem_base;
  unsigned long long stat = 0;
  if (warp >= kProducerWarp0 && warp < kMmaWarp) {
    producer<kProbe>(warp - kProducerWarp0, &xmap, a, sh, tiles, n, ntiles, kbc, S, stat);
    if (!kProbe && lane_id() == 0 && stat) atomicAdd(&a.ib.counters[1], stat);
  } else if (warp == kMmaWarp) {
    if (lane_id() == 0) mma_issuer(sh, tiles, tmem, ntiles, kbc, a.idesc, a.err);
    __syncwarp();
  } else {
    epilogue<kProbe>(a, sh, tmem, n, ntiles, stat);
    if (!kProbe) {
#pragma unroll
      for (int o = 16; o; o >>= 1) stat += __shfl_xor_sync(0xffffffffu, stat, o);
      if (lane_id() == 0 && stat) atomicAdd(&a.ib.counters[2], stat);
    }
  }
  tc_fence_before();
  __syncthreads();
  // drain, once every role is done: the copies of the last armed use of each
  // stage have landed before the CTA's shared memory goes away
  if (threadIdx.x == 32 * kProducerWarp0) {
    for (int s = 0; s < kStages; s++) {
      const uint32_t u = sh.armed[s];
      if (u > 0 && !mbar_wait(&sh.full[s], (u - 1) & 1, nullptr)) atomicOr(a.err, DEVERR_TIMEOUT);
    }
    for (int m = 0; m < kMetaSlots; m++) {  // the norm / worst[] copies as well
      const uint32_t u = sh.marmed[m];
      if (u > 0 && !mbar_wait(&sh.mfull[m], (u - 1) & 1, nullptr)) atomicOr(a.err, DEVERR_TIMEOUT);
    }
  }
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// ---- host ----------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

size_t smem_bytes() {
  size_t b = 1024 + (size_t)kStages * kKBlockBytes + sizeof(Shared);
  return b < kMinSmem ? kMinSmem : b;
}

template <bool kProbe>
void launch(Context *ctx, const TcJoin &tj, int64_t ntiles, int S, const JoinArgs &a) {
  const int kbc = tj.dpad / kTcKBlock;
  HDB_CUDA(cudaFuncSetAttribute(k_join_tc<kProbe>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_bytes()));
  const int64_t g = std::min<int64_t>(ntiles, 2 * (int64_t)ctx->num_sms);
  if (g <= 0) return;
  k_join_tc<kProbe><<<(int)g, kThreads, tj.smem, ctx->stream>>>(tj.xmap, tj.n, ntiles, kbc, S, a);
  ctx->launches++;
  HDB_CHECK_LAUNCH();
}

}  // namespace

void tc_join_prepare(Context *ctx, const uint16_t *Xb, int64_t n, int dpad, bool fp16, float dscale,
                     TcJoin *tj) {
  HDB_REQUIRE(dpad % kTcKBlock == 0 && dpad >= kTcKBlock && dpad <= kTcMaxDpad, HDB_ERR_ARG,
              "tensor-core join: padded dimension must be a multiple of 64 in [64, 256]");
  HDB_REQUIRE(n >= 1 && n < (int64_t(1) << 31), HDB_ERR_ARG, "tensor-core join: bad row count");
  HDB_REQUIRE((reinterpret_cast<uintptr_t>(Xb) & 15) == 0, HDB_ERR_INTERNAL,
              "tensor-core join: rows not 16-byte aligned");
  auto fn = encode_tiled();
  HDB_REQUIRE(fn != nullptr, HDB_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  cuuint64_t gdim[2] = {(cuuint64_t)dpad, (cuuint64_t)n};
  cuuint64_t gstride[1] = {(cuuint64_t)dpad * sizeof(uint16_t)};
  cuuint32_t box[2] = {(cuuint32_t)kTcKBlock, 1};  // one row high (gather4)
  cuuint32_t estride[2] = {1, 1};
  CUresult r = fn(&tj->xmap, fp16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16,
                  2, const_cast<uint16_t *>(Xb),
                  gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  HDB_REQUIRE(r == CUDA_SUCCESS, HDB_ERR_CUDA,
              "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  tj->n = n;
  tj->dpad = dpad;
  tj->smem = smem_bytes();
  tj->idesc = idesc_for(fp16);
  tj->dscale = dscale;
  (void)ctx;
}

void tc_join_launch(Context *ctx, const TcJoin &tj, int S, const float *nrm, const int32_t *newS,
                    const int32_t *oldS, const int8_t *nf, const int8_t *of, int32_t *nrev,
                    int32_t *orev, const float *worst, const Inbox &ib) {
  HDB_REQUIRE(S >= 1 && 2 * S <= 32, HDB_ERR_ARG, "tensor-core join: need 2 * SAMPLE_NUM <= 32");
  k_join_lists<<<grid_for(ctx, tj.n, 8, 8), 256, 0, ctx->stream>>>(
      tj.n, S, const_cast<int32_t *>(newS), const_cast<int32_t *>(oldS),
      const_cast<int8_t *>(nf), const_cast<int8_t *>(of), nrev, orev);
  ctx->launches++;
  HDB_CHECK_LAUNCH();
  JoinArgs a{nrm,     newS,    oldS,    nf,           of,       nrev,     orev,
             worst,   ib,      nullptr, nullptr,      nullptr,  ctx->dev_err, tj.idesc,
             tj.dscale};
  launch<false>(ctx, tj, (tj.n + 1) / 2, S, a);
}

void tc_gram_probe(Context *ctx, const uint16_t *Xb, const float *nrm, int64_t n, int dpad,
                   const int32_t *ids, const int32_t *counts, int64_t tiles, float *out) {
  TcJoin tj;
  tc_join_prepare(ctx, Xb, n, dpad, false, -2.0f, &tj);
  JoinArgs a{nrm,     nullptr, nullptr, nullptr, nullptr, nullptr,      nullptr,
             nullptr, Inbox{}, ids,     counts,  out,     ctx->dev_err, tj.idesc,
             tj.dscale};
  launch<true>(ctx, tj, tiles, 1, a);
}

}  // namespace hdb
