/*
 * CPU oracle for the HDBSCAN hot path -- TEST INFRASTRUCTURE ONLY (see
 * hdb_oracle.h).  Plain C11 + OpenMP.  Every function restates the reference
 * algorithm of gorlando04/GPU_HDBSCAN and cites the file:line it follows.
 * Nothing here is shipped or called by the product library.
 */
#include "hdb_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void orc_free(void *p) { free(p); }

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Distances                                                                */
/* ------------------------------------------------------------------------ */

/* gpuknn/nndescent.cu:1086-1093 (and the tiled form :1242-1250): squared L2 as
 * a sequential "difference sum" in one thread.  nvcc contracts
 * `sum += diff * diff` into fmaf(diff, diff, sum); diff itself is rounded. */
float orc_diffsum(const float *a, const float *b, int32_t d) {
  float sum = 0.0f;
  for (int32_t j = 0; j < d; j++) {
    float diff = a[j] - b[j]; /* rounded: built with -ffp-contract=off */
    sum = fmaf(diff, diff, sum);
  }
  return sum;
}

/* build_kNNG.cu:4-13 and HDBSCAN/calculates/calculates.cu:275-283:
 * soma (float) += pow(a-b, 2) (double), then sqrt of the float sum. */
float orc_euclid_ref(const float *a, const float *b, int32_t d) {
  float soma = 0.0f;
  for (int32_t i = 0; i < d; i++) {
    float diff = a[i] - b[i];
    double sq = (double)diff * (double)diff; /* pow(float, 2) promotes; exact */
    soma = (float)((double)soma + sq);
  }
  return sqrtf(soma);
}

/* build_kNNG.cu:131-174: every kNN distance rewritten as sqrt-L2. */
void orc_fix_distances(const float *X, int64_t n, int32_t d, const int32_t *ids, int32_t k,
                       float *dist_out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++)
    for (int32_t j = 0; j < k; j++)
      dist_out[i * k + j] =
          orc_euclid_ref(X + i * (int64_t)d, X + (int64_t)ids[i * k + j] * d, d);
}

/* ------------------------------------------------------------------------ */
/* NN-Descent (gpuknn/nndescent.cu)                                          */
/* ------------------------------------------------------------------------ */

/* gpuknn/knncuda_tools.cu:126-132 */
uint64_t orc_xorshift64star(uint64_t x) {
  x += 42;
  x ^= x >> 12;
  x ^= x << 25;
  x ^= x >> 27;
  return x * 0x2545F4914F6CDD1DULL;
}

typedef struct { float d; int32_t id; } orc_nb; /* NNDElement (tools/nndescent_element.cuh:9) */

static int nb_less(orc_nb a, orc_nb b) { return a.d < b.d || (a.d == b.d && a.id < b.id); }

static int cmp_nb(const void *x, const void *y) {
  orc_nb a = *(const orc_nb *)x, b = *(const orc_nb *)y;
  if (nb_less(a, b)) return -1;
  if (nb_less(b, a)) return 1;
  return 0;
}

static int cmp_i32(const void *x, const void *y) {
  int32_t a = *(const int32_t *)x, b = *(const int32_t *)y;
  return (a > b) - (a < b);
}

typedef struct { int32_t target, id; float d; } orc_cand;

/* Candidate distances of a precision form inside the local join (the
 * evaluation of the BF16, FP16 and FP8 e4m3 forms; the reference computes
 * every candidate distance as the FP32 difference sum).  q holds each row's
 * quantised coordinates (of the column-centred rows), scale a per-row scale
 * (NULL: 1), nrm the squared norm of the dequantised row; a pair's distance
 * is nrm_u + nrm_v - 2 s_u s_v (q_u . q_v), clamped at 0, in FP32. */
typedef struct {
  const float *q, *scale, *nrm;
} orc_qrows;

static float pair_dist(const float *X, int32_t d, const orc_qrows *Q, int32_t u, int32_t v) {
  if (!Q) return orc_diffsum(X + (int64_t)u * d, X + (int64_t)v * d, d);
  const float *a = Q->q + (int64_t)u * d, *b = Q->q + (int64_t)v * d;
  float dot = 0.0f;
  for (int32_t j = 0; j < d; j++) dot = fmaf(a[j], b[j], dot);
  const float s = Q->scale ? Q->scale[u] * Q->scale[v] : 1.0f;
  const float r = Q->nrm[u] + Q->nrm[v] - 2.0f * s * dot;
  return r > 0.0f ? r : 0.0f;
}

/* `iterations` rounds of sampling + local join + merge on G (n rows of k,
 * sorted by (distance, id)) with its new/old flags.  split > 0 is the merge of
 * the point sets [0, split) and [split, n) (NNDescentForMerge,
 * nndescent.cu:1999-2087): old entries are sampled only from the row's own
 * set (PrepareGraphForMerge :100-166) and the join compares new x old pairs
 * only (TiledNewOldNeighborsCompareKernelForMerge :1328-1383 without the
 * new x new kernel, UpdateGraphForMerge :1582-1640). */
static int nnd_iterate(const float *X, int64_t n, int32_t d, int32_t k, int32_t S,
                       int32_t iterations, int64_t split, orc_nb *G, uint8_t *isnew,
                       const orc_qrows *Q) {
  int32_t *newl = (int32_t *)malloc(sizeof(int32_t) * n * 2 * S);
  int32_t *oldl = (int32_t *)malloc(sizeof(int32_t) * n * 2 * S);
  int32_t *nfwd = (int32_t *)calloc(n, 4), *ofwd = (int32_t *)calloc(n, 4);
  int32_t *nrev = (int32_t *)calloc(n, 4), *orev = (int32_t *)calloc(n, 4);
  const int64_t cap = 3 * 2 * (int64_t)S; /* candidates per joined row */
  orc_cand *cand = (orc_cand *)malloc(sizeof(orc_cand) * n * cap);
  int32_t *ncand = (int32_t *)calloc(n, 4);
  int64_t *off = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
  orc_cand *bucket = (orc_cand *)malloc(sizeof(orc_cand) * n * cap);
  if (!newl || !oldl || !nfwd || !ofwd || !nrev || !orev || !cand || !ncand || !off || !bucket) {
    free(newl); free(oldl); free(nfwd); free(ofwd); free(nrev);
    free(orev); free(cand); free(ncand); free(off); free(bucket);
    return ORC_ERR_ALLOC;
  }
  const int cross_only = split > 0;

  for (int32_t it = 0; it < iterations; it++) {
    /* PrepareGraph (:44-98): first S new / first S old by position. */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      int32_t cn = 0, co = 0;
      for (int32_t t = 0; t < k; t++) {
        const int32_t id = G[i * k + t].id;
        if (isnew[i * k + t]) {
          if (cn < S) newl[i * 2 * S + cn++] = id;
        } else if (split <= 0 || ((i < split) == (id < split))) {
          if (co < S) oldl[i * 2 * S + co++] = id;
        }
      }
      nfwd[i] = cn;
      ofwd[i] = co;
      nrev[i] = 0;
      orev[i] = 0;
    }
    /* PrepareReverseGraph (:293-346): slots [S, 2S), at most S per row. */
    for (int64_t i = 0; i < n; i++) {
      for (int32_t t = 0; t < nfwd[i]; t++) {
        int32_t u = newl[i * 2 * S + t];
        if (nrev[u] < S) newl[(int64_t)u * 2 * S + S + nrev[u]++] = (int32_t)i;
      }
      for (int32_t t = 0; t < ofwd[i]; t++) {
        int32_t u = oldl[i * 2 * S + t];
        if (orev[u] < S) oldl[(int64_t)u * 2 * S + S + orev[u]++] = (int32_t)i;
      }
    }
    /* MarkAllToOld (:1398-1403) happens before the join. */
    memset(isnew, 0, (size_t)n * k);

    /* ShrinkGraph (:405-510) + join (:1030-1108, :1259-1326). */
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
      int32_t nv[64], ov[64], nn = 0, no = 0;
      for (int32_t t = 0; t < nfwd[i]; t++) nv[nn++] = newl[i * 2 * S + t];
      for (int32_t t = 0; t < nrev[i]; t++) nv[nn++] = newl[i * 2 * S + S + t];
      for (int32_t t = 0; t < ofwd[i]; t++) ov[no++] = oldl[i * 2 * S + t];
      for (int32_t t = 0; t < orev[i]; t++) ov[no++] = oldl[i * 2 * S + S + t];
      qsort(nv, nn, 4, cmp_i32);
      qsort(ov, no, 4, cmp_i32);
      int32_t m = 0; /* RemoveDuplicates (:285-291) */
      for (int32_t t = 0; t < nn; t++) if (m == 0 || nv[t] != nv[m - 1]) nv[m++] = nv[t];
      nn = m;
      m = 0;
      for (int32_t t = 0; t < no; t++) if (m == 0 || ov[t] != ov[m - 1]) ov[m++] = ov[t];
      no = m;
      m = 0; /* new \ old (:468-486) */
      for (int32_t t = 0; t < nn; t++) {
        int hit = 0;
        for (int32_t u = 0; u < no && !hit; u++) hit = (nv[t] == ov[u]);
        if (!hit) nv[m++] = nv[t];
      }
      nn = m;
      orc_cand *cb = cand + i * cap;
      int32_t nc = 0;
      float dno[64][64];
      for (int32_t a = 0; a < nn; a++)
        for (int32_t b = 0; b < no; b++)
          dno[a][b] = pair_dist(X, d, Q, nv[a], ov[b]);
      for (int32_t a = 0; a < nn; a++) {
        if (!cross_only) {
          orc_nb best = {1e10f, INT_MAX};
          for (int32_t b = 0; b < nn; b++) {
            if (b == a) continue;
            orc_nb c = {pair_dist(X, d, Q, nv[a], nv[b]), nv[b]};
            if (nb_less(c, best)) best = c;
          }
          if (best.id != INT_MAX) cb[nc++] = (orc_cand){nv[a], best.id, best.d};
        }
        orc_nb best2 = {1e10f, INT_MAX};
        for (int32_t b = 0; b < no; b++) {
          orc_nb c = {dno[a][b], ov[b]};
          if (nb_less(c, best2)) best2 = c;
        }
        if (best2.id != INT_MAX) cb[nc++] = (orc_cand){nv[a], best2.id, best2.d};
      }
      for (int32_t b = 0; b < no; b++) {
        orc_nb best = {1e10f, INT_MAX};
        for (int32_t a = 0; a < nn; a++) {
          orc_nb c = {dno[a][b], nv[a]};
          if (nb_less(c, best)) best = c;
        }
        if (best.id != INT_MAX) cb[nc++] = (orc_cand){ov[b], best.id, best.d};
      }
      ncand[i] = nc;
    }
    /* Group candidates by target, then merge: the list becomes the k best of
     * (list U candidates) -- the order-independent result of repeated
     * InsertToGlobalGraph calls. */
    memset(off, 0, sizeof(int64_t) * (n + 1));
    for (int64_t i = 0; i < n; i++)
      for (int32_t t = 0; t < ncand[i]; t++) off[cand[i * cap + t].target + 1]++;
    for (int64_t i = 0; i < n; i++) off[i + 1] += off[i];
    {
      int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * n);
      memcpy(fill, off, sizeof(int64_t) * n);
      for (int64_t i = 0; i < n; i++)
        for (int32_t t = 0; t < ncand[i]; t++) {
          orc_cand c = cand[i * cap + t];
          bucket[fill[c.target]++] = c;
        }
      free(fill);
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t x = 0; x < n; x++) {
      orc_nb *row = G + x * k;
      uint8_t *fl = isnew + x * k;
      for (int64_t q = off[x]; q < off[x + 1]; q++) {
        orc_nb c = {bucket[q].d, bucket[q].id};
        if (c.id == (int32_t)x || !nb_less(c, row[k - 1])) continue;
        int dup = 0;
        for (int32_t u = 0; u < k && !dup; u++) dup = (row[u].id == c.id);
        if (dup) continue;
        int32_t p = k - 1;
        while (p > 0 && nb_less(c, row[p - 1])) { row[p] = row[p - 1]; fl[p] = fl[p - 1]; p--; }
        row[p] = c;
        fl[p] = 1;
      }
    }
  }
  free(newl); free(oldl); free(nfwd); free(ofwd); free(nrev);
  free(orev); free(cand); free(ncand); free(off); free(bucket);
  return ORC_OK;
}

/*
 * Sequential restatement of gpuknn::NNDescent (nndescent.cu:2088-2199):
 *   InitRandomKNNGraph (:1800-1871; ids from xorshift64star(pos) % n, :1673-1692),
 *   then `iterations` rounds of PrepareForUpdate (:624-671) + UpdateGraph
 *   (:1487-1580).  Candidate semantics follow the join kernels: every new
 *   neighbour x is offered its closest other new neighbour (:1030-1108) and its
 *   closest old neighbour, every old neighbour its closest new one
 *   (:1259-1326); InsertToGlobalGraph (:969-1028) keeps a sorted, duplicate-free
 *   list of k.  Flags: all entries become "old" before the join (MarkAllToOld
 *   :1398), inserted candidates are "new".
 * Deterministic choices where the reference races: forward samples are the
 * first S new / old entries by list position; reverse samples keep the first S
 * sources in row order; ties order by (distance, id).  The initial distance is
 * the same sequential difference sum as the join (the reference's warp-tree sum
 * at :1694-1726 rounds differently), and an initial id already present in the
 * row is advanced like a self id, so rows never hold duplicates.
 * Output ids carry no old/new flag; distances are squared L2.
 */
/* InitKNNGraphIndexKernel (:1673-1692) + distances + per-row sort. */
static void nnd_init(const float *X, int64_t n, int32_t d, int32_t k, orc_nb *G, uint8_t *isnew) {
  const int32_t NB = (k + 31) / 32;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    orc_nb *row = G + i * k;
    for (int32_t t = 0; t < k; t++) {
      int64_t pos = i * k + t;
      int32_t blk = t / 32;
      int64_t label = (int64_t)(orc_xorshift64star((uint64_t)pos) % (uint64_t)n);
      for (;;) {
        int bad = (label % NB != blk) || label == i;
        for (int32_t u = 0; u < t && !bad; u++) bad = (row[u].id == label);
        if (!bad) break;
        label = (label + 1) % n;
      }
      row[t].id = (int32_t)label;
      row[t].d = orc_diffsum(X + i * (int64_t)d, X + label * d, d);
    }
    qsort(row, k, sizeof(orc_nb), cmp_nb);
    memset(isnew + i * k, 1, k);
  }
}

int orc_nndescent(const float *X, int64_t n, int32_t d, int32_t k, int32_t S,
                  int32_t iterations, int32_t *ids_out, float *dist_out) {
  return orc_nndescent_form(X, n, d, k, S, iterations, ORC_FORM_FP32, ids_out, dist_out);
}

/* Round to the nearest BF16 value, ties to even. */
static float round_bf16(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

/* Round to the nearest FP8 e4m3 value (OCP FP8: 4 exponent bits, bias 7, 3
 * mantissa bits, largest finite 448, subnormal step 2^-9), ties to even,
 * saturating at +-448. */
static float round_e4m3(float x) {
  const float a = fabsf(x);
  float q;
  if (a >= 448.0f) {
    q = 448.0f;
  } else if (a < 0.015625f) {  /* below 2^-6: subnormal, step 2^-9 */
    q = rintf(a * 512.0f) / 512.0f;
  } else {
    int e;
    frexpf(a, &e);                       /* a = m 2^e, m in [0.5, 1) */
    const float step = ldexpf(1.0f, e - 4);  /* 3 mantissa bits below the leading one */
    q = rintf(a / step) * step;
    if (q > 448.0f) q = 448.0f;
  }
  return copysignf(q, x);
}

/* Round to the nearest FP16 value (5 exponent bits, bias 15, 10 mantissa
 * bits; subnormal step 2^-24), ties to even; the callers scale rows so that
 * nothing overflows. */
static float round_fp16(float x) {
  const float a = fabsf(x);
  float q;
  if (a < 6.103515625e-05f) {  /* below 2^-14: subnormal, step 2^-24 */
    q = rintf(a * 16777216.0f) / 16777216.0f;
  } else {
    int e;
    frexpf(a, &e);
    const float step = ldexpf(1.0f, e - 11);  /* 10 mantissa bits below the leading one */
    q = rintf(a / step) * step;
  }
  return copysignf(q, x);
}

/*
 * NN-Descent with the local join's candidate distances taken in a precision
 * form (ORC_FORM_FP32: the reference's difference sum, as orc_nndescent;
 * ORC_FORM_BF16: the Gram form of the column-centred rows rounded to BF16;
 * ORC_FORM_FP8: the Gram form of the column-centred rows in FP8 e4m3 with a
 * per-row scale max|x| / 448; ORC_FORM_FP16: in FP16 with one power-of-two
 * scale for all rows), the initial distances exact, and every kept
 * neighbour re-ranked with the exact FP32 difference sum at the end -- the
 * structure of the library's BF16 tensor-core form, used to measure what a
 * form does to the final graph's recall.  Output as orc_nndescent.
 */
int orc_nndescent_form(const float *X, int64_t n, int32_t d, int32_t k, int32_t S,
                       int32_t iterations, int32_t form, int32_t *ids_out, float *dist_out) {
  if (n < 2 || k < 1 || k > 1024 || S < 1 || 2 * S > k || n <= k) return ORC_ERR_ARG;
  if (form < ORC_FORM_FP32 || form > ORC_FORM_FP16) return ORC_ERR_ARG;
  orc_nb *G = (orc_nb *)malloc(sizeof(orc_nb) * n * k);
  uint8_t *isnew = (uint8_t *)malloc((size_t)n * k);
  float *q = NULL, *scale = NULL, *nrm = NULL;
  if (form != ORC_FORM_FP32) {
    q = (float *)malloc(sizeof(float) * n * d);
    nrm = (float *)malloc(sizeof(float) * n);
    if (form == ORC_FORM_FP8 || form == ORC_FORM_FP16) scale = (float *)malloc(sizeof(float) * n);
  }
  if (!G || !isnew || (form != ORC_FORM_FP32 && (!q || !nrm)) ||
      ((form == ORC_FORM_FP8 || form == ORC_FORM_FP16) && !scale)) {
    free(G); free(isnew); free(q); free(scale); free(nrm);
    return ORC_ERR_ALLOC;
  }
  nnd_init(X, n, d, k, G, isnew);
  orc_qrows Q = {q, scale, nrm};
  if (form != ORC_FORM_FP32) {
    double *mean = (double *)calloc(d, sizeof(double));
    for (int64_t i = 0; i < n; i++)
      for (int32_t j = 0; j < d; j++) mean[j] += X[i * d + j];
    for (int32_t j = 0; j < d; j++) mean[j] /= (double)n;
    /* FP16: one power-of-two scale for all rows, max |x| / s in [2^14, 2^15) */
    float gmax = 0.0f, gscale = 1.0f;
    for (int64_t i = 0; i < n * d; i++) gmax = fmaxf(gmax, fabsf(X[i] - (float)mean[i % d]));
    if (gmax > 0.0f) {
      int e = 0;
      frexpf(gmax, &e);
      gscale = ldexpf(1.0f, e - 15);
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      float mx = 0.0f, s = 1.0f, acc = 0.0f;
      for (int32_t j = 0; j < d; j++) mx = fmaxf(mx, fabsf(X[i * d + j] - (float)mean[j]));
      if (form == ORC_FORM_FP8) {
        s = mx > 0.0f ? mx / 448.0f : 1.0f;
        scale[i] = s;
      } else if (form == ORC_FORM_FP16) {
        s = gscale;
        scale[i] = s;
      }
      for (int32_t j = 0; j < d; j++) {
        const float c = X[i * d + j] - (float)mean[j];
        const float v = form == ORC_FORM_BF16 ? round_bf16(c)
                        : form == ORC_FORM_FP8 ? round_e4m3(c / s) : round_fp16(c / s);
        q[i * d + j] = v;
        acc = fmaf(v * s, v * s, acc);
      }
      nrm[i] = acc;
    }
    free(mean);
  }
  int rc = nnd_iterate(X, n, d, k, S, iterations, 0, G, isnew,
                       form == ORC_FORM_FP32 ? NULL : &Q);
  if (rc == ORC_OK && form != ORC_FORM_FP32) {
    /* re-rank every kept neighbour with the exact difference sum */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      orc_nb *row = G + i * k;
      for (int32_t t = 0; t < k; t++) row[t].d = orc_diffsum(X + i * d, X + (int64_t)row[t].id * d, d);
      qsort(row, k, sizeof(orc_nb), cmp_nb);
    }
  }
  if (rc == ORC_OK)
    for (int64_t i = 0; i < n * k; i++) {
      ids_out[i] = G[i].id;
      dist_out[i] = G[i].d;
    }
  free(G); free(isnew); free(q); free(scale); free(nrm);
  return rc;
}

/*
 * Sequential restatement of gpuknn::KNNMerge (knnmerge.cu:401-437): the kNN
 * graph of the union of the point sets A = X[0, n1) and B = X[n1, n1 + n2)
 * (X holds them back to back, as MergeVectors :358-399 lays them out) from
 * the graphs of each (ids1 [n1, k] local to A, ids2 [n2, k] local to B).
 * Initial rows (InitRandomBlockedKNNGraph :80-185, k <= 32, one block): the
 * first k - k/2 entries of the row's own subgraph row, shifted into the
 * merged numbering and old (MarkAllToOld of both subgraphs, :408-410), then
 * k/2 ids of the other set, xorshift64star(local row * (k/2) + t) % |other|,
 * new.  An id drawn twice is advanced to the next free one (the reference
 * keeps repeats).  All k distances are recomputed (InitRandomKNNGraph with
 * start_from_random_index = false, nndescent.cu:2013) as the join's sequential
 * difference sum, and each row is sorted by (distance, id).  Then
 * `iterations` merge rounds (nnd_iterate with split = n1).  The subgraph ids
 * must be valid: in their set, no self id, no repeat (ORC_ERR_ARG otherwise).
 */
int orc_knn_merge(const float *X, int64_t n1, int64_t n2, int32_t d, const int32_t *ids1,
                  const int32_t *ids2, int32_t k, int32_t S, int32_t iterations,
                  int32_t *ids_out, float *dist_out) {
  if (k < 1 || k > 32 || S < 1 || 2 * S > k || n1 <= k || n2 <= k) return ORC_ERR_ARG;
  const int64_t n = n1 + n2;
  const int32_t h = k - k / 2, r = k / 2;
  for (int64_t i = 0; i < n; i++) {
    const int inb = i >= n1;
    const int64_t local = inb ? i - n1 : i, own_n = inb ? n2 : n1;
    const int32_t *own = inb ? ids2 : ids1;
    for (int32_t t = 0; t < h; t++) {
      const int32_t v = own[local * k + t];
      if (v < 0 || v >= own_n || v == local) return ORC_ERR_ARG;
      for (int32_t u = 0; u < t; u++)
        if (own[local * k + u] == v) return ORC_ERR_ARG;
    }
  }
  orc_nb *G = (orc_nb *)malloc(sizeof(orc_nb) * n * k);
  uint8_t *isnew = (uint8_t *)malloc((size_t)n * k);
  if (!G || !isnew) {
    free(G); free(isnew);
    return ORC_ERR_ALLOC;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    const int inb = i >= n1;
    const int64_t local = inb ? i - n1 : i;
    const int64_t own_off = inb ? n1 : 0, oth_n = inb ? n1 : n2, oth_off = inb ? 0 : n1;
    const int32_t *own = inb ? ids2 : ids1;
    orc_nb *row = G + i * k;
    for (int32_t t = 0; t < h; t++) row[t].id = (int32_t)(own[local * k + t] + own_off);
    for (int32_t t = 0; t < r; t++) {
      int64_t label = (int64_t)(orc_xorshift64star((uint64_t)(local * r + t)) % (uint64_t)oth_n);
      for (;;) {
        int dup = 0;
        for (int32_t u = 0; u < t && !dup; u++) dup = (row[h + u].id == label + oth_off);
        if (!dup) break;
        label = (label + 1) % oth_n;
      }
      row[h + t].id = (int32_t)(label + oth_off);
    }
    for (int32_t t = 0; t < k; t++)
      row[t].d = orc_diffsum(X + i * (int64_t)d, X + (int64_t)row[t].id * d, d);
    qsort(row, k, sizeof(orc_nb), cmp_nb);
    for (int32_t t = 0; t < k; t++) isnew[i * k + t] = (uint8_t)((row[t].id >= n1) != inb);
  }
  int rc = nnd_iterate(X, n, d, k, S, iterations, n1, G, isnew, NULL);
  if (rc == ORC_OK)
    for (int64_t i = 0; i < n * k; i++) {
      ids_out[i] = G[i].id;
      dist_out[i] = G[i].d;
    }
  free(G); free(isnew);
  return rc;
}

/* Exact kNN in FP64 (the ground truth cmake/eval.py:57 reads from outside the
 * repository): for each query row, the k nearest other rows by squared L2
 * computed in double, ties by id. */
int orc_bruteforce_knn(const float *X, int64_t n, int32_t d, int32_t k, const int64_t *queries,
                       int64_t nq, int32_t *ids_out, double *dist_out) {
  if (k < 1 || k >= n) return ORC_ERR_ARG;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t qi = 0; qi < nq; qi++) {
    int64_t q = queries ? queries[qi] : qi;
    double bd[1024];
    int32_t bi[1024];
    int32_t cnt = 0;
    const float *xq = X + q * d;
    for (int64_t j = 0; j < n; j++) {
      if (j == q) continue;
      const float *xj = X + j * d;
      double s = 0.0;
      for (int32_t t = 0; t < d; t++) {
        double df = (double)xq[t] - (double)xj[t];
        s += df * df;
      }
      if (cnt == k && !(s < bd[k - 1] || (s == bd[k - 1] && j < bi[k - 1]))) continue;
      int32_t p = cnt < k ? cnt++ : k - 1;
      while (p > 0 && (s < bd[p - 1] || (s == bd[p - 1] && j < bi[p - 1]))) {
        bd[p] = bd[p - 1];
        bi[p] = bi[p - 1];
        p--;
      }
      bd[p] = s;
      bi[p] = (int32_t)j;
    }
    for (int32_t t = 0; t < k; t++) {
      ids_out[qi * k + t] = bi[t];
      if (dist_out) dist_out[qi * k + t] = bd[t];
    }
  }
  return ORC_OK;
}

/* tools/evaluate.hpp:13-52: recall@r as the size of the set intersection of the
 * first r ids of each row, summed over rows, over rows * r. */
double orc_recall(const int32_t *ids, int32_t k_ids, const int32_t *gt, int32_t k_gt,
                  int64_t rows, int32_t r) {
  int64_t tp = 0;
  for (int64_t i = 0; i < rows; i++) {
    int32_t a[1024], b[1024];
    for (int32_t j = 0; j < r; j++) {
      int32_t v = ids[i * k_ids + j];
      a[j] = v < 0 ? -v - 1 : v; /* NNDElement::label() decodes the old flag */
      b[j] = gt[i * k_gt + j];
    }
    qsort(a, r, 4, cmp_i32);
    qsort(b, r, 4, cmp_i32);
    int32_t x = 0, y = 0;
    while (x < r && y < r) {
      if (a[x] == b[y]) { tp++; x++; y++; }
      else if (a[x] < b[y]) x++;
      else y++;
    }
  }
  return rows ? (double)tp / ((double)rows * r) : 0.0;
}

/* ------------------------------------------------------------------------ */
/* Enhanced kNN graph                                                       */
/* ------------------------------------------------------------------------ */

/* Input contract shared with the CUDA path: every id in [0, n), no self id,
 * no id twice in one row.  (The reference's own driver checks the duplicate
 * case and only prints, HDBSCAN/_new.cu:234-242; its CSR sizing is only
 * consistent without duplicates, calculates.cu:286-338.) */
int orc_validate_knn(const int32_t *ids, int64_t n, int32_t k) {
  for (int64_t i = 0; i < n; i++)
    for (int32_t j = 0; j < k; j++) {
      int32_t v = ids[i * k + j];
      if (v < 0 || v >= n || v == i) return ORC_ERR_ARG;
      for (int32_t u = 0; u < j; u++)
        if (ids[i * k + u] == v) return ORC_ERR_ARG;
    }
  return ORC_OK;
}

/* HDBSCAN/counts/count.cu:10-19 + :36-110 (all shards summed). */
void orc_degrees(const int32_t *ids, int64_t n, int32_t k, int32_t *deg) {
  memset(deg, 0, sizeof(int32_t) * n);
  for (int64_t e = 0; e < n * k; e++) deg[ids[e]]++;
}

typedef struct { int32_t key, index; } orc_vk;
static int cmp_vk(const void *x, const void *y) {
  const orc_vk *a = (const orc_vk *)x, *b = (const orc_vk *)y;
  if (a->key != b->key) return (a->key > b->key) - (a->key < b->key);
  return (a->index > b->index) - (a->index < b->index);
}

/*
 * buildEnhancedKNNG antihub selection, HDBSCAN/graphs/graph.cu:113-151:
 * P = get_NumThreshold(n) = (int)sqrt(n) (getters/getters.cu:6-9) vertices of
 * lowest in-degree; vertices tied at the threshold degree are ranked by
 * calculateScore = sum of their neighbours' degrees (calculates.cu:21-36,
 * 491-523).  Output sorted by index (graph.cu:151).  The reference's
 * std::partial_sort leaves equal keys unordered; ties go to the lower index.
 */
int32_t orc_select_antihubs(const int32_t *ids, const int32_t *deg, int64_t n, int32_t k,
                            int32_t *out) {
  int32_t P = (int32_t)sqrt((double)n);
  if (P < 1) return 0;
  orc_vk *v = (orc_vk *)malloc(sizeof(orc_vk) * n);
  for (int64_t i = 0; i < n; i++) v[i] = (orc_vk){deg[i], (int32_t)i};
  qsort(v, n, sizeof(orc_vk), cmp_vk);
  int32_t thr = v[P - 1].key;
  int64_t ties = 0;
  for (int64_t i = 0; i < n; i++) ties += (deg[i] == thr);
  int32_t cnt = 0;
  if (ties > 1) {
    int32_t not_ties = 0; /* get_TiedVertexes, getters.cu:11-24 */
    while (not_ties < P && v[not_ties].key != thr) not_ties++;
    int32_t missing = P - not_ties;
    for (int32_t i = 0; i < not_ties; i++) out[cnt++] = v[i].index;
    orc_vk *u = (orc_vk *)malloc(sizeof(orc_vk) * ties);
    int64_t m = 0;
    for (int64_t i = 0; i < n; i++)
      if (deg[i] == thr) {
        int32_t score = 0;
        for (int32_t j = 0; j < k; j++) score += deg[ids[i * k + j]];
        u[m++] = (orc_vk){score, (int32_t)i};
      }
    qsort(u, m, sizeof(orc_vk), cmp_vk);
    for (int32_t i = 0; i < missing; i++) out[cnt++] = u[i].index;
    free(u);
  } else {
    for (int32_t i = 0; i < P; i++) out[cnt++] = v[i].index;
  }
  free(v);
  qsort(out, cnt, 4, cmp_i32);
  return cnt;
}

/*
 * buildECLgraph, HDBSCAN/graphs/graph.cu:16-103:
 *  calculate_nindex (calculates.cu:286-338, findKNNlist getters.cu:41-49):
 *    row sizes, including the antihub clique;
 *  calculate_nlist (calculates.cu:340-410): row i = its k kNN ids in list
 *    order, then i' for every non-mutual edge i'->i in ascending i', then the
 *    other antihubs in ascending order (antihub rows only);
 *  calculateCoreDistance(dist, core, n, k, k-1) (graph.cu:77, calculates.cu:185-197);
 *  calculateMRD (calculates.cu:61-82): w = max(core[src], core[dst]);
 *  calculate_coreDistance_antihubs (calculates.cu:412-446): clique edges take
 *    max(w, sqrt-L2) with the float/pow recipe of calculates.cu:275-283.
 */
int64_t orc_enhanced_knng(const int32_t *ids, const float *dist, const float *X, int64_t n,
                          int32_t d, int32_t k, int64_t **nindex_out, int32_t **nlist_out,
                          float **eweight_out, int32_t **antihubs_out, int32_t *num_ah_out) {
  if (orc_validate_knn(ids, n, k) != ORC_OK) return -1;
  int32_t *deg = (int32_t *)malloc(sizeof(int32_t) * n);
  orc_degrees(ids, n, k, deg);
  int32_t P = (int32_t)sqrt((double)n);
  int32_t *ah = (int32_t *)malloc(sizeof(int32_t) * (P > 0 ? P : 1));
  int32_t nah = orc_select_antihubs(ids, deg, n, k, ah);
  free(deg);

  int64_t *nindex = (int64_t *)calloc(n + 1, sizeof(int64_t));
  int32_t *flag = (int32_t *)malloc(sizeof(int32_t) * n * k);
  for (int64_t i = 0; i < n; i++) {
    int64_t soma = 0;
    for (int32_t j = 0; j < k; j++) {
      int64_t neig = ids[i * k + j];
      int32_t FLAG = 0;
      for (int32_t t = 0; t < k; t++) FLAG += (ids[neig * k + t] == i);
      flag[i * k + j] = FLAG;
      if (FLAG > 1) { nindex[neig + 1] += FLAG - 1; nindex[i + 1] -= (FLAG - 1); }
      nindex[neig + 1] += 1;
      if (!FLAG) soma += 1;
    }
    nindex[i + 1] += soma;
  }
  {
    int32_t c = 0;
    for (int64_t i = 0; i < n; i++)
      if (c < nah && i == ah[c]) { c++; nindex[i + 1] += (nah - 1); }
  }
  for (int64_t i = 1; i < n + 1; i++) nindex[i] = nindex[i - 1] + nindex[i];
  int64_t E = nindex[n];

  int32_t *nlist = (int32_t *)malloc(sizeof(int32_t) * (E > 0 ? E : 1));
  int64_t *aux = (int64_t *)calloc(n, sizeof(int64_t));
  for (int64_t i = 0; i < n; i++) {
    int64_t pos = nindex[i] + aux[i];
    for (int32_t j = 0; j < k; j++) { nlist[pos++] = ids[i * k + j]; aux[i]++; }
  }
  for (int64_t i = 0; i < n; i++)
    for (int32_t j = 0; j < k; j++) {
      int64_t neig = ids[i * k + j];
      if (!flag[i * k + j]) nlist[nindex[neig] + aux[neig]++] = (int32_t)i;
    }
  for (int32_t i = 0; i < nah; i++) {
    int32_t cur = ah[i];
    int64_t pos = nindex[cur], o = aux[cur];
    for (int32_t j = 0; j < nah; j++)
      if (ah[j] != cur) nlist[pos + o++] = ah[j];
  }
  free(flag);

  float *core = (float *)malloc(sizeof(float) * n);
  for (int64_t i = 0; i < n; i++) core[i] = dist[i * k + (k - 1)];
  float *ew = (float *)malloc(sizeof(float) * (E > 0 ? E : 1));
  for (int64_t i = 0; i < n; i++)
    for (int64_t e = nindex[i]; e < nindex[i + 1]; e++) {
      float a = core[i], b = core[nlist[e]];
      ew[e] = a > b ? a : b;
    }
  free(core);
  for (int32_t i = 0; i < nah; i++) {
    int32_t ia = ah[i];
    int64_t pb = nindex[ia] + aux[ia];
    for (int32_t j = i; j < nah - 1; j++) {
      int32_t ib = ah[j + 1];
      float eu = orc_euclid_ref(X + (int64_t)ia * d, X + (int64_t)ib * d, d);
      if (ew[pb + j] < eu) {
        ew[pb + j] = eu;
        ew[nindex[ib] + aux[ib] + i] = eu;
      }
    }
  }
  free(aux);
  *nindex_out = nindex;
  *nlist_out = nlist;
  *eweight_out = ew;
  if (antihubs_out) *antihubs_out = ah; else free(ah);
  if (num_ah_out) *num_ah_out = nah;
  return E;
}

/*
 * Core-SG, HDBSCAN/core-sg/core-sg.cu: the union of the kNN graph and the MST
 * of the enhanced kNN graph, as build_CoreSG (:477-571) leaves it.
 *  core_sg_calculate_nindex (:101-145): row i has its k kNN ids, one entry
 *    i' for every non-mutual edge i'->i, and one entry per incident MST edge;
 *  core_sg_calculate_nlist (:148-237): kNN ids in list order, then the
 *    non-mutual sources in ascending order, then the MST neighbours in the
 *    order of the (sorted, buildMST mst.cu:291-336) MST edge list, the
 *    to_node row taking from_node before the from_node row takes to_node;
 *  the weights finally held are the Euclidean ones (update_core_sg_weights,
 *    :432-471, replaces the MRD weights by the vector written by
 *    core_sg_calculate_MRD_mst :242-285): the kNN distance for kNN and
 *    reverse entries (dist[i][j] of the listing row), and the float/pow
 *    Euclidean distance (calculates.cu:275-283) for MST entries.
 */
int64_t orc_core_sg(const int32_t *ids, const float *dist, const float *X, int64_t n, int32_t d,
                    int32_t k, const orc_mst_edge *mst, int64_t **nindex_out, int32_t **nlist_out,
                    float **eweight_out) {
  if (orc_validate_knn(ids, n, k) != ORC_OK) return -1;
  int64_t *nindex = (int64_t *)calloc(n + 1, sizeof(int64_t));
  int32_t *flag = (int32_t *)malloc(sizeof(int32_t) * n * k);
  for (int64_t i = 0; i < n; i++) {
    int64_t soma = 0;
    for (int32_t j = 0; j < k; j++) {
      int64_t neig = ids[i * k + j];
      int32_t FLAG = 0;
      for (int32_t t = 0; t < k; t++) FLAG += (ids[neig * k + t] == i);
      flag[i * k + j] = FLAG;
      if (FLAG > 1) { nindex[neig + 1] += FLAG - 1; nindex[i + 1] -= (FLAG - 1); }
      nindex[neig + 1] += 1;
      if (!FLAG) soma += 1;
    }
    nindex[i + 1] += soma;
  }
  for (int64_t e = 0; e < n - 1; e++) {
    nindex[mst[e].to_node + 1] += 1;
    nindex[mst[e].from_node + 1] += 1;
  }
  for (int64_t i = 1; i < n + 1; i++) nindex[i] = nindex[i - 1] + nindex[i];
  int64_t E = nindex[n];
  int32_t *nlist = (int32_t *)malloc(sizeof(int32_t) * (E > 0 ? E : 1));
  float *ew = (float *)malloc(sizeof(float) * (E > 0 ? E : 1));
  int64_t *aux = (int64_t *)calloc(n, sizeof(int64_t));
  for (int64_t i = 0; i < n; i++) {
    int64_t pos = nindex[i] + aux[i];
    for (int32_t j = 0; j < k; j++) {
      ew[pos] = dist[i * k + j];
      nlist[pos++] = ids[i * k + j];
      aux[i]++;
    }
  }
  for (int64_t i = 0; i < n; i++)
    for (int32_t j = 0; j < k; j++) {
      int64_t neig = ids[i * k + j];
      if (!flag[i * k + j]) {
        int64_t p = nindex[neig] + aux[neig]++;
        nlist[p] = (int32_t)i;
        ew[p] = dist[i * k + j];
      }
    }
  for (int64_t e = 0; e < n - 1; e++) {
    int32_t to = mst[e].to_node, from = mst[e].from_node;
    float eu = orc_euclid_ref(X + (int64_t)from * d, X + (int64_t)to * d, d);
    int64_t pt = nindex[to] + aux[to]++, pf = nindex[from] + aux[from]++;
    nlist[pt] = from;
    ew[pt] = eu;
    nlist[pf] = to;
    ew[pf] = eu;
  }
  free(flag);
  free(aux);
  *nindex_out = nindex;
  *nlist_out = nlist;
  *eweight_out = ew;
  return E;
}

/* ------------------------------------------------------------------------ */
/* MST                                                                       */
/* ------------------------------------------------------------------------ */

/* mst.cu:7-19 */
static int32_t serial_find(int32_t idx, int32_t *parent) {
  int32_t curr = parent[idx];
  if (curr != idx) {
    int32_t next, prev = idx;
    while (curr != (next = parent[curr])) {
      parent[prev] = next;
      prev = curr;
      curr = next;
    }
  }
  return curr;
}

typedef struct { float w; int64_t j; int32_t a, b; } orc_kedge;
static int cmp_kedge(const void *x, const void *y) {
  const orc_kedge *p = (const orc_kedge *)x, *q = (const orc_kedge *)y;
  if (p->w < q->w) return -1;
  if (q->w < p->w) return 1;
  return (p->j > q->j) - (p->j < q->j);
}

/* cpuMST, mst.cu:34-78: Kruskal over (weight, CSR edge index) of the entries
 * whose target is larger than their row, serial union-find. */
int orc_kruskal(const int64_t *nindex, const int32_t *nlist, const float *eweight, int32_t nodes,
                int64_t edges, uint8_t *in_mst) {
  memset(in_mst, 0, (size_t)edges);
  int32_t *parent = (int32_t *)malloc(sizeof(int32_t) * nodes);
  for (int32_t i = 0; i < nodes; i++) parent[i] = i;
  int64_t m = 0;
  for (int32_t i = 0; i < nodes; i++)
    for (int64_t j = nindex[i]; j < nindex[i + 1]; j++) m += (nlist[j] > i);
  orc_kedge *list = (orc_kedge *)malloc(sizeof(orc_kedge) * (m > 0 ? m : 1));
  m = 0;
  for (int32_t i = 0; i < nodes; i++)
    for (int64_t j = nindex[i]; j < nindex[i + 1]; j++)
      if (nlist[j] > i) list[m++] = (orc_kedge){eweight[j], j, i, nlist[j]};
  qsort(list, m, sizeof(orc_kedge), cmp_kedge);
  int32_t count = nodes - 1;
  for (int64_t p = 0; p < m && count > 0; p++) {
    int32_t ar = serial_find(list[p].a, parent), br = serial_find(list[p].b, parent);
    if (ar != br) {
      in_mst[list[p].j] = 1;
      if (ar > br) parent[br] = ar; else parent[ar] = br; /* serial_join, mst.cu:22-31 */
      count--;
    }
  }
  free(list);
  free(parent);
  return count == 0 ? ORC_OK : ORC_ERR_DISCONNECTED;
}

/* (weight, min id, max id, edge index): a canonical entry's row is its min id
 * and its target its max id. */
static int cmp_kedge_ids(const void *x, const void *y) {
  const orc_kedge *p = (const orc_kedge *)x, *q = (const orc_kedge *)y;
  if (p->w < q->w) return -1;
  if (q->w < p->w) return 1;
  if (p->a != q->a) return p->a < q->a ? -1 : 1;
  if (p->b != q->b) return p->b < q->b ? -1 : 1;
  return (p->j > q->j) - (p->j < q->j);
}

/* The float MST under a tie order: ORC_ORDER_EDGE is cpuMST's (weight, CSR
 * edge index), mst.cu:34-78; ORC_ORDER_IDS is (weight, min id, max id, edge
 * index).  Kruskal over the canonical entries (target > row) in that order;
 * out[nodes - 1] receives the chosen edges in the order they were taken,
 * which for ORC_ORDER_EDGE is the list orc_build_mst + orc_sort_edges give.
 * in_mst [edges] (optional) receives the bool-per-edge result. */
int orc_mst_ordered(const int64_t *nindex, const int32_t *nlist, const float *eweight,
                    int32_t nodes, int64_t edges, int32_t order, uint8_t *in_mst,
                    orc_mst_edge *out) {
  if (in_mst) memset(in_mst, 0, (size_t)edges);
  int32_t *parent = (int32_t *)malloc(sizeof(int32_t) * nodes);
  for (int32_t i = 0; i < nodes; i++) parent[i] = i;
  int64_t m = 0;
  for (int32_t i = 0; i < nodes; i++)
    for (int64_t j = nindex[i]; j < nindex[i + 1]; j++) m += (nlist[j] > i);
  orc_kedge *list = (orc_kedge *)malloc(sizeof(orc_kedge) * (m > 0 ? m : 1));
  m = 0;
  for (int32_t i = 0; i < nodes; i++)
    for (int64_t j = nindex[i]; j < nindex[i + 1]; j++)
      if (nlist[j] > i) list[m++] = (orc_kedge){eweight[j], j, i, nlist[j]};
  qsort(list, m, sizeof(orc_kedge), order == ORC_ORDER_IDS ? cmp_kedge_ids : cmp_kedge);
  int64_t taken = 0;
  for (int64_t p = 0; p < m && taken < nodes - 1; p++) {
    int32_t ar = serial_find(list[p].a, parent), br = serial_find(list[p].b, parent);
    if (ar != br) {
      if (in_mst) in_mst[list[p].j] = 1;
      out[taken++] = (orc_mst_edge){list[p].a, list[p].b, list[p].w};
      if (ar > br) parent[br] = ar; else parent[ar] = br;
    }
  }
  free(list);
  free(parent);
  return taken == nodes - 1 ? ORC_OK : ORC_ERR_DISCONNECTED;
}

/* buildMST, mst.cu:291-336 (before the sort): MST edges in CSR index order. */
int orc_build_mst(const int64_t *nindex, const int32_t *nlist, const float *eweight,
                  int32_t nodes, int64_t edges, const uint8_t *in_mst, orc_mst_edge *out) {
  int64_t soma = 0;
  for (int32_t i = 0; i < nodes; i++)
    for (int64_t j = nindex[i]; j < nindex[i + 1]; j++)
      if (in_mst[j]) {
        if (soma >= nodes - 1) return ORC_ERR_DISCONNECTED;
        out[soma++] = (orc_mst_edge){i, nlist[j], eweight[j]};
      }
  return soma == nodes - 1 ? ORC_OK : ORC_ERR_DISCONNECTED;
}

/* sort_edges / mergeSort, merge_sort.cu:27-116, 226-244: a stable ascending
 * sort on the weight alone (merge keeps the left element on equal weights). */
void orc_sort_edges(orc_mst_edge *e, int64_t m) {
  orc_mst_edge *tmp = (orc_mst_edge *)malloc(sizeof(orc_mst_edge) * (m > 0 ? m : 1));
  for (int64_t width = 1; width < m; width *= 2) {
    for (int64_t l = 0; l < m; l += 2 * width) {
      int64_t mid = l + width < m ? l + width : m;
      int64_t r = l + 2 * width < m ? l + 2 * width : m;
      int64_t i = l, j = mid, o = l;
      while (i < mid && j < r) tmp[o++] = (e[i].weight <= e[j].weight) ? e[i++] : e[j++];
      while (i < mid) tmp[o++] = e[i++];
      while (j < r) tmp[o++] = e[j++];
    }
    memcpy(e, tmp, sizeof(orc_mst_edge) * m);
  }
  free(tmp);
}

/* The mst_gpu = 1 MST of build_CoreSG (core-sg.cu:533-540).
 *  - GetMinDistanceFromKNNG (tools/filetool.hpp:312-347): the smallest
 *    positive first-neighbour distance of the .kgraph rows (start 999.0; row
 *    0's distance replaces it outright when positive); first_dist[i] is row
 *    i's first distance.
 *  - buildGPUgraph (core-sg.cu:8-44): multiplier m = ceil(-log10|min|) + 2,
 *    integer weights (int)(10^m * w).  A product outside the int range takes
 *    the value x86's truncating conversion gives it, INT_MIN.
 *  - gpuMST (mst.cu:210-288): Boruvka over the entries j with nlist[j] > row,
 *    keyed by ((uint32)q << 32 | j) -- unique keys, so the tree is Kruskal's
 *    under that order.
 *  - buildMST_gpu (mst.cu:338-380): chosen edges in CSR order with weight
 *    (float)(q / 10^m), then sort_edges (stable by weight).
 * Returns ORC_ERR_DISCONNECTED when the tree has fewer than nodes-1 edges. */
typedef struct { uint64_t key; int32_t a, b; } orc_qedge;
static int cmp_qedge(const void *x, const void *y) {
  uint64_t a = ((const orc_qedge *)x)->key, b = ((const orc_qedge *)y)->key;
  return a < b ? -1 : a > b;
}

int orc_mst_quantised(const int64_t *nindex, const int32_t *nlist, const float *eweight,
                      int32_t nodes, int64_t edges, const float *first_dist, orc_mst_edge *out,
                      int32_t *mult_out) {
  double min_value = 999.0;
  for (int32_t i = 0; i < nodes; i++) {
    double d = (double)first_dist[i];
    if (i == 0 && d > 0.0) min_value = d;
    else if (min_value > d && d > 0.0) min_value = d;
  }
  int32_t m = (int32_t)(ceil(-log10(fabs(min_value))) + 2);
  double p10 = pow(10.0, m);
  int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (edges > 0 ? edges : 1));
  for (int64_t j = 0; j < edges; j++) {
    double v = p10 * (double)eweight[j] / 1;
    q[j] = (v < 2147483648.0 && v > -2147483649.0) ? (int32_t)v : INT32_MIN;
  }
  int64_t cnt = 0;
  for (int32_t i = 0; i < nodes; i++)
    for (int64_t j = nindex[i]; j < nindex[i + 1]; j++) cnt += (nlist[j] > i);
  orc_qedge *list = (orc_qedge *)malloc(sizeof(orc_qedge) * (cnt > 0 ? cnt : 1));
  cnt = 0;
  for (int32_t i = 0; i < nodes; i++)
    for (int64_t j = nindex[i]; j < nindex[i + 1]; j++)
      if (nlist[j] > i)
        list[cnt++] = (orc_qedge){((uint64_t)(uint32_t)q[j] << 32) | (uint64_t)j, i, nlist[j]};
  qsort(list, cnt, sizeof(orc_qedge), cmp_qedge);
  int32_t *parent = (int32_t *)malloc(sizeof(int32_t) * nodes);
  for (int32_t i = 0; i < nodes; i++) parent[i] = i;
  uint8_t *in = (uint8_t *)calloc(edges > 0 ? edges : 1, 1);
  int32_t left = nodes - 1;
  for (int64_t p = 0; p < cnt && left > 0; p++) {
    int32_t ar = serial_find(list[p].a, parent), br = serial_find(list[p].b, parent);
    if (ar != br) {
      in[(uint32_t)list[p].key] = 1;
      if (ar > br) parent[br] = ar; else parent[ar] = br;
      left--;
    }
  }
  int64_t soma = 0;
  for (int32_t i = 0; i < nodes && left == 0; i++)
    for (int64_t j = nindex[i]; j < nindex[i + 1]; j++)
      if (in[j]) out[soma++] = (orc_mst_edge){i, nlist[j], (float)((1.0 * q[j]) / p10)};
  free(list); free(parent); free(in); free(q);
  if (left != 0) return ORC_ERR_DISCONNECTED;
  orc_sort_edges(out, nodes - 1);
  if (mult_out) *mult_out = m;
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Trees                                                                     */
/* ------------------------------------------------------------------------ */

/* UnionFind::FastFind, tree.cu:75-88 (the reference's compression loop also
 * writes parent_arr[-1] when called on a root; the result does not depend on
 * it). */
static int32_t uf_fastfind(int32_t *parent, int32_t n) {
  int32_t p = n;
  while (parent[n] != -1) n = parent[n];
  while (p != n && parent[p] != n) {
    int32_t q = parent[p];
    parent[p] = n;
    p = q;
  }
  return n;
}

/* build_Linkage_tree, tree.cu:171-202, UnionFind tree.cu:9-73: node N+i is the
 * merge made by sorted MST edge i; left/right are the current roots of its
 * endpoints. */
void orc_linkage_tree(const orc_mst_edge *mst, int64_t N, orc_linkage_node *out) {
  int32_t *parent = (int32_t *)malloc(sizeof(int32_t) * (2 * N - 1));
  int32_t *size = (int32_t *)malloc(sizeof(int32_t) * (2 * N - 1));
  for (int64_t i = 0; i < 2 * N - 1; i++) { parent[i] = -1; size[i] = i < N ? 1 : 0; }
  int32_t next = (int32_t)N;
  for (int64_t i = 0; i < N - 1; i++) {
    int32_t aa = uf_fastfind(parent, mst[i].from_node);
    int32_t bb = uf_fastfind(parent, mst[i].to_node);
    out[i] = (orc_linkage_node){aa, bb, mst[i].weight, size[aa] + size[bb]};
    size[next] = size[aa] + size[bb];
    parent[aa] = next;
    parent[bb] = next;
    next++;
  }
  free(parent);
  free(size);
}

/* BFS_from_hierarchy, tree.cu:206-252 (num_nodes = N-1, num_points = N). */
static int64_t bfs_hier(const orc_linkage_node *h, int32_t root, int64_t N, int32_t *out) {
  int64_t head = 0, tail = 0;
  out[tail++] = root;
  while (head < tail) {
    int32_t x = out[head++];
    if (x >= N) {
      out[tail++] = h[x - N].left_node;
      out[tail++] = h[x - N].right_node;
    }
  }
  return tail;
}

/* build_Condensed_tree, tree.cu:255-442. */
int64_t orc_condensed_tree(const orc_linkage_node *h, int64_t N, int32_t mpts,
                           orc_condensed_node **out_p) {
  int32_t root = (int32_t)(2 * (N - 1));
  int32_t num_points = (int32_t)N;
  int32_t nextlabel = num_points + 1;
  int64_t total = 2 * N - 1;
  int32_t *node_list = (int32_t *)malloc(sizeof(int32_t) * total);
  int32_t *sub = (int32_t *)malloc(sizeof(int32_t) * total);
  bfs_hier(h, root, N, node_list);
  int32_t *relabel = (int32_t *)malloc(sizeof(int32_t) * (root + 1));
  uint8_t *ignore = (uint8_t *)calloc(total, 1);
  orc_condensed_node *res = (orc_condensed_node *)malloc(sizeof(orc_condensed_node) * (2 * N + 2));
  relabel[root] = num_points;
  int64_t app = 0;
  for (int64_t i = 0; i < total; i++) {
    int32_t node = node_list[i];
    if (ignore[node] || node < num_points) continue;
    const orc_linkage_node *hn = &h[node - num_points];
    int32_t left = hn->left_node, right = hn->right_node;
    float lambda_value = (float)INT_MAX; /* INFINITE, tree.cuh:10 */
    if (hn->weight > 0.0) lambda_value = (float)(1.0 / (double)hn->weight);
    int32_t lc = left >= num_points ? h[left - num_points].node_size : 1;
    int32_t rc = right >= num_points ? h[right - num_points].node_size : 1;
    int32_t sides[2] = {left, right};
    if (lc >= mpts && rc >= mpts) {
      relabel[left] = nextlabel++;
      res[app++] = (orc_condensed_node){relabel[node], relabel[left], lambda_value, lc};
      relabel[right] = nextlabel++;
      res[app++] = (orc_condensed_node){relabel[node], relabel[right], lambda_value, rc};
      continue;
    }
    int first = 0, last = 1;
    if (lc < mpts && rc < mpts) { first = 0; last = 1; }
    else if (lc < mpts) { relabel[right] = relabel[node]; first = last = 0; }
    else { relabel[left] = relabel[node]; first = last = 1; }
    for (int s = first; s <= last; s++) {
      int64_t m = bfs_hier(h, sides[s], N, sub);
      for (int64_t t = 0; t < m; t++) {
        if (sub[t] < num_points)
          res[app++] = (orc_condensed_node){relabel[node], sub[t], lambda_value, 1};
        ignore[sub[t]] = 1;
      }
    }
  }
  free(node_list); free(sub); free(relabel); free(ignore);
  *out_p = res;
  return app;
}

typedef struct { int32_t child; float lambda; } orc_cl;
static int cmp_cl(const void *x, const void *y) {
  const orc_cl *a = (const orc_cl *)x, *b = (const orc_cl *)y;
  if (a->child != b->child) return (a->child > b->child) - (a->child < b->child);
  return (a->lambda > b->lambda) - (a->lambda < b->lambda);
}

/* compute_stability, tree.cu:444-528: birth = min lambda of each child row;
 * stability[parent] += (lambda - birth[parent]) * child_size in FP32, in row
 * order.  When out64 is given the same sums are also accumulated in double
 * (the FP64 stability mode). */
int64_t orc_stability(const orc_condensed_node *t, int64_t size, orc_stab **out,
                      double **out64) {
  int32_t max_child = t[0].child, max_parent = t[0].parent, min_parent = t[0].parent;
  for (int64_t i = 0; i < size; i++) {
    if (t[i].child > max_child) max_child = t[i].child;
    if (t[i].parent > max_parent) max_parent = t[i].parent;
    if (t[i].parent < min_parent) min_parent = t[i].parent;
  }
  int32_t largest_child = max_child > min_parent ? max_child : min_parent;
  int32_t num_clusters = max_parent - min_parent + 1;
  orc_cl *sorted = (orc_cl *)malloc(sizeof(orc_cl) * size);
  for (int64_t i = 0; i < size; i++) sorted[i] = (orc_cl){t[i].child, t[i].lambda_val};
  qsort(sorted, size, sizeof(orc_cl), cmp_cl);
  float *birth = (float *)calloc((size_t)largest_child + 1, sizeof(float));
  int32_t cur = -1;
  float minl = 0.0f;
  for (int64_t i = 0; i < size; i++) {
    if (sorted[i].child == cur) minl = minl < sorted[i].lambda ? minl : sorted[i].lambda;
    else if (cur != -1) { birth[cur] = minl; cur = sorted[i].child; minl = sorted[i].lambda; }
    else { cur = sorted[i].child; minl = sorted[i].lambda; }
  }
  if (cur != -1) birth[cur] = minl;
  birth[min_parent] = 0.0f;
  float *res = (float *)calloc(num_clusters, sizeof(float));
  double *res64 = (double *)calloc(num_clusters, sizeof(double));
  for (int64_t i = 0; i < size; i++) {
    int32_t p = t[i].parent;
    res[p - min_parent] += ((t[i].lambda_val - birth[p]) * (float)t[i].child_size);
    res64[p - min_parent] += ((double)t[i].lambda_val - (double)birth[p]) * (double)t[i].child_size;
  }
  int64_t sz = max_parent + 1 - min_parent;
  orc_stab *r = (orc_stab *)malloc(sizeof(orc_stab) * sz);
  for (int64_t i = 0; i < sz; i++) r[i] = (orc_stab){min_parent + (int32_t)i, res[i]};
  free(sorted); free(birth); free(res);
  if (out64) *out64 = res64; else free(res64);
  *out = r;
  return sz;
}

/* TreeUnionFind, tree.cu:103-169 */
static int32_t tuf_find(int32_t *d0, int32_t x) {
  int32_t r = x;
  while (d0[r] != r) r = d0[r];
  while (d0[x] != r) { int32_t nx = d0[x]; d0[x] = r; x = nx; }
  return r;
}
static void tuf_union(int32_t *d0, int32_t *d1, int32_t x, int32_t y) {
  int32_t xr = tuf_find(d0, x), yr = tuf_find(d0, y);
  if (d1[xr] < d1[yr]) d0[xr] = yr;
  else if (d1[xr] > d1[yr]) d0[yr] = xr;
  else { d0[yr] = xr; d1[xr] += 1; }
}

/* get_clusters + do_labelling + BFS_from_cluster_tree, tree.cu:535-746,
 * initializeHash initialize.cu:89-109: excess-of-mass selection, processing
 * clusters in descending id, then labels with the rule of tree.cu:599-621. */
int orc_get_clusters(const orc_condensed_node *t, int64_t size, orc_stab *stab,
                     double *s64, int64_t stab_size, int64_t num_points, int32_t *labels,
                     int32_t *num_clusters_out) {
  int32_t max_parent = t[0].parent, min_parent = t[0].parent;
  for (int64_t i = 0; i < size; i++) {
    if (t[i].parent > max_parent) max_parent = t[i].parent;
    if (t[i].parent < min_parent) min_parent = t[i].parent;
  }
  int64_t nc = max_parent + 1;
  uint8_t *is_cluster = (uint8_t *)malloc(nc);
  for (int64_t i = 0; i < nc; i++) is_cluster[i] = (i > min_parent);
  /* cluster rows (child_size > 1) per parent, in row order */
  int64_t *first = (int64_t *)malloc(sizeof(int64_t) * (nc + 1));
  for (int64_t i = 0; i <= nc; i++) first[i] = 0;
  for (int64_t i = 0; i < size; i++) if (t[i].child_size > 1) first[t[i].parent + 1]++;
  for (int64_t i = 0; i < nc; i++) first[i + 1] += first[i];
  int32_t *kids = (int32_t *)malloc(sizeof(int32_t) * (first[nc] > 0 ? first[nc] : 1));
  {
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * nc);
    memcpy(fill, first, sizeof(int64_t) * nc);
    for (int64_t i = 0; i < size; i++)
      if (t[i].child_size > 1) kids[fill[t[i].parent]++] = t[i].child;
    free(fill);
  }
  int32_t *stack = (int32_t *)malloc(sizeof(int32_t) * (nc + 1));
  for (int64_t i = stab_size - 1; i > 0; i--) {
    int32_t node = stab[i].cluster_id;
    int64_t pos = node - stab[0].cluster_id; /* buscaBinaria on contiguous ids */
    int over;
    if (s64) {
      double sub = 0.0;
      for (int64_t q = first[node]; q < first[node + 1]; q++) sub += s64[kids[q] - stab[0].cluster_id];
      over = sub > s64[pos];
      if (over) { s64[pos] = sub; stab[pos].lambda = (float)sub; }
    } else {
      float sub = 0.0f;
      for (int64_t q = first[node]; q < first[node + 1]; q++) sub += stab[kids[q] - stab[0].cluster_id].lambda;
      over = sub > stab[pos].lambda;
      if (over) stab[pos].lambda = sub;
    }
    if (over) {
      is_cluster[node] = 0;
    } else {
      int64_t sp = 0;
      for (int64_t q = first[node]; q < first[node + 1]; q++) stack[sp++] = kids[q];
      while (sp > 0) {
        int32_t c = stack[--sp];
        is_cluster[c] = 0;
        for (int64_t q = first[c]; q < first[c + 1]; q++) stack[sp++] = kids[q];
      }
    }
  }
  free(stack);
  /* cluster_map: selected ids ascending -> 0.. */
  int32_t *map = (int32_t *)malloc(sizeof(int32_t) * nc);
  int32_t ncl = 0;
  for (int64_t i = 0; i < nc; i++) map[i] = is_cluster[i] ? ncl++ : -1;
  /* initializeHash: lambda of each child's row; root gets a root row lambda */
  int32_t max_child = 0;
  for (int64_t i = 0; i < size; i++) if (t[i].child > max_child) max_child = t[i].child;
  int64_t hl = (max_child > max_parent ? max_child : max_parent) + 1;
  float *lam = (float *)calloc(hl, sizeof(float));
  for (int64_t i = 0; i < size; i++) {
    lam[t[i].child] = t[i].lambda_val;
    if (t[i].parent == min_parent) lam[min_parent] = t[i].lambda_val;
  }
  /* do_labelling: union every row whose child is not a selected cluster */
  int32_t *d0 = (int32_t *)malloc(sizeof(int32_t) * nc);
  int32_t *d1 = (int32_t *)calloc(nc, sizeof(int32_t));
  for (int64_t i = 0; i < nc; i++) d0[i] = (int32_t)i;
  for (int64_t i = 0; i < size; i++) {
    int32_t child = t[i].child;
    if (!(child < nc && is_cluster[child])) tuf_union(d0, d1, t[i].parent, child);
  }
  for (int64_t p = 0; p < num_points; p++) {
    int32_t c = tuf_find(d0, (int32_t)p);
    if (c <= min_parent) labels[p] = -1;
    else labels[p] = (lam[p] > lam[c]) ? map[c] : -1;
  }
  if (num_clusters_out) *num_clusters_out = ncl;
  free(is_cluster); free(first); free(kids); free(map); free(lam); free(d0); free(d1);
  return ORC_OK;
}

/* The _new.cu call order (HDBSCAN/_new.cu:251-347) from a given kNN graph. */
int orc_hdbscan_from_knn(const int32_t *ids, const float *dist, const float *X, int64_t n,
                         int32_t d, int32_t k, int32_t mpts, int32_t fp64,
                         orc_mst_edge *mst_out, int32_t *labels, int32_t *ncl) {
  return orc_hdbscan_from_knn_order(ids, dist, X, n, d, k, mpts, fp64, ORC_ORDER_EDGE, mst_out,
                                    labels, ncl);
}

int orc_hdbscan_from_knn_order(const int32_t *ids, const float *dist, const float *X, int64_t n,
                               int32_t d, int32_t k, int32_t mpts, int32_t fp64, int32_t order,
                               orc_mst_edge *mst_out, int32_t *labels, int32_t *ncl) {
  int64_t *nindex; int32_t *nlist; float *ew;
  int64_t E = orc_enhanced_knng(ids, dist, X, n, d, k, &nindex, &nlist, &ew, NULL, NULL);
  if (E < 0) return ORC_ERR_ARG;
  orc_mst_edge *m = mst_out ? mst_out : (orc_mst_edge *)malloc(sizeof(orc_mst_edge) * (n - 1));
  int rc;
  if (order == ORC_ORDER_IDS) {
    rc = orc_mst_ordered(nindex, nlist, ew, (int32_t)n, E, order, NULL, m);
    free(nindex); free(nlist); free(ew);
    if (rc != ORC_OK) { if (!mst_out) free(m); return rc; }
  } else {
    uint8_t *in = (uint8_t *)malloc(E > 0 ? E : 1);
    rc = orc_kruskal(nindex, nlist, ew, (int32_t)n, E, in);
    if (rc == ORC_OK) rc = orc_build_mst(nindex, nlist, ew, (int32_t)n, E, in, m);
    free(in); free(nindex); free(nlist); free(ew);
    if (rc != ORC_OK) { if (!mst_out) free(m); return rc; }
    orc_sort_edges(m, n - 1);
  }
  orc_linkage_node *h = (orc_linkage_node *)malloc(sizeof(orc_linkage_node) * (n - 1));
  orc_linkage_tree(m, n, h);
  if (!mst_out) free(m);
  orc_condensed_node *ct;
  int64_t cs = orc_condensed_tree(h, n, mpts, &ct);
  free(h);
  orc_stab *st;
  double *s64 = NULL;
  int64_t ss = orc_stability(ct, cs, &st, fp64 ? &s64 : NULL);
  rc = orc_get_clusters(ct, cs, st, s64, ss, n, labels, ncl);
  free(ct); free(st); free(s64);
  return rc;
}
