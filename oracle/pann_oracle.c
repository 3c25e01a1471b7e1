/*
 * pann_oracle.c -- CPU restatement of ParlayANN's hot path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY. This is the oracle: the parity tests, smoke() and
 * bench.py's cpu_baseline leg compare the CUDA path against it. The product
 * never links or calls it. Each function cites the reference file:line it
 * restates (paths relative to the ParlayANN checkout). The restatement is
 * pinned by tests/test_oracle_pin.py against the reference's own code compiled
 * in place (oracle/_ref/libpann_ref.so) and against tests/golden/ fixtures
 * generated from that library by tests/golden/make_golden.py.
 *
 * dtype: 0 = uint8, 1 = int8, 2 = float32.   metric: 0 = Euclidian, 1 = mips.
 * Vectors are dense row-major n x d (no padding). Graph rows are the
 * reference layout: n x (R+1) uint32, slot 0 = degree (graph.h:138-145,239-247).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EMPTY32 0xFFFFFFFFu

/* ------------------------------------------------------------ distances */
/* euclidian_point.h:54-62 (uint8), :74-81 (int8), :83-90 (float);
 * mips_point.h:44-50 (uint8), :52-58 (int8), :60-66 (float). The float sums
 * are sequential in dimension order with no fused multiply-add: this file is
 * compiled with -std=c11 -ffp-contract=off, as the reference is under
 * -std=c++17 (algorithms/bench/parallelDefsANN:8). */
static float dist_u8_l2(const uint8_t* p, const uint8_t* q, unsigned d) {
  int32_t r = 0;
  for (unsigned i = 0; i < d; i++) { int32_t a = p[i], b = q[i]; r += (a - b) * (a - b); }
  return (float)r;
}
static float dist_i8_l2(const int8_t* p, const int8_t* q, unsigned d) {
  int32_t r = 0;
  for (unsigned i = 0; i < d; i++) { int32_t x = (int32_t)((int16_t)q[i] - (int16_t)p[i]); r += x * x; }
  return (float)r;
}
static float dist_f32_l2(const float* p, const float* q, unsigned d) {
  float r = 0.0f;
  for (unsigned i = 0; i < d; i++) r += (q[i] - p[i]) * (q[i] - p[i]);
  return r;
}
static float dist_u8_ip(const uint8_t* p, const uint8_t* q, unsigned d) {
  int32_t r = 0;
  for (unsigned i = 0; i < d; i++) r += (int32_t)q[i] * (int32_t)p[i];
  return -((float)r);
}
static float dist_i8_ip(const int8_t* p, const int8_t* q, unsigned d) {
  int32_t r = 0;
  for (unsigned i = 0; i < d; i++) r += (int32_t)q[i] * (int32_t)p[i];
  return -((float)r);
}
static float dist_f32_ip(const float* p, const float* q, unsigned d) {
  float r = 0.0f;
  for (unsigned i = 0; i < d; i++) r += q[i] * p[i];
  return -r;
}

typedef struct {
  int dtype, metric;
  unsigned d;
  size_t row_bytes;
  const uint8_t* base;
} pts_t;

static inline const void* row(const pts_t* P, uint32_t i) { return P->base + (size_t)i * P->row_bytes; }

/* a.distance(b) with a's values as the first argument (euclidian_point.h:115-117) */
static float dist(const pts_t* P, const void* a, const void* b) {
  unsigned d = P->d;
  if (P->metric == 0) {
    if (P->dtype == 0) return dist_u8_l2(a, b, d);
    if (P->dtype == 1) return dist_i8_l2(a, b, d);
    return dist_f32_l2(a, b, d);
  } else {
    if (P->dtype == 0) return dist_u8_ip(a, b, d);
    if (P->dtype == 1) return dist_i8_ip(a, b, d);
    return dist_f32_ip(a, b, d);
  }
}

static size_t elem_size(int dtype) { return dtype == 2 ? 4 : 1; }

float oracle_distance(int dtype, int metric, unsigned d, const void* a, const void* b) {
  pts_t P = {dtype, metric, d, d * elem_size(dtype), NULL};
  return dist(&P, a, b);
}

/* ------------------------------------------------------------ hashset */
/* hashset.h:13-55, including its growth behaviour (the probe after growth
 * starts from the slot computed with the old mask, and num_entries keeps the
 * re-inserted keys' count). grew counts growth events. */
typedef struct {
  int bits;
  uint32_t* e;
  size_t size;
  size_t mask;
  long num_entries;
  int grew;
} hset_t;

static inline size_t hs_hash(uint32_t k) { return (size_t)((uint64_t)k * UINT64_C(0xbf58476d1ce4e5b9)); }

static void hs_init(hset_t* h, long n) {
  h->bits = (int)ceil(log2((double)n));
  h->size = (size_t)1 << h->bits;
  h->e = (uint32_t*)malloc(h->size * sizeof(uint32_t));
  memset(h->e, 0xFF, h->size * sizeof(uint32_t));
  h->mask = h->size - 1;
  h->num_entries = 0;
  h->grew = 0;
}
static void hs_free(hset_t* h) { free(h->e); }

/* returns 1 if a was present, else inserts a and returns 0 (hashset.h:22-48) */
static int hs_test_insert(hset_t* h, uint32_t a) {
  int loc = (int)(hs_hash(a) & h->mask);
  if (h->e[loc] == a) return 1;
  if (h->num_entries > (long)(h->size / 2)) {
    size_t old_size = h->size;
    uint32_t* old = h->e;
    h->bits += 1;
    h->size = (size_t)1 << h->bits;
    h->e = (uint32_t*)malloc(h->size * sizeof(uint32_t));
    memset(h->e, 0xFF, h->size * sizeof(uint32_t));
    h->mask = h->size - 1;
    for (size_t i = 0; i < old_size; i++) {
      uint32_t k = old[i];
      if (k != EMPTY32) {
        int l2 = (int)(hs_hash(k) & h->mask);
        while (h->e[l2] != EMPTY32 && h->e[l2] != k) l2 = (int)((l2 + 1) & h->mask);
        h->e[l2] = k;
        h->num_entries++;
      }
    }
    free(old);
    h->grew++;
  }
  if (h->e[loc] != EMPTY32) {
    loc = (int)((loc + 1) & h->mask);
    while (h->e[loc] != EMPTY32 && h->e[loc] != a) loc = (int)((loc + 1) & h->mask);
    if (h->e[loc] == a) return 1;
  }
  h->e[loc] = a;
  h->num_entries++;
  return 0;
}

/* ------------------------------------------------------------ beam search */
typedef struct { uint32_t id; float d; } pair_t;

/* (dist, id) lexicographic order (beamSearch.h:62-64) */
static inline int pless(pair_t a, pair_t b) { return a.d < b.d || (a.d == b.d && a.id < b.id); }

static int cmp_pair(const void* x, const void* y) {
  pair_t a = *(const pair_t*)x, b = *(const pair_t*)y;
  if (pless(a, b)) return -1;
  if (pless(b, a)) return 1;
  return 0;
}

typedef struct {
  uint32_t k, L, degree_limit;
  uint64_t limit;
  double batch_factor;
  /* early stopping (earlyStopping.h:19-29); es_count == 0 disables it */
  double es_count;  /* QP.early_stopping_count */
  double es_radius; /* QP.radius as the early-stopping rule sees it */
  double es_esr;    /* QP.early_stopping_radius */
} qparams_t;

typedef struct {
  pair_t* frontier; uint32_t frontier_n; /* sorted, <= L */
  pair_t* visited;  uint32_t visited_n;  /* sorted */
  uint64_t cmps;                         /* full_dist_cmps */
  int hash_grew;                         /* seen-set growth events */
} bs_out_t;

/* filtered_beam_search with use_filtering = false (beamSearch.h:33-228), with
 * the early_stopping functor of range search when QP->es_count > 0
 * (earlyStopping.h:19-29, called at beamSearch.h:120-121). self != EMPTY32 marks the build-time query point:
 * Points[a].same_as(p) is pointer equality, i.e. a == self (euclidian_point.h:184-186).
 * Returns 0, or -1 on invalid start points (beamSearch.h:51-57). */
static int beam_search_one(const pts_t* P, const uint32_t* G, uint32_t R, const void* q,
                           uint32_t self, const uint32_t* starts, uint32_t n_start,
                           const qparams_t* QP, bs_out_t* out) {
  long beamSize = QP->L;
  if (n_start == 0 || (long)n_start > beamSize) return -1;
  hset_t seen;
  hs_init(&seen, 2 * (10 + beamSize) * (long)QP->degree_limit); /* :66 */

  pair_t* frontier = (pair_t*)malloc(sizeof(pair_t) * (beamSize + 1));
  size_t fn = 0;
  for (uint32_t i = 0; i < n_start; i++) { /* :73-76 */
    pair_t e = {starts[i], dist(P, row(P, starts[i]), q)};
    frontier[fn++] = e;
    hs_test_insert(&seen, starts[i]);
  }
  qsort(frontier, fn, sizeof(pair_t), cmp_pair); /* :77 */

  pair_t* unvisited = (pair_t*)malloc(sizeof(pair_t) * (beamSize + 1));
  for (size_t i = 0; i < fn; i++) unvisited[i] = frontier[i]; /* :81-83 */

  size_t vcap = 2 * beamSize + 16, vn = 0;
  pair_t* visited = (pair_t*)malloc(sizeof(pair_t) * vcap);

  uint64_t full_dist_cmps = n_start; /* :91 */
  long remain = (long)fn;
  long num_visited = 0;
  size_t new_cap = 2 * (size_t)(beamSize > (long)n_start ? beamSize : (long)n_start) + R;
  pair_t* new_frontier = (pair_t*)malloc(sizeof(pair_t) * (new_cap + 1));
  size_t ccap = R + beamSize + 16, cn = 0;
  pair_t* cand = (pair_t*)malloc(sizeof(pair_t) * ccap);
  uint32_t* pruned = (uint32_t*)malloc(sizeof(uint32_t) * (R + 1));
  long offset = 0;

  while (remain > offset && (uint64_t)num_visited < QP->limit) { /* :116 */
    pair_t current = unvisited[offset];
    /* early_stopping(frontier, unvisited_frontier, visited, QP): it reads
     * unvisited_frontier[0], which is only refreshed at a merge */
    if (QP->es_count > 0 && (double)vn >= QP->es_count && !((double)frontier[0].d <= QP->es_radius) &&
        !((double)unvisited[0].d <= QP->es_esr))
      break;
    /* insert into the sorted visited list (:125-127) */
    if (vn == vcap) { vcap *= 2; visited = (pair_t*)realloc(visited, sizeof(pair_t) * vcap); }
    size_t pos = vn;
    { /* upper_bound */
      size_t lo = 0, hi = vn;
      while (lo < hi) { size_t mid = (lo + hi) / 2; if (pless(current, visited[mid])) hi = mid; else lo = mid + 1; }
      pos = lo;
    }
    memmove(visited + pos + 1, visited + pos, sizeof(pair_t) * (vn - pos));
    visited[pos] = current;
    vn++;
    num_visited++;
    int frontier_full = (long)fn == beamSize; /* :128 */

    /* neighbours not yet seen (:151-160) */
    const uint32_t* gr = G + (size_t)current.id * (R + 1);
    long deg = gr[0];
    long num_elts = deg < (long)QP->degree_limit ? deg : (long)QP->degree_limit;
    size_t pn = 0;
    for (long i = 0; i < num_elts; i++) {
      uint32_t a = gr[1 + i];
      if (hs_test_insert(&seen, a) || a == self) continue;
      pruned[pn++] = a;
    }
    /* distances, cutoff (:173-182) */
    float cutoff = frontier_full ? frontier[fn - 1].d : 3.40282346638528859812e+38F;
    for (size_t i = 0; i < pn; i++) {
      float dd = dist(P, row(P, pruned[i]), q);
      full_dist_cmps++;
      if (dd >= cutoff) continue;
      if (cn == ccap) { ccap *= 2; cand = (pair_t*)realloc(cand, sizeof(pair_t) * ccap); }
      pair_t e = {pruned[i], dd};
      cand[cn++] = e;
    }
    /* deferral (:185-192) */
    if (cn == 0 || (QP->limit >= 2 * (uint64_t)beamSize && (double)cn < QP->batch_factor * (double)beamSize &&
                    offset + 1 < remain)) {
      offset++;
      continue;
    }
    offset = 0;
    /* sort + unique by id (:197-199) */
    qsort(cand, cn, sizeof(pair_t), cmp_pair);
    size_t un = 0;
    for (size_t i = 0; i < cn; i++) if (un == 0 || cand[un - 1].id != cand[i].id) cand[un++] = cand[i];
    /* set_union(frontier, cand) (:202-205) */
    size_t need = fn + un;
    if (need > new_cap) { new_cap = need; new_frontier = (pair_t*)realloc(new_frontier, sizeof(pair_t) * (new_cap + 1)); }
    size_t i = 0, j = 0, m = 0;
    while (i < fn && j < un) {
      if (pless(frontier[i], cand[j])) new_frontier[m++] = frontier[i++];
      else if (pless(cand[j], frontier[i])) new_frontier[m++] = cand[j++];
      else { new_frontier[m++] = frontier[i++]; j++; }
    }
    while (i < fn) new_frontier[m++] = frontier[i++];
    while (j < un) new_frontier[m++] = cand[j++];
    cn = 0;
    /* trim to beamSize (:209-214) */
    if ((long)m > beamSize) m = (size_t)beamSize;
    for (size_t t = 0; t < m; t++) frontier[t] = new_frontier[t];
    fn = m;
    /* set_difference(frontier, visited) (:217-222) */
    size_t a = 0, b = 0, r = 0;
    while (a < fn && b < vn) {
      if (pless(frontier[a], visited[b])) unvisited[r++] = frontier[a++];
      else if (pless(visited[b], frontier[a])) b++;
      else { a++; b++; }
    }
    while (a < fn) unvisited[r++] = frontier[a++];
    remain = (long)r;
  }
  out->frontier = frontier;
  out->frontier_n = (uint32_t)fn;
  out->visited = visited;
  out->visited_n = (uint32_t)vn;
  out->cmps = full_dist_cmps;
  out->hash_grew = seen.grew;
  hs_free(&seen);
  free(unvisited);
  free(new_frontier);
  free(cand);
  free(pruned);
  return 0;
}

/* Batch search: beam_search per query from the given start points, then the
 * first k of the frontier (beam_search_rerank without quantization,
 * beamSearch.h:588-596; the recomputed distance equals the stored one).
 * Optional outputs may be NULL. Returns 0, -1 (bad params), or -2 when a query
 * returned fewer than k results (beamSearch.h:557-562). */
int oracle_search(int dtype, int metric, uint32_t n, uint32_t d, const void* base,
                  uint32_t nq, const void* queries, uint32_t R, const uint32_t* graph,
                  uint32_t k, uint32_t L, uint64_t limit, uint32_t degree_limit,
                  double batch_factor, uint32_t n_start, const uint32_t* starts,
                  uint32_t* out_ids, float* out_dists, uint32_t* out_visited, uint32_t* out_cmps,
                  int32_t* out_hash_grew, uint32_t* out_frontier_n, uint32_t* out_frontier_ids,
                  float* out_frontier_d, uint32_t visited_cap, uint32_t* out_visited_ids,
                  float* out_visited_d) {
  (void)n;
  if (k > L || degree_limit == 0) return -1; /* beamSearch.h:612-616 */
  pts_t P = {dtype, metric, d, d * elem_size(dtype), (const uint8_t*)base};
  pts_t Q = {dtype, metric, d, d * elem_size(dtype), (const uint8_t*)queries};
  qparams_t QP = {k, L, degree_limit, limit, batch_factor};
  int rc = 0;
  for (uint32_t i = 0; i < nq; i++) {
    bs_out_t o;
    if (beam_search_one(&P, graph, R, row(&Q, i), EMPTY32, starts, n_start, &QP, &o) != 0) return -1;
    if (o.frontier_n < k) rc = -2;
    for (uint32_t j = 0; j < k; j++) {
      out_ids[(size_t)i * k + j] = j < o.frontier_n ? o.frontier[j].id : EMPTY32;
      out_dists[(size_t)i * k + j] = j < o.frontier_n ? o.frontier[j].d : 0.0f;
    }
    if (out_visited) out_visited[i] = o.visited_n;
    if (out_cmps) out_cmps[i] = (uint32_t)o.cmps;
    if (out_hash_grew) out_hash_grew[i] = o.hash_grew;
    if (out_frontier_n) {
      out_frontier_n[i] = o.frontier_n;
      for (uint32_t j = 0; j < o.frontier_n; j++) {
        out_frontier_ids[(size_t)i * L + j] = o.frontier[j].id;
        out_frontier_d[(size_t)i * L + j] = o.frontier[j].d;
      }
    }
    if (out_visited_ids) {
      for (uint32_t j = 0; j < o.visited_n && j < visited_cap; j++) {
        out_visited_ids[(size_t)i * visited_cap + j] = o.visited[j].id;
        out_visited_d[(size_t)i * visited_cap + j] = o.visited[j].d;
      }
    }
    free(o.frontier);
    free(o.visited);
  }
  return rc;
}

/* ------------------------------------------------------------ range search */
/* greedy_search (rangeSearch.h:21-55): a breadth-first expansion over points
 * within `radius`, seeded with the beam's in-range frontier, with the
 * reference's growing hashset of initial capacity 2 * |seeds| * 64. Appends
 * to *res (grown with realloc); returns the distance comparisons. */
static uint64_t greedy_one(const pts_t* P, const uint32_t* G, uint32_t R, const void* q, const pair_t* seeds,
                           uint32_t m, double radius, uint32_t** res, size_t* rn, size_t* rcap, int* grew) {
  hset_t seen;
  hs_init(&seen, 2 * (long)m * 64);
#define PUSH(v) do { if (*rn == *rcap) { *rcap = *rcap * 2 + 16; *res = (uint32_t*)realloc(*res, 4 * *rcap); } \
                     (*res)[(*rn)++] = (v); } while (0)
  for (uint32_t i = 0; i < m; i++) { /* :30-33 */
    if (hs_test_insert(&seen, seeds[i].id) || (double)seeds[i].d > radius) continue;
    PUSH(seeds[i].id);
  }
  uint64_t cmps = 0;
  uint32_t* unseen = (uint32_t*)malloc(4 * (R + 1));
  size_t position = 0;
  while (position < *rn) { /* :38-52 */
    uint32_t next = (*res)[position++];
    const uint32_t* gr = G + (size_t)next * (R + 1);
    uint32_t deg = gr[0], un = 0;
    for (uint32_t i = 0; i < deg; i++) {
      uint32_t v = gr[1 + i];
      if (hs_test_insert(&seen, v)) continue;
      unseen[un++] = v;
    }
    for (uint32_t i = 0; i < un; i++) {
      cmps++;
      if ((double)dist(P, row(P, unseen[i]), q) <= radius) PUSH(unseen[i]);
    }
  }
#undef PUSH
  free(unseen);
  *grew += seen.grew;
  hs_free(&seen);
  return cmps;
}

/* Range search per query from one start point:
 *   type 1 (Greedy) / 3 (Beam): RangeSearch (rangeSearch.h:183-276) without
 *     quantization: a beam search of width `beam` (k = beam, limit = n,
 *     degree_limit = R, batch_factor .125) with early stopping, where the
 *     early-stopping radii pass through Point::translate_distance (a float
 *     rounding for unquantized points, euclidian_point.h:119-123,
 *     mips_point.h:90-92); the frontier entries with distance <= radius are
 *     the answer unless all `beam` of them are in range and the type is Greedy,
 *     in which case greedy_search from them (radius rounded the same way)
 *     gives the answer, in its discovery order.
 *   type 2 (Doubling): DoubleBeamRangeSearch (doublingSearch.h:50-148). Its
 *     first round is the same beam search with the radius not rounded. When
 *     every frontier entry is in range it runs beam_search again from them
 *     with QueryParams(2 beam, 2 beam, 0.0, G.size(), G.max_degree()), whose
 *     third argument is the visit limit: with limit 0 that search visits
 *     nothing and returns the start points sorted, so the answer stays the
 *     in-range frontier, visited gains 0 and comparisons gain `beam`.
 * visited / cmps accumulate as QueryStats does (rangeSearch.h:258-267,
 * doublingSearch.h:88-89,138-139). Per query, out_count gets the answer's
 * size and out_ids (rows of `cap`) its first cap ids. */
int oracle_range_search(int dtype, int metric, uint32_t n, uint32_t d, const void* base, uint32_t nq,
                        const void* queries, uint32_t R, const uint32_t* graph, uint32_t beam, uint32_t start,
                        int type, double radius, double esr, uint32_t esc, uint64_t* out_count, uint32_t* out_ids,
                        uint64_t cap, uint32_t* out_visited, uint64_t* out_cmps, int32_t* out_grew) {
  if (beam == 0 || type < 1 || type > 3) return -1;
  pts_t P = {dtype, metric, d, d * elem_size(dtype), (const uint8_t*)base};
  pts_t Q = {dtype, metric, d, d * elem_size(dtype), (const uint8_t*)queries};
  const double r_f = (double)(float)radius, esr_f = (double)(float)esr;
  qparams_t QP = {beam, beam, R, (uint64_t)n, 0.125, (double)esc, type == 2 ? radius : r_f, esr_f};
  size_t rcap = 0;
  uint32_t* res = NULL;
  for (uint32_t i = 0; i < nq; i++) {
    const void* q = row(&Q, i);
    bs_out_t o;
    if (beam_search_one(&P, graph, R, q, EMPTY32, &start, 1, &QP, &o) != 0) { free(res); return -1; }
    uint64_t visited = o.visited_n, cmps = o.cmps;
    int grew = o.hash_grew;
    uint32_t c = 0;
    while (c < o.frontier_n && (double)o.frontier[c].d <= radius) c++; /* the sorted frontier's in-range prefix */
    size_t rn = 0;
    if (c < beam || type == 3) {
      for (uint32_t j = 0; j < c; j++) { if (rn == rcap) { rcap = rcap * 2 + 16; res = (uint32_t*)realloc(res, 4 * rcap); } res[rn++] = o.frontier[j].id; }
    } else if (type == 2) {
      for (uint32_t j = 0; j < c; j++) { if (rn == rcap) { rcap = rcap * 2 + 16; res = (uint32_t*)realloc(res, 4 * rcap); } res[rn++] = o.frontier[j].id; }
      cmps += c; /* the limit-0 second round: start points only */
    } else {
      cmps += greedy_one(&P, graph, R, q, o.frontier, c, r_f, &res, &rn, &rcap, &grew);
      visited += rn;
    }
    out_count[i] = rn;
    for (size_t j = 0; j < rn && j < cap; j++) out_ids[(size_t)i * cap + j] = res[j];
    if (out_visited) out_visited[i] = (uint32_t)visited;
    if (out_cmps) out_cmps[i] = cmps;
    if (out_grew) out_grew[i] = grew;
    free(o.frontier);
    free(o.visited);
  }
  free(res);
  return 0;
}

/* ------------------------------------------------------------ quantized search + re-rank */
/* Euclidian_Point<uint8_t>::generate_parameters (euclidian_point.h:214-240):
 * min and max over every value with 0.0 as the starting point of both; when
 * every value is a non-negative integer, [0, 255]. parameters(min, max, d)
 * (:104-107): slope = 255 / (max - min) in float, offset = round(min * slope). */
void oracle_quant_params(uint32_t n, uint32_t d, const float* base, float* slope, int32_t* offset) {
  float mn = 0.0f, mx = 0.0f;
  int all_ints = 1;
  for (size_t i = 0; i < (size_t)n * d; i++) {
    const float x = base[i];
    all_ints = all_ints && (x >= 0) && (x - (float)(long)x) == 0;
    if (x < mn) mn = x;
    if (x > mx) mx = x;
  }
  if (all_ints) {
    if (mx < 256) mx = 255;
    mn = 0;
  }
  const float s = 255.0f / (mx - mn);
  *slope = s;
  *offset = (int32_t)roundf(mn * s);
}

/* translate_point (euclidian_point.h:188-212): round(x * slope) - offset,
 * clamped to [0, 255]. */
static void quant_row(const float* x, uint32_t d, float slope, int32_t offset, uint8_t* out) {
  for (uint32_t j = 0; j < d; j++) {
    if (slope == 1.0f && offset == 0) { out[j] = (uint8_t)x[j]; continue; }
    int64_t r = (int64_t)roundf(x[j] * slope) - offset;
    if (r < 0) r = 0;
    if (r > 255) r = 255;
    out[j] = (uint8_t)r;
  }
}

/* Quantized_Mips_Point<8, true>::generate_parameters (mips_point.h:438-499):
 * per point the minimum and maximum of its values (0.0 the starting point of
 * both); trimmed: the minimum of rank (size_t)(1e-4 n) among the points'
 * minima and the maximum of rank (size_t)((1 - 1e-4)(n - 1)) among their
 * maxima; bound = max(max, -min); parameters(bound, d) (:303-308): scale =
 * 127 / bound in float. */
static int cmp_float(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}
void oracle_quant_params_mips(uint32_t n, uint32_t d, const float* base, float* scale, float* bound) {
  float* mins = (float*)malloc(sizeof(float) * (n ? n : 1));
  float* maxs = (float*)malloc(sizeof(float) * (n ? n : 1));
  for (uint32_t i = 0; i < n; i++) {
    float mn = 0.0f, mx = 0.0f;
    for (uint32_t j = 0; j < d; j++) {
      const float x = base[(size_t)i * d + j];
      if (x < mn) mn = x;
      if (x > mx) mx = x;
    }
    mins[i] = mn;
    maxs[i] = mx;
  }
  const double cutoff = .0001;
  const size_t min_rank = (size_t)(cutoff * n);
  const size_t max_rank = (size_t)((1.0 - cutoff) * (n - 1));
  qsort(mins, n, sizeof(float), cmp_float);
  qsort(maxs, n, sizeof(float), cmp_float);
  const float mn = mins[min_rank], mx = maxs[max_rank];
  const float b = mx > -mn ? mx : -mn;
  *bound = b;
  *scale = 127 / b;
  free(mins);
  free(maxs);
}

/* translate_point (mips_point.h:421-436): -127 below -bound, 127 above bound,
 * else round(x * scale), as int8. */
static void quant_row_mips(const float* x, uint32_t d, float scale, float bound, int8_t* out) {
  for (uint32_t j = 0; j < d; j++) {
    const float pj = x[j];
    if (pj < -bound) out[j] = -127;
    else if (pj > bound) out[j] = 127;
    else out[j] = (int8_t)(int32_t)roundf(pj * scale);
  }
}

/* beam_search_rerank (beamSearch.h:529-597) for a float index with one-byte
 * quantized points, no filtering: the beam search runs on the quantized
 * points and query (uint8 Euclidian for metric 0, int8 mips for metric 1);
 * the first min(k * rerank_factor, |frontier|) frontier entries are re-scored
 * with the float distance, sorted by (distance, id), and the first k kept.
 * Returns -2 if the frontier holds fewer than k entries (the reference
 * aborts). */
int oracle_search_quantized(int metric, uint32_t n, uint32_t d, const float* base, uint32_t nq, const float* queries,
                            uint32_t R, const uint32_t* graph, uint32_t k, uint32_t L, uint64_t limit,
                            uint32_t degree_limit, double rerank_factor, double batch_factor, uint32_t start,
                            uint32_t* out_ids, float* out_dists, uint32_t* out_visited, uint32_t* out_cmps) {
  float slope = 1.0f, scale = 1.0f, bound = 1.0f;
  int32_t offset = 0;
  if (metric == 0) oracle_quant_params(n, d, base, &slope, &offset);
  else oracle_quant_params_mips(n, d, base, &scale, &bound);
  uint8_t* qb = (uint8_t*)malloc((size_t)n * d);
  for (uint32_t i = 0; i < n; i++) {
    if (metric == 0) quant_row(base + (size_t)i * d, d, slope, offset, qb + (size_t)i * d);
    else quant_row_mips(base + (size_t)i * d, d, scale, bound, (int8_t*)(qb + (size_t)i * d));
  }
  pts_t QP8 = {metric == 0 ? 0 : 1, metric, d, d, qb};
  pts_t PF = {2, metric, d, 4 * (size_t)d, (const uint8_t*)base};
  qparams_t QP = {k, L, degree_limit, limit, batch_factor, 0.0, 0.0, 0.0};
  uint8_t* qq = (uint8_t*)malloc(d);
  int rc = 0;
  for (uint32_t i = 0; i < nq && rc == 0; i++) {
    const float* q = queries + (size_t)i * d;
    if (metric == 0) quant_row(q, d, slope, offset, qq);
    else quant_row_mips(q, d, scale, bound, (int8_t*)qq);
    bs_out_t o;
    if (beam_search_one(&QP8, graph, R, qq, EMPTY32, &start, 1, &QP, &o) != 0) { rc = -1; break; }
    if (o.frontier_n < k) rc = -2;
    int num_check = (int)(k * rerank_factor);
    if ((uint32_t)num_check > o.frontier_n) num_check = (int)o.frontier_n;
    pair_t* pts = (pair_t*)malloc(sizeof(pair_t) * (num_check > 0 ? num_check : 1));
    for (int j = 0; j < num_check; j++) {
      uint32_t id = o.frontier[j].id;
      pair_t e = {id, dist(&PF, q, row(&PF, id))};
      pts[j] = e;
    }
    qsort(pts, (size_t)num_check, sizeof(pair_t), cmp_pair);
    for (uint32_t j = 0; j < k; j++) {
      out_ids[(size_t)i * k + j] = (int)j < num_check ? pts[j].id : EMPTY32;
      out_dists[(size_t)i * k + j] = (int)j < num_check ? pts[j].d : 0.0f;
    }
    out_visited[i] = o.visited_n;
    out_cmps[i] = (uint32_t)o.cmps;
    free(pts);
    free(o.frontier);
    free(o.visited);
  }
  free(qq);
  free(qb);
  return rc;
}

/* ------------------------------------------------------------ range groundtruth */
/* compute_range_groundtruth (data_tools/compute_range_groundtruth.cpp:14-30):
 * answer i = every base id j, in increasing order, whose float distance
 * Q[i].distance(B[j]) is <= the float radius. out_offsets has nq + 1 entries;
 * ids past cap are counted, not written. Returns 1 if they did not fit. */
int oracle_range_groundtruth(int dtype, int metric, uint32_t n, uint32_t d, const void* base, uint32_t nq,
                             const void* queries, float radius, uint64_t* out_offsets, uint32_t* out_ids,
                             uint64_t cap) {
  pts_t P = {dtype, metric, d, d * elem_size(dtype), (const uint8_t*)base};
  pts_t Q = {dtype, metric, d, d * elem_size(dtype), (const uint8_t*)queries};
  uint64_t total = 0;
  for (uint32_t i = 0; i < nq; i++) {
    out_offsets[i] = total;
    const void* q = row(&Q, i);
    for (uint32_t j = 0; j < n; j++) {
      const float dd = dist(&P, q, row(&P, j));
      if (dd <= radius) {
        if (total < cap) out_ids[total] = j;
        total++;
      }
    }
  }
  out_offsets[nq] = total;
  return total > cap ? 1 : 0;
}

/* ------------------------------------------------------------ robustPrune */
/* knn_index::robustPrune (index.h:63-120): candidates = cand ++ (if add) the
 * current out-neighbours of p with their distances; sort by (dist, id);
 * unique by id; greedy selection up to R with the alpha test in double.
 * Returns the number of new neighbours written to out; *cmps gets the
 * distance-comparison count. */
static uint32_t robust_prune(const pts_t* P, const uint32_t* G, uint32_t R, uint32_t p,
                             const pair_t* cand, size_t cn, double alpha, int add,
                             uint32_t* out, long* cmps) {
  const uint32_t* gp = G + (size_t)p * (R + 1);
  size_t out_size = gp[0];
  size_t total = cn + (add ? out_size : 0);
  pair_t* c = (pair_t*)malloc(sizeof(pair_t) * (total + 1));
  long dc = 0;
  size_t m = 0;
  for (size_t i = 0; i < cn; i++) c[m++] = cand[i];
  if (add) {
    for (size_t i = 0; i < out_size; i++) {
      dc++;
      uint32_t nb = gp[1 + i];
      pair_t e = {nb, dist(P, row(P, nb), row(P, p))};
      c[m++] = e;
    }
  }
  qsort(c, m, sizeof(pair_t), cmp_pair);
  size_t un = 0;
  for (size_t i = 0; i < m; i++) if (un == 0 || c[un - 1].id != c[i].id) c[un++] = c[i];
  uint32_t nn = 0;
  size_t idx = 0;
  while (nn < R && idx < un) {
    uint32_t p_star = c[idx].id;
    idx++;
    if (p_star == p || p_star == EMPTY32) continue;
    out[nn++] = p_star;
    for (size_t i = idx; i < un; i++) {
      uint32_t p_prime = c[i].id;
      if (p_prime != EMPTY32) {
        dc++;
        float d_sp = dist(P, row(P, p_star), row(P, p_prime));
        float d_pp = c[i].d;
        if (alpha * (double)d_sp <= (double)d_pp) c[i].id = EMPTY32;
      }
    }
  }
  free(c);
  *cmps = dc;
  return nn;
}

int oracle_robust_prune(int dtype, int metric, uint32_t d, const void* base, uint32_t R,
                        const uint32_t* graph, uint32_t p, uint32_t n_cand,
                        const uint32_t* cand_ids, const float* cand_d, double alpha, int add,
                        uint32_t* out_nbrs, uint32_t* out_n, long* out_cmps) {
  pts_t P = {dtype, metric, d, d * elem_size(dtype), (const uint8_t*)base};
  pair_t* c = (pair_t*)malloc(sizeof(pair_t) * (n_cand + 1));
  for (uint32_t i = 0; i < n_cand; i++) { c[i].id = cand_ids[i]; c[i].d = cand_d[i]; }
  *out_n = robust_prune(&P, graph, R, p, c, n_cand, alpha, add, out_nbrs, out_cmps);
  free(c);
  return 0;
}

/* ------------------------------------------------------------ build */
static uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
typedef struct { uint64_t key; uint32_t idx; } permkey_t;
static int cmp_permkey(const void* x, const void* y) {
  const permkey_t* a = x; const permkey_t* b = y;
  if (a->key < b->key) return -1;
  if (a->key > b->key) return 1;
  return (a->idx > b->idx) - (a->idx < b->idx);
}
/* The insertion order: indices ordered by splitmix64(seed + i). This is the
 * definition the oracle's ParlayLib shim gives random_permutation (index.h:212),
 * so the reference build, this oracle and the GPU build insert in one order. */
void oracle_permutation(uint32_t m, uint64_t seed, uint32_t* out) {
  permkey_t* k = (permkey_t*)malloc(sizeof(permkey_t) * (m + 1));
  for (uint32_t i = 0; i < m; i++) { k[i].key = splitmix64(seed + i); k[i].idx = i; }
  qsort(k, m, sizeof(permkey_t), cmp_permkey);
  for (uint32_t i = 0; i < m; i++) out[i] = k[i].idx;
  free(k);
}

typedef struct { uint32_t key, val, ord; } edge_t;
static int cmp_edge(const void* x, const void* y) {
  const edge_t* a = x; const edge_t* b = y;
  if (a->key != b->key) return a->key < b->key ? -1 : 1;
  return (a->ord > b->ord) - (a->ord < b->ord); /* stable: input order */
}

/* Batch schedule of knn_index::batch_insert (index.h:206-240): batch i covers
 * [2^i - 1, 2^(i+1) - 1) until 2^i exceeds max_batch = min(0.02 n, 1e6), then
 * fixed-size batches. Writes up to cap (floor, ceiling) pairs; returns count. */
uint32_t oracle_batch_schedule(uint64_t n, uint64_t m, double base, double max_fraction,
                               uint64_t* floors, uint64_t* ceilings, uint32_t cap) {
  uint64_t max_batch = (uint64_t)(max_fraction * (double)(float)n);
  if (max_batch > 1000000ull) max_batch = 1000000ull;
  if (max_batch == 0) max_batch = n;
  uint64_t count = 0, inc = 0;
  uint32_t nb = 0;
  while (count < m) {
    uint64_t fl, ce;
    if (pow(base, (double)inc) <= (double)max_batch) {
      fl = (uint64_t)pow(base, (double)inc) - 1;
      uint64_t c2 = (uint64_t)pow(base, (double)(inc + 1)) - 1;
      ce = c2 < m ? c2 : m;
      count = ce;
    } else {
      fl = count;
      ce = count + max_batch < m ? count + max_batch : m;
      count += max_batch;
    }
    if (nb < cap) { floors[nb] = fl; ceilings[nb] = ce; }
    nb++;
    inc++;
  }
  return nb;
}

/* One pass of knn_index::batch_insert over all points in perm order
 * (index.h:188-319). G is updated in place. Returns 0 or -1. */
static int batch_insert(const pts_t* P, uint32_t n, uint32_t* G, uint32_t R, uint32_t L,
                        double alpha, double batch_factor, const uint32_t* perm,
                        uint64_t* dist_total) {
  uint64_t floors[4096], ceilings[4096];
  uint32_t nb = oracle_batch_schedule(n, n, 2.0, 0.02, floors, ceilings, 4096);
  if (nb > 4096) return -1;
  qparams_t QP = {0, L, R, (uint64_t)n, batch_factor}; /* index.h:251-252 */
  uint32_t start = 0;
  for (uint32_t b = 0; b < nb; b++) {
    uint64_t fl = floors[b], ce = ceilings[b];
    uint64_t bs = ce - fl;
    uint32_t* new_out = (uint32_t*)malloc(sizeof(uint32_t) * bs * R + 4);
    uint32_t* new_n = (uint32_t*)malloc(sizeof(uint32_t) * bs + 4);
    /* search + prune against the pre-batch graph (:247-269) */
    for (uint64_t i = fl; i < ce; i++) {
      uint32_t index = perm[i];
      bs_out_t o;
      if (beam_search_one(P, G, R, row(P, index), index, &start, 1, &QP, &o) != 0) return -1;
      long pc = 0;
      new_n[i - fl] = robust_prune(P, G, R, index, o.visited, o.visited_n, alpha, 1,
                                   new_out + (i - fl) * R, &pc);
      if (dist_total) *dist_total += o.cmps + (uint64_t)pc;
      free(o.frontier);
      free(o.visited);
    }
    /* write the new out-lists (:271-273) */
    for (uint64_t i = fl; i < ce; i++) {
      uint32_t* gr = G + (size_t)perm[i] * (R + 1);
      gr[0] = new_n[i - fl];
      for (uint32_t j = 0; j < R; j++) gr[1 + j] = j < new_n[i - fl] ? new_out[(i - fl) * R + j] : 0;
    }
    /* reverse edges (ngh, index), grouped by ngh, stable (:281-285) */
    size_t ne = 0;
    for (uint64_t i = 0; i < bs; i++) ne += new_n[i];
    edge_t* E = (edge_t*)malloc(sizeof(edge_t) * (ne + 1));
    size_t t = 0;
    for (uint64_t i = 0; i < bs; i++)
      for (uint32_t j = 0; j < new_n[i]; j++) { E[t].key = new_out[i * R + j]; E[t].val = perm[fl + i]; E[t].ord = (uint32_t)t; t++; }
    qsort(E, ne, sizeof(edge_t), cmp_edge);
    /* per target: append without repeats, or robustPrune (:292-303) */
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * (ne + R + 1));
    size_t s = 0;
    while (s < ne) {
      size_t e = s;
      while (e < ne && E[e].key == E[s].key) e++;
      uint32_t index = E[s].key;
      size_t nc = e - s;
      uint32_t* gr = G + (size_t)index * (R + 1);
      size_t newsize = nc + gr[0];
      if (newsize <= R) {
        /* add_neighbors_without_repeats(G[index], candidates) (:140-146) */
        size_t m2 = 0;
        for (size_t u = s; u < e; u++) tmp[m2++] = E[u].val;
        for (uint32_t u = 0; u < gr[0]; u++) {
          uint32_t x = gr[1 + u];
          int dup = 0;
          for (size_t w = s; w < e; w++) if (E[w].val == x) { dup = 1; break; }
          if (!dup) tmp[m2++] = x;
        }
        if (m2 > R) return -1; /* update_neighbors would abort (graph.h:79-83) */
        gr[0] = (uint32_t)m2;
        for (size_t u = 0; u < R; u++) gr[1 + u] = u < m2 ? tmp[u] : 0;
      } else {
        /* robustPrune(index, ids, ...) computes each candidate's distance
         * first (index.h:124-137) */
        pair_t* c = (pair_t*)malloc(sizeof(pair_t) * (nc + 1));
        for (size_t u = 0; u < nc; u++) { c[u].id = E[s + u].val; c[u].d = dist(P, row(P, c[u].id), row(P, index)); }
        long pc = 0;
        uint32_t nn = robust_prune(P, G, R, index, c, nc, alpha, 1, tmp, &pc);
        if (dist_total) *dist_total += nc + (uint64_t)pc;
        gr[0] = nn;
        for (uint32_t u = 0; u < R; u++) gr[1 + u] = u < nn ? tmp[u] : 0;
        free(c);
      }
      s = e;
    }
    free(tmp);
    free(E);
    free(new_out);
    free(new_n);
  }
  return 0;
}

/* knn_index::build_index (index.h:150-186) without the final neighbour sort
 * when sort_neighbors == 0. Passes use alpha 1.0 except the last (:173-178).
 * perm may be NULL (then oracle_permutation(n, seed)). The final sort
 * (:180-185) orders each list by distance; ties are ordered by id here (the
 * reference's std::sort leaves them unspecified). */
int oracle_build(int dtype, int metric, uint32_t n, uint32_t d, const void* base, uint32_t R,
                 uint32_t L, double alpha, int passes, double batch_factor, const uint32_t* perm,
                 uint64_t perm_seed, int sort_neighbors, uint32_t* out_graph,
                 uint64_t* out_dist_total) {
  pts_t P = {dtype, metric, d, d * elem_size(dtype), (const uint8_t*)base};
  memset(out_graph, 0, sizeof(uint32_t) * (size_t)n * (R + 1));
  uint32_t* pm = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  if (perm) memcpy(pm, perm, sizeof(uint32_t) * n);
  else oracle_permutation(n, perm_seed, pm);
  uint64_t dt = 0;
  for (int pass = 0; pass < passes; pass++) {
    double a = (pass == passes - 1) ? alpha : 1.0;
    if (batch_insert(&P, n, out_graph, R, L, a, batch_factor, pm, &dt) != 0) { free(pm); return -1; }
  }
  if (sort_neighbors) {
    pair_t* tmp = (pair_t*)malloc(sizeof(pair_t) * (R + 1));
    for (uint32_t v = 0; v < n; v++) {
      uint32_t* gr = out_graph + (size_t)v * (R + 1);
      for (uint32_t j = 0; j < gr[0]; j++) { tmp[j].id = gr[1 + j]; tmp[j].d = dist(&P, row(&P, v), row(&P, gr[1 + j])); }
      qsort(tmp, gr[0], sizeof(pair_t), cmp_pair);
      for (uint32_t j = 0; j < gr[0]; j++) gr[1 + j] = tmp[j].id;
    }
    free(tmp);
  }
  if (out_dist_total) *out_dist_total = dt;
  free(pm);
  return 0;
}

/* ------------------------------------------------------------ brute force */
/* compute_groundtruth (data_tools/compute_groundtruth.cpp:22-60): exact top-k
 * by a full scan. Integer types use the exact integer distance; float uses
 * FP64 arithmetic (this project's FP64 oracle). Ties are ordered by id. */
typedef struct { double d; uint32_t id; } dpair_t;
static int cmp_dpair(const void* x, const void* y) {
  const dpair_t* a = x; const dpair_t* b = y;
  if (a->d < b->d) return -1;
  if (a->d > b->d) return 1;
  return (a->id > b->id) - (a->id < b->id);
}
static double dist64(int dtype, int metric, unsigned d, const void* a, const void* b) {
  double r = 0.0;
  for (unsigned i = 0; i < d; i++) {
    double x, y;
    if (dtype == 0) { x = ((const uint8_t*)a)[i]; y = ((const uint8_t*)b)[i]; }
    else if (dtype == 1) { x = ((const int8_t*)a)[i]; y = ((const int8_t*)b)[i]; }
    else { x = ((const float*)a)[i]; y = ((const float*)b)[i]; }
    r += metric == 0 ? (x - y) * (x - y) : x * y;
  }
  return metric == 0 ? r : -r;
}
int oracle_groundtruth(int dtype, int metric, uint32_t n, uint32_t d, const void* base,
                       uint32_t nq, const void* queries, uint32_t k, uint32_t* out_ids,
                       double* out_d) {
  size_t rb = d * elem_size(dtype);
  dpair_t* best = (dpair_t*)malloc(sizeof(dpair_t) * (k + 1));
  for (uint32_t q = 0; q < nq; q++) {
    const uint8_t* qp = (const uint8_t*)queries + (size_t)q * rb;
    uint32_t cnt = 0;
    for (uint32_t j = 0; j < n; j++) {
      dpair_t e = {dist64(dtype, metric, d, qp, (const uint8_t*)base + (size_t)j * rb), j};
      if (cnt < k) {
        best[cnt++] = e;
        for (uint32_t t = cnt - 1; t > 0 && cmp_dpair(&best[t], &best[t - 1]) < 0; t--) {
          dpair_t s = best[t]; best[t] = best[t - 1]; best[t - 1] = s;
        }
      } else if (cmp_dpair(&e, &best[k - 1]) < 0) {
        best[k - 1] = e;
        for (uint32_t t = k - 1; t > 0 && cmp_dpair(&best[t], &best[t - 1]) < 0; t--) {
          dpair_t s = best[t]; best[t] = best[t - 1]; best[t - 1] = s;
        }
      }
    }
    for (uint32_t t = 0; t < k; t++) {
      out_ids[(size_t)q * k + t] = t < cnt ? best[t].id : EMPTY32;
      if (out_d) out_d[(size_t)q * k + t] = t < cnt ? best[t].d : 0.0;
    }
  }
  free(best);
  return 0;
}
