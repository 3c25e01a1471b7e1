// Warp-per-query beam search: the device form of ParlayANN's
// filtered_beam_search with use_filtering = false and no early stopping
// (algorithms/utils/beamSearch.h:33-228).
//
// One warp owns one query at a time and keeps all of its search state in
// shared memory:
//   qs    the query vector (row stride bytes)
//   fr    the frontier, <= L 64-bit (dist, id) keys, sorted; bit 31 of the id
//         word marks a visited entry. The reference's separate sorted
//         `visited` list and `unvisited_frontier` (set_difference, :217-222)
//         are represented by that flag: the next node to expand is the first
//         unflagged frontier entry, exactly unvisited_frontier[offset] (:119),
//         because between merges the frontier is unchanged and the flagged
//         entries are precisely unvisited_frontier[0..offset).
//   cand  candidates accumulated since the last merge (deferred batching,
//         :185-192); sorted by rank into cand2 and merged into the frontier
//         (set_union + trim to L, :197-214).
//   table the seen-set (:66, hashset.h). The reference's hashset is exact
//         until it grows; this table is exact, and the kernel counts inserts
//         against the reference's growth threshold (capacity/2) to flag
//         queries on which the reference's growth could change its result.
// Lanes split the adjacency row (one id per lane), test-and-insert ids with
// shared-memory CAS, compact the new ids, and compute one distance per lane
// (so float sums keep the reference's sequential order).
#pragma once
#include "common.cuh"
#include "lowprec.cuh"

namespace pann {

struct SearchArgs {
  // index
  const uint8_t* points;
  uint64_t stride;  // bytes per row (multiple of 16)
  uint32_t d;
  uint32_t nchunks;  // stride / 16
  const uint32_t* graph;
  uint32_t R;
  // queries
  const uint8_t* queries;  // nq rows of `stride` bytes; null in build mode
  const uint32_t* self_ids;  // build mode: query j is point self_ids[j] and skips itself
  uint32_t nq;
  const uint32_t* job_list;   // optional: job j is query job_list[j]
  const uint32_t* njobs_dev;  // optional: number of jobs read from device memory
  uint32_t* job_counter;      // dynamic work distribution (zeroed before launch)
  // query parameters (QueryParams, types.h:233-252); k and L are the maxima
  // when qk / qL give per-query values (the batched form)
  uint32_t k, L, dl;
  const uint32_t* qk;  // optional per-query k
  const uint32_t* qL;  // optional per-query beam
  uint32_t kstride;    // output row stride (>= every k)
  uint64_t limit;
  double batch_factor;
  uint32_t ref_half;  // the reference hashset's growth threshold: capacity/2
  const uint32_t* starts;
  uint32_t n_start;
  // per-warp shared-memory layout
  uint32_t Ccap;  // candidate buffer capacity
  uint32_t S;     // seen-table slots (power of two)
  uint32_t warp_bytes;
  uint32_t* gtables;  // global seen tables (TABLE_GLOBAL form), S slots per resident warp
  uint32_t* gspill;   // shared-memory form: per resident warp, Sg-slot table taking inserts
  uint32_t Sg;        // once the shared table is 3/4 full (0 = no spill: re-run instead)
  // outputs
  uint32_t* out_ids;
  float* out_dists;
  uint32_t* out_visited;
  uint32_t* out_cmps;
  uint32_t* out_status;
  uint64_t* vis_keys;  // build mode: visited (dist,id) keys, vis_cap per query
  uint32_t vis_cap;
  uint32_t* redo_list;  // queries whose seen table filled up
  uint32_t* redo_count;
  uint32_t* emu_list;   // queries on which the reference's hashset would grow
  uint32_t* emu_rec;    // per emu_list entry: resume record index, or PAD to re-run from scratch
  uint32_t* emu_count;
  uint64_t opaque_zero;  // always 0; see f32_chunk2
  // Hand-off to the emulation tier. Before the visit in which a query could
  // push the reference's seen-set past its growth threshold, tier 0 stops the
  // query and saves its exact state in a resume record; the emulation tier
  // rebuilds the reference's table from the insertion log and continues.
  uint32_t* inslog;     // per resident warp: logcap ids, inserted in call order
  uint32_t logcap;
  uint32_t* vislog;     // per resident warp: viscap visited ids, in visit order
  uint32_t viscap;
  uint32_t* rec_pool;   // rec_cap records of rec_words words (layout: resume_layout)
  uint32_t rec_cap;
  uint32_t rec_words;
  uint32_t* rec_count;
  // precision form (float32 indexes): low-precision rows steer the search,
  // the best `rerank` frontier entries are re-scored exactly at the end
  const uint8_t* lp_rows;
  uint64_t lp_stride;
  uint32_t lp_chunks;
  const float* lp_scales;
  const float* lp_norms;  // squared norm of every low-precision row (tensor-core tile scoring)
  uint32_t rerank;
  // early stopping of range search (earlyStopping.h:19-29); es_count == 0 disables it
  double es_count;   // QP.early_stopping_count
  double es_radius;  // QP.radius as the rule sees it
  double es_esr;     // QP.early_stopping_radius
};

// The reference's seen-set capacity for beam L and degree limit dl is
// 2^ceil(log2(2 (10 + L) dl)) (beamSearch.h:66, hashset.h:50-54); it grows
// above half of that.
__host__ __device__ inline uint32_t ref_bits(uint32_t L, uint32_t dl) {
  const uint64_t n = 2ull * (10ull + L) * dl;
  uint32_t b = 0;
  while ((1ull << b) < n) b++;
  return b;
}

// Resume record: 8-word header (query, fn, cn, visits, cmps, entries), the
// frontier (2L words), the candidates (2 Ccap words), the insertion log
// (logcap words) and the visited ids (viscap words).
struct ResumeLayout {
  uint32_t fr, cand, log, vis, words;
};
__host__ __device__ inline ResumeLayout resume_layout(uint32_t L, uint32_t Ccap, uint32_t logcap, uint32_t viscap) {
  ResumeLayout r;
  r.fr = 8;
  r.cand = r.fr + 2 * L;
  r.log = r.cand + 2 * Ccap;
  r.vis = r.log + logcap;
  r.words = (r.vis + viscap + 3) & ~3u;
  return r;
}

__host__ __device__ inline uint32_t search_warp_bytes(uint64_t stride, uint32_t L, uint32_t Ccap, uint32_t R,
                                                      uint32_t S, bool table_global) {
  uint64_t b = stride;                 // query
  b += 16ull * L;                      // fr + fr2
  b += 16ull * Ccap;                   // cand + cand2
  b += 4ull * ((R + 3) & ~3u);         // compacted new ids
  if (!table_global) b += 4ull * S;    // seen table
  return (uint32_t)((b + 15) & ~15ull);
}

// Sort n distinct keys from `in` into `out` by rank (warp-cooperative).
__device__ __forceinline__ void warp_rank_sort(const uint64_t* in, uint64_t* out, int n, int lane) {
  for (int i = lane; i < n; i += 32) {
    uint64_t ki = in[i] & PANN_KEYMASK;
    int r = 0;
    for (int j = 0; j < n; j++) {
      uint64_t kj = in[j] & PANN_KEYMASK;
      r += (kj < ki) | ((kj == ki) & (j < i));
    }
    out[r] = in[i];
  }
}

// Merge sorted frontier fr[0..fn) with sorted candidates c[0..cn) into out,
// keeping the first L (std::set_union then trim, beamSearch.h:202-214). Keys
// of the two inputs are disjoint (the seen-set admits each id once).
__device__ __forceinline__ int warp_merge(const uint64_t* fr, int fn, const uint64_t* c, int cn, uint64_t* out,
                                          int L, int lane) {
  for (int i = lane; i < fn; i += 32) {
    uint64_t k = fr[i] & PANN_KEYMASK;
    int lo = 0, hi = cn;
    while (lo < hi) { int mid = (lo + hi) >> 1; if ((c[mid] & PANN_KEYMASK) < k) lo = mid + 1; else hi = mid; }
    int pos = i + lo;
    if (pos < L) out[pos] = fr[i];
  }
  for (int j = lane; j < cn; j += 32) {
    uint64_t k = c[j] & PANN_KEYMASK;
    int lo = 0, hi = fn;
    while (lo < hi) { int mid = (lo + hi) >> 1; if ((fr[mid] & PANN_KEYMASK) < k) lo = mid + 1; else hi = mid; }
    int pos = j + lo;
    if (pos < L) out[pos] = c[j];
  }
  int t = fn + cn;
  return t < L ? t : L;
}

// Lookup without insert (linear probing): 1 if present.
__device__ __forceinline__ int table_has(const uint32_t* table, uint32_t mask, uint32_t id) {
  uint32_t h = hash_slot(id, mask);
  for (uint32_t probe = 0; probe <= mask; probe++) {
    uint32_t v = table[h];
    if (v == id) return 1;
    if (v == PANN_PAD) return 0;
    h = (h + 1) & mask;
  }
  return 0;
}

// Test-and-insert into an open-addressing table (linear probing). Returns 1 if
// id was inserted (first sighting), 0 if it was already present. The caller
// keeps the load below 1 so the probe always ends.
__device__ __forceinline__ int table_insert(uint32_t* table, uint32_t mask, uint32_t id) {
  uint32_t h = hash_slot(id, mask);
  for (uint32_t probe = 0; probe <= mask; probe++) {
    uint32_t old = atomicCAS(table + h, PANN_PAD, id);
    if (old == PANN_PAD) return 1;
    if (old == id) return 0;
    h = (h + 1) & mask;
  }
  return 0;
}

// Chunks of a float32 row a tier-0 lane has in flight at once.
constexpr int T0_ROW_CHUNKS = 12;

// MINB: blocks of 128 threads the register budget is fitted to (3: 168
// registers a thread; 4: 128).
template <int DT, int MT, bool TABLE_GLOBAL, int PREC = PREC_F32, int MINB = 3>
__global__ void __launch_bounds__(128, MINB) search_kernel(SearchArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const unsigned FULL = 0xFFFFFFFFu;

  uint8_t* wbase = smem + (size_t)warp * a.warp_bytes;
  uint8_t* qs = wbase;
  uint64_t* frA = reinterpret_cast<uint64_t*>(wbase + a.stride);
  uint64_t* frB = frA + a.L;
  uint64_t* cand = frB + a.L;
  uint64_t* cand2 = cand + a.Ccap;
  uint32_t* nbuf = reinterpret_cast<uint32_t*>(cand2 + a.Ccap);
  uint32_t* table;
  if (TABLE_GLOBAL) {
    table = a.gtables + ((size_t)blockIdx.x * wpb + warp) * a.S;
  } else {
    table = nbuf + ((a.R + 3) & ~3u);
  }
  const uint32_t mask = a.S - 1;
  const uint32_t table_limit = (a.S >> 2) * 3;  // abort above 3/4 load
  uint32_t* spill = (!TABLE_GLOBAL && a.gspill) ? a.gspill + ((size_t)blockIdx.x * wpb + warp) * a.Sg : nullptr;
  const uint32_t smask = a.Sg - 1;
  const uint32_t spill_limit = (a.Sg >> 2) * 3;
  const uint32_t njobs = a.njobs_dev ? *a.njobs_dev : a.nq;
  const bool handoff = PREC == PREC_F32 && a.inslog != nullptr && a.emu_list != nullptr;
  uint32_t* const wlog = handoff ? a.inslog + ((size_t)blockIdx.x * wpb + warp) * a.logcap : nullptr;
  uint32_t* const wvis = handoff ? a.vislog + ((size_t)blockIdx.x * wpb + warp) * a.viscap : nullptr;

  for (;;) {
    uint32_t job = 0;
    if (lane == 0) job = atomicAdd(a.job_counter, 1u);
    job = __shfl_sync(FULL, job, 0);
    if (job >= njobs) break;
    const uint32_t qi = a.job_list ? a.job_list[job] : job;
    const uint32_t self = a.self_ids ? a.self_ids[qi] : PANN_PAD;
    const uint8_t* qsrc = a.self_ids ? a.points + (uint64_t)self * a.stride : a.queries + (uint64_t)qi * a.stride;
    const uint32_t L = a.qL ? a.qL[qi] : a.L;  // this query's beam (<= a.L, the buffer size)
    const uint32_t kq = a.qk ? a.qk[qi] : a.k;
    const uint32_t ref_half = a.qL ? (1u << ref_bits(L, a.dl)) / 2 : a.ref_half;

    // stage the query, clear the seen table
    stage_query<DT, MT>(qs, qsrc, (int)a.nchunks, lane);
    {
      uint4 e = make_uint4(PANN_PAD, PANN_PAD, PANN_PAD, PANN_PAD);
      for (uint32_t c = lane; c < (a.S >> 2); c += 32) reinterpret_cast<uint4*>(table)[c] = e;
    }
    if (TABLE_GLOBAL) __threadfence_block();
    __syncwarp();
    int32_t qq = 0;
    if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), a.nchunks);

    // starting points (:73-77); n_start <= L, staged in frB then sorted into frA
    for (uint32_t s = lane; s < a.n_start; s += 32) {
      uint32_t id = a.starts[s];
      float dd, dummy;
      if (PREC == PREC_F32) dd = point_dist<DT, MT>(a.points + (uint64_t)id * a.stride, qs, a.d, a.nchunks, qq);
      else lp_dist2<MT, PREC>(a.lp_rows + (uint64_t)id * a.lp_stride, nullptr, reinterpret_cast<const float*>(qs),
                              a.lp_scales, (int)a.d, (int)a.lp_chunks, dd, dummy);
      frB[s] = make_key(dd, id);
      table_insert(table, mask, id);
      if (handoff) wlog[s] = id;
    }
    __syncwarp();
    uint64_t* fr = frA;
    uint64_t* fr2 = frB;
    warp_rank_sort(frB, fr, (int)a.n_start, lane);
    __syncwarp();
    int fn = (int)a.n_start;
    int cn = 0;
    uint32_t entries = a.n_start;    // distinct ids inserted (the reference's num_entries)
    uint32_t entries_sh = a.n_start;  // of which in the shared-memory table
    bool spilled = false;
    uint32_t cmps = a.n_start;
    uint64_t nvis = 0;
    uint32_t status = 0;
    bool hand_over = false;
    const uint32_t nel = a.dl < a.R ? a.dl : a.R;
    // the reference's early-stopping rule reads unvisited_frontier[0], which is
    // refreshed only at a merge: its distance, taken at the first scan after one
    float u0 = 0.0f;
    bool u0_fresh = true;

    for (;;) {
      __syncwarp();
      // first unvisited frontier entry and the number of unvisited entries
      int first = -1, second = -1, cnt = 0;
      for (int b = 0; b < fn; b += 32) {
        int i = b + lane;
        bool unv = (i < fn) && !(fr[i] & PANN_VFLAG);
        unsigned m = __ballot_sync(FULL, unv);
        if (first < 0 && m) {
          first = b + __ffs(m) - 1;
          m &= m - 1;
        }
        if (first >= 0 && second < 0 && m) second = b + __ffs(m) - 1;
        cnt += __popc(m);
      }
      if (first >= 0) cnt += 1;
      if (first < 0 || nvis >= a.limit) break;  // :116
      if (u0_fresh) {
        u0 = key_dist(fr[first]);
        u0_fresh = false;
      }
      if (a.es_count > 0.0 && (double)nvis >= a.es_count && !((double)key_dist(fr[0]) <= a.es_radius) &&
          !((double)u0 <= a.es_esr))
        break;  // early_stopping (earlyStopping.h:19-29), checked at beamSearch.h:120-121
      if (handoff && entries + nel > ref_half) {
        // this visit could cross the reference's growth threshold
        status |= QS_REF_WOULD_GROW;
        hand_over = true;
        break;
      }
      const uint64_t cur = fr[first];
      // the next node to expand is most often the following unvisited entry:
      // start its adjacency row on its way to L2
      if (second >= 0 && lane == 0)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a.graph + (uint64_t)key_id(fr[second]) * a.R));
      __syncwarp();
      if (lane == 0) fr[first] = cur | PANN_VFLAG;
      nvis++;
      if (a.vis_keys && lane == 0) {
        if (nvis <= a.vis_cap) a.vis_keys[(uint64_t)qi * a.vis_cap + (nvis - 1)] = cur & PANN_KEYMASK;
      }
      if (nvis > a.vis_cap && a.vis_keys) status |= QS_VISIT_OVERFLOW;
      const bool full = (fn == (int)L);
      const float cutoff = full ? key_dist(fr[fn - 1]) : 3.40282346638528859812e+38F;  // :173-175
      const uint32_t cid = key_id(cur);
      if (handoff && lane == 0 && nvis <= a.viscap) wvis[nvis - 1] = cid;

      // neighbours not seen before (:151-160), compacted into nbuf
      const uint32_t* grow = a.graph + (uint64_t)cid * a.R;
      if (!spilled && entries_sh + nel > table_limit) {
        if (!spill) { status |= QS_TABLE_FULL; break; }
        // the shared table is frozen from here on; new ids go to the global spill table
        spilled = true;
        uint4 e4 = make_uint4(PANN_PAD, PANN_PAD, PANN_PAD, PANN_PAD);
        for (uint32_t c = lane; c < (a.Sg >> 2); c += 32) reinterpret_cast<uint4*>(spill)[c] = e4;
        __threadfence_block();
        __syncwarp();
      }
      if (spilled && entries - entries_sh + nel > spill_limit) { status |= QS_TABLE_FULL; break; }
      int nnew = 0;
      uint32_t ins = 0;
      // the next 32 ids are loaded before this chunk's seen-set work, so a
      // row longer than one warp costs one round trip, not one per chunk
      uint32_t vnext = (uint32_t)lane < nel ? __ldg(grow + lane) : PANN_PAD;
      for (uint32_t b = 0; b < nel; b += 32) {
        const uint32_t v = vnext;
        vnext = (b + 32 + lane < nel) ? __ldg(grow + b + 32 + lane) : PANN_PAD;
        int inserted = 0;
        if (v != PANN_PAD) {
          if (!spilled) inserted = table_insert(table, mask, v);
          else if (!table_has(table, mask, v)) inserted = table_insert(spill, smask, v);
        }
        bool isnew = inserted && (v != self);
        unsigned mi = __ballot_sync(FULL, inserted);
        unsigned mn = __ballot_sync(FULL, isnew);
        if (handoff && inserted) wlog[entries + ins + __popc(mi & ((1u << lane) - 1))] = v;  // call order
        ins += __popc(mi);
        if (isnew) nbuf[nnew + __popc(mn & ((1u << lane) - 1))] = v;
        nnew += __popc(mn);
      }
      entries += ins;
      if (!spilled) entries_sh += ins;
      if (entries > ref_half) status |= QS_REF_WOULD_GROW;
      __syncwarp();

      // distances; keep those below the cutoff (:176-182)
      cmps += (uint32_t)nnew;
      if ((uint32_t)(cn + nnew) > a.Ccap) { status |= QS_INTERNAL; break; }
      // float32 rows: one row per lane per round, T0_ROW_CHUNKS chunks of it
      // in flight at once (the rest of the row prefetched to L2 first). On the
      // 1M x 96 workload this is 2.29 M QPS against 2.11 M for two rows per
      // lane in batches of 8 chunks (PAIR_CHUNKS), 2.29 M with 16 chunks, and
      // 1.89 M with all 24 chunks at once, which spills (A/B on one box).
      if (PREC == PREC_F32 && DT == DT_F32) {
        for (int b = 0; b < nnew; b += 32) {
          const int i0 = b + lane;
          float d0 = 0.0f;
          uint32_t v0 = 0;
          if (i0 < nnew) {
            v0 = nbuf[i0];
            const float4* row = reinterpret_cast<const float4*>(a.points + (uint64_t)v0 * a.stride);
            const float4* q = reinterpret_cast<const float4*>(qs);
            const int nv = (int)a.nchunks;
            if (nv > T0_ROW_CHUNKS) prefetch_row_l2(row, nv);
            float r = 0.0f;
            for (int c0 = 0; c0 < nv; c0 += T0_ROW_CHUNKS) {
              float4 buf[T0_ROW_CHUNKS];
#pragma unroll
              for (int c = 0; c < T0_ROW_CHUNKS; c++)
                if (c0 + c < nv) buf[c] = __ldg(row + c0 + c);
#pragma unroll
              for (int c = 0; c < T0_ROW_CHUNKS; c++)
                if (c0 + c < nv) r = f32_chunk<MT>(r, buf[c], q[c0 + c]);
            }
            d0 = MT == MT_L2 ? r : -r;
          }
          const bool keep0 = i0 < nnew && !(d0 >= cutoff);
          const unsigned m0 = __ballot_sync(FULL, keep0);
          if (keep0) cand[cn + __popc(m0 & ((1u << lane) - 1))] = make_key(d0, v0);
          cn += __popc(m0);
        }
      } else
      // two rows per lane per round: rows b+lane and b+32+lane
      for (int b = 0; b < nnew; b += 64) {
        const int i0 = b + lane, i1 = b + 32 + lane;
        float d0 = 0.0f, d1 = 0.0f;
        uint32_t v0 = 0, v1 = 0;
        if (i0 < nnew) {
          v0 = nbuf[i0];
          v1 = i1 < nnew ? nbuf[i1] : 0u;
          if (PREC == PREC_F32)
            point_dist2<DT, MT>(a.points + (uint64_t)v0 * a.stride,
                                i1 < nnew ? a.points + (uint64_t)v1 * a.stride : nullptr, qs, a.nchunks, qq, d0, d1,
                                a.opaque_zero);
          else
            lp_dist2<MT, PREC>(a.lp_rows + (uint64_t)v0 * a.lp_stride,
                               i1 < nnew ? a.lp_rows + (uint64_t)v1 * a.lp_stride : nullptr,
                               reinterpret_cast<const float*>(qs), a.lp_scales, (int)a.d, (int)a.lp_chunks, d0, d1);
        }
        bool keep0 = i0 < nnew && !(d0 >= cutoff);
        unsigned m0 = __ballot_sync(FULL, keep0);
        if (keep0) cand[cn + __popc(m0 & ((1u << lane) - 1))] = make_key(d0, v0);
        cn += __popc(m0);
        bool keep1 = i1 < nnew && !(d1 >= cutoff);
        unsigned m1 = __ballot_sync(FULL, keep1);
        if (keep1) cand[cn + __popc(m1 & ((1u << lane) - 1))] = make_key(d1, v1);
        cn += __popc(m1);
      }
      // deferred batching (:185-192): cnt - 1 unvisited entries remain after this one
      if (cn == 0 || (a.limit >= 2ull * L && (double)cn < a.batch_factor * (double)L && cnt - 1 >= 1)) continue;
      __syncwarp();
      warp_rank_sort(cand, cand2, cn, lane);
      __syncwarp();
      fn = warp_merge(fr, fn, cand2, cn, fr2, (int)L, lane);
      u0_fresh = true;
      uint64_t* t = fr; fr = fr2; fr2 = t;
      cn = 0;
      __syncwarp();
    }

    if (status & (QS_TABLE_FULL | QS_INTERNAL)) {
      if (status & QS_INTERNAL) {
        if (lane == 0 && a.out_status) a.out_status[qi] = status;
        __syncwarp();
        continue;
      }
      if (lane == 0 && a.redo_list) a.redo_list[atomicAdd(a.redo_count, 1u)] = qi;
      if (lane == 0 && a.out_status) a.out_status[qi] = status;
      __syncwarp();
      continue;
    }
    if ((status & QS_REF_WOULD_GROW) && a.emu_list) {
      // continued (or re-run) by the exact-emulation tier, which writes this query's outputs
      uint32_t r = PANN_PAD;
      if (hand_over) {
        if (lane == 0) r = atomicAdd(a.rec_count, 1u);
        r = __shfl_sync(FULL, r, 0);
        if (r < a.rec_cap && nvis <= a.viscap) {
          const ResumeLayout ly = resume_layout(a.L, a.Ccap, a.logcap, a.viscap);
          uint32_t* rec = a.rec_pool + (size_t)r * a.rec_words;
          if (lane == 0) {
            rec[0] = qi; rec[1] = (uint32_t)fn; rec[2] = (uint32_t)cn; rec[3] = (uint32_t)nvis;
            rec[4] = cmps; rec[5] = entries; rec[6] = __float_as_uint(u0);
          }
          uint64_t* rfr = reinterpret_cast<uint64_t*>(rec + ly.fr);
          uint64_t* rcand = reinterpret_cast<uint64_t*>(rec + ly.cand);
          for (int i = lane; i < fn; i += 32) rfr[i] = fr[i];
          for (int i = lane; i < cn; i += 32) rcand[i] = cand[i];
          __syncwarp();
          for (uint32_t i = lane; i < entries; i += 32) rec[ly.log + i] = wlog[i];
          for (uint32_t i = lane; i < (uint32_t)nvis; i += 32) rec[ly.vis + i] = wvis[i];
        } else {
          r = PANN_PAD;  // no room: the emulation re-runs the query from the start
        }
      }
      // publish: the record and the list entry before the record index, which
      // an emulation pass running beside this kernel reads as "ready"
      __threadfence();
      __syncwarp();
      if (lane == 0) {
        uint32_t pos = atomicAdd(a.emu_count, 1u);
        a.emu_list[pos] = qi;
        __threadfence();
        atomicExch(a.emu_rec + pos, r);
      }
      __syncwarp();
      continue;
    }
    if ((uint32_t)fn < kq) status |= QS_SHORT;
    uint32_t* const oid = a.out_ids + (uint64_t)qi * a.kstride;
    float* const odist = a.out_dists ? a.out_dists + (uint64_t)qi * a.kstride : nullptr;
    if (PREC != PREC_F32) {
      // re-rank the best min(rerank, fn) entries by exact float32 distance
      // (beam_search_rerank's full-precision pass, beamSearch.h:569-587)
      const uint32_t rr = a.rerank ? a.rerank : 4 * kq;  // 0: 4k of this query
      const int nr = (int)min((uint32_t)fn, rr > kq ? rr : kq);
      for (int b = 0; b < nr; b += 64) {
        const int i0 = b + lane, i1 = b + 32 + lane;
        float d0 = 0.f, d1 = 0.f;
        uint32_t v0 = 0, v1 = 0;
        if (i0 < nr) {
          v0 = key_id(fr[i0]);
          v1 = i1 < nr ? key_id(fr[i1]) : 0u;
          point_dist2<DT, MT>(a.points + (uint64_t)v0 * a.stride,
                              i1 < nr ? a.points + (uint64_t)v1 * a.stride : nullptr, qs, a.nchunks, qq, d0, d1,
                              a.opaque_zero);
          fr2[i0] = make_key(d0, v0);
          if (i1 < nr) fr2[i1] = make_key(d1, v1);
        }
      }
      __syncwarp();
      for (int i = lane; i < nr; i += 32) {
        const uint64_t ki = fr2[i];
        int r = 0;
        for (int j = 0; j < nr; j++) r += fr2[j] < ki;
        if ((uint32_t)r < kq) {
          oid[r] = key_id(ki);
          if (odist) odist[r] = key_dist(ki);
        }
      }
      for (uint32_t j = min((uint32_t)nr, kq) + lane; j < a.kstride; j += 32) {
        oid[j] = PANN_PAD;
        if (odist) odist[j] = 0.0f;
      }
    } else {
      for (uint32_t j = lane; j < a.kstride; j += 32) {
        bool ok = j < (uint32_t)fn && j < kq;
        oid[j] = ok ? key_id(fr[j]) : PANN_PAD;
        if (odist) odist[j] = ok ? key_dist(fr[j]) : 0.0f;
      }
    }
    if (lane == 0) {
      if (a.out_visited) a.out_visited[qi] = (uint32_t)nvis;
      if (a.out_cmps) a.out_cmps[qi] = cmps;
      if (a.out_status) a.out_status[qi] = status;
    }
    __syncwarp();
  }
}

}  // namespace pann
