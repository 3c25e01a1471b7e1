// Batched form: many queries with their own k and beam in one launch sequence
// (include/parlayann_b200.h, pann_batch_*).
//
// The reference serves such a mix as a parlay::parallel_for over beam_search
// calls, each with its own QueryParams (beamSearch.h:492-526). Here the tiers
// of the exact search run once per batch: every query carries its k and beam
// (SearchArgs::qk / qL), the shared-memory state is sized for the largest, and
// the persistent first tier takes queries longest-beam first so that the long
// searches do not trail at the end. The buffers are allocated when the batch
// is created, so the device launch sequence has fixed arguments and can be
// captured once as a CUDA graph and replayed. The tier-0 seen-table size and
// warps per block, the two knobs that trade occupancy against table
// overflow, can be picked by timing them on the first batch.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "index.cuh"
#include "tiers.cuh"

struct pann_batch {
  pann_index* idx = nullptr;
  pann::SearchPlan plan{};
  uint32_t max_q = 0;
  int prec = 0;
  uint32_t rerank = 0;
  uint32_t parents = 0;
  uint32_t scorer = 0;
  uint32_t tile_rows = 0;  // tile search: rows staged per round (0 = chosen for occupancy)
  pann_batch_options bopt{};
  pann::TierSizes z{};
  // device buffers, allocated at creation
  pann::DevBuf q, qk, qL, order, ids, dists, vis, cmps, status, counters, redo, spill, handoff, gt2, ge2, starts;
  pann::DevBuf oscratch;  // keys and sort scratch of the device-side job order
  // pinned host staging for the per-query arrays (k, beam; nq in the last word)
  uint32_t* h_stage = nullptr;
  cudaEvent_t staged = nullptr;  // the last upload from h_stage has completed
  cudaStream_t cap = nullptr;    // capture stream
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int runs = 0;
};

namespace pann {

int make_plan(const pann_index* idx, const pann_query_params* qp, uint32_t n_start, SearchPlan* plan);

static int ensure_tier_buffers(pann_batch* b, const TierSizes& z) {
  PANN_CUDA(b->spill.ensure(std::max<size_t>(z.spill_bytes, 16)));
  if (b->prec == PREC_F32) PANN_CUDA(b->handoff.ensure(std::max<size_t>(z.handoff_bytes, 16)));
  PANN_CUDA(b->gt2.ensure(z.t2_bytes));
  if (b->prec == PREC_F32) PANN_CUDA(b->ge2.ensure(z.e2_bytes));
  return PANN_OK;
}

static TierBufs tier_bufs(pann_batch* b) {
  const uint32_t m = b->max_q;
  TierBufs t{};
  t.cnt = b->counters.as<uint32_t>();
  t.redo0 = b->redo.as<uint32_t>();
  t.redo1 = t.redo0 + m;
  t.emu = t.redo1 + m;
  t.ovf = t.emu + m;
  t.emu_rec = t.ovf + m;
  t.ovf_rec = t.emu_rec + m;
  t.gspill = b->spill.as<uint32_t>();
  t.handoff = b->prec == PREC_F32 ? b->handoff.as<uint32_t>() : nullptr;
  t.gt2 = b->gt2.as<uint32_t>();
  t.ge2 = b->prec == PREC_F32 ? b->ge2.as<uint32_t>() : nullptr;
  t.job_list0 = b->order.as<uint32_t>();
  t.njobs0 = b->counters.as<uint32_t>() + 32;  // outside the words every enqueue clears
  return t;
}

// The device launch sequence of one run over the batch's own buffers; the
// number of queries is read from device memory, so one capture serves every nq.
static int enqueue(pann_batch* b, const TierSizes& z, cudaStream_t st) {
  pann_index* idx = b->idx;
  SearchArgs a = base_args(idx, b->plan, b->q.as<uint8_t>(), nullptr, b->max_q, b->starts.as<uint32_t>(),
                           b->ids.as<uint32_t>(), b->dists.as<float>(), b->vis.as<uint32_t>(), b->cmps.as<uint32_t>(),
                           b->status.as<uint32_t>(), nullptr, 0);
  a.qk = b->qk.as<uint32_t>();
  a.qL = b->qL.as<uint32_t>();
  a.kstride = b->plan.k;
  // job order: longest beam first, then the queries farthest from the start point
  int orc = order_batch(idx, b->q.as<uint8_t>(), b->starts.as<uint32_t>(), b->qL.as<uint32_t>(),
                        b->counters.as<uint32_t>() + 32, b->max_q, b->oscratch.p, b->oscratch.bytes,
                        b->order.as<uint32_t>(), st);
  if (orc) return orc;
  if (b->parents > 0 && b->prec != PREC_F32) {
    a.job_list = b->order.as<uint32_t>();
    a.njobs_dev = b->counters.as<uint32_t>() + 32;
    int rc = enqueue_tile(idx, b->plan, a, b->parents, b->counters.as<uint32_t>() + 10, b->prec, b->rerank, st,
                          b->scorer, b->tile_rows);
    if (rc != PANN_EINVAL) return rc;  // EINVAL: does not fit; the single-parent tiers below
  }
  return enqueue_tiers(idx, b->plan, a, z, tier_bufs(b), st, b->prec, b->rerank);
}

// Picks how the batch maps onto the GPU by timing each candidate on the
// staged batch (three runs each, the first warming the caches, the faster of
// the other two counts). Every candidate gives the same answers:
//  * exact search, warp per query: the first tier's seen-table slots
//    ({1/2, 1, 2} x the estimate), warps per block ({2, 4}) and register
//    budget (fitted to 3 or 4 resident blocks);
//  * exact search, CTA per query: every query on one block of the
//    exact-emulation kernel (when its tables fit in shared memory);
//  * tile search (precision form, parents > 0): the rows staged and scored per
//    round (the tile's height: all the step's candidates, 3/4, 1/2 or 1/4).
static int autotune(pann_batch* b, cudaStream_t st) {
  struct Cand {
    TierSizes z;
    uint32_t tile_rows;
  };
  std::vector<Cand> cands;
  const bool tile = b->parents > 0 && b->prec != PREC_F32;
  if (tile) {
    const uint32_t cw = std::max<uint32_t>(1, std::min<uint32_t>(b->parents, 4)) * std::min(b->plan.dl, b->idx->R);
    for (uint32_t f : {4u, 3u, 2u, 1u}) cands.push_back({b->z, std::max<uint32_t>(16, cw * f / 4)});
  } else {
    const uint32_t base_S = b->z.S;
    const uint32_t floor_S = 4 * (b->idx->R + 1);
    for (uint32_t S : {base_S / 2, base_S, base_S * 2})
      for (int w : {2, 4})
        for (int minb : {3, 4}) {
          if (S < floor_S || S > 16384) continue;
          if (minb == 4 && b->prec != PREC_F32) continue;
          TierSizes z;
          if (size_tiers(b->idx, b->plan, b->max_q, b->prec, S, w, &z, minb) != PANN_OK) continue;
          if (z.S != S || z.wpb != w) continue;  // did not fit as asked
          cands.push_back({z, 0});
        }
    if (b->prec == PREC_F32 && b->z.emu_smem) {
      TierSizes z = b->z;
      z.cta = true;
      cands.push_back({z, 0});
    }
  }
  cudaEvent_t e0, e1;
  PANN_CUDA(cudaEventCreate(&e0));
  PANN_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  Cand best_c{b->z, b->tile_rows};
  int rc = PANN_OK;
  for (auto& c : cands) {
    if ((rc = ensure_tier_buffers(b, c.z)) != PANN_OK) break;
    b->tile_rows = c.tile_rows;
    float t_min = 1e30f;
    for (int rep = 0; rep < 3 && rc == PANN_OK; rep++) {
      cudaEventRecord(e0, st);
      rc = enqueue(b, c.z, st);
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "autotune run");
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) t_min = std::min(t_min, ms);  // the first run warms the caches
    }
    if (rc) break;
    if (t_min < best) {
      best = t_min;
      best_c = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  b->z = best_c.z;
  b->tile_rows = best_c.tile_rows;
  return PANN_OK;
}

// ---------------------------------------------------------------------------
// Batches laid out in an arena (index.cuh: batch_scratch_bytes, run_in_arena).

namespace {

struct ArenaLayout {
  SearchPlan plan;
  TierSizes z;
  size_t cnt, starts, q, qk, qL, order, okeys, okeys_bytes, ids, dists, vis, cmps, status, redo, spill, handoff, gt2,
      ge2, bytes;
};

size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

int arena_layout(const pann_index* idx, const pann_query_params* bounds, uint32_t n_start, uint32_t nq, int prec,
                 ArenaLayout* y) {
  int rc = make_plan(idx, bounds, n_start, &y->plan);
  if (rc) return rc;
  // any query may defer candidates (its own beam is at most the bound)
  y->plan.Ccap = (uint32_t)std::floor(y->plan.bf * (double)y->plan.L) + std::min(y->plan.dl, idx->R) + 1;
  rc = size_tiers(idx, y->plan, nq, prec, 0, 0, &y->z);
  if (rc) return rc;
  // batches that overlap on the device: the emulation tier keeps its tables in
  // global memory (the shared-memory tier's blocks each need a whole SM and
  // would wait for the other batches' blocks to leave one)
  y->z.emu_smem = false;
  const size_t k = y->plan.k;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o += a256(std::max<size_t>(bytes, 16));
    return at;
  };
  y->cnt = take(4 * 64);
  y->starts = take(4ull * std::max<uint32_t>(n_start, 1));
  y->q = take(idx->stride * (size_t)nq);
  y->qk = take(4ull * nq);
  y->qL = take(4ull * nq);
  y->order = take(4ull * nq);
  y->okeys_bytes = batch_order_scratch_bytes(nq);
  y->okeys = take(y->okeys_bytes);
  y->ids = take(4ull * nq * k);
  y->dists = take(4ull * nq * k);
  y->vis = take(4ull * nq);
  y->cmps = take(4ull * nq);
  y->status = take(4ull * nq);
  y->redo = take(4ull * 6 * nq);
  y->spill = take(y->z.spill_bytes);
  y->handoff = prec == PREC_F32 ? take(y->z.handoff_bytes) : o;
  y->gt2 = take(y->z.t2_bytes);
  y->ge2 = prec == PREC_F32 ? take(y->z.e2_bytes) : o;
  y->bytes = o;
  return PANN_OK;
}

}  // namespace

int batch_scratch_bytes(const pann_index* idx, const pann_query_params* bounds, uint32_t n_start, uint32_t nq,
                        int precision, uint32_t parents, size_t* bytes) {
  (void)parents;  // the tile search needs no scratch beyond the single-parent tiers' own
  ArenaLayout y;
  int rc = arena_layout(idx, bounds, n_start, std::max<uint32_t>(nq, 1), precision, &y);
  if (rc) return rc;
  *bytes = y.bytes;
  return PANN_OK;
}

int run_in_arena(pann_index* idx, uint8_t* arena, size_t arena_bytes, const pann_query_params* bounds,
                 const uint32_t* h_starts, uint32_t n_start, const uint8_t* h_queries, uint32_t nq, const uint32_t* h_k,
                 const uint32_t* h_beam, const uint32_t* h_order, int precision, uint32_t rerank, uint32_t parents,
                 uint32_t scorer, uint32_t* h_ids, float* h_dists, cudaStream_t st) {
  if (nq == 0) return PANN_OK;
  ArenaLayout y;
  int rc = arena_layout(idx, bounds, n_start, nq, precision, &y);
  if (rc) return rc;
  if (y.bytes > arena_bytes)
    return fail(PANN_EINVAL, "batch needs " + std::to_string(y.bytes) + " bytes of scratch; the arena holds " +
                                 std::to_string(arena_bytes));
  auto at = [&](size_t off) { return arena + off; };
  uint32_t* cnt = reinterpret_cast<uint32_t*>(at(y.cnt));
  const size_t rb = (size_t)idx->d * idx->esize;
  // the job count comes from the pinned order array's tail word, so every copy is from pinned memory
  PANN_CUDA(cudaMemsetAsync(cnt, 0, 4 * 64, st));
  PANN_CUDA(cudaMemcpyAsync(at(y.starts), h_starts, 4ull * n_start, cudaMemcpyHostToDevice, st));
  if (rb != idx->stride) PANN_CUDA(cudaMemsetAsync(at(y.q), 0, idx->stride * (size_t)nq, st));
  PANN_CUDA(cudaMemcpy2DAsync(at(y.q), idx->stride, h_queries, rb, rb, nq, cudaMemcpyHostToDevice, st));
  PANN_CUDA(cudaMemcpyAsync(at(y.qk), h_k, 4ull * nq, cudaMemcpyHostToDevice, st));
  PANN_CUDA(cudaMemcpyAsync(at(y.qL), h_beam, 4ull * nq, cudaMemcpyHostToDevice, st));
  PANN_CUDA(cudaMemcpyAsync(cnt + 32, h_order + nq, 4, cudaMemcpyHostToDevice, st));
  // job order on the device: longest beam first, then farthest from the start point
  rc = order_batch(idx, at(y.q), reinterpret_cast<const uint32_t*>(at(y.starts)),
                   reinterpret_cast<const uint32_t*>(at(y.qL)), cnt + 32, nq, at(y.okeys), y.okeys_bytes,
                   reinterpret_cast<uint32_t*>(at(y.order)), st);
  if (rc) return rc;
  SearchArgs a = base_args(idx, y.plan, at(y.q), nullptr, nq, reinterpret_cast<const uint32_t*>(at(y.starts)),
                           reinterpret_cast<uint32_t*>(at(y.ids)), reinterpret_cast<float*>(at(y.dists)),
                           reinterpret_cast<uint32_t*>(at(y.vis)), reinterpret_cast<uint32_t*>(at(y.cmps)),
                           reinterpret_cast<uint32_t*>(at(y.status)), nullptr, 0);
  a.qk = reinterpret_cast<const uint32_t*>(at(y.qk));
  a.qL = reinterpret_cast<const uint32_t*>(at(y.qL));
  a.kstride = y.plan.k;
  rc = PANN_EINVAL;
  if (parents > 0 && precision != PREC_F32) {
    a.job_list = reinterpret_cast<const uint32_t*>(at(y.order));
    a.njobs_dev = cnt + 32;
    rc = enqueue_tile(idx, y.plan, a, parents, cnt + 10, precision, rerank, st, scorer);
    if (rc != PANN_OK && rc != PANN_EINVAL) return rc;
  }
  if (rc == PANN_EINVAL) {
    TierBufs t{};
    t.cnt = cnt;
    t.redo0 = reinterpret_cast<uint32_t*>(at(y.redo));
    t.redo1 = t.redo0 + nq;
    t.emu = t.redo1 + nq;
    t.ovf = t.emu + nq;
    t.emu_rec = t.ovf + nq;
    t.ovf_rec = t.emu_rec + nq;
    t.gspill = reinterpret_cast<uint32_t*>(at(y.spill));
    t.handoff = precision == PREC_F32 ? reinterpret_cast<uint32_t*>(at(y.handoff)) : nullptr;
    t.gt2 = reinterpret_cast<uint32_t*>(at(y.gt2));
    t.ge2 = precision == PREC_F32 ? reinterpret_cast<uint32_t*>(at(y.ge2)) : nullptr;
    t.job_list0 = reinterpret_cast<const uint32_t*>(at(y.order));
    t.njobs0 = cnt + 32;
    rc = enqueue_tiers(idx, y.plan, a, y.z, t, st, precision, rerank);
    if (rc) return rc;
  }
  const size_t kb = 4ull * y.plan.k * nq;
  PANN_CUDA(cudaMemcpyAsync(h_ids, at(y.ids), kb, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(h_dists, at(y.dists), kb, cudaMemcpyDeviceToHost, st));
  return PANN_OK;
}

}  // namespace pann

using namespace pann;

extern "C" {

int pann_batch_create(pann_batch** out, pann_index* idx, uint32_t max_queries, const pann_query_params* bounds,
                      const uint32_t* starts, uint32_t n_start, const pann_search_options* opt,
                      const pann_batch_options* bopt) {
  if (!out) return fail(PANN_EINVAL, "out is NULL");
  *out = nullptr;
  if (!idx || !idx->points_set) return fail(PANN_EINVAL, "index has no points (pann_index_set_points)");
  if (max_queries == 0) return fail(PANN_EINVAL, "max_queries must be positive");
  if (!starts) return fail(PANN_EINVAL, "start points are NULL");
  for (uint32_t i = 0; i < n_start; i++) {
    if ((uint64_t)starts[i] >= idx->n) return fail(PANN_EINVAL, "start point id out of range");
    for (uint32_t j = 0; j < i; j++)
      if (starts[j] == starts[i]) return fail(PANN_EINVAL, "duplicate start point");
  }
  SearchPlan plan;
  int rc = make_plan(idx, bounds, n_start, &plan);
  if (rc) return rc;
  if (plan.k == 0) return fail(PANN_EINVAL, "bounds->k must be positive");
  // any query may defer candidates (its own beam is at most the bound)
  plan.Ccap = (uint32_t)std::floor(plan.bf * (double)plan.L) + std::min(plan.dl, idx->R) + 1;
  const int prec = opt ? opt->precision : PANN_PREC_F32;
  if (prec != PANN_PREC_F32 && idx->lp_prec != prec)
    return fail(PANN_EINVAL, "call pann_index_set_precision for this precision first");

  pann_batch* b = new pann_batch();
  b->idx = idx;
  b->plan = plan;
  b->max_q = max_queries;
  b->prec = prec;
  b->rerank = opt ? opt->rerank : 0;
  b->parents = opt ? opt->parents : 0;
  b->scorer = opt ? opt->scorer : 0;
  if (bopt) b->bopt = *bopt;
  auto bail = [&](int code) {
    pann_batch_destroy(b);
    return code;
  };
  rc = size_tiers(idx, plan, max_queries, prec, b->bopt.seen_slots, (int)b->bopt.warps_per_block, &b->z);
  if (rc) return bail(rc);
  if (b->bopt.cta_per_query) {
    if (prec != PANN_PREC_F32 || !b->z.emu_smem)
      return bail(fail(PANN_EINVAL, "CTA per query needs the exact search and emulated tables that fit in shared "
                                    "memory at this beam"));
    b->z.cta = true;
  }
  const size_t m = max_queries;
  cudaError_t e = cudaSuccess;
  auto need = [&](DevBuf& d, size_t bytes) {
    if (e == cudaSuccess) e = d.ensure(std::max<size_t>(bytes, 16));
  };
  need(b->q, idx->stride * m);
  need(b->qk, 4 * m);
  need(b->qL, 4 * m);
  need(b->order, 4 * m);
  need(b->oscratch, batch_order_scratch_bytes((uint32_t)m));
  need(b->ids, 4 * m * plan.k);
  need(b->dists, 4 * m * plan.k);
  need(b->vis, 4 * m);
  need(b->cmps, 4 * m);
  need(b->status, 4 * m);
  need(b->counters, 4 * 64);
  need(b->redo, 4 * 6 * m);
  need(b->starts, 4ull * std::max<uint32_t>(n_start, 1));
  if (e != cudaSuccess) return bail(cuda_fail(e, "batch buffers"));
  if ((rc = ensure_tier_buffers(b, b->z)) != PANN_OK) return bail(rc);
  e = cudaMallocHost(&b->h_stage, 4 * (3 * m + 1));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMemcpy(b->starts.p, starts, 4ull * n_start, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->q.p, 0, idx->stride * m);  // zero row padding once
  if (e != cudaSuccess) return bail(cuda_fail(e, "batch setup"));
  *out = b;
  return PANN_OK;
}

int pann_batch_run(pann_batch* b, const void* queries, uint32_t nq, const uint32_t* k, const uint32_t* beam,
                   uint32_t* out_ids, float* out_dists, uint32_t* out_visited, uint32_t* out_cmps,
                   uint32_t* out_flags, int on_device, void* stream) {
  if (!b) return fail(PANN_EINVAL, "batch is NULL");
  if (nq > b->max_q) return fail(PANN_EINVAL, "nq = " + std::to_string(nq) + " exceeds the batch's max_queries = " +
                                                  std::to_string(b->max_q));
  if (nq == 0) return PANN_OK;
  if (!queries || !out_ids || !k || !beam) return fail(PANN_EINVAL, "queries, out_ids, k or beam is NULL");
  const SearchPlan& p = b->plan;
  for (uint32_t i = 0; i < nq; i++) {
    if (k[i] == 0 || k[i] > p.k) return fail(PANN_EINVAL, "query " + std::to_string(i) + ": k must be in [1, bounds->k]");
    if (beam[i] < k[i])
      return fail(PANN_EINVAL, "query " + std::to_string(i) + ": beam search parameter Q = " + std::to_string(beam[i]) +
                                   " same size or smaller than k = " + std::to_string(k[i]));
    if (beam[i] > p.L) return fail(PANN_EINVAL, "query " + std::to_string(i) + ": beam exceeds bounds->beam");
    if (beam[i] < p.n_start)
      return fail(PANN_EINVAL, "query " + std::to_string(i) + ": beam search has more starting points than beam size");
  }
  pann_index* idx = b->idx;
  cudaStream_t st = on_device ? static_cast<cudaStream_t>(stream) : idx->stream;
  // stage k, beam and nq (the job order is made on the device by the launch sequence)
  PANN_CUDA(cudaEventSynchronize(b->staged));  // the previous run's upload is done with h_stage
  uint32_t* hk = b->h_stage;
  uint32_t* hL = hk + b->max_q;
  uint32_t* hn = hL + 2 * b->max_q;
  std::memcpy(hk, k, 4ull * nq);
  std::memcpy(hL, beam, 4ull * nq);
  *hn = nq;
  const size_t rb = (size_t)idx->d * idx->esize;
  PANN_CUDA(cudaMemcpy2DAsync(b->q.p, idx->stride, queries, rb, rb, nq,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  PANN_CUDA(cudaMemcpyAsync(b->qk.p, hk, 4ull * nq, cudaMemcpyHostToDevice, st));
  PANN_CUDA(cudaMemcpyAsync(b->qL.p, hL, 4ull * nq, cudaMemcpyHostToDevice, st));
  PANN_CUDA(cudaMemcpyAsync(b->counters.as<uint32_t>() + 32, hn, 4, cudaMemcpyHostToDevice, st));
  PANN_CUDA(cudaEventRecord(b->staged, st));

  int rc = PANN_OK;
  if (b->runs == 0 && b->bopt.autotune && !b->bopt.seen_slots && !b->bopt.warps_per_block && !b->bopt.cta_per_query) {
    rc = autotune(b, st);
    if (rc) return rc;
  }
  if (b->exec) {
    PANN_CUDA(cudaGraphLaunch(b->exec, st));
  } else {
    rc = enqueue(b, b->z, st);
    if (rc) return rc;
    if (b->bopt.use_graph) {
      // capture after an eager run, so every kernel is already loaded
      PANN_CUDA(cudaStreamSynchronize(st));
      PANN_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
      rc = enqueue(b, b->z, b->cap);
      cudaGraph_t g = nullptr;
      cudaError_t ce = cudaStreamEndCapture(b->cap, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
      ce = cudaGraphInstantiate(&b->exec, g, 0);
      if (ce != cudaSuccess) {
        cudaGraphDestroy(g);
        b->exec = nullptr;
        return cuda_fail(ce, "cudaGraphInstantiate");
      }
      b->graph = g;
    }
  }
  b->runs++;
  // results out of the batch's buffers
  const size_t kb = 4ull * p.k * nq;
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  PANN_CUDA(cudaMemcpyAsync(out_ids, b->ids.p, kb, kind, st));
  if (out_dists) PANN_CUDA(cudaMemcpyAsync(out_dists, b->dists.p, kb, kind, st));
  if (out_visited) PANN_CUDA(cudaMemcpyAsync(out_visited, b->vis.p, 4ull * nq, kind, st));
  if (out_cmps) PANN_CUDA(cudaMemcpyAsync(out_cmps, b->cmps.p, 4ull * nq, kind, st));
  if (on_device) {
    if (out_flags) PANN_CUDA(cudaMemcpyAsync(out_flags, b->status.p, 4ull * nq, kind, st));
    return PANN_OK;
  }
  std::vector<uint32_t> status(nq);
  PANN_CUDA(cudaMemcpyAsync(status.data(), b->status.p, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  int rc2 = PANN_OK;
  for (uint32_t i = 0; i < nq; i++) {
    uint32_t s = status[i];
    if (out_flags) out_flags[i] = ((s & QS_REF_WOULD_GROW) ? 1u : 0u) | ((s & 32u) ? 2u : 0u);
    if (s & (QS_TABLE_FULL | QS_INTERNAL)) rc2 = PANN_EOVERFLOW;
    else if ((s & QS_SHORT) && rc2 == PANN_OK) rc2 = PANN_ESHORT;
  }
  if (rc2 == PANN_EOVERFLOW) return fail(rc2, "a query's seen-set outgrew the largest table");
  if (rc2 == PANN_ESHORT) return fail(rc2, "beam search returned fewer than k results");
  return PANN_OK;
}

int pann_batch_config(const pann_batch* b, uint32_t* seen_slots, uint32_t* warps_per_block, uint32_t* blocks,
                      int32_t* graph_captured) {
  if (!b) return fail(PANN_EINVAL, "batch is NULL");
  if (seen_slots) *seen_slots = b->z.S;
  if (warps_per_block) *warps_per_block = (uint32_t)b->z.wpb;
  if (blocks) *blocks = (uint32_t)b->z.blocks;
  if (graph_captured) *graph_captured = b->exec != nullptr;
  return PANN_OK;
}

int pann_batch_mapping(const pann_batch* b, uint32_t* cta_per_query, uint32_t* register_blocks, uint32_t* tile_rows) {
  if (!b) return fail(PANN_EINVAL, "batch is NULL");
  if (cta_per_query) *cta_per_query = b->z.cta ? 1u : 0u;
  if (register_blocks) *register_blocks = (uint32_t)b->z.minb;
  if (tile_rows) *tile_rows = b->tile_rows;
  return PANN_OK;
}

int pann_batch_destroy(pann_batch* b) {
  if (!b) return PANN_OK;
  // the index may already be gone: touch only the batch's own objects
  if (b->cap) cudaStreamSynchronize(b->cap);
  if (b->staged) cudaEventSynchronize(b->staged);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (DevBuf* d : {&b->q, &b->qk, &b->qL, &b->order, &b->oscratch, &b->ids, &b->dists, &b->vis, &b->cmps, &b->status, &b->counters,
                    &b->redo, &b->spill, &b->handoff, &b->gt2, &b->ge2, &b->starts})
    d->release();
  if (b->h_stage) cudaFreeHost(b->h_stage);
  if (b->staged) cudaEventDestroy(b->staged);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
  return PANN_OK;
}

}  // extern "C"
