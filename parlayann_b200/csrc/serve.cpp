// Serving form (include/parlayann_b200.h, pann_server_*): a request loop over
// one resident index with continuous batching and admission by scratch memory.
//
// The reference answers queries in closed batches (qsearchAll,
// beamSearch.h:599-646; RangeSearch, rangeSearch.h:183-276); it has no request
// loop. Here requests arrive one by one from any thread. A dispatcher thread
// owns `inflight` slots, each a device arena of scratch_bytes with its own
// stream and pinned host buffers. Whenever a slot is free it takes the waiting
// k-NN requests in arrival order while the batch they form still fits the
// arena: the bytes a batch needs (its queries, outputs, per-query work lists,
// the per-warp seen tables and hand-off logs of the first tier, the hand-off
// records of the queries that may need them, the later tiers' tables) follow
// from its query count and its largest k and beam (batch_scratch_bytes), so
// small-k, short-beam requests pack many more queries into a slot than
// k = 100, beam = 200 ones. The batch is laid out in the arena and run
// (run_in_arena); requests that arrive while other batches are on the GPU go
// into the next free slot, so batches overlap on the device. Finished slots
// are retired by polling their events; each request's latency runs from its
// submission to the moment its results are in host memory. Range requests run
// on a second worker through pann_range_search, concurrently with the k-NN
// batches. Results of a request are the same as that request run alone (same
// kernels, per-query parameters).
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "index.cuh"

namespace {

using clk = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  int kind = 0;  // 0 = k-NN, 1 = range
  uint32_t nq = 0, k = 0, beam = 0;
  std::vector<uint8_t> queries;
  pann_range_params rp{};
  uint32_t start = 0;
  // results
  std::vector<uint32_t> ids;
  std::vector<float> dists;
  std::vector<uint64_t> offsets;
  int rc = PANN_OK;
  std::string err;
  bool done = false;
  clk::time_point t_submit, t_done;
};

struct Slot {
  uint8_t* arena = nullptr;  // device scratch of one batch
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  uint8_t* h_q = nullptr;  // pinned: queries, per-query k / beam / job order, results
  uint32_t* h_k = nullptr;
  uint32_t* h_L = nullptr;
  uint32_t* h_order = nullptr;  // word nq: the job count (pinned, copied with the batch)
  uint32_t* h_ids = nullptr;
  float* h_d = nullptr;
  std::vector<Request*> reqs;
  uint32_t nq = 0, kmax = 0;
  bool busy = false;
};

}  // namespace

struct pann_server {
  pann_index* idx = nullptr;
  pann_server_options opt{};
  size_t row_bytes = 0;
  std::vector<uint32_t> starts;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> knn_q, range_q;
  std::unordered_map<uint64_t, Request*> reqs;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::thread dispatcher, ranger;
  int device = 0;
  // statistics since the last reset
  std::vector<double> lat;
  uint64_t done_queries = 0;
  clk::time_point stats_t0;
  std::string fatal;
  // admission
  size_t scratch = 0;  // bytes of each slot's arena
  uint64_t batches = 0, batched_queries = 0;
  size_t scratch_peak = 0;
};

namespace {

void finish(pann_server* s, Request* r, int rc, const std::string& err) {
  r->rc = rc;
  r->err = err;
  r->t_done = clk::now();
  r->done = true;
  s->lat.push_back(std::chrono::duration<double>(r->t_done - r->t_submit).count());
  s->done_queries += r->nq;
}

// Copies a finished slot's results into its requests (called with s->mu held).
void retire(pann_server* s, Slot& sl) {
  uint32_t off = 0;
  const uint32_t K = sl.kmax;  // the batch's output rows hold its largest k
  for (Request* r : sl.reqs) {
    r->ids.resize((size_t)r->nq * r->k);
    r->dists.resize((size_t)r->nq * r->k);
    for (uint32_t i = 0; i < r->nq; i++) {
      std::memcpy(&r->ids[(size_t)i * r->k], sl.h_ids + (size_t)(off + i) * K, 4ull * r->k);
      std::memcpy(&r->dists[(size_t)i * r->k], sl.h_d + (size_t)(off + i) * K, 4ull * r->k);
    }
    off += r->nq;
    finish(s, r, PANN_OK, "");
  }
  sl.reqs.clear();
  sl.busy = false;
}

// Bytes a batch of nq queries with largest k and beam needs in an arena.
size_t batch_bytes(const pann_server* s, uint32_t nq, uint32_t kmax, uint32_t Lmax) {
  pann_query_params b{kmax, Lmax, s->opt.limit, s->opt.degree_limit, s->opt.batch_factor};
  size_t bytes = 0;
  if (pann::batch_scratch_bytes(s->idx, &b, (uint32_t)s->starts.size(), nq, s->opt.precision, s->opt.parents,
                                &bytes) != PANN_OK)
    return SIZE_MAX;
  return bytes;
}

// Launches the waiting k-NN requests that fit into a free slot (s->mu held on
// entry; released during the launch). Requests are taken in arrival order
// while the batch stays within max_batch_queries and its scratch within the
// slot's arena (see below for the beam rule). Returns true if something was
// launched.
bool launch(pann_server* s, Slot& sl, std::unique_lock<std::mutex>& lk) {
  if (s->knn_q.empty()) return false;
  uint32_t nq = 0, kmax = 0, Lmax = 0;
  size_t used = 0;
  // The oldest request always goes in; later ones join while the batch fits,
  // taken in arrival order among those whose beam is within 5/4 of the oldest
  // one's (a batch's shared-memory state is sized for its largest beam, so a
  // long-beam request would slow every short-beam query beside it); the
  // requests passed over keep their place and lead the next batch.
  const uint32_t beam0 = s->knn_q.front()->beam;
  size_t scanned = 0;
  for (auto it = s->knn_q.begin(); it != s->knn_q.end() && scanned < 512; scanned++) {
    const Request* r = *it;
    if (!sl.reqs.empty() && 4ull * r->beam > 5ull * beam0) {
      ++it;
      continue;
    }
    const uint32_t n2 = nq + r->nq, k2 = std::max(kmax, r->k), L2 = std::max(Lmax, r->beam);
    if (n2 > s->opt.max_batch_queries) break;
    const size_t need = batch_bytes(s, n2, k2, L2);
    if (need > s->scratch) break;
    it = s->knn_q.erase(it);
    sl.reqs.push_back(const_cast<Request*>(r));
    nq = n2;
    kmax = k2;
    Lmax = L2;
    used = need;
  }
  if (sl.reqs.empty()) return false;
  sl.busy = true;
  sl.nq = nq;
  sl.kmax = kmax;
  s->batches++;
  s->batched_queries += nq;
  s->scratch_peak = std::max(s->scratch_peak, used);
  lk.unlock();
  uint32_t at = 0;
  for (Request* r : sl.reqs) {
    std::memcpy(sl.h_q + (size_t)at * s->row_bytes, r->queries.data(), (size_t)r->nq * s->row_bytes);
    for (uint32_t i = 0; i < r->nq; i++) {
      sl.h_k[at + i] = r->k;
      sl.h_L[at + i] = r->beam;
    }
    at += r->nq;
  }
  // the job count (the job order, longest beam first, is made on the device)
  sl.h_order[nq] = nq;
  pann_query_params bounds{kmax, Lmax, s->opt.limit, s->opt.degree_limit, s->opt.batch_factor};
  int rc = pann::run_in_arena(s->idx, sl.arena, s->scratch, &bounds, s->starts.data(), (uint32_t)s->starts.size(),
                              sl.h_q, nq, sl.h_k, sl.h_L, sl.h_order, s->opt.precision, 0, s->opt.parents,
                              s->opt.scorer, sl.h_ids, sl.h_d, sl.st);
  cudaError_t e = cudaSuccess;
  if (rc == PANN_OK) e = cudaEventRecord(sl.done, sl.st);
  lk.lock();
  if (e != cudaSuccess || rc != PANN_OK) {
    std::string msg = e != cudaSuccess ? std::string("CUDA error: ") + cudaGetErrorString(e) : pann_last_error();
    cudaStreamSynchronize(sl.st);
    for (Request* r : sl.reqs) finish(s, r, rc != PANN_OK ? rc : PANN_EDEVICE, msg);
    sl.reqs.clear();
    sl.busy = false;
    s->cv_done.notify_all();
  }
  return true;
}

void dispatcher_main(pann_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    bool progress = false;
    // retire finished batches
    for (Slot& sl : s->slots) {
      if (sl.busy && !sl.reqs.empty() && cudaEventQuery(sl.done) == cudaSuccess) {
        retire(s, sl);
        progress = true;
      }
    }
    if (progress) s->cv_done.notify_all();
    // fill free slots
    for (Slot& sl : s->slots)
      if (!sl.busy && launch(s, sl, lk)) progress = true;
    bool any_busy = false;
    for (Slot& sl : s->slots) any_busy |= sl.busy;
    if (s->stop && !any_busy && s->knn_q.empty()) break;
    if (!progress) {
      // batches on the device: poll their events at a short interval; idle:
      // sleep until a request arrives
      if (any_busy) s->cv_work.wait_for(lk, std::chrono::microseconds(20));
      else s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
    }
  }
}

void ranger_main(pann_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    if (s->range_q.empty()) {
      if (s->stop) break;
      s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
      continue;
    }
    // the waiting range requests with the same parameters, up to 16 queries,
    // as one search (the answers of a group stay within the reserved pool)
    std::vector<Request*> group;
    uint32_t gq = 0;
    for (auto it = s->range_q.begin(); it != s->range_q.end();) {
      Request* r = *it;
      const Request* f = group.empty() ? r : group.front();
      if (group.empty() || (gq + r->nq <= 16 && r->start == f->start &&
                            std::memcmp(&r->rp, &f->rp, sizeof(pann_range_params)) == 0)) {
        gq += r->nq;
        group.push_back(r);
        it = s->range_q.erase(it);
      } else {
        ++it;
      }
    }
    lk.unlock();
    uint32_t nq = 0;
    for (Request* r : group) nq += r->nq;
    std::vector<uint8_t> qs((size_t)nq * s->row_bytes);
    {
      size_t at = 0;
      for (Request* r : group) {
        std::memcpy(qs.data() + at, r->queries.data(), r->queries.size());
        at += r->queries.size();
      }
    }
    const Request* f = group.front();
    std::vector<uint64_t> offs((size_t)nq + 1, 0);
    std::vector<uint32_t> ids((size_t)nq * f->rp.beam * 4 + 16);
    int rc = pann_range_search(s->idx, qs.data(), nq, &f->rp, f->start, offs.data(), ids.data(), ids.size(), nullptr,
                               nullptr, nullptr);
    if (rc == PANN_EOVERFLOW && offs[nq] > ids.size()) {
      ids.resize(offs[nq]);
      rc = pann_range_fetch(s->idx, ids.data(), ids.size());
    }
    std::string msg = rc ? pann_last_error() : "";
    lk.lock();
    uint32_t q0 = 0;
    for (Request* r : group) {
      if (rc == PANN_OK) {
        r->offsets.resize((size_t)r->nq + 1);
        for (uint32_t i = 0; i <= r->nq; i++) r->offsets[i] = offs[q0 + i] - offs[q0];
        r->ids.assign(ids.begin() + (ptrdiff_t)offs[q0], ids.begin() + (ptrdiff_t)offs[q0 + r->nq]);
      }
      q0 += r->nq;
      finish(s, r, rc, msg);
    }
    s->cv_done.notify_all();
  }
}

int submit(pann_server* s, Request* r, uint64_t* ticket) {
  r->t_submit = clk::now();
  std::lock_guard<std::mutex> g(s->mu);
  if (s->stop) {
    delete r;
    return pann::fail(PANN_EINVAL, "server is stopping");
  }
  r->ticket = s->next_ticket++;
  s->reqs[r->ticket] = r;
  (r->kind == 0 ? s->knn_q : s->range_q).push_back(r);
  *ticket = r->ticket;
  s->cv_work.notify_all();
  return PANN_OK;
}

// Waits for a ticket and removes it (s->mu not held on entry).
Request* take(pann_server* s, uint64_t ticket, int* rc) {
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) {
    *rc = pann::fail(PANN_EINVAL, "unknown ticket");
    return nullptr;
  }
  Request* r = it->second;
  s->cv_done.wait(lk, [&] { return r->done; });
  s->reqs.erase(it);
  *rc = PANN_OK;
  return r;
}

double quantile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  size_t i = (size_t)std::min<double>((double)v.size() - 1, std::floor(q * (double)(v.size() - 1) + 0.5));
  return v[i];
}

}  // namespace

extern "C" {

int pann_server_create(pann_server** out, pann_index* idx, const pann_server_options* opt, const uint32_t* starts,
                       uint32_t n_start) {
  if (!out || !idx || !opt || !starts) return pann::fail(PANN_EINVAL, "NULL argument");
  if (!idx->points_set) return pann::fail(PANN_EINVAL, "index has no points (pann_index_set_points)");
  *out = nullptr;
  if (opt->max_batch_queries == 0 || opt->inflight == 0 || opt->inflight > 16)
    return pann::fail(PANN_EINVAL, "max_batch_queries must be positive and inflight in [1, 16]");
  pann_server* s = new pann_server();
  s->idx = idx;
  s->opt = *opt;
  s->starts.assign(starts, starts + n_start);
  cudaGetDevice(&s->device);
  if (opt->precision != PANN_PREC_F32 && idx->lp_prec != opt->precision) {
    delete s;
    return pann::fail(PANN_EINVAL, "call pann_index_set_precision for this precision first");
  }
  s->row_bytes = (size_t)idx->d * idx->esize;
  // the arena: the option, or what a full batch at the bounds needs
  s->scratch = opt->scratch_bytes ? (size_t)opt->scratch_bytes
                                  : batch_bytes(s, opt->max_batch_queries, opt->max_k, opt->max_beam);
  if (s->scratch == SIZE_MAX || batch_bytes(s, 1, opt->max_k, opt->max_beam) > s->scratch) {
    const size_t one = batch_bytes(s, 1, opt->max_k, opt->max_beam);
    delete s;
    return pann::fail(PANN_EINVAL, "scratch_bytes is below the " + std::to_string(one) +
                                       " bytes one query at max_k and max_beam needs");
  }
  s->slots.resize(opt->inflight);
  auto bail = [&](int rc) {
    pann_server_destroy(s);
    return rc;
  };
  for (Slot& sl : s->slots) {
    const size_t m = opt->max_batch_queries;
    cudaError_t e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&sl.arena, s->scratch);
    if (e == cudaSuccess) e = cudaMallocHost(&sl.h_q, m * s->row_bytes);
    if (e == cudaSuccess) e = cudaMallocHost(&sl.h_k, 4 * m);
    if (e == cudaSuccess) e = cudaMallocHost(&sl.h_L, 4 * m);
    if (e == cudaSuccess) e = cudaMallocHost(&sl.h_order, 4 * (m + 1));
    if (e == cudaSuccess) e = cudaMallocHost(&sl.h_ids, 4 * m * opt->max_k);
    if (e == cudaSuccess) e = cudaMallocHost(&sl.h_d, 4 * m * opt->max_k);
    if (e != cudaSuccess) return bail(pann::cuda_fail(e, "server slot"));
  }
  // range search's scratch taken now, not while k-NN batches run
  if (pann::range_reserve(idx) != PANN_OK) cudaGetLastError();  // without it range search allocates as it goes
  s->stats_t0 = clk::now();
  s->dispatcher = std::thread(dispatcher_main, s);
  s->ranger = std::thread(ranger_main, s);
  *out = s;
  return PANN_OK;
}

int pann_server_submit_knn(pann_server* s, const void* queries, uint32_t nq, uint32_t k, uint32_t beam,
                           uint64_t* ticket) {
  if (!s || !queries || !ticket) return pann::fail(PANN_EINVAL, "NULL argument");
  if (nq == 0 || nq > s->opt.max_batch_queries)
    return pann::fail(PANN_EINVAL, "a request needs 1 to max_batch_queries queries");
  if (k == 0 || k > s->opt.max_k || beam < k || beam > s->opt.max_beam || beam < s->starts.size())
    return pann::fail(PANN_EINVAL, "k / beam outside the server's bounds (1 <= k <= beam <= max_beam, k <= max_k)");
  const size_t need = batch_bytes(s, nq, k, beam);
  if (need > s->scratch)
    return pann::fail(PANN_EINVAL, "the request needs " + std::to_string(need) + " bytes of scratch; a slot holds " +
                                       std::to_string(s->scratch) + " (split it)");
  Request* r = new Request();
  r->kind = 0;
  r->nq = nq;
  r->k = k;
  r->beam = beam;
  r->queries.assign(static_cast<const uint8_t*>(queries), static_cast<const uint8_t*>(queries) + (size_t)nq * s->row_bytes);
  return submit(s, r, ticket);
}

int pann_server_submit_range(pann_server* s, const void* queries, uint32_t nq, const pann_range_params* rp,
                             uint32_t start_point, uint64_t* ticket) {
  if (!s || !queries || !rp || !ticket) return pann::fail(PANN_EINVAL, "NULL argument");
  if (nq == 0) return pann::fail(PANN_EINVAL, "a request needs at least one query");
  Request* r = new Request();
  r->kind = 1;
  r->nq = nq;
  r->rp = *rp;
  r->start = start_point;
  r->queries.assign(static_cast<const uint8_t*>(queries), static_cast<const uint8_t*>(queries) + (size_t)nq * s->row_bytes);
  return submit(s, r, ticket);
}

int pann_server_wait_knn(pann_server* s, uint64_t ticket, uint32_t* out_ids, float* out_dists, double* latency_s) {
  if (!s) return pann::fail(PANN_EINVAL, "server is NULL");
  int rc;
  Request* r = take(s, ticket, &rc);
  if (!r) return rc;
  if (r->kind != 0) {
    delete r;
    return pann::fail(PANN_EINVAL, "ticket is a range request");
  }
  rc = r->rc;
  if (rc == PANN_OK) {
    if (out_ids) std::memcpy(out_ids, r->ids.data(), 4 * r->ids.size());
    if (out_dists) std::memcpy(out_dists, r->dists.data(), 4 * r->dists.size());
  } else {
    pann::fail(rc, r->err);
  }
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  delete r;
  return rc;
}

int pann_server_wait_range(pann_server* s, uint64_t ticket, uint64_t* out_offsets, uint32_t* out_ids, uint64_t ids_cap,
                           double* latency_s) {
  if (!s) return pann::fail(PANN_EINVAL, "server is NULL");
  int rc;
  Request* r = take(s, ticket, &rc);
  if (!r) return rc;
  if (r->kind != 1) {
    delete r;
    return pann::fail(PANN_EINVAL, "ticket is a k-NN request");
  }
  rc = r->rc;
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  if (rc == PANN_OK) {
    if (out_offsets) std::memcpy(out_offsets, r->offsets.data(), 8 * r->offsets.size());
    if (r->ids.size() > ids_cap) {
      rc = pann::fail(PANN_EOVERFLOW, "range answers need " + std::to_string(r->ids.size()) + " ids");
    } else if (out_ids && !r->ids.empty()) {
      std::memcpy(out_ids, r->ids.data(), 4 * r->ids.size());
    }
  } else {
    pann::fail(rc, r->err);
  }
  delete r;
  return rc;
}

int pann_server_stats(pann_server* s, int reset, uint64_t* requests, uint64_t* queries, double* seconds, double* p50_s,
                      double* p99_s) {
  if (!s) return pann::fail(PANN_EINVAL, "server is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  if (requests) *requests = s->lat.size();
  if (queries) *queries = s->done_queries;
  if (seconds) *seconds = std::chrono::duration<double>(clk::now() - s->stats_t0).count();
  if (p50_s) *p50_s = quantile(s->lat, 0.50);
  if (p99_s) *p99_s = quantile(s->lat, 0.99);
  if (reset) {
    s->lat.clear();
    s->done_queries = 0;
    s->stats_t0 = clk::now();
  }
  return PANN_OK;
}

int pann_server_admission(pann_server* s, int reset, uint64_t* batches, uint64_t* queries, uint64_t* scratch_peak,
                          uint64_t* scratch_bytes) {
  if (!s) return pann::fail(PANN_EINVAL, "server is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  if (batches) *batches = s->batches;
  if (queries) *queries = s->batched_queries;
  if (scratch_peak) *scratch_peak = s->scratch_peak;
  if (scratch_bytes) *scratch_bytes = s->scratch;
  if (reset) {
    s->batches = 0;
    s->batched_queries = 0;
    s->scratch_peak = 0;
  }
  return PANN_OK;
}

int pann_server_destroy(pann_server* s) {
  if (!s) return PANN_OK;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if (s->dispatcher.joinable()) s->dispatcher.join();
  if (s->ranger.joinable()) s->ranger.join();
  for (auto& kv : s->reqs) delete kv.second;
  for (Slot& sl : s->slots) {
    if (sl.st) cudaStreamSynchronize(sl.st);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.st) cudaStreamDestroy(sl.st);
    if (sl.arena) cudaFree(sl.arena);
    for (void* h : {(void*)sl.h_q, (void*)sl.h_k, (void*)sl.h_L, (void*)sl.h_order, (void*)sl.h_ids, (void*)sl.h_d})
      if (h) cudaFreeHost(h);
  }
  delete s;
  return PANN_OK;
}

// Open-loop load generator: submits request i at arrival_s[i] seconds after the
// call starts (k-NN when kind[i] == 0, else range with *rp), from queries
// pool rows q_row[i] .. q_row[i] + nq[i] - 1, waits for all, and reports each
// request's latency and the wall time from the first submission to the last
// completion.
int pann_server_replay(pann_server* s, uint32_t nreq, const double* arrival_s, const uint32_t* kind,
                       const uint32_t* nq, const uint32_t* k, const uint32_t* beam, const uint64_t* q_row,
                       const void* query_pool, const pann_range_params* rp, uint32_t range_start, double* out_latency_s,
                       double* out_wall_s) {
  if (!s || (nreq && (!arrival_s || !kind || !nq || !q_row || !query_pool))) return pann::fail(PANN_EINVAL, "NULL argument");
  std::vector<uint64_t> tickets(nreq, 0);
  std::vector<int> rcs(nreq, PANN_OK);
  std::atomic<uint32_t> submitted{0};
  const uint8_t* pool = static_cast<const uint8_t*>(query_pool);
  const auto t0 = clk::now();
  std::thread waiter([&] {
    for (uint32_t i = 0; i < nreq; i++) {
      while (submitted.load(std::memory_order_acquire) <= i) std::this_thread::yield();
      if (rcs[i] != PANN_OK) continue;
      double lat = 0;
      if (kind[i] == 0) {
        rcs[i] = pann_server_wait_knn(s, tickets[i], nullptr, nullptr, &lat);
      } else {
        rcs[i] = pann_server_wait_range(s, tickets[i], nullptr, nullptr, ~0ull, &lat);
      }
      if (out_latency_s) out_latency_s[i] = lat;
    }
  });
  for (uint32_t i = 0; i < nreq; i++) {
    const auto when = t0 + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(arrival_s[i]));
    while (clk::now() < when) {
      auto left = when - clk::now();
      if (left > std::chrono::microseconds(200)) std::this_thread::sleep_for(left - std::chrono::microseconds(100));
    }
    const void* q = pool + (size_t)q_row[i] * s->row_bytes;
    rcs[i] = kind[i] == 0 ? pann_server_submit_knn(s, q, nq[i], k[i], beam[i], &tickets[i])
                          : pann_server_submit_range(s, q, nq[i], rp, range_start, &tickets[i]);
    submitted.store(i + 1, std::memory_order_release);
  }
  waiter.join();
  if (out_wall_s) *out_wall_s = std::chrono::duration<double>(clk::now() - t0).count();
  for (uint32_t i = 0; i < nreq; i++)
    if (rcs[i] != PANN_OK) return pann::fail(rcs[i], "request " + std::to_string(i) + " failed");
  return PANN_OK;
}

}  // extern "C"
