// Range search (include/parlayann_b200.h, pann_range_search): RangeSearch
// (rangeSearch.h:183-276) and DoubleBeamRangeSearch (doublingSearch.h:50-157)
// on unquantized points.
//
//   1. The beam search of width `beam` with early stopping runs through the
//      tiers of the exact search (search.cuh / search_emu.cuh, with
//      SearchArgs::es_*), k = beam.
//   2. range_classify_kernel: the frontier is sorted by (distance, id), so the
//      entries within the radius are a prefix. A Greedy query whose whole
//      frontier is in range becomes an expansion job; every other query's
//      answer is that prefix.
//   3. range_expand_kernel: greedy_search (rangeSearch.h:21-55), one warp per
//      query. Its FIFO order is the answer's order and its hashset
//      (hashset.h:13-55, initial capacity 2 * beam * 64) decides which
//      neighbours count as new, so the warp runs the reference's sequence of
//      hashset calls exactly (the ordered emulation of search_emu.cuh, tables
//      in global memory) and evaluates distances in parallel: it takes the
//      neighbours of every node already in the queue (up to a key budget) in
//      queue order, tests them 32 at a time, then scores the new ones and
//      appends those in range in order. Processing several queued nodes at
//      once is the same computation: a node's appends never change which
//      nodes were queued before it, and its hashset calls come after those of
//      the nodes ahead of it.
//   4. range_assemble_kernel: answers gathered into one CSR array.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "index.cuh"
#include "tiers.cuh"

namespace pann {

enum RangeStatus : uint32_t { RS_RETRY = 1u, RS_GREW = 2u };
constexpr int HOME_BATCH = 8;      // table loads in flight per thread
constexpr int EXPAND_THREADS = 256;  // one block per expansion

struct RangeArgs {
  const uint8_t* points;
  uint64_t stride;
  uint32_t d, nchunks;
  const uint32_t* graph;
  uint32_t R;
  const uint8_t* queries;
  const uint32_t* fr_ids;  // beam search frontiers, `beam` entries per query (PAD past the end)
  const float* fr_d;
  uint32_t beam;
  double radius;           // the expansion's radius (rangeSearch.h:236-240)
  const uint32_t* jobs;
  const uint32_t* njobs;
  uint32_t* job_counter;
  uint32_t bits0;          // ceil(log2(2 * beam * 64)) (rangeSearch.h:27, hashset.h:50-54)
  uint32_t* tabs;          // per slot: two tables of `cap` slots
  uint32_t cap;
  uint32_t* queues;        // per slot: qcap ids
  uint32_t qcap;
  uint32_t keybuf;         // keys gathered per round (shared memory)
  uint32_t* pool;
  unsigned long long pool_cap;
  unsigned long long* pool_count;
  unsigned long long* res_off;  // per query
  uint32_t* res_n;
  uint32_t* res_cmps;
  uint32_t* res_status;
  uint32_t* retry;
  uint32_t* retry_count;
};

// Per query: the answer is the in-range prefix of the frontier, or an
// expansion (Greedy, whole frontier in range). src[i] = 1 marks the latter.
__global__ void range_classify_kernel(const uint32_t* __restrict__ fr_ids, const float* __restrict__ fr_d, uint32_t nq,
                                      uint32_t beam, double radius, int type, uint32_t* jobs, uint32_t* njobs,
                                      uint32_t* res_n, uint32_t* src, uint32_t* extra_cmps, uint32_t* res_status) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
    const uint32_t* ids = fr_ids + (uint64_t)i * beam;
    const float* ds = fr_d + (uint64_t)i * beam;
    uint32_t c = 0;
    while (c < beam && ids[c] != PANN_PAD && (double)ds[c] <= radius) c++;
    const bool full = c == beam;
    res_status[i] = 0;
    extra_cmps[i] = 0;
    if (full && type == PANN_RANGE_GREEDY) {
      jobs[atomicAdd(njobs, 1u)] = i;
      res_n[i] = 0;
      src[i] = 1;
    } else {
      res_n[i] = c;
      src[i] = 0;
      // Doubling's second round: beam_search with limit 0 from the in-range
      // frontier visits nothing and counts its start points
      if (full && type == PANN_RANGE_DOUBLING) extra_cmps[i] = beam;
    }
  }
}

// Block-wide ordered compaction: the entries of tmp[0, n) other than PAD, in
// order, to out[0, cap); returns how many there are (possibly above cap) to
// every thread. ccnt holds n / 32 + 1 words of shared memory, tot one.
__device__ __forceinline__ uint32_t block_compact(const uint32_t* tmp, uint32_t n, uint32_t* out, uint32_t cap,
                                                  uint32_t* ccnt, uint32_t* tot) {
  const unsigned FULL = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const uint32_t nch = (n + 31) / 32;
  for (uint32_t c = warp; c < nch; c += nw) {
    const uint32_t i = c * 32 + lane;
    const unsigned m = __ballot_sync(FULL, i < n && tmp[i] != PANN_PAD);
    if (lane == 0) ccnt[c] = __popc(m);
  }
  __syncthreads();
  if (warp == 0) {  // exclusive scan of the chunk counts
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < nch; c0 += 32) {
      const uint32_t v = c0 + lane < nch ? ccnt[c0 + lane] : 0u;
      uint32_t incl = v;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, incl, d);
        if (lane >= d) incl += t;
      }
      if (c0 + lane < nch) ccnt[c0 + lane] = carry + incl - v;
      carry += __shfl_sync(FULL, incl, 31);
    }
    if (lane == 0) *tot = carry;
  }
  __syncthreads();
  for (uint32_t c = warp; c < nch; c += nw) {
    const uint32_t i = c * 32 + lane;
    const bool keep = i < n && tmp[i] != PANN_PAD;
    const unsigned m = __ballot_sync(FULL, keep);
    const uint32_t o = ccnt[c] + __popc(m & lt);
    if (keep && o < cap) out[o] = tmp[i];
  }
  const uint32_t total = *tot;
  __syncthreads();
  return total;
}

// Block control words in shared memory; CTL_CUR (the table pointer) and
// CTL_OFF (the answer pool offset) are 64-bit, at 8-byte aligned words.
enum : uint32_t {
  CTL_JOB = 0, CTL_OK, CTL_COUNT, CTL_NUN, CTL_FILTERED = 5, CTL_BITS, CTL_TOT, CTL_CUR = 8, CTL_OFF = 10, CTL_WORDS = 16
};

// One block per query (EXPAND_THREADS threads). Warp 0 owns the emulated
// hashset and makes its calls in order; every warp gathers adjacency rows,
// looks keys up in the table as it stands, scores new neighbours and takes
// part in the ordered compactions.
template <int DT, int MT>
__global__ void __launch_bounds__(EXPAND_THREADS) range_expand_kernel(RangeArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const unsigned FULL = 0xFFFFFFFFu;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t nthr = blockDim.x;
  const unsigned lt = (1u << lane) - 1u;
  uint8_t* qs = smem;
  uint32_t* kbuf = reinterpret_cast<uint32_t*>(smem + a.stride);
  uint32_t* ubuf = kbuf + a.keybuf;
  uint32_t* kraw = ubuf + a.keybuf;  // a round's adjacency rows as loaded
  uint32_t* ctl = kraw + a.keybuf;
  uint32_t* ccnt = ctl + CTL_WORDS;
  uint32_t* tabA = a.tabs + (size_t)blockIdx.x * 2 * a.cap;
  uint32_t* tabB = tabA + a.cap;
  uint32_t* Q = a.queues + (size_t)blockIdx.x * a.qcap;
  const uint32_t njobs = *a.njobs;

  for (;;) {
    __syncthreads();
    if (tid == 0) ctl[CTL_JOB] = atomicAdd(a.job_counter, 1u);
    __syncthreads();
    const uint32_t job = ctl[CTL_JOB];
    if (job >= njobs) break;
    const uint32_t qi = a.jobs[job];
    if (warp == 0) stage_query<DT, MT>(qs, a.queries + (uint64_t)qi * a.stride, (int)a.nchunks, lane);
    for (uint32_t i = tid; i < (1u << a.bits0); i += nthr) tabA[i] = PANN_PAD;
    __syncthreads();
    int32_t qq = 0;
    if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), a.nchunks);
    EmuHash h;  // warp 0's copy is the hashset; the others read bits and table from ctl
    h.cur = tabA; h.other = tabB; h.cur_cap = a.cap; h.other_cap = a.cap;
    h.bits = a.bits0; h.num_entries = 0;
    uint32_t cmps = 0;

    // seeds: every frontier entry goes through the hashset; new and in range
    // ones start the queue (rangeSearch.h:30-33)
    if (warp == 0) {
      bool ok = true;
      uint32_t count = 0;
      for (uint32_t s0 = 0; s0 < a.beam && ok; s0 += 32) {
        const bool valid = s0 + lane < a.beam;
        const uint32_t id = valid ? a.fr_ids[(uint64_t)qi * a.beam + s0 + lane] : PANN_PAD;
        const float dd = valid ? a.fr_d[(uint64_t)qi * a.beam + s0 + lane] : 0.0f;
        bool seen = false;
        ok = emu_batch(h, id, valid, lane, &seen);
        if (!ok) break;
        const bool keep = valid && !seen && !((double)dd > a.radius);
        const unsigned m = __ballot_sync(FULL, keep);
        if (keep && count + __popc(m & lt) < a.qcap) Q[count + __popc(m & lt)] = id;
        count += __popc(m);
        if (count > a.qcap) ok = false;
      }
      if (lane == 0) {
        ctl[CTL_OK] = ok;
        ctl[CTL_COUNT] = count;
        ctl[CTL_BITS] = h.bits;
        *reinterpret_cast<uint32_t**>(ctl + CTL_CUR) = h.cur;
      }
    }
    __syncthreads();
    bool ok = ctl[CTL_OK] != 0;
    uint32_t count = ctl[CTL_COUNT];

    // breadth-first expansion (rangeSearch.h:36-52), up to gn queued nodes a
    // round: their adjacency rows are gathered together (one memory round
    // trip), the hash homes of all their neighbours and the next round's rows
    // are prefetched into L2, the hashset calls run in order, and the rows of
    // the new neighbours are prefetched as the calls find them
    const uint32_t gn = a.keybuf / a.R > 0 ? a.keybuf / a.R : 1;
    const uint32_t row_lines = (a.R * 4 + 127) / 128;
    uint32_t pos = 0;
    while (ok && pos < count) {
      const uint32_t end = count - pos < gn ? count : pos + gn;
      const uint32_t nraw = (end - pos) * a.R;
      const uint32_t bits = ctl[CTL_BITS];
      const uint32_t* tab = *reinterpret_cast<uint32_t* const*>(ctl + CTL_CUR);
      const uint32_t mask0 = (1u << bits) - 1u;
      for (uint32_t i = tid; i < nraw; i += nthr) {
        const uint32_t node = Q[pos + i / a.R];
        const uint32_t v = __ldg(a.graph + (uint64_t)node * a.R + (i % a.R));
        kraw[i] = v;
        if (v != PANN_PAD) asm volatile("prefetch.global.L2 [%0];" ::"l"(tab + ref_slot(v, mask0)));
      }
      {  // the next round's rows (nodes queued so far)
        const uint32_t nend = count - end < gn ? count : end + gn;
        for (uint32_t i = tid; i < (nend - end) * row_lines; i += nthr) {
          const uint32_t node = Q[end + i / row_lines];
          asm volatile("prefetch.global.L2 [%0];" ::"l"(a.graph + (uint64_t)node * a.R + 32 * (i % row_lines)));
        }
      }
      __syncthreads();
      // the neighbours in order (a row's live entries are those before PAD)
      const uint32_t nk = block_compact(kraw, nraw, kbuf, a.keybuf, ccnt, ctl + CTL_TOT);
      // A call whose key the table already holds on its probe path (its home
      // slot, then the slots after it up to the first empty one) returns true
      // and changes nothing (hashset.h:22-24,39-44) unless the table grows
      // first (hashset.h:25). Slots are only ever emptied by a growth, and the
      // table cannot grow while num_entries stays at or below half its size.
      // So the round's calls are looked up against the table as it stands;
      // when even every call not found there inserting keeps num_entries at
      // or below half, only those calls run, in order; otherwise all of them.
      for (uint32_t b0 = 0; b0 < nk; b0 += nthr * HOME_BATCH) {
        uint32_t hv[HOME_BATCH];
#pragma unroll
        for (int j = 0; j < HOME_BATCH; j++) {
          const uint32_t i = b0 + nthr * j + tid;
          hv[j] = i < nk ? tab[ref_slot(kbuf[i], mask0)] : PANN_PAD;
        }
#pragma unroll
        for (int j = 0; j < HOME_BATCH; j++) {
          const uint32_t i = b0 + nthr * j + tid;
          if (i < nk) {
            const uint32_t key = kbuf[i];
            uint32_t v = hv[j];
            uint32_t p = ref_slot(key, mask0);
            for (uint32_t s = 0; v != PANN_PAD && v != key && s < mask0; s++) {
              p = (p + 1) & mask0;
              v = tab[p];
            }
            kraw[i] = v == key ? PANN_PAD : key;
          }
        }
      }
      __syncthreads();
      // warp 0 decides; the kept calls replace kbuf only on the fast path
      if (warp == 0) {
        uint32_t nf = 0;
        for (uint32_t c0 = 0; c0 < nk; c0 += 32)
          nf += __popc(__ballot_sync(FULL, c0 + lane < nk && kraw[c0 + lane] != PANN_PAD));
        if (lane == 0) ctl[CTL_FILTERED] = h.num_entries + (long long)nf <= (long long)((1u << h.bits) / 2);
      }
      __syncthreads();
      uint32_t ncalls = nk;
      if (ctl[CTL_FILTERED]) ncalls = block_compact(kraw, nk, kbuf, a.keybuf, ccnt, ctl + CTL_TOT);
      // the hashset calls, in order (warp 0)
      if (warp == 0) {
        uint32_t nun = 0;
        bool wok = true;
        for (uint32_t k0 = 0; k0 < ncalls && wok; k0 += 32) {
          const bool valid = k0 + lane < ncalls;
          const uint32_t key = valid ? kbuf[k0 + lane] : PANN_PAD;
          bool seen = false;
          wok = emu_batch(h, key, valid, lane, &seen);
          const bool un = wok && valid && !seen;
          const unsigned m = __ballot_sync(FULL, un);
          if (un) {
            ubuf[nun + __popc(m & lt)] = key;
            const char* row = reinterpret_cast<const char*>(a.points + (uint64_t)key * a.stride);
            for (uint32_t o = 0; o < a.stride; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(row + o));
          }
          nun += __popc(m);
        }
        if (lane == 0) {
          ctl[CTL_OK] = wok;
          ctl[CTL_NUN] = nun;
          ctl[CTL_BITS] = h.bits;
          *reinterpret_cast<uint32_t**>(ctl + CTL_CUR) = h.cur;
        }
      }
      __syncthreads();
      ok = ctl[CTL_OK] != 0;
      if (!ok) break;
      const uint32_t nun = ctl[CTL_NUN];
      cmps += nun;
      // distances of the new neighbours; in-range ones join the queue in order
      for (uint32_t u = tid; u < nun; u += nthr) {
        const uint32_t id = ubuf[u];
        const float dd = point_dist<DT, MT>(a.points + (uint64_t)id * a.stride, qs, (int)a.d, (int)a.nchunks, qq);
        kbuf[u] = (double)dd <= a.radius ? id : PANN_PAD;
      }
      __syncthreads();
      count += block_compact(kbuf, nun, Q + count, a.qcap - count, ccnt, ctl + CTL_TOT);
      if (count > a.qcap) ok = false;
      pos = end;
    }

    if (!ok) {
      // the table or the queue outgrew this tier: the next tier re-runs it
      if (tid == 0) {
        if (a.retry) a.retry[atomicAdd(a.retry_count, 1u)] = qi;
        a.res_status[qi] |= RS_RETRY;
      }
      continue;
    }
    if (tid == 0) *reinterpret_cast<unsigned long long*>(ctl + CTL_OFF) = atomicAdd(a.pool_count, (unsigned long long)count);
    __syncthreads();
    const unsigned long long off = *reinterpret_cast<unsigned long long*>(ctl + CTL_OFF);
    if (off + count <= a.pool_cap)
      for (uint32_t i = tid; i < count; i += nthr) a.pool[off + i] = Q[i];
    if (tid == 0) {
      a.res_off[qi] = off;
      a.res_n[qi] = count;
      a.res_cmps[qi] = cmps;
      a.res_status[qi] = ctl[CTL_BITS] != a.bits0 ? RS_GREW : 0u;
    }
  }
}

// Answers into one CSR array: query i's ids at out[offsets[i] ..].
__global__ void range_assemble_kernel(uint32_t nq, const unsigned long long* __restrict__ offsets,
                                      const uint32_t* __restrict__ src, const uint32_t* __restrict__ res_n,
                                      const unsigned long long* __restrict__ res_off, const uint32_t* __restrict__ pool,
                                      const uint32_t* __restrict__ fr_ids, uint32_t beam, uint32_t* out) {
  const int lane = threadIdx.x & 31;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nq; i += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t* from = src[i] ? pool + res_off[i] : fr_ids + (uint64_t)i * beam;
    uint32_t* to = out + offsets[i];
    for (uint32_t j = lane; j < res_n[i]; j += 32) to[j] = from[j];
  }
}

template <int DT, int MT>
static cudaError_t launch_expand_t(const RangeArgs& a, int slots, size_t smem, cudaStream_t st) {
  auto k = range_expand_kernel<DT, MT>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max());
  if (e != cudaSuccess) return e;
  k<<<slots, EXPAND_THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

static cudaError_t launch_expand(int dtype, int metric, const RangeArgs& a, int slots, size_t smem, cudaStream_t st) {
#define PANN_RANGE_CASE(DT, MT) \
  if (dtype == DT && metric == MT) return launch_expand_t<DT, MT>(a, slots, smem, st);
  PANN_RANGE_CASE(DT_U8, MT_L2)
  PANN_RANGE_CASE(DT_U8, MT_IP)
  PANN_RANGE_CASE(DT_I8, MT_L2)
  PANN_RANGE_CASE(DT_I8, MT_IP)
  PANN_RANGE_CASE(DT_F32, MT_L2)
  PANN_RANGE_CASE(DT_F32, MT_IP)
#undef PANN_RANGE_CASE
  return cudaErrorInvalidValue;
}

// A small device-to-host read of a result the stream is still producing.
// The stream is waited on first, so the copy into pageable memory (which
// the driver completes synchronously) never waits on a long kernel itself:
// other threads' launches on other streams (the serving loop's batches)
// are not held up meanwhile.
static cudaError_t to_host(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

static uint32_t ceil_log2(uint64_t x) {
  uint32_t b = 0;
  while ((1ull << b) < x) b++;
  return b;
}

}  // namespace pann

using namespace pann;

namespace pann {
// Range search's largest device scratch taken once: the expansion tables at
// their design cap (4 GB across a tier's slots) and a pool of 4M answers.
// A serving loop calls it at creation, so the range requests it groups never
// reallocate (a free drains the whole device, stalling the k-NN batches
// beside it).
int range_reserve(pann_index* idx) {
  PANN_CUDA(idx->range_tabs.ensure_grow(4ull << 30));
  PANN_CUDA(idx->range_pool.ensure_grow(4ull << 22));
  PANN_CUDA(idx->range_out.ensure_grow(4ull << 22));
  return PANN_OK;
}
}  // namespace pann

extern "C" int pann_range_search(pann_index* idx, const void* queries, uint32_t nq, const pann_range_params* rp,
                                 uint32_t start_point, uint64_t* out_offsets, uint32_t* out_ids, uint64_t ids_cap,
                                 uint32_t* out_visited, uint32_t* out_cmps, uint32_t* out_flags) {
  if (!idx || !idx->points_set) return fail(PANN_EINVAL, "index has no points (pann_index_set_points)");
  idx->range_held = 0;
  if (!rp) return fail(PANN_EINVAL, "range params are NULL");
  if (rp->type < PANN_RANGE_GREEDY || rp->type > PANN_RANGE_BEAM)
    return fail(PANN_EINVAL, "range type must be PANN_RANGE_GREEDY, PANN_RANGE_DOUBLING or PANN_RANGE_BEAM");
  if (!out_offsets) return fail(PANN_EINVAL, "out_offsets is NULL");
  if (nq && !queries) return fail(PANN_EINVAL, "queries is NULL");
  // QueryParams QP1(beam, beam, G.size(), G.max_degree(), ...) (rangeSearch.h:207-210)
  pann_query_params qp{rp->beam, rp->beam, idx->n, idx->R, 0.125};
  SearchPlan plan;
  int rc = make_plan(idx, &qp, 1, &plan);
  if (rc) return rc;
  out_offsets[0] = 0;
  if (nq == 0) return PANN_OK;
  cudaStream_t st = idx->stream;
  rc = stage_starts(idx, &start_point, 1, st);
  if (rc) return rc;
  const uint32_t beam = rp->beam;
  const size_t rb = (size_t)idx->d * idx->esize;
  PANN_CUDA(idx->q.ensure_grow(idx->stride * (size_t)nq));
  PANN_CUDA(idx->ids.ensure_grow(4ull * beam * nq));
  PANN_CUDA(idx->dists.ensure_grow(4ull * beam * nq));
  PANN_CUDA(idx->vis.ensure_grow(4ull * nq));
  PANN_CUDA(idx->cmps.ensure_grow(4ull * nq));
  PANN_CUDA(idx->status.ensure_grow(4ull * nq));
  if (rb != idx->stride) PANN_CUDA(cudaMemsetAsync(idx->q.p, 0, idx->stride * (size_t)nq, st));
  PANN_CUDA(cudaMemcpy2DAsync(idx->q.p, idx->stride, queries, rb, rb, nq, cudaMemcpyHostToDevice, st));

  // ---- 1. beam search with early stopping. The rule's radii pass through
  // Point::translate_distance, a float rounding for unquantized points
  // (euclidian_point.h:119-123, mips_point.h:90-92); Doubling passes the
  // radius itself (doublingSearch.h:77-81).
  const double r_f = (double)(float)rp->radius;
  const double esr_f = (double)(float)rp->early_stopping_radius;
  {
    TierSizes z;
    rc = size_tiers(idx, plan, nq, PREC_F32, 0, 0, &z);
    if (rc) return rc;
    TierBufs b{};
    rc = index_tier_buffers(idx, z, nq, PREC_F32, &b);
    if (rc) return rc;
    SearchArgs a = base_args(idx, plan, idx->q.as<uint8_t>(), nullptr, nq, idx->starts.as<uint32_t>(),
                             idx->ids.as<uint32_t>(), idx->dists.as<float>(), idx->vis.as<uint32_t>(),
                             idx->cmps.as<uint32_t>(), idx->status.as<uint32_t>(), nullptr, 0);
    a.es_count = (double)rp->early_stopping_count;
    a.es_radius = rp->type == PANN_RANGE_DOUBLING ? rp->radius : r_f;
    a.es_esr = esr_f;
    rc = enqueue_tiers(idx, plan, a, z, b, st, PREC_F32, 0);
    if (rc) return rc;
  }

  // ---- 2. classify; per-query metadata in one buffer
  // words: jobs nq | res_n nq | src nq | extra nq | rstatus nq | res_cmps nq | retry nq | res_off 2nq | offsets 2(nq+1) | counters 8
  const size_t meta_words = 11ull * nq + 2 + 8 + 8;
  PANN_CUDA(idx->range_meta.ensure_grow(4 * meta_words));
  uint32_t* jobs = idx->range_meta.as<uint32_t>();
  uint32_t* res_n = jobs + nq;
  uint32_t* src = res_n + nq;
  uint32_t* extra = src + nq;
  uint32_t* rstat = extra + nq;
  uint32_t* rcmps = rstat + nq;
  uint32_t* retry = rcmps + nq;
  uint32_t* after = retry + nq;
  if (reinterpret_cast<uintptr_t>(after) & 7) after++;  // 8-byte alignment for the 64-bit arrays
  unsigned long long* res_off = reinterpret_cast<unsigned long long*>(after);
  unsigned long long* d_offsets = res_off + nq;
  uint32_t* cnt = reinterpret_cast<uint32_t*>(d_offsets + nq + 1);  // [0] njobs [1] job ctr [2] retry n [4..5] pool count
  unsigned long long* pool_count = reinterpret_cast<unsigned long long*>(cnt + 4);
  PANN_CUDA(cudaMemsetAsync(cnt, 0, 32, st));
  PANN_CUDA(cudaMemsetAsync(rcmps, 0, 4ull * nq, st));
  {
    int blocks = (int)std::min<uint64_t>((nq + 255) / 256, 4096);
    range_classify_kernel<<<blocks, 256, 0, st>>>(idx->ids.as<uint32_t>(), idx->dists.as<float>(), nq, beam,
                                                  rp->radius, rp->type, jobs, cnt, res_n, src, extra, rstat);
    PANN_CUDA(cudaGetLastError());
  }
  uint32_t h_njobs = 0;
  PANN_CUDA(to_host(&h_njobs, cnt, 4, st));

  // ---- 3. expansions, in tiers of growing per-query room; the answers go to
  // a pool sized up front and grown (with a re-run) if they do not fit
  const uint32_t bits0 = ceil_log2(2ull * beam * 64);
  if (h_njobs > 0) {
    // The first tier gives each of its slots (a warp running one expansion
    // after another) the largest tables that fit 4 GB at that slot count, so
    // that only rare, very large expansions fail there and re-run from the
    // start in the second tier's 2^24-slot tables. The queue holds a quarter
    // of a table: a table outgrows its slots before its queue fills.
    struct Tier { uint32_t cap_bits, qcap_bits; int max_slots; };
    const int slots0 = (int)std::min<uint64_t>(h_njobs, 2ull * idx->sm_count);
    uint32_t cap0 = 18;
    while (cap0 < 22 && (uint64_t)slots0 * 4ull * (2ull * (2ull << cap0) + (1ull << (cap0 - 1))) <= (4ull << 30)) cap0++;
    cap0 = std::max(cap0, bits0 + 2);
    const Tier tiers[2] = {{cap0, cap0 - 2, 2 * idx->sm_count}, {std::max<uint32_t>(24, bits0 + 2), 22, 16}};
    const uint32_t keybuf = (std::max<uint32_t>(2048, idx->R) + 31) & ~31u;  // 8-byte aligned control words
    const size_t smem = idx->stride + 12ull * keybuf + 4ull * (CTL_WORDS + keybuf / 32 + 2);
    unsigned long long pool_cap = std::max<unsigned long long>(1ull << 22, 256ull * h_njobs);
    for (int attempt = 0; attempt < 3; attempt++) {
      PANN_CUDA(idx->range_pool.ensure_grow(4 * pool_cap));
      PANN_CUDA(cudaMemsetAsync(pool_count, 0, 8, st));
      const uint32_t* tier_jobs = jobs;
      const uint32_t* tier_n = cnt;
      uint32_t pending = h_njobs;
      for (int t = 0; t < 2 && pending > 0; t++) {
        const uint32_t cap = 1u << tiers[t].cap_bits, qcap = 1u << tiers[t].qcap_bits;
        const size_t per_slot = 4ull * (2ull * cap + qcap);
        int slots = (int)std::max<uint64_t>(1, std::min<uint64_t>({(uint64_t)pending, (uint64_t)tiers[t].max_slots,
                                                                   (4ull << 30) / per_slot}));
        PANN_CUDA(idx->range_tabs.ensure_grow(per_slot * slots));
        PANN_CUDA(cudaMemsetAsync(cnt + 1, 0, 8, st));  // job counter, retry count
        RangeArgs ra{};
        ra.points = idx->d_points;
        ra.stride = idx->stride;
        ra.d = idx->d;
        ra.nchunks = idx->nchunks;
        ra.graph = idx->d_graph;
        ra.R = idx->R;
        ra.queries = idx->q.as<uint8_t>();
        ra.fr_ids = idx->ids.as<uint32_t>();
        ra.fr_d = idx->dists.as<float>();
        ra.beam = beam;
        ra.radius = r_f;  // greedy_search(…, QP1.radius) (rangeSearch.h:236-240)
        ra.jobs = tier_jobs;
        ra.njobs = tier_n;
        ra.job_counter = cnt + 1;
        ra.bits0 = bits0;
        ra.tabs = idx->range_tabs.as<uint32_t>();
        ra.cap = cap;
        ra.queues = ra.tabs + (size_t)slots * 2 * cap;
        // per-slot queues follow the tables of all slots
        ra.qcap = qcap;
        ra.keybuf = keybuf;
        ra.pool = idx->range_pool.as<uint32_t>();
        ra.pool_cap = pool_cap;
        ra.pool_count = pool_count;
        ra.res_off = res_off;
        ra.res_n = res_n;
        ra.res_cmps = rcmps;
        ra.res_status = rstat;
        ra.retry = t == 0 ? retry : nullptr;  // the last tier's failures stay flagged
        ra.retry_count = cnt + 2;
        PANN_CUDA(launch_expand(idx->dtype, idx->metric, ra, slots, smem, st));
        if (t == 0) {
          uint32_t h_retry = 0;
          PANN_CUDA(to_host(&h_retry, cnt + 2, 4, st));
          pending = h_retry;
          if (pending) {
            // the retry list becomes the next tier's job list
            PANN_CUDA(cudaMemcpyAsync(cnt + 3, cnt + 2, 4, cudaMemcpyDeviceToDevice, st));
            tier_jobs = retry;
            tier_n = cnt + 3;
          }
        }
      }
      unsigned long long used = 0;
      PANN_CUDA(to_host(&used, pool_count, 8, st));
      if (used <= pool_cap) break;
      pool_cap = used;  // the answers did not fit: size the pool for them and run again
      PANN_CUDA(cudaMemsetAsync(rstat, 0, 4ull * nq, st));
    }
  }

  // ---- 4. counts, offsets, the CSR gather
  std::vector<uint32_t> h_n(nq), h_src(nq), h_extra(nq), h_rst(nq), h_rcmps(nq), h_vis(nq), h_cmps(nq), h_st(nq);
  PANN_CUDA(cudaStreamSynchronize(st));
  PANN_CUDA(cudaMemcpyAsync(h_n.data(), res_n, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(h_src.data(), src, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(h_extra.data(), extra, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(h_rst.data(), rstat, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(h_rcmps.data(), rcmps, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(h_vis.data(), idx->vis.p, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(h_cmps.data(), idx->cmps.p, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(h_st.data(), idx->status.p, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < nq; i++) {
    if (h_st[i] & (QS_TABLE_FULL | QS_INTERNAL)) return fail(PANN_EOVERFLOW, "a query's seen-set outgrew the largest table");
    if (h_rst[i] & RS_RETRY) return fail(PANN_EOVERFLOW, "a range expansion outgrew the largest table");
  }
  uint64_t total = 0;
  for (uint32_t i = 0; i < nq; i++) {
    out_offsets[i] = total;
    total += h_n[i];
    // QueryStats: the beam's visited + cmps, plus the expansion's (rangeSearch.h:258-267)
    if (out_visited) out_visited[i] = h_vis[i] + (h_src[i] ? h_n[i] : 0u);
    if (out_cmps) out_cmps[i] = h_cmps[i] + h_extra[i] + (h_src[i] ? h_rcmps[i] : 0u);
    if (out_flags) out_flags[i] = ((h_st[i] & QS_REF_WOULD_GROW) ? 1u : 0u) | ((h_rst[i] & RS_GREW) ? 2u : 0u);
  }
  out_offsets[nq] = total;
  if (total == 0) return PANN_OK;
  if (total <= ids_cap && !out_ids) return fail(PANN_EINVAL, "out_ids is NULL");
  PANN_CUDA(idx->range_out.ensure_grow(4 * total));
  PANN_CUDA(cudaMemcpyAsync(d_offsets, out_offsets, 8ull * (nq + 1), cudaMemcpyHostToDevice, st));
  {
    int blocks = (int)std::min<uint64_t>((nq + 7) / 8, 8192);
    range_assemble_kernel<<<blocks, 256, 0, st>>>(nq, d_offsets, src, res_n, res_off,
                                                  idx->range_pool.p ? idx->range_pool.as<uint32_t>() : nullptr,
                                                  idx->ids.as<uint32_t>(), beam, idx->range_out.as<uint32_t>());
    PANN_CUDA(cudaGetLastError());
  }
  if (total > ids_cap) {
    PANN_CUDA(cudaStreamSynchronize(st));
    idx->range_held = total;
    return fail(PANN_EOVERFLOW, "range answers need " + std::to_string(total) + " ids; out_ids holds " +
                                    std::to_string(ids_cap) + " (pann_range_fetch copies them)");
  }
  PANN_CUDA(cudaStreamSynchronize(st));
  PANN_CUDA(cudaMemcpyAsync(out_ids, idx->range_out.p, 4 * total, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  return PANN_OK;
}

extern "C" int pann_range_fetch(pann_index* idx, uint32_t* out_ids, uint64_t ids_cap) {
  if (!idx) return fail(PANN_EINVAL, "index is NULL");
  if (idx->range_held == 0) return fail(PANN_EINVAL, "no range answers are held (pann_range_fetch follows a "
                                                     "pann_range_search that returned PANN_EOVERFLOW)");
  const uint64_t total = idx->range_held;
  if (ids_cap < total)
    return fail(PANN_EOVERFLOW, "range answers need " + std::to_string(total) + " ids; out_ids holds " +
                                    std::to_string(ids_cap));
  if (!out_ids) return fail(PANN_EINVAL, "out_ids is NULL");
  PANN_CUDA(cudaMemcpyAsync(out_ids, idx->range_out.p, 4 * total, cudaMemcpyDeviceToHost, idx->stream));
  PANN_CUDA(cudaStreamSynchronize(idx->stream));
  idx->range_held = 0;
  return PANN_OK;
}
