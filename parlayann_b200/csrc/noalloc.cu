// pann_search_device_noalloc: the exact beam search of pann_search_device with
// every piece of its working memory carved out of one fixed, statically
// declared device array instead of buffers the index allocates on demand.
//
// Why: cudaMalloc and cudaFree are not free to call from everywhere. cudaFree
// waits for the whole device to go idle, so a serving thread that shares the
// GPU with other streams would stall all of them; a process whose framework
// allocator has already reserved the device's memory may find nothing left to
// allocate; and a request path with a latency bound cannot take the chance of
// an allocation that only its first large batch would trigger. Such callers
// get a search here whose device memory is fixed when the library's module
// is loaded, and which never asks the driver for more.
//
// The array is PANN_NOALLOC_SCRATCH_BYTES (32 MiB) per device, held from the
// module's load until the process exits. It holds the per-call counters, the
// start points, the per-query work lists and status words, a padded copy of
// the queries when the row size is not a multiple of 16 bytes, the per-warp
// global seen tables of the large-table tier and the per-warp emulated
// hashsets of the global emulation tier. A call whose layout does not fit is
// rejected with PANN_EINVAL and a message; nothing is truncated. The tiers run
// the same kernels as pann_search_device minus two optional buffers (the
// first tier's spill table and its hand-off logs), so the results are the
// same: queries whose small table fills re-run in the large-table tier, and
// queries on which the reference's hashset grows are re-run from the start by
// the emulation tiers.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <string>

#include "common.cuh"
#include "index.cuh"
#include "search.cuh"
#include "search_emu.cuh"

namespace pann {

// defined in capi.cu
cudaError_t launch_search(int dtype, int metric, bool global_table, const SearchArgs& a, int blocks, int threads,
                          size_t smem, cudaStream_t st, int prec, int minb = 3);
cudaError_t launch_emulate(int dtype, int metric, bool smem_tables, const SearchArgs& a, const EmuArgs& e,
                           int blocks, size_t smem, cudaStream_t st);
int search_occupancy(int dtype, int metric, bool g, int threads, size_t smem, int minb = 3);
uint32_t tier0_slots(const SearchPlan& p, uint32_t R);

constexpr size_t kNoallocScratchBytes = PANN_NOALLOC_SCRATCH_BYTES;

// The scratch itself. Every call on a device shares it and finds in it what
// the previous call left there.
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoallocScratchBytes];

// Device address of the array on `dev`, which must be the current device.
// Looked up on every call, not cached: the lookup costs little next to the
// launches, and a process that resets the device (which tears down the
// context holding the array) gets the new context's address instead of a
// stale one. The first lookup on a device may load this file's module onto
// it. Host code only ever passes this address on: the array's own name is a
// host-side stand-in, not a device pointer.
static int noalloc_scratch(int dev, uint8_t** out) {
  if (dev < 0) return fail(PANN_EINVAL, "no current device for the static scratch");
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr) {
    cudaGetLastError();
    return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress(static search scratch)");
  }
  *out = static_cast<uint8_t*>(p);
  return PANN_OK;
}

static uint32_t pow2_ceil(uint64_t x) {
  uint32_t p = 1;
  while (p < x && p < (1u << 30)) p <<= 1;
  return p;
}

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Bump allocation inside the scratch, 256-byte aligned.
struct Carve {
  uint8_t* base;
  size_t used = 0;
  uint8_t* take(size_t bytes) {
    uint8_t* p = base + used;
    used += align256(bytes);
    return p;
  }
};

}  // namespace pann

using namespace pann;

extern "C" int pann_search_device_noalloc(pann_index* idx, const void* d_queries, uint32_t nq,
                                          const pann_query_params* qp, const uint32_t* starts, uint32_t n_start,
                                          uint32_t* d_out_ids, float* d_out_dists, uint32_t* d_out_visited,
                                          uint32_t* d_out_cmps, uint32_t* d_out_flags, void* stream) {
  if (!idx) return fail(PANN_EINVAL, "index is NULL");
  if (!idx->points_set) return fail(PANN_EINVAL, "index has no points (pann_index_set_points)");
  if (nq && (!d_queries || !d_out_ids)) return fail(PANN_EINVAL, "queries or out_ids is NULL");
  SearchPlan plan;
  int rc = make_plan(idx, qp, n_start, &plan);
  if (rc) return rc;
  if (!starts) return fail(PANN_EINVAL, "start points are NULL");
  for (uint32_t i = 0; i < n_start; i++) {
    if ((uint64_t)starts[i] >= idx->n) return fail(PANN_EINVAL, "start point id out of range");
    for (uint32_t j = 0; j < i; j++)
      if (starts[j] == starts[i]) return fail(PANN_EINVAL, "duplicate start point");
  }
  if (nq == 0) return PANN_OK;

  // ---- layout, sized before anything runs so an oversized call is refused whole
  const size_t rb = (size_t)idx->d * idx->esize;
  const bool pad_queries = rb != idx->stride;
  const double cap_n = 2.0 * (10.0 + (double)plan.L) * (double)plan.dl;
  const uint32_t bits0 = (uint32_t)std::ceil(std::log2(cap_n));
  const uint64_t S0 = 1ull << bits0;
  const uint32_t S2 = std::min<uint32_t>(std::max<uint32_t>(1u << 16, pow2_ceil(4ull * plan.ref_half)), 1u << 24);
  const uint64_t capA = 16 * S0, capB = 8 * S0;
  const size_t t2_slot = 4ull * S2;              // one large-table tier seen table
  const size_t e2_slot = 4ull * (capA + capB);   // one global emulation table pair
  const size_t fixed = align256(256) + align256(4ull * n_start) + align256(4ull * 7 * nq) +
                       (pad_queries ? align256(idx->stride * (size_t)nq) : 0);
  if (fixed + t2_slot + e2_slot > kNoallocScratchBytes) {
    const size_t per_q = 28 + (pad_queries ? idx->stride : 0);
    const size_t slack = t2_slot + e2_slot + 4096 + align256(4ull * n_start);
    const size_t room = kNoallocScratchBytes > slack ? (kNoallocScratchBytes - slack) / per_q : 0;
    return fail(PANN_EINVAL, "pann_search_device_noalloc: this call needs " + std::to_string(fixed + t2_slot + e2_slot) +
                                 " bytes of scratch but the static scratch holds " +
                                 std::to_string(kNoallocScratchBytes) + " (at most " + std::to_string(room) +
                                 " queries per call at this beam, degree limit and row size); split the batch"
                                 " or use pann_search_device");
  }
  const size_t rem = kNoallocScratchBytes - fixed;
  // up to half of the rest to the emulation tier, never the large-table tier's one slot
  const int e2_slots =
      (int)std::max<uint64_t>(1, std::min<uint64_t>(idx->sm_count, std::min(rem / 2, rem - t2_slot) / e2_slot));
  const int t2_slots = (int)std::max<uint64_t>(
      1, std::min<uint64_t>(2ull * idx->sm_count, (rem - (size_t)e2_slots * e2_slot) / t2_slot));

  int dev = -1;
  PANN_CUDA(cudaGetDevice(&dev));
  if (dev != idx->device)
    return fail(PANN_EINVAL, "pann_search_device_noalloc must be called with the index's device current");
  uint8_t* base = nullptr;
  rc = noalloc_scratch(dev, &base);
  if (rc) return rc;
  Carve cv{base};
  uint32_t* cnt = reinterpret_cast<uint32_t*>(cv.take(256));
  uint32_t* d_starts = reinterpret_cast<uint32_t*>(cv.take(4ull * n_start));
  uint32_t* redo0 = reinterpret_cast<uint32_t*>(cv.take(4ull * 7 * nq));
  uint32_t* redo1 = redo0 + nq;
  uint32_t* emu = redo1 + nq;
  uint32_t* ovf = emu + nq;
  uint32_t* emu_rec = ovf + nq;
  uint32_t* ovf_rec = emu_rec + nq;
  uint32_t* own_status = ovf_rec + nq;
  uint8_t* qpad = pad_queries ? cv.take(idx->stride * (size_t)nq) : nullptr;
  uint32_t* gt2 = reinterpret_cast<uint32_t*>(cv.take((size_t)t2_slots * t2_slot));
  uint32_t* ge2 = reinterpret_cast<uint32_t*>(cv.take((size_t)e2_slots * e2_slot));
  if (cv.used > kNoallocScratchBytes) return fail(PANN_EDEVICE, "static scratch layout overran its array");

  cudaStream_t st = static_cast<cudaStream_t>(stream);  // 0 is the legacy default stream
  // The counters are the only scratch that must start at zero (the previous
  // call left its own there); every other region is written before it is read.
  PANN_CUDA(cudaMemsetAsync(cnt, 0, 256, st));
  PANN_CUDA(cudaMemcpyAsync(d_starts, starts, 4ull * n_start, cudaMemcpyHostToDevice, st));
  const uint8_t* q = static_cast<const uint8_t*>(d_queries);
  if (pad_queries) {
    PANN_CUDA(cudaMemsetAsync(qpad, 0, idx->stride * (size_t)nq, st));
    PANN_CUDA(cudaMemcpy2DAsync(qpad, idx->stride, d_queries, rb, rb, nq, cudaMemcpyDeviceToDevice, st));
    q = qpad;
  }
  uint32_t* status = d_out_flags ? d_out_flags : own_status;

  SearchArgs a{};
  a.points = idx->d_points;
  a.stride = idx->stride;
  a.d = idx->d;
  a.nchunks = idx->nchunks;
  a.graph = idx->d_graph;
  a.R = idx->R;
  a.queries = q;
  a.nq = nq;
  a.k = plan.k;
  a.L = plan.L;
  a.kstride = plan.k;
  a.dl = plan.dl;
  a.limit = plan.limit;
  a.batch_factor = plan.bf;
  a.ref_half = plan.ref_half;
  a.starts = d_starts;
  a.n_start = plan.n_start;
  a.Ccap = plan.Ccap;
  a.out_ids = d_out_ids;
  a.out_dists = d_out_dists;
  a.out_visited = d_out_visited;
  a.out_cmps = d_out_cmps;
  a.out_status = status;
  a.emu_list = emu;
  a.emu_rec = emu_rec;
  a.emu_count = cnt + 6;

  const size_t smem_cap = idx->smem_optin;
  // ---- first tier: shared-memory seen tables, no spill table, no hand-off
  {
    uint32_t S = tier0_slots(plan, idx->R);
    uint32_t wb = search_warp_bytes(idx->stride, plan.L, plan.Ccap, idx->R, S, false);
    int wpb = 4;
    while (wpb > 1 && (size_t)wb * wpb > smem_cap) wpb >>= 1;
    while ((size_t)wb * wpb > smem_cap && S > pow2_ceil(4ull * (idx->R + 1))) {
      S >>= 1;
      wb = search_warp_bytes(idx->stride, plan.L, plan.Ccap, idx->R, S, false);
    }
    if ((size_t)wb * wpb > smem_cap) return fail(PANN_EINVAL, "search state for this beam does not fit in shared memory");
    int occ = search_occupancy(idx->dtype, idx->metric, false, 32 * wpb, (size_t)wb * wpb);
    if (occ <= 0) occ = 1;
    uint64_t want = (nq + wpb - 1) / wpb;
    int blocks = (int)std::min<uint64_t>(want, (uint64_t)occ * idx->sm_count);
    SearchArgs t = a;
    t.S = S;
    t.warp_bytes = wb;
    t.job_counter = cnt + 0;
    t.redo_list = redo0;
    t.redo_count = cnt + 3;
    t.gspill = nullptr;
    t.Sg = 0;
    t.inslog = nullptr;
    PANN_CUDA(launch_search(idx->dtype, idx->metric, false, t, blocks, 32 * wpb, (size_t)wb * wpb, st, PREC_F32));
  }
  // ---- large-table tier: one global seen table per warp, in the scratch
  {
    uint32_t wb = search_warp_bytes(idx->stride, plan.L, plan.Ccap, idx->R, S2, true);
    SearchArgs t = a;
    t.S = S2;
    t.warp_bytes = wb;
    t.gtables = gt2;
    t.inslog = nullptr;
    t.job_list = redo0;
    t.njobs_dev = cnt + 3;
    t.job_counter = cnt + 2;
    t.redo_list = nullptr;
    t.redo_count = nullptr;
    PANN_CUDA(launch_search(idx->dtype, idx->metric, true, t, t2_slots, 32, wb, st, PREC_F32));
  }
  // ---- emulation tiers: the reference's hashset emulated exactly, first in
  // shared memory, then (queries that outgrow it) in the scratch
  {
    uint32_t vs = pow2_ceil(8ull * plan.L + 64);
    uint32_t basew = search_warp_bytes(idx->stride, plan.L, plan.Ccap, idx->R, 0, true);
    SearchArgs t = a;
    t.redo_list = nullptr;
    t.redo_count = nullptr;
    t.emu_list = nullptr;
    t.emu_count = nullptr;
    EmuArgs e{};
    e.bits0 = bits0;
    e.vs_slots = vs;
    e.base_bytes = basew;
    size_t smem_need = emu_smem_bytes(basew, vs, (uint32_t)(4 * S0), (uint32_t)(2 * S0), true);
    const uint32_t* glist = emu;
    uint32_t* gcount = cnt + 6;
    const uint32_t* grec = emu_rec;
    if (smem_need <= smem_cap && 4 * S0 < (1ull << 31)) {
      e.capA = (uint32_t)(4 * S0);
      e.capB = (uint32_t)(2 * S0);
      e.overflow_list = ovf;
      e.overflow_rec = ovf_rec;
      e.overflow_count = cnt + 8;
      e.job_rec = emu_rec;
      t.job_list = emu;
      t.njobs_dev = cnt + 6;
      t.job_counter = cnt + 5;
      PANN_CUDA(launch_emulate(idx->dtype, idx->metric, true, t, e, 2 * idx->sm_count, smem_need, st));
      glist = ovf;
      grec = ovf_rec;
      gcount = cnt + 8;
    }
    e.gA = ge2;
    e.gB = ge2 + (size_t)e2_slots * capA;
    e.capA = (uint32_t)capA;
    e.capB = (uint32_t)capB;
    e.overflow_list = nullptr;
    e.overflow_rec = nullptr;
    e.overflow_count = nullptr;
    e.job_rec = grec;
    t.job_list = glist;
    t.njobs_dev = gcount;
    t.job_counter = cnt + 7;
    PANN_CUDA(launch_emulate(idx->dtype, idx->metric, false, t, e, e2_slots, emu_smem_bytes(basew, vs, 0, 0, false), st));
  }
  return PANN_OK;
}
