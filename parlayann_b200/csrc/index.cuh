// Internal definition of the index handle behind the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <string>
#include "../../include/parlayann_b200.h"

namespace pann {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define PANN_CUDA(call)                                   \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) return ::pann::cuda_fail(_e, #call); \
  } while (0)

// Largest dynamic shared memory a block may use on the current device. Every
// kernel gets this as its cudaFuncAttributeMaxDynamicSharedMemorySize, whatever
// one launch needs, so threads that launch the same kernel with different
// shared-memory sizes never undo each other's setting.
int smem_attr_max();

// Device scratch buffer that only grows.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want) {
    if (want <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  // as ensure, with room for growth (a buffer whose size follows the
  // request mix is not reallocated, and the device not drained, each time
  // a slightly larger request arrives)
  cudaError_t ensure_grow(size_t want) {
    if (want <= bytes) return cudaSuccess;
    const size_t grown = std::max(want, bytes + bytes / 2);
    if (grown > want && ensure(grown) == cudaSuccess) return cudaSuccess;
    cudaGetLastError();  // no room to spare: exactly what is asked
    return ensure(want);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace pann

struct pann_index {
  int dtype = 0, metric = 0;
  uint64_t n = 0;
  uint32_t d = 0, R = 0;
  uint32_t esize = 1;
  uint64_t stride = 0;  // bytes per device row
  uint32_t nchunks = 0;
  int device = 0;
  int sm_count = 0;
  size_t smem_optin = 0;
  uint8_t* d_points = nullptr;
  uint32_t* d_graph = nullptr;
  bool points_set = false;
  cudaStream_t stream = nullptr;
  // a low-priority stream and two events for the emulation pass that runs
  // beside tier 0's tail (created on first use by a plain search)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // search scratch
  pann::DevBuf q, ids, dists, vis, cmps, status, redo, counters, gtables, gtables2, emu, handoff, starts, tmp;
  // range search: per-query metadata, expansion tables and queues, answer pool, CSR output
  pann::DevBuf range_meta, range_tabs, range_pool, range_out;
  uint64_t range_held = 0;  // ids in range_out left for pann_range_fetch (0: none)
  // precision form: low-precision copy of float32 points (lowprec.cuh)
  pann::DevBuf lp_rows, lp_scales, lp_norms;
  pann::DevBuf order;  // tier-0 job order of a plain search (order.cu)
  int lp_prec = 0;
  uint64_t lp_stride = 0;
  uint32_t lp_chunks = 0;
  // quantized search: an internal uint8 Euclidean index over the one-byte
  // quantized points that reads this index's graph (quant.cu)
  pann_index* quant = nullptr;
  float q_slope = 1.0f;  // mips: the scale
  int32_t q_offset = 0;
  float q_bound = 1.0f;  // mips: the trimmed bound
  bool graph_borrowed = false;  // d_graph belongs to another index
  uint32_t gt_fallbacks = 0;  // queries of the last float groundtruth recomputed by the plain kernel
  uint32_t starts_cached_n = 0;
  uint32_t starts_cached[64] = {};
};

namespace pann {

struct SearchPlan {
  uint32_t k, L, dl;
  uint64_t limit;
  double bf;
  uint32_t n_start;
  uint32_t ref_half;
  uint32_t Ccap;
};

int make_plan(const pann_index* idx, const pann_query_params* qp, uint32_t n_start, SearchPlan* plan);

// Run the tiered search on device buffers (queries already in index row layout).
// self_ids (device, nullable) selects build mode: query j is point self_ids[j].
// precision != 0 runs the precision form (low-precision traversal, exact
// re-rank of the best `rerank` entries).
int run_search(pann_index* idx, const SearchPlan& plan, const uint8_t* d_queries, const uint32_t* d_self_ids,
               uint32_t nq, const uint32_t* d_starts, uint32_t* d_ids, float* d_dists, uint32_t* d_vis,
               uint32_t* d_cmps, uint32_t* d_status, uint64_t* d_vis_keys, uint32_t vis_cap, cudaStream_t st,
               int precision = 0, uint32_t rerank = 0, uint32_t parents = 0, uint32_t scorer = 0);

// A batch laid out in a caller's device arena (the serving form's admission
// by scratch memory): every buffer of one run of nq queries, whose k and beam
// are at most bounds->k and bounds->beam, carved from one allocation.
// batch_scratch_bytes gives the bytes such a run needs; run_in_arena stages
// the inputs (pinned host arrays: nq query rows of d * element bytes, per-query
// k and beam, the job order), enqueues the search on `st` and the copies of
// its ids and distances (nq rows of bounds->k) to pinned host memory.
// Takes range search's largest scratch up front (range.cu).
int range_reserve(pann_index* idx);
int batch_scratch_bytes(const pann_index* idx, const pann_query_params* bounds, uint32_t n_start, uint32_t nq,
                        int precision, uint32_t parents, size_t* bytes);
// A batch laid out in a caller's arena (the serving loop's slots): h_order[nq]
// holds nq in pinned memory; the job order itself is made on the device.
int run_in_arena(pann_index* idx, uint8_t* arena, size_t arena_bytes, const pann_query_params* bounds,
                 const uint32_t* h_starts, uint32_t n_start, const uint8_t* h_queries, uint32_t nq, const uint32_t* h_k,
                 const uint32_t* h_beam, const uint32_t* h_order, int precision, uint32_t rerank, uint32_t parents,
                 uint32_t scorer, uint32_t* h_ids, float* h_dists, cudaStream_t st);

}  // namespace pann
