// C ABI: index lifetime, data upload, graph formats, and the search entry
// points (include/parlayann_b200.h).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "index.cuh"
#include "search.cuh"
#include "search_emu.cuh"
#include "lowprec.cuh"
#include "tiers.cuh"

namespace pann {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  g_last_error = m;
  return e == cudaErrorMemoryAllocation ? PANN_ENOMEM : PANN_EDEVICE;
}

// ------------------------------------------------------------ graph layout kernels
// reference rows (deg, e0..e_{R-1}) -> flat rows (e0..e_{deg-1}, PAD...)
__global__ void graph_from_ref_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint64_t rows,
                                      uint32_t R, uint64_t n_total, uint32_t* bad) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t total = rows * R;
  for (; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t r = t / R;
    uint32_t j = (uint32_t)(t - r * R);
    const uint32_t* src = in + r * (R + 1);
    uint32_t deg = src[0];
    if (deg > R) { atomicOr(bad, 1u); deg = R; }
    uint32_t v = PANN_PAD;
    if (j < deg) {
      v = src[1 + j];
      if ((uint64_t)v >= n_total) { atomicOr(bad, 2u); v = PANN_PAD; }
    }
    out[t] = v;
  }
}
// flat rows -> reference rows
__global__ void graph_to_ref_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint64_t rows,
                                    uint32_t R) {
  uint64_t r = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x & 31;
  for (; r < rows; r += (uint64_t)gridDim.x * (blockDim.x / 32)) {
    const uint32_t* src = in + r * R;
    uint32_t deg = 0;
    for (uint32_t b = 0; b < R; b += 32) {
      uint32_t j = b + lane;
      uint32_t v = j < R ? src[j] : PANN_PAD;
      deg += __popc(__ballot_sync(0xFFFFFFFFu, v != PANN_PAD));
      if (j < R) out[r * (R + 1) + 1 + j] = (v != PANN_PAD) ? v : 0u;
    }
    if (lane == 0) out[r * (R + 1)] = deg;
  }
}

// ------------------------------------------------------------ precision-form conversions
__global__ void to_bf16_kernel(const float* __restrict__ src, uint64_t src_stride_f, uint16_t* dst,
                               uint64_t dst_stride_h, uint64_t n, uint32_t d) {
  uint64_t total = n * (uint64_t)d;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = t / d;
    uint32_t j = (uint32_t)(t - i * d);
    __nv_bfloat16 b = __float2bfloat16_rn(src[i * src_stride_f + j]);
    dst[i * dst_stride_h + j] = *reinterpret_cast<uint16_t*>(&b);
  }
}

// per-dimension max |x| (as float bits: non-negative floats order like unsigned ints)
__global__ void absmax_kernel(const float* __restrict__ src, uint64_t src_stride_f, uint64_t n, uint32_t d,
                              uint32_t* out_bits) {
  for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) {
    float m = 0.0f;
    for (uint64_t i = blockIdx.x; i < n; i += gridDim.x) m = fmaxf(m, fabsf(src[i * src_stride_f + j]));
    atomicMax(out_bits + j, __float_as_uint(m));
  }
}

__global__ void to_fp8_kernel(const float* __restrict__ src, uint64_t src_stride_f, uint8_t* dst, uint64_t dst_stride,
                              uint64_t n, uint32_t d, const float* __restrict__ inv_scale) {
  uint64_t total = n * (uint64_t)d;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = t / d;
    uint32_t j = (uint32_t)(t - i * d);
    __nv_fp8_e4m3 v(src[i * src_stride_f + j] * inv_scale[j]);
    dst[i * dst_stride + j] = *reinterpret_cast<uint8_t*>(&v);
  }
}

// Squared norm of every low-precision row as the tensor-core tile scoring
// uses it: the row dequantized exactly (bfloat16, or E4M3 x the dimension's
// scale), squared and summed in float32.
template <int PREC>
__global__ void lp_norms_kernel(const uint8_t* __restrict__ rows, uint64_t stride, uint64_t n, uint32_t d,
                                const float* __restrict__ scales, float* out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint8_t* r = rows + i * stride;
    float s = 0.0f;
    for (uint32_t t = 0; t < d; t++) {
      float x;
      if (PREC == PREC_BF16) {
        x = __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(r)[t]);
      } else {
        __nv_fp8_e4m3 f;
        *reinterpret_cast<uint8_t*>(&f) = r[t];
        x = float(f) * scales[t];
      }
      s = fmaf(x, x, s);
    }
    out[i] = s;
  }
}

int smem_attr_max() {
  static int cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 48 * 1024;
  if (cached[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || v <= 0) v = 48 * 1024;
    cached[dev] = v;  // the same value from every thread: a benign race
  }
  return cached[dev];
}

int make_plan(const pann_index* idx, const pann_query_params* qp, uint32_t n_start, SearchPlan* plan) {
  if (!qp) return fail(PANN_EINVAL, "query params are NULL");
  if (qp->beam == 0) return fail(PANN_EINVAL, "beam (L) must be positive");
  if (qp->k > qp->beam)
    return fail(PANN_EINVAL, "beam search parameter Q = " + std::to_string(qp->beam) +
                                 " same size or smaller than k = " + std::to_string(qp->k));
  if (qp->degree_limit == 0) return fail(PANN_EINVAL, "degree_limit must be positive");
  if (n_start == 0) return fail(PANN_EINVAL, "beam search expects at least one start point");
  if (n_start > qp->beam) return fail(PANN_EINVAL, "beam search has more starting points than beam size");
  if (!(qp->batch_factor >= 0.0) || qp->batch_factor > 64.0) return fail(PANN_EINVAL, "batch_factor out of range");
  if (qp->beam > 4096) return fail(PANN_EINVAL, "beam (L) above 4096 is not supported");
  plan->k = qp->k;
  plan->L = qp->beam;
  plan->dl = qp->degree_limit;
  plan->limit = qp->limit;
  plan->bf = qp->batch_factor;
  plan->n_start = n_start;
  // hashset<indexType> has_been_seen(2 * (10 + beamSize) * max_degree) (beamSearch.h:66):
  // capacity 2^ceil(log2(n)) (hashset.h:50-54); it grows above capacity/2 entries.
  double cap_n = 2.0 * (10.0 + (double)qp->beam) * (double)qp->degree_limit;
  int bits = (int)std::ceil(std::log2(cap_n));
  uint64_t cap = 1ull << bits;
  plan->ref_half = (uint32_t)std::min<uint64_t>(cap / 2, 0xFFFFFFFFull);
  uint32_t nel = std::min(qp->degree_limit, idx->R);
  uint64_t defer = (uint64_t)std::floor(qp->batch_factor * (double)qp->beam);
  if (qp->limit < 2ull * qp->beam) defer = 0;  // no deferral: candidates are merged every step
  plan->Ccap = (uint32_t)(defer + nel + 1);
  return PANN_OK;
}

static uint32_t pow2_at_least(uint64_t x) {
  uint32_t p = 1;
  while (p < x && p < (1u << 30)) p <<= 1;
  return p;
}

// Tier-0 register budget for float32 Euclidean search: PANN_T0_MINB=4 fits the
// kernel to four 128-thread blocks per SM (128 registers) instead of three.
static int t0_minb() {
  static const int v = [] {
    const char* e = std::getenv("PANN_T0_MINB");
    return e && std::atoi(e) == 4 ? 4 : 3;
  }();
  return v;
}

// The first tier's kernel fitted to `minb` resident 128-thread blocks (3 or 4).
template <int DT, int MT, bool G, int PREC = PREC_F32>
static auto search_kernel_ptr(int minb) {
  if constexpr (!G && PREC == PREC_F32)
    if (minb == 4) return search_kernel<DT, MT, G, PREC, 4>;
  return search_kernel<DT, MT, G, PREC, 3>;
}

template <int DT, int MT, bool G, int PREC = PREC_F32>
static cudaError_t launch_search_t(const SearchArgs& a, int blocks, int threads, size_t smem, cudaStream_t st,
                                   int minb) {
  auto k = search_kernel_ptr<DT, MT, G, PREC>(minb);
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max());
  if (e != cudaSuccess) return e;
  k<<<blocks, threads, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_search(int dtype, int metric, bool global_table, const SearchArgs& a, int blocks,
                                 int threads, size_t smem, cudaStream_t st, int prec, int minb) {
  if (prec != PREC_F32) {
    if (dtype != DT_F32) return cudaErrorInvalidValue;
#define PANN_LP_CASE(MT, PR)                                                               \
    if (metric == MT && prec == PR)                                                        \
      return global_table ? launch_search_t<DT_F32, MT, true, PR>(a, blocks, threads, smem, st, 3) \
                          : launch_search_t<DT_F32, MT, false, PR>(a, blocks, threads, smem, st, 3);
    PANN_LP_CASE(MT_L2, PREC_BF16)
    PANN_LP_CASE(MT_IP, PREC_BF16)
    PANN_LP_CASE(MT_L2, PREC_FP8)
    PANN_LP_CASE(MT_IP, PREC_FP8)
#undef PANN_LP_CASE
    return cudaErrorInvalidValue;
  }
#define PANN_SEARCH_CASE(DT, MT)                                                        \
  if (dtype == DT && metric == MT)                                                      \
    return global_table ? launch_search_t<DT, MT, true>(a, blocks, threads, smem, st, 3)   \
                        : launch_search_t<DT, MT, false>(a, blocks, threads, smem, st, minb);
  PANN_SEARCH_CASE(DT_U8, MT_L2)
  PANN_SEARCH_CASE(DT_U8, MT_IP)
  PANN_SEARCH_CASE(DT_I8, MT_L2)
  PANN_SEARCH_CASE(DT_I8, MT_IP)
  PANN_SEARCH_CASE(DT_F32, MT_L2)
  PANN_SEARCH_CASE(DT_F32, MT_IP)
#undef PANN_SEARCH_CASE
  return cudaErrorInvalidValue;
}

template <int DT, int MT, bool SM>
static cudaError_t launch_emulate_t(const SearchArgs& a, const EmuArgs& e, int blocks, size_t smem, cudaStream_t st) {
  auto k = search_emulate_kernel<DT, MT, SM>;
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max());
  if (err != cudaSuccess) return err;
  k<<<blocks, 32, smem, st>>>(a, e);
  return cudaGetLastError();
}
cudaError_t launch_emulate(int dtype, int metric, bool smem_tables, const SearchArgs& a, const EmuArgs& e,
                                  int blocks, size_t smem, cudaStream_t st) {
#define PANN_EMU_CASE(DT, MT)                                                              \
  if (dtype == DT && metric == MT)                                                         \
    return smem_tables ? launch_emulate_t<DT, MT, true>(a, e, blocks, smem, st)            \
                       : launch_emulate_t<DT, MT, false>(a, e, blocks, smem, st);
  PANN_EMU_CASE(DT_U8, MT_L2)
  PANN_EMU_CASE(DT_U8, MT_IP)
  PANN_EMU_CASE(DT_I8, MT_L2)
  PANN_EMU_CASE(DT_I8, MT_IP)
  PANN_EMU_CASE(DT_F32, MT_L2)
  PANN_EMU_CASE(DT_F32, MT_IP)
#undef PANN_EMU_CASE
  return cudaErrorInvalidValue;
}

template <int DT, int MT>
static cudaError_t launch_emulate_block_t(const SearchArgs& a, const EmuArgs& e, int blocks, size_t smem,
                                          cudaStream_t st) {
  auto k = search_emulate_block_kernel<DT, MT, EMU_BLOCK_WARPS, 24>;
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max());
  if (err != cudaSuccess) return err;
  k<<<blocks, 32 * EMU_BLOCK_WARPS, smem, st>>>(a, e);
  return cudaGetLastError();
}
cudaError_t launch_emulate_block(int dtype, int metric, const SearchArgs& a, const EmuArgs& e, int blocks, size_t smem,
                                 cudaStream_t st) {
#define PANN_EMUB_CASE(DT, MT) \
  if (dtype == DT && metric == MT) return launch_emulate_block_t<DT, MT>(a, e, blocks, smem, st);
  PANN_EMUB_CASE(DT_U8, MT_L2)
  PANN_EMUB_CASE(DT_U8, MT_IP)
  PANN_EMUB_CASE(DT_I8, MT_L2)
  PANN_EMUB_CASE(DT_I8, MT_IP)
  PANN_EMUB_CASE(DT_F32, MT_L2)
  PANN_EMUB_CASE(DT_F32, MT_IP)
#undef PANN_EMUB_CASE
  return cudaErrorInvalidValue;
}

template <int DT, int MT, bool G, int PREC = PREC_F32>
static int occupancy_t(int threads, size_t smem, int minb = 3) {
  int nb = 0;
  auto k = search_kernel_ptr<DT, MT, G, PREC>(minb);
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max());
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, threads, smem) != cudaSuccess) return 0;
  return nb;
}
int search_occupancy(int dtype, int metric, bool g, int threads, size_t smem, int minb) {
#define PANN_OCC_CASE(DT, MT) \
  if (dtype == DT && metric == MT) \
    return g ? occupancy_t<DT, MT, true>(threads, smem) : occupancy_t<DT, MT, false>(threads, smem, minb);
  PANN_OCC_CASE(DT_U8, MT_L2)
  PANN_OCC_CASE(DT_U8, MT_IP)
  PANN_OCC_CASE(DT_I8, MT_L2)
  PANN_OCC_CASE(DT_I8, MT_IP)
  PANN_OCC_CASE(DT_F32, MT_L2)
  PANN_OCC_CASE(DT_F32, MT_IP)
#undef PANN_OCC_CASE
  return 0;
}

static int lp_occupancy(int metric, int prec, int threads, size_t smem) {
  if (metric == MT_L2 && prec == PREC_BF16) return occupancy_t<DT_F32, MT_L2, false, PREC_BF16>(threads, smem);
  if (metric == MT_IP && prec == PREC_BF16) return occupancy_t<DT_F32, MT_IP, false, PREC_BF16>(threads, smem);
  if (metric == MT_L2 && prec == PREC_FP8) return occupancy_t<DT_F32, MT_L2, false, PREC_FP8>(threads, smem);
  if (metric == MT_IP && prec == PREC_FP8) return occupancy_t<DT_F32, MT_IP, false, PREC_FP8>(threads, smem);
  return 0;
}

// Shared-memory seen-table slots of tier 0: the PANN_SEEN_SLOTS environment
// variable, else the power of two at or above (L + 16) * min(dl, R) * 2/3
// (about 3/4-load room for the ids a search typically sees), between 4 (R + 1)
// and 8192 slots; queries that need more continue in the per-warp global
// spill table. Doubling the table halves the warps that fit on an SM, so the
// estimate errs small.
uint32_t tier0_slots(const SearchPlan& p, uint32_t R) {
  uint32_t floor_s = pow2_at_least(4ull * (R + 1));
  if (const char* e = std::getenv("PANN_SEEN_SLOTS")) {
    long v = std::atol(e);
    if (v > 0) return std::max<uint32_t>(pow2_at_least((uint64_t)v), floor_s);
  }
  uint32_t nel = std::min(p.dl, R);
  uint64_t est = (uint64_t)(p.L + 16) * nel * 2 / 3;
  uint32_t s = pow2_at_least(est);
  s = std::min<uint32_t>(s, 8192);
  return std::max<uint32_t>(s, floor_s);
}

// Tiers: (0) every query, many warps per SM, shared-memory seen table with a
// global spill table; (2) queries whose tables still filled up, with one large
// global table per warp; (E) queries on which the reference's hashset grows,
// re-run with that hashset emulated exactly.
int size_tiers(const pann_index* idx, const SearchPlan& plan, uint64_t nq, int precision, uint32_t S_force,
               int wpb_force, TierSizes* z, int minb_force) {
  const size_t smem_cap = idx->smem_optin;
  TierSizes& t = *z;
  t = TierSizes{};
  // ---- tier 0
  uint32_t S = S_force ? std::max<uint32_t>(pow2_at_least(S_force), pow2_at_least(4ull * (idx->R + 1)))
                       : tier0_slots(plan, idx->R);
  uint32_t wb = search_warp_bytes(idx->stride, plan.L, plan.Ccap, idx->R, S, false);
  int wpb = wpb_force > 0 ? std::min(wpb_force, 4) : 4;
  while (wpb > 1 && (size_t)wb * wpb > smem_cap) wpb >>= 1;
  while ((size_t)wb * wpb > smem_cap && S > pow2_at_least(4ull * (idx->R + 1))) {
    S >>= 1;
    wb = search_warp_bytes(idx->stride, plan.L, plan.Ccap, idx->R, S, false);
  }
  if ((size_t)wb * wpb > smem_cap) return fail(PANN_EINVAL, "search state for this beam does not fit in shared memory");
  t.minb = precision == PREC_F32 ? (minb_force == 4 || (minb_force == 0 && t0_minb() == 4) ? 4 : 3) : 3;
  int occ = precision == PREC_F32 ? search_occupancy(idx->dtype, idx->metric, false, 32 * wpb, (size_t)wb * wpb, t.minb)
                                  : lp_occupancy(idx->metric, precision, 32 * wpb, (size_t)wb * wpb);
  if (occ <= 0) occ = 1;
  uint64_t want = (std::max<uint64_t>(nq, 1) + wpb - 1) / wpb;
  t.S = S;
  t.wb = wb;
  t.wpb = wpb;
  t.blocks = (int)std::min<uint64_t>(want, (uint64_t)occ * idx->sm_count);
  t.slots = (size_t)t.blocks * wpb;
  uint32_t Sg = std::max<uint32_t>(4 * S, pow2_at_least(2ull * plan.ref_half));
  while (Sg > 4 * S && t.slots * Sg * 4 > (1ull << 30)) Sg >>= 1;
  t.Sg = Sg;
  t.spill_bytes = t.slots * Sg * 4;
  // ---- hand-off buffers: per-warp insertion/visit logs and the resume records
  t.logcap = plan.ref_half;
  t.viscap = pow2_at_least(8ull * plan.L + 64);
  t.ly = resume_layout(plan.L, plan.Ccap, t.logcap, t.viscap);
  t.rec_cap = std::min<uint64_t>(std::max<uint64_t>(nq, 1), std::max<uint64_t>(64, (256ull << 20) / (4ull * t.ly.words)));
  t.handoff_bytes = 4ull * (t.slots * (size_t)(t.logcap + t.viscap) + t.rec_cap * t.ly.words);
  // ---- tier 2
  t.S2 = std::min<uint32_t>(std::max<uint32_t>(1u << 16, pow2_at_least(4ull * plan.ref_half)), 1u << 24);
  t.t2_slots = (int)std::max<uint64_t>(1, std::min<uint64_t>(2ull * idx->sm_count, (256ull << 20) / (4ull * t.S2)));
  t.wb2 = search_warp_bytes(idx->stride, plan.L, plan.Ccap, idx->R, t.S2, true);
  t.t2_bytes = (size_t)t.t2_slots * t.S2 * 4;
  // ---- emulation tiers
  double cap_n = 2.0 * (10.0 + (double)plan.L) * (double)plan.dl;
  t.bits0 = (uint32_t)std::ceil(std::log2(cap_n));
  t.S0 = 1ull << t.bits0;
  t.vs = pow2_at_least(8ull * plan.L + 64);
  t.base = search_warp_bytes(idx->stride, plan.L, plan.Ccap, idx->R, 0, true);
  t.emu_smem_need = emu_block_layout(idx->stride, plan.L, plan.Ccap, idx->R, t.vs, (uint32_t)(4 * t.S0),
                                     (uint32_t)(2 * t.S0)).bytes;
  t.emu_smem = 4 * t.S0 < (1ull << 30) && t.emu_smem_need <= smem_cap;
  t.capA = 16 * t.S0;
  t.capB = 8 * t.S0;
  size_t per_slot = 4ull * (t.capA + t.capB);
  t.e2_slots = (int)std::max<uint64_t>(1, std::min<uint64_t>(idx->sm_count, (1ull << 30) / per_slot));
  t.e2_bytes = per_slot * t.e2_slots;
  return PANN_OK;
}

int enqueue_tiers(const pann_index* idx, const SearchPlan& plan, const SearchArgs& a0, const TierSizes& z,
                  const TierBufs& b, cudaStream_t st, int precision, uint32_t rerank, cudaStream_t side) {
  uint32_t* cnt = b.cnt;
  PANN_CUDA(cudaMemsetAsync(cnt, 0, 64, st));
  // an emulation pass beside tier 0's tail: its blocks need most of an SM's
  // shared memory, so they start only as tier 0's blocks leave the SMs
  const bool early = side && idx->ev_fork && idx->ev_join && precision == PREC_F32 && z.emu_smem && !z.cta;
  if (early) {
    PANN_CUDA(cudaMemsetAsync(b.emu_rec, 0xFE, sizeof(uint32_t) * (size_t)std::max<uint32_t>(a0.nq, 1), st));
    PANN_CUDA(cudaEventRecord(idx->ev_fork, st));
    PANN_CUDA(cudaStreamWaitEvent(side, idx->ev_fork, 0));
  }
  SearchArgs a = a0;
  a.emu_list = b.emu;
  a.emu_rec = b.emu_rec;
  a.emu_count = cnt + 6;
  if (precision != PREC_F32) {
    if (idx->lp_prec != precision) return fail(PANN_EINVAL, "pann_index_set_precision was not called for this precision");
    a.emu_list = nullptr;  // the precision form is not a reference path: no hashset emulation
    a.lp_rows = idx->lp_rows.as<uint8_t>();
    a.lp_stride = idx->lp_stride;
    a.lp_chunks = idx->lp_chunks;
    a.lp_scales = idx->lp_scales.as<float>();
    a.rerank = rerank;  // 0: 4k per query
  }
  // ---- tier 0: many warps per SM, a modest shared-memory seen table that
  // spills into a per-warp global table for the queries that outgrow it
  {
    SearchArgs t = a;
    t.S = z.S;
    t.warp_bytes = z.wb;
    t.job_counter = cnt + 0;
    t.job_list = b.job_list0;
    t.njobs_dev = b.njobs0;
    t.redo_list = b.redo0;
    t.redo_count = cnt + 3;
    if (b.handoff) {
      t.inslog = b.handoff;
      t.logcap = z.logcap;
      t.vislog = t.inslog + z.slots * (size_t)z.logcap;
      t.viscap = z.viscap;
      t.rec_pool = t.vislog + z.slots * (size_t)z.viscap;
      t.rec_cap = (uint32_t)z.rec_cap;
      t.rec_words = z.ly.words;
      t.rec_count = cnt + 9;
      a.logcap = z.logcap;  // the emulation tiers read the record layout
      a.viscap = z.viscap;
      a.rec_pool = t.rec_pool;
      a.rec_words = z.ly.words;
    } else {
      t.inslog = nullptr;
    }
    t.gspill = b.gspill;
    t.Sg = b.gspill ? z.Sg : 0;
    if (z.cta && precision == PREC_F32 && z.emu_smem) {
      // CTA per query: every query on a block of the exact-emulation kernel from its start points
      // (the same answers: that kernel is the reference's search with its hashset as written);
      // queries whose emulated table outgrows shared memory continue in the global tier below
      SearchArgs c = a;
      c.redo_list = nullptr;
      c.redo_count = nullptr;
      c.emu_list = nullptr;
      c.emu_count = nullptr;
      c.job_list = b.job_list0;
      c.njobs_dev = b.njobs0;
      c.job_counter = cnt + 5;
      EmuArgs e{};
      e.bits0 = z.bits0;
      e.vs_slots = z.vs;
      e.base_bytes = z.base;
      e.capA = (uint32_t)(4 * z.S0);
      e.capB = (uint32_t)(2 * z.S0);
      e.overflow_list = b.ovf;
      e.overflow_rec = b.ovf_rec;
      e.overflow_count = cnt + 8;
      e.job_rec = nullptr;
      PANN_CUDA(launch_emulate_block(idx->dtype, idx->metric, c, e, (int)std::min<uint64_t>(idx->sm_count, a.nq),
                                     z.emu_smem_need, st));
      EmuArgs e2 = e;
      e2.gA = b.ge2;
      e2.gB = e2.gA + (size_t)z.e2_slots * z.capA;
      e2.capA = (uint32_t)z.capA;
      e2.capB = (uint32_t)z.capB;
      e2.overflow_list = nullptr;
      e2.overflow_rec = nullptr;
      e2.overflow_count = nullptr;
      e2.job_rec = b.ovf_rec;
      c.job_list = b.ovf;
      c.njobs_dev = cnt + 8;
      c.job_counter = cnt + 7;
      PANN_CUDA(launch_emulate(idx->dtype, idx->metric, false, c, e2, z.e2_slots,
                               emu_smem_bytes(z.base, z.vs, 0, 0, false), st));
      return PANN_OK;
    }
    PANN_CUDA(launch_search(idx->dtype, idx->metric, false, t, z.blocks, 32 * z.wpb, (size_t)z.wb * z.wpb, st, precision,
                            z.minb));
  }
  if (early) {
    SearchArgs t = a;
    t.redo_list = nullptr;
    t.redo_count = nullptr;
    t.emu_list = nullptr;
    t.emu_count = nullptr;
    t.job_list = b.emu;
    t.njobs_dev = cnt + 6;
    t.job_counter = cnt + 5;
    EmuArgs e{};
    e.bits0 = z.bits0;
    e.vs_slots = z.vs;
    e.base_bytes = z.base;
    e.capA = (uint32_t)(4 * z.S0);
    e.capB = (uint32_t)(2 * z.S0);
    e.overflow_list = b.ovf;
    e.overflow_rec = b.ovf_rec;
    e.overflow_count = cnt + 8;
    e.job_rec = b.emu_rec;
    e.early = 1;
    PANN_CUDA(launch_emulate_block(idx->dtype, idx->metric, t, e, (int)std::min<uint64_t>(idx->sm_count, a.nq),
                                   z.emu_smem_need, side));
    PANN_CUDA(cudaEventRecord(idx->ev_join, side));
  }
  // ---- tier 2: queries whose tables still filled up, with one global-memory
  // seen table per warp sized above the reference's own capacity
  {
    SearchArgs t = a;
    t.S = z.S2;
    t.warp_bytes = z.wb2;
    t.gtables = b.gt2;
    t.inslog = nullptr;
    t.job_list = b.redo0;
    t.njobs_dev = cnt + 3;
    t.job_counter = cnt + 2;
    t.redo_list = nullptr;
    t.redo_count = nullptr;
    PANN_CUDA(launch_search(idx->dtype, idx->metric, true, t, z.t2_slots, 32, z.wb2, st, precision));
  }
  if (precision != PREC_F32) return PANN_OK;
  // ---- tier E: exact emulation of the reference's hashset for flagged queries,
  // first with the emulated table in shared memory (capacities 4 S0 / 2 S0),
  // then, for queries that outgrow it, in global memory (16 S0 / 8 S0)
  {
    SearchArgs t = a;
    t.redo_list = nullptr;
    t.redo_count = nullptr;
    t.emu_list = nullptr;
    t.emu_count = nullptr;
    EmuArgs e{};
    e.bits0 = z.bits0;
    e.vs_slots = z.vs;
    e.base_bytes = z.base;
    const uint32_t* glist = b.emu;
    uint32_t* gcount = cnt + 6;
    const uint32_t* grec = b.emu_rec;
    if (z.emu_smem) {
      e.capA = (uint32_t)(4 * z.S0);
      e.capB = (uint32_t)(2 * z.S0);
      e.overflow_list = b.ovf;
      e.overflow_rec = b.ovf_rec;
      e.overflow_count = cnt + 8;
      e.job_rec = b.emu_rec;
      t.job_list = b.emu;
      t.njobs_dev = cnt + 6;
      t.job_counter = cnt + 5;
      // no more blocks than queries: each needs most of an SM's shared memory,
      // so a small search beside other work on the device asks for few SMs
      PANN_CUDA(launch_emulate_block(idx->dtype, idx->metric, t, e, (int)std::min<uint64_t>(idx->sm_count, a.nq),
                                     z.emu_smem_need, st));
      glist = b.ovf;
      grec = b.ovf_rec;
      gcount = cnt + 8;
    }
    // the pass beside tier 0 adds to the overflow list too
    if (early) PANN_CUDA(cudaStreamWaitEvent(st, idx->ev_join, 0));
    e.gA = b.ge2;
    e.gB = e.gA + (size_t)z.e2_slots * z.capA;
    e.capA = (uint32_t)z.capA;
    e.capB = (uint32_t)z.capB;
    e.overflow_list = nullptr;
    e.overflow_rec = nullptr;
    e.overflow_count = nullptr;
    e.job_rec = grec;
    t.job_list = glist;
    t.njobs_dev = gcount;
    t.job_counter = cnt + 7;
    PANN_CUDA(launch_emulate(idx->dtype, idx->metric, false, t, e, z.e2_slots, emu_smem_bytes(z.base, z.vs, 0, 0, false),
                             st));
  }
  return PANN_OK;
}

// Fills the search arguments every tier shares.
SearchArgs base_args(const pann_index* idx, const SearchPlan& plan, const uint8_t* d_queries,
                     const uint32_t* d_self_ids, uint32_t nq, const uint32_t* d_starts, uint32_t* d_ids,
                     float* d_dists, uint32_t* d_vis, uint32_t* d_cmps, uint32_t* d_status, uint64_t* d_vis_keys,
                     uint32_t vis_cap) {
  SearchArgs a{};
  a.points = idx->d_points;
  a.stride = idx->stride;
  a.d = idx->d;
  a.nchunks = idx->nchunks;
  a.graph = idx->d_graph;
  a.R = idx->R;
  a.queries = d_queries;
  a.self_ids = d_self_ids;
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
  a.out_ids = d_ids;
  a.out_dists = d_dists;
  a.out_visited = d_vis;
  a.out_cmps = d_cmps;
  a.out_status = d_status;
  a.vis_keys = d_vis_keys;
  a.vis_cap = vis_cap;
  a.opaque_zero = 0;
  return a;
}

// PANN_T0_ORDER=0: search jobs in the given query order.
static bool t0_keep_order() {
  static const bool keep = [] {
    const char* e = std::getenv("PANN_T0_ORDER");
    return e && e[0] == '0';
  }();
  return keep;
}

// The index's side stream (lowest priority) and its fork / join events,
// created on first use; nullptr if they cannot be created (the emulation
// then runs only after the search tiers). PANN_EMU_OVERLAP=0 turns the
// overlapped pass off.
static cudaStream_t side_stream(pann_index* idx) {
  static const bool off = [] {
    const char* e = std::getenv("PANN_EMU_OVERLAP");
    return e && e[0] == '0';
  }();
  if (off) return nullptr;
  if (!idx->side) {
    int lo = 0, hi = 0;
    if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) lo = 0;
    cudaStream_t s = nullptr;
    cudaEvent_t f = nullptr, j = nullptr;
    if (cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, lo) != cudaSuccess ||
        cudaEventCreateWithFlags(&f, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&j, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      if (s) cudaStreamDestroy(s);
      if (f) cudaEventDestroy(f);
      if (j) cudaEventDestroy(j);
      return nullptr;
    }
    idx->side = s;
    idx->ev_fork = f;
    idx->ev_join = j;
  }
  return idx->side;
}

int run_search(pann_index* idx, const SearchPlan& plan, const uint8_t* d_queries, const uint32_t* d_self_ids,
               uint32_t nq, const uint32_t* d_starts, uint32_t* d_ids, float* d_dists, uint32_t* d_vis,
               uint32_t* d_cmps, uint32_t* d_status, uint64_t* d_vis_keys, uint32_t vis_cap, cudaStream_t st,
               int precision, uint32_t rerank, uint32_t parents, uint32_t scorer) {
  if (nq == 0) return PANN_OK;
  if (precision != PREC_F32 && idx->lp_prec != precision)
    return fail(PANN_EINVAL, "pann_index_set_precision was not called for this precision");
  if (parents > 0 && precision != PREC_F32 && d_self_ids == nullptr) {
    PANN_CUDA(idx->counters.ensure(64));
    SearchArgs a = base_args(idx, plan, d_queries, nullptr, nq, d_starts, d_ids, d_dists, d_vis, d_cmps, d_status,
                             nullptr, 0);
    if (!t0_keep_order() && nq > 4u * (uint32_t)idx->sm_count) {
      const uint32_t* order = nullptr;
      int orc = order_far_first(idx, d_queries, nullptr, d_starts, nq, st, &order);
      if (orc) return orc;
      a.job_list = order;  // one CTA per query: the far queries first as well
    }
    int rc = enqueue_tile(idx, plan, a, parents, idx->counters.as<uint32_t>() + 10, precision, rerank, st, scorer);
    if (rc != PANN_EINVAL) return rc;  // EINVAL: does not fit; take the single-parent path
  }
  TierSizes z;
  int rc = size_tiers(idx, plan, nq, precision, 0, 0, &z);
  if (rc) return rc;
  TierBufs b{};
  rc = index_tier_buffers(idx, z, nq, precision, &b);
  if (rc) return rc;
  SearchArgs a = base_args(idx, plan, d_queries, d_self_ids, nq, d_starts, d_ids, d_dists, d_vis, d_cmps, d_status,
                           d_vis_keys, vis_cap);
  // queries far from the start point first, where they queue for tier 0's warps
  if (!t0_keep_order() && nq > z.slots) {
    const uint32_t* order = nullptr;
    rc = order_far_first(idx, d_queries, d_self_ids, d_starts, nq, st, &order);
    if (rc) return rc;
    b.job_list0 = order;
  }
  return enqueue_tiers(idx, plan, a, z, b, st, precision, rerank, side_stream(idx));
}

int index_tier_buffers(pann_index* idx, const TierSizes& z, uint32_t nq, int precision, TierBufs* out) {
  // counters: [0..2] job counters per tier, [3] redo count 0, [4] redo count 1,
  // [5] shared-memory emulation job counter, [6] emulation list length,
  // [7] global emulation job counter, [8] emulation overflow count,
  // [9] resume records taken
  PANN_CUDA(idx->counters.ensure(64));
  PANN_CUDA(idx->redo.ensure_grow(sizeof(uint32_t) * 6 * (size_t)std::max<uint32_t>(nq, 1)));
  TierBufs& b = *out;
  b = TierBufs{};
  b.cnt = idx->counters.as<uint32_t>();
  b.redo0 = idx->redo.as<uint32_t>();
  b.redo1 = b.redo0 + nq;
  b.emu = b.redo1 + nq;
  b.ovf = b.emu + nq;
  b.emu_rec = b.ovf + nq;
  b.ovf_rec = b.emu_rec + nq;
  // the spill table and the hand-off buffers are optional: without them
  // queries re-run in the later tiers
  if (precision == PREC_F32) {
    if (idx->handoff.ensure_grow(z.handoff_bytes) == cudaSuccess) b.handoff = idx->handoff.as<uint32_t>();
    else cudaGetLastError();
  }
  if (idx->gtables.ensure_grow(z.spill_bytes) == cudaSuccess) b.gspill = idx->gtables.as<uint32_t>();
  else cudaGetLastError();
  PANN_CUDA(idx->gtables2.ensure_grow(z.t2_bytes));
  b.gt2 = idx->gtables2.as<uint32_t>();
  if (precision == PREC_F32) {
    PANN_CUDA(idx->emu.ensure_grow(z.e2_bytes));
    b.ge2 = idx->emu.as<uint32_t>();
  }
  return PANN_OK;
}

static int check_index(const pann_index* idx, bool need_graph) {
  if (!idx) return fail(PANN_EINVAL, "index is NULL");
  if (!idx->points_set) return fail(PANN_EINVAL, "index has no points (pann_index_set_points)");
  (void)need_graph;
  return PANN_OK;
}

int stage_starts(pann_index* idx, const uint32_t* starts, uint32_t n_start, cudaStream_t st) {
  if (!starts) return fail(PANN_EINVAL, "start points are NULL");
  for (uint32_t i = 0; i < n_start; i++) {
    if ((uint64_t)starts[i] >= idx->n) return fail(PANN_EINVAL, "start point id out of range");
    for (uint32_t j = 0; j < i; j++)
      if (starts[j] == starts[i]) return fail(PANN_EINVAL, "duplicate start point");
  }
  bool same = n_start == idx->starts_cached_n && n_start <= 64 &&
              std::memcmp(starts, idx->starts_cached, sizeof(uint32_t) * n_start) == 0;
  if (same) return PANN_OK;
  PANN_CUDA(idx->starts.ensure(sizeof(uint32_t) * std::max<uint32_t>(n_start, 16)));
  PANN_CUDA(cudaMemcpyAsync(idx->starts.p, starts, sizeof(uint32_t) * n_start, cudaMemcpyHostToDevice, st));
  PANN_CUDA(cudaStreamSynchronize(st));  // starts may live on the caller's stack
  if (n_start <= 64) {
    std::memcpy(idx->starts_cached, starts, sizeof(uint32_t) * n_start);
    idx->starts_cached_n = n_start;
  } else {
    idx->starts_cached_n = 0;
  }
  return PANN_OK;
}

// status bits -> caller flags: bit0 = reference hashset would grow
static int summarize_status(const uint32_t* status, uint32_t nq, uint32_t* out_flags) {
  int rc = PANN_OK;
  for (uint32_t i = 0; i < nq; i++) {
    uint32_t s = status[i];
    if (out_flags) out_flags[i] = ((s & QS_REF_WOULD_GROW) ? 1u : 0u) | ((s & 32u) ? 2u : 0u);
    if (s & (QS_TABLE_FULL | QS_INTERNAL)) rc = PANN_EOVERFLOW;
    else if ((s & QS_SHORT) && rc == PANN_OK) rc = PANN_ESHORT;
  }
  if (rc == PANN_EOVERFLOW) set_error("a query's seen-set outgrew the largest table");
  if (rc == PANN_ESHORT) set_error("beam search returned fewer than k results");
  return rc;
}

}  // namespace pann

using namespace pann;

extern "C" {

const char* pann_last_error(void) { return g_last_error.c_str(); }

int pann_index_create(pann_index** out, int dtype, int metric, uint64_t n, uint32_t d, uint32_t R) {
  if (!out) return fail(PANN_EINVAL, "out is NULL");
  *out = nullptr;
  if (dtype < 0 || dtype > 2) return fail(PANN_EINVAL, "dtype must be PANN_U8, PANN_I8 or PANN_F32");
  if (metric < 0 || metric > 1) return fail(PANN_EINVAL, "metric must be PANN_L2 or PANN_MIPS");
  if (n == 0 || n >= 0x7FFFFFFFull) return fail(PANN_EINVAL, "n must be in [1, 2^31-1)");
  if (d == 0 || d > 8192) return fail(PANN_EINVAL, "dimension must be in [1, 8192]");
  if (R == 0 || R > 1024) return fail(PANN_EINVAL, "max degree R must be in [1, 1024]");
  int dev = 0;
  PANN_CUDA(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  PANN_CUDA(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10) return fail(PANN_EDEVICE, "this library is built for sm_100a (B200); device is sm_" +
                                                     std::to_string(prop.major) + std::to_string(prop.minor));
  pann_index* idx = new pann_index();
  idx->dtype = dtype;
  idx->metric = metric;
  idx->n = n;
  idx->d = d;
  idx->R = R;
  idx->esize = dtype == PANN_F32 ? 4 : 1;
  idx->stride = ((uint64_t)d * idx->esize + 15) & ~15ull;
  idx->nchunks = (uint32_t)(idx->stride / 16);
  idx->device = dev;
  idx->sm_count = prop.multiProcessorCount;
  idx->smem_optin = prop.sharedMemPerBlockOptin;
  cudaError_t e = cudaStreamCreateWithFlags(&idx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&idx->d_points, idx->stride * n);
  if (e == cudaSuccess) e = cudaMalloc(&idx->d_graph, sizeof(uint32_t) * (size_t)R * n);
  if (e == cudaSuccess) e = cudaMemset(idx->d_graph, 0xFF, sizeof(uint32_t) * (size_t)R * n);
  if (e != cudaSuccess) {
    int rc = cuda_fail(e, "index allocation");
    pann_index_destroy(idx);
    return rc;
  }
  *out = idx;
  return PANN_OK;
}

int pann_index_destroy(pann_index* idx) {
  if (!idx) return PANN_OK;
  if (idx->stream) cudaStreamSynchronize(idx->stream);
  if (idx->side) cudaStreamSynchronize(idx->side);
  if (idx->quant) pann_index_destroy(idx->quant);
  if (idx->d_points) cudaFree(idx->d_points);
  if (idx->d_graph && !idx->graph_borrowed) cudaFree(idx->d_graph);
  for (DevBuf* b : {&idx->q, &idx->ids, &idx->dists, &idx->vis, &idx->cmps, &idx->status, &idx->redo,
                    &idx->counters, &idx->gtables, &idx->gtables2, &idx->emu, &idx->handoff, &idx->starts,
                    &idx->tmp, &idx->lp_rows, &idx->lp_scales, &idx->range_meta, &idx->range_tabs,
                    &idx->range_pool, &idx->range_out})
    b->release();
  idx->lp_norms.release();
  idx->order.release();
  if (idx->ev_fork) cudaEventDestroy(idx->ev_fork);
  if (idx->ev_join) cudaEventDestroy(idx->ev_join);
  if (idx->side) cudaStreamDestroy(idx->side);
  if (idx->stream) cudaStreamDestroy(idx->stream);
  delete idx;
  return PANN_OK;
}

int pann_index_set_points(pann_index* idx, const void* vectors, int on_device) {
  if (!idx || !vectors) return fail(PANN_EINVAL, "index or vectors is NULL");
  size_t rb = (size_t)idx->d * idx->esize;
  PANN_CUDA(cudaMemsetAsync(idx->d_points, 0, idx->stride * idx->n, idx->stream));
  PANN_CUDA(cudaMemcpy2DAsync(idx->d_points, idx->stride, vectors, rb, rb, idx->n,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, idx->stream));
  PANN_CUDA(cudaStreamSynchronize(idx->stream));
  idx->points_set = true;
  return PANN_OK;
}

int pann_graph_upload(pann_index* idx, const uint32_t* rows, int on_device) {
  if (!idx || !rows) return fail(PANN_EINVAL, "index or rows is NULL");
  const uint64_t R = idx->R, n = idx->n;
  const uint64_t chunk = std::max<uint64_t>(1, (256ull << 20) / (4 * (R + 1)));
  PANN_CUDA(idx->tmp.ensure(4 * (R + 1) * std::min(chunk, n) + 64));
  uint32_t* bad = reinterpret_cast<uint32_t*>(idx->tmp.as<uint8_t>() + 4 * (R + 1) * std::min(chunk, n));
  PANN_CUDA(cudaMemsetAsync(bad, 0, 4, idx->stream));
  for (uint64_t r0 = 0; r0 < n; r0 += chunk) {
    uint64_t rows_here = std::min(chunk, n - r0);
    PANN_CUDA(cudaMemcpyAsync(idx->tmp.p, rows + r0 * (R + 1), 4 * (R + 1) * rows_here,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, idx->stream));
    int blocks = (int)std::min<uint64_t>((rows_here * R + 255) / 256, 65535ull * 4);
    graph_from_ref_kernel<<<blocks, 256, 0, idx->stream>>>(idx->tmp.as<uint32_t>(), idx->d_graph + r0 * R,
                                                            rows_here, (uint32_t)R, n, bad);
    PANN_CUDA(cudaGetLastError());
  }
  uint32_t hbad = 0;
  PANN_CUDA(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, idx->stream));
  PANN_CUDA(cudaStreamSynchronize(idx->stream));
  if (hbad & 1u) return fail(PANN_EINVAL, "graph row degree exceeds max degree");
  if (hbad & 2u) return fail(PANN_EINVAL, "graph neighbour id out of range");
  return PANN_OK;
}

int pann_graph_download(pann_index* idx, uint32_t* rows) {
  if (!idx || !rows) return fail(PANN_EINVAL, "index or rows is NULL");
  const uint64_t R = idx->R, n = idx->n;
  const uint64_t chunk = std::max<uint64_t>(1, (256ull << 20) / (4 * (R + 1)));
  PANN_CUDA(idx->tmp.ensure(4 * (R + 1) * std::min(chunk, n) + 64));
  PANN_CUDA(cudaMemsetAsync(idx->tmp.p, 0, 4 * (R + 1) * std::min(chunk, n), idx->stream));
  for (uint64_t r0 = 0; r0 < n; r0 += chunk) {
    uint64_t rows_here = std::min(chunk, n - r0);
    int blocks = (int)std::min<uint64_t>((rows_here + 7) / 8, 65535ull * 4);
    graph_to_ref_kernel<<<blocks, 256, 0, idx->stream>>>(idx->d_graph + r0 * R, idx->tmp.as<uint32_t>(), rows_here,
                                                          (uint32_t)R);
    PANN_CUDA(cudaGetLastError());
    PANN_CUDA(cudaMemcpyAsync(rows + r0 * (R + 1), idx->tmp.p, 4 * (R + 1) * rows_here, cudaMemcpyDeviceToHost,
                              idx->stream));
  }
  PANN_CUDA(cudaStreamSynchronize(idx->stream));
  return PANN_OK;
}

int pann_graph_save(pann_index* idx, const char* path) {
  if (!idx || !path) return fail(PANN_EINVAL, "index or path is NULL");
  const uint64_t R = idx->R, n = idx->n;
  std::vector<uint32_t> rows((size_t)(n * (R + 1)));
  int rc = pann_graph_download(idx, rows.data());
  if (rc) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(PANN_EINVAL, std::string("cannot open graph file for writing: ") + path);
  uint32_t pre[2] = {(uint32_t)n, (uint32_t)R};
  bool ok = std::fwrite(pre, 4, 2, f) == 2;
  std::vector<uint32_t> deg((size_t)n);
  for (uint64_t i = 0; i < n; i++) deg[i] = rows[i * (R + 1)];
  ok = ok && std::fwrite(deg.data(), 4, (size_t)n, f) == (size_t)n;
  for (uint64_t i = 0; i < n && ok; i++)
    if (deg[i]) ok = std::fwrite(&rows[i * (R + 1) + 1], 4, deg[i], f) == deg[i];
  std::fclose(f);
  if (!ok) return fail(PANN_EINVAL, std::string("short write to graph file: ") + path);
  return PANN_OK;
}

int pann_graph_load(pann_index* idx, const char* path) {
  if (!idx || !path) return fail(PANN_EINVAL, "index or path is NULL");
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(PANN_EINVAL, std::string("graph file ") + path + " not found");
  uint32_t pre[2];
  if (std::fread(pre, 4, 2, f) != 2) { std::fclose(f); return fail(PANN_EINVAL, "graph file too short"); }
  const uint64_t n = pre[0], R = pre[1];
  if (n != idx->n || R > idx->R) {
    std::fclose(f);
    return fail(PANN_EINVAL, "graph file has n=" + std::to_string(n) + ", maxDeg=" + std::to_string(R) +
                                 " but the index has n=" + std::to_string(idx->n) + ", R=" + std::to_string(idx->R));
  }
  const uint64_t RI = idx->R;
  std::vector<uint32_t> deg((size_t)n);
  if (std::fread(deg.data(), 4, (size_t)n, f) != (size_t)n) { std::fclose(f); return fail(PANN_EINVAL, "graph file truncated"); }
  std::vector<uint32_t> rows((size_t)(n * (RI + 1)), 0);
  for (uint64_t i = 0; i < n; i++) {
    if (deg[i] > R) { std::fclose(f); return fail(PANN_EINVAL, "graph file degree exceeds maxDeg"); }
    rows[i * (RI + 1)] = deg[i];
    if (deg[i] && std::fread(&rows[i * (RI + 1) + 1], 4, deg[i], f) != deg[i]) {
      std::fclose(f);
      return fail(PANN_EINVAL, "graph file truncated");
    }
  }
  std::fclose(f);
  return pann_graph_upload(idx, rows.data(), 0);
}

int pann_search_device(pann_index* idx, const void* d_queries, uint32_t nq, const pann_query_params* qp,
                       const uint32_t* starts, uint32_t n_start, uint32_t* d_out_ids, float* d_out_dists,
                       uint32_t* d_out_visited, uint32_t* d_out_cmps, uint32_t* d_out_flags, void* stream) {
  int rc = check_index(idx, true);
  if (rc) return rc;
  if (nq && (!d_queries || !d_out_ids)) return fail(PANN_EINVAL, "queries or out_ids is NULL");
  SearchPlan plan;
  rc = make_plan(idx, qp, n_start, &plan);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);  // 0 is the legacy default stream
  rc = stage_starts(idx, starts, n_start, st);
  if (rc) return rc;
  const uint8_t* q = static_cast<const uint8_t*>(d_queries);
  size_t rb = (size_t)idx->d * idx->esize;
  if (rb != idx->stride) {
    PANN_CUDA(idx->q.ensure(idx->stride * (size_t)nq));
    PANN_CUDA(cudaMemsetAsync(idx->q.p, 0, idx->stride * (size_t)nq, st));
    PANN_CUDA(cudaMemcpy2DAsync(idx->q.p, idx->stride, d_queries, rb, rb, nq, cudaMemcpyDeviceToDevice, st));
    q = idx->q.as<uint8_t>();
  }
  uint32_t* status = d_out_flags;
  if (!status) {
    PANN_CUDA(idx->status.ensure(sizeof(uint32_t) * (size_t)std::max<uint32_t>(nq, 1)));
    status = idx->status.as<uint32_t>();
  }
  return run_search(idx, plan, q, nullptr, nq, idx->starts.as<uint32_t>(), d_out_ids, d_out_dists, d_out_visited,
                    d_out_cmps, status, nullptr, 0, st);
}

int pann_search(pann_index* idx, const void* queries, uint32_t nq, const pann_query_params* qp,
                const uint32_t* starts, uint32_t n_start, uint32_t* out_ids, float* out_dists,
                uint32_t* out_visited, uint32_t* out_cmps, uint32_t* out_flags) {
  int rc = check_index(idx, true);
  if (rc) return rc;
  if (nq && (!queries || !out_ids)) return fail(PANN_EINVAL, "queries or out_ids is NULL");
  SearchPlan plan;
  rc = make_plan(idx, qp, n_start, &plan);
  if (rc) return rc;
  if (nq == 0) return PANN_OK;
  cudaStream_t st = idx->stream;
  rc = stage_starts(idx, starts, n_start, st);
  if (rc) return rc;
  const size_t k = plan.k;
  size_t rb = (size_t)idx->d * idx->esize;
  PANN_CUDA(idx->q.ensure(idx->stride * (size_t)nq));
  PANN_CUDA(idx->ids.ensure(4 * std::max<size_t>(1, k * nq)));
  PANN_CUDA(idx->dists.ensure(4 * std::max<size_t>(1, k * nq)));
  PANN_CUDA(idx->vis.ensure(4 * (size_t)nq));
  PANN_CUDA(idx->cmps.ensure(4 * (size_t)nq));
  PANN_CUDA(idx->status.ensure(4 * (size_t)nq));
  if (rb != idx->stride) PANN_CUDA(cudaMemsetAsync(idx->q.p, 0, idx->stride * (size_t)nq, st));
  PANN_CUDA(cudaMemcpy2DAsync(idx->q.p, idx->stride, queries, rb, rb, nq, cudaMemcpyHostToDevice, st));
  rc = run_search(idx, plan, idx->q.as<uint8_t>(), nullptr, nq, idx->starts.as<uint32_t>(), idx->ids.as<uint32_t>(),
                  idx->dists.as<float>(), idx->vis.as<uint32_t>(), idx->cmps.as<uint32_t>(),
                  idx->status.as<uint32_t>(), nullptr, 0, st);
  if (rc) return rc;
  if (k) {
    PANN_CUDA(cudaMemcpyAsync(out_ids, idx->ids.p, 4 * k * nq, cudaMemcpyDeviceToHost, st));
    if (out_dists) PANN_CUDA(cudaMemcpyAsync(out_dists, idx->dists.p, 4 * k * nq, cudaMemcpyDeviceToHost, st));
  }
  if (out_visited) PANN_CUDA(cudaMemcpyAsync(out_visited, idx->vis.p, 4 * (size_t)nq, cudaMemcpyDeviceToHost, st));
  if (out_cmps) PANN_CUDA(cudaMemcpyAsync(out_cmps, idx->cmps.p, 4 * (size_t)nq, cudaMemcpyDeviceToHost, st));
  std::vector<uint32_t> status(nq);
  PANN_CUDA(cudaMemcpyAsync(status.data(), idx->status.p, 4 * (size_t)nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  return summarize_status(status.data(), nq, out_flags);
}

int pann_index_set_precision(pann_index* idx, int precision) {
  if (!idx || !idx->points_set) return fail(PANN_EINVAL, "index has no points");
  if (precision == PANN_PREC_F32) {
    idx->lp_rows.release();
    idx->lp_scales.release();
    idx->lp_norms.release();
    idx->lp_prec = 0;
    return PANN_OK;
  }
  if (idx->dtype != PANN_F32) return fail(PANN_EINVAL, "the precision form needs float32 points");
  if (precision != PANN_PREC_BF16 && precision != PANN_PREC_FP8) return fail(PANN_EINVAL, "unknown precision");
  cudaStream_t st = idx->stream;
  const uint64_t n = idx->n;
  const uint32_t d = idx->d;
  const uint64_t vals = precision == PANN_PREC_BF16 ? 2 : 1;
  idx->lp_stride = ((uint64_t)d * vals + 15) & ~15ull;
  idx->lp_chunks = (uint32_t)(idx->lp_stride / 16);
  PANN_CUDA(idx->lp_rows.ensure(idx->lp_stride * n));
  PANN_CUDA(cudaMemsetAsync(idx->lp_rows.p, 0, idx->lp_stride * n, st));
  const uint32_t dpad = (d + 15) & ~15u;
  PANN_CUDA(idx->lp_scales.ensure(4ull * dpad * 2));
  PANN_CUDA(cudaMemsetAsync(idx->lp_scales.p, 0, 4ull * dpad * 2, st));
  int blocks = (int)std::min<uint64_t>((n * d + 255) / 256, 65535ull * 4);
  if (precision == PANN_PREC_BF16) {
    to_bf16_kernel<<<blocks, 256, 0, st>>>(reinterpret_cast<const float*>(idx->d_points), idx->stride / 4,
                                           idx->lp_rows.as<uint16_t>(), idx->lp_stride / 2, n, d);
    PANN_CUDA(cudaGetLastError());
  } else {
    uint32_t* bits = idx->lp_scales.as<uint32_t>() + dpad;  // scratch: per-dimension max |x|
    absmax_kernel<<<1024, 128, 0, st>>>(reinterpret_cast<const float*>(idx->d_points), idx->stride / 4, n, d, bits);
    PANN_CUDA(cudaGetLastError());
    std::vector<uint32_t> hb(d);
    PANN_CUDA(cudaMemcpyAsync(hb.data(), bits, 4ull * d, cudaMemcpyDeviceToHost, st));
    PANN_CUDA(cudaStreamSynchronize(st));
    std::vector<float> scale(dpad, 0.0f), inv(d);
    for (uint32_t j = 0; j < d; j++) {
      float m;
      std::memcpy(&m, &hb[j], 4);
      scale[j] = m > 0.0f ? m / 448.0f : 1.0f;
      inv[j] = 1.0f / scale[j];
    }
    DevBuf dinv;
    PANN_CUDA(dinv.ensure(4ull * d));
    PANN_CUDA(cudaMemcpyAsync(dinv.p, inv.data(), 4ull * d, cudaMemcpyHostToDevice, st));
    PANN_CUDA(cudaMemcpyAsync(idx->lp_scales.p, scale.data(), 4ull * dpad, cudaMemcpyHostToDevice, st));
    to_fp8_kernel<<<blocks, 256, 0, st>>>(reinterpret_cast<const float*>(idx->d_points), idx->stride / 4,
                                          idx->lp_rows.as<uint8_t>(), idx->lp_stride, n, d, dinv.as<float>());
    PANN_CUDA(cudaGetLastError());
    PANN_CUDA(cudaStreamSynchronize(st));
    dinv.release();
  }
  PANN_CUDA(idx->lp_norms.ensure(4ull * std::max<uint64_t>(n, 1)));
  const int nb = (int)std::min<uint64_t>((n + 255) / 256, 65535ull);
  if (precision == PANN_PREC_BF16)
    lp_norms_kernel<PREC_BF16><<<nb, 256, 0, st>>>(idx->lp_rows.as<uint8_t>(), idx->lp_stride, n, d,
                                                   idx->lp_scales.as<float>(), idx->lp_norms.as<float>());
  else
    lp_norms_kernel<PREC_FP8><<<nb, 256, 0, st>>>(idx->lp_rows.as<uint8_t>(), idx->lp_stride, n, d,
                                                  idx->lp_scales.as<float>(), idx->lp_norms.as<float>());
  PANN_CUDA(cudaGetLastError());
  PANN_CUDA(cudaStreamSynchronize(st));
  idx->lp_prec = precision;
  return PANN_OK;
}

int pann_search_ex(pann_index* idx, const void* queries, uint32_t nq, const pann_query_params* qp,
                   const pann_search_options* opt, const uint32_t* starts, uint32_t n_start, uint32_t* out_ids,
                   float* out_dists, uint32_t* out_visited, uint32_t* out_cmps, uint32_t* out_flags, int on_device,
                   void* stream) {
  int rc = check_index(idx, true);
  if (rc) return rc;
  if (nq && (!queries || !out_ids)) return fail(PANN_EINVAL, "queries or out_ids is NULL");
  const int prec = opt ? opt->precision : PANN_PREC_F32;
  const uint32_t rerank = opt ? opt->rerank : 0;
  const uint32_t parents = opt ? opt->parents : 0;
  const uint32_t scorer = opt ? opt->scorer : 0;
  SearchPlan plan;
  rc = make_plan(idx, qp, n_start, &plan);
  if (rc) return rc;
  if (prec != PANN_PREC_F32 && idx->lp_prec != prec)
    return fail(PANN_EINVAL, "call pann_index_set_precision for this precision first");
  if (nq == 0) return PANN_OK;
  cudaStream_t st = on_device ? static_cast<cudaStream_t>(stream) : idx->stream;
  rc = stage_starts(idx, starts, n_start, st);
  if (rc) return rc;
  const size_t k = plan.k;
  size_t rb = (size_t)idx->d * idx->esize;
  const uint8_t* q = static_cast<const uint8_t*>(queries);
  if (!on_device || rb != idx->stride) {
    PANN_CUDA(idx->q.ensure(idx->stride * (size_t)nq));
    if (rb != idx->stride) PANN_CUDA(cudaMemsetAsync(idx->q.p, 0, idx->stride * (size_t)nq, st));
    PANN_CUDA(cudaMemcpy2DAsync(idx->q.p, idx->stride, queries, rb, rb, nq,
                                on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    q = idx->q.as<uint8_t>();
  }
  uint32_t *d_ids = out_ids, *d_vis = out_visited, *d_cmps = out_cmps, *d_status = out_flags;
  float* d_dists = out_dists;
  if (!on_device) {
    PANN_CUDA(idx->ids.ensure(4 * std::max<size_t>(1, k * nq)));
    PANN_CUDA(idx->dists.ensure(4 * std::max<size_t>(1, k * nq)));
    PANN_CUDA(idx->vis.ensure(4 * (size_t)nq));
    PANN_CUDA(idx->cmps.ensure(4 * (size_t)nq));
    d_ids = idx->ids.as<uint32_t>();
    d_dists = idx->dists.as<float>();
    d_vis = idx->vis.as<uint32_t>();
    d_cmps = idx->cmps.as<uint32_t>();
  }
  if (!on_device || !d_status) {
    PANN_CUDA(idx->status.ensure(4 * (size_t)nq));
    d_status = idx->status.as<uint32_t>();
  }
  rc = run_search(idx, plan, q, nullptr, nq, idx->starts.as<uint32_t>(), d_ids, d_dists, d_vis, d_cmps, d_status,
                  nullptr, 0, st, prec, rerank, parents, scorer);
  if (rc || on_device) return rc;
  if (k) {
    PANN_CUDA(cudaMemcpyAsync(out_ids, d_ids, 4 * k * nq, cudaMemcpyDeviceToHost, st));
    if (out_dists) PANN_CUDA(cudaMemcpyAsync(out_dists, d_dists, 4 * k * nq, cudaMemcpyDeviceToHost, st));
  }
  if (out_visited) PANN_CUDA(cudaMemcpyAsync(out_visited, d_vis, 4 * (size_t)nq, cudaMemcpyDeviceToHost, st));
  if (out_cmps) PANN_CUDA(cudaMemcpyAsync(out_cmps, d_cmps, 4 * (size_t)nq, cudaMemcpyDeviceToHost, st));
  std::vector<uint32_t> status(nq);
  PANN_CUDA(cudaMemcpyAsync(status.data(), d_status, 4 * (size_t)nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  return summarize_status(status.data(), nq, out_flags);
}

int pann_search_lists(pann_index* idx, const void* queries, uint32_t nq, const pann_query_params* qp,
                      const uint32_t* starts, uint32_t n_start, uint32_t* frontier_ids, float* frontier_d,
                      uint32_t* frontier_n, uint32_t visited_cap, uint32_t* visited_ids, float* visited_d,
                      uint32_t* visited_n, uint32_t* out_cmps) {
  int rc = check_index(idx, true);
  if (rc) return rc;
  if (nq && (!queries || !frontier_ids || !frontier_n || !visited_n)) return fail(PANN_EINVAL, "NULL output buffer");
  if (visited_cap && (!visited_ids || !visited_d)) return fail(PANN_EINVAL, "NULL visited buffer");
  if (!qp) return fail(PANN_EINVAL, "query params are NULL");
  pann_query_params q2 = *qp;
  q2.k = qp->beam;  // the whole frontier
  SearchPlan plan;
  rc = make_plan(idx, &q2, n_start, &plan);
  if (rc) return rc;
  if (nq == 0) return PANN_OK;
  cudaStream_t st = idx->stream;
  rc = stage_starts(idx, starts, n_start, st);
  if (rc) return rc;
  const size_t L = plan.L, vc = std::max<uint32_t>(visited_cap, 1);
  size_t rb = (size_t)idx->d * idx->esize;
  PANN_CUDA(idx->q.ensure(idx->stride * (size_t)nq));
  PANN_CUDA(idx->ids.ensure(4 * L * nq));
  PANN_CUDA(idx->dists.ensure(4 * L * nq));
  PANN_CUDA(idx->vis.ensure(4 * (size_t)nq));
  PANN_CUDA(idx->cmps.ensure(4 * (size_t)nq));
  PANN_CUDA(idx->status.ensure(4 * (size_t)nq));
  PANN_CUDA(idx->tmp.ensure(8 * vc * nq));
  if (rb != idx->stride) PANN_CUDA(cudaMemsetAsync(idx->q.p, 0, idx->stride * (size_t)nq, st));
  PANN_CUDA(cudaMemcpy2DAsync(idx->q.p, idx->stride, queries, rb, rb, nq, cudaMemcpyHostToDevice, st));
  rc = run_search(idx, plan, idx->q.as<uint8_t>(), nullptr, nq, idx->starts.as<uint32_t>(), idx->ids.as<uint32_t>(),
                  idx->dists.as<float>(), idx->vis.as<uint32_t>(), idx->cmps.as<uint32_t>(),
                  idx->status.as<uint32_t>(), idx->tmp.as<uint64_t>(), (uint32_t)vc, st);
  if (rc) return rc;
  std::vector<uint32_t> fid(L * nq), status(nq), vn(nq);
  std::vector<float> fd(L * nq);
  std::vector<uint64_t> vk(vc * nq);
  PANN_CUDA(cudaMemcpyAsync(fid.data(), idx->ids.p, 4 * L * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(fd.data(), idx->dists.p, 4 * L * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(vn.data(), idx->vis.p, 4 * (size_t)nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(status.data(), idx->status.p, 4 * (size_t)nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(vk.data(), idx->tmp.p, 8 * vc * nq, cudaMemcpyDeviceToHost, st));
  if (out_cmps) PANN_CUDA(cudaMemcpyAsync(out_cmps, idx->cmps.p, 4 * (size_t)nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < nq; i++) {
    if (status[i] & (QS_TABLE_FULL | QS_INTERNAL)) return fail(PANN_EOVERFLOW, "a query's seen-set outgrew the largest table");
    if (vn[i] > visited_cap) return fail(PANN_EOVERFLOW, "a query visited more nodes than visited_cap");
    uint32_t fn = 0;
    for (size_t j = 0; j < L; j++) {
      uint32_t id = fid[i * L + j];
      frontier_ids[i * L + j] = id;
      frontier_d[i * L + j] = fd[i * L + j];
      if (id != PANN_PAD) fn = (uint32_t)j + 1;
    }
    frontier_n[i] = fn;
    visited_n[i] = vn[i];
    // the reference keeps `visited` sorted by (distance, id) (beamSearch.h:125-126)
    uint64_t* v = &vk[(size_t)i * vc];
    std::sort(v, v + vn[i]);
    for (uint32_t j = 0; j < vn[i]; j++) {
      visited_ids[(size_t)i * visited_cap + j] = key_id(v[j]);
      visited_d[(size_t)i * visited_cap + j] = key_dist(v[j]);
    }
  }
  return PANN_OK;
}

}  // extern "C"
