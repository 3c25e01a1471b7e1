// Exact brute-force top-k (compute_groundtruth, data_tools/compute_groundtruth.cpp:22-60).
// Integer types: exact integer distance. float32: FP64 arithmetic (the FP64
// oracle recall is measured against). Results ordered by (distance, id).
//
// A block of 8 warps serves 8 queries; the warps sweep the base points in the
// same order, one point per lane, so each 32-row tile is read from HBM once
// and served to the other warps from L1. Each warp keeps its query's top-k
// as a sorted list in shared memory.
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"
#include "index.cuh"

namespace pann {

template <int DT, int MT>
__device__ __forceinline__ double exact_dist(const uint8_t* __restrict__ row, const uint8_t* q, int d) {
  if (DT == DT_F32) {
    const float* x = reinterpret_cast<const float*>(row);
    const float* y = reinterpret_cast<const float*>(q);
    double r = 0.0;
    for (int i = 0; i < d; i++) {
      double a = (double)y[i], b = (double)__ldg(x + i);
      r = MT == MT_L2 ? __dadd_rn(r, __dmul_rn(__dsub_rn(a, b), __dsub_rn(a, b))) : __dadd_rn(r, __dmul_rn(a, b));
    }
    return MT == MT_L2 ? r : -r;
  } else {
    long long r = 0;
    for (int i = 0; i < d; i++) {
      int a = DT == DT_U8 ? (int)q[i] : (int)(int8_t)q[i];
      int b = DT == DT_U8 ? (int)__ldg(row + i) : (int)(int8_t)__ldg(row + i);
      r += MT == MT_L2 ? (long long)(a - b) * (a - b) : (long long)a * b;
    }
    return MT == MT_L2 ? (double)r : -(double)r;
  }
}

__device__ __forceinline__ bool dless(double a, uint32_t ia, double b, uint32_t ib) {
  return a < b || (a == b && ia < ib);
}

template <int DT, int MT>
__global__ void __launch_bounds__(256) bruteforce_kernel(const uint8_t* __restrict__ points, uint64_t n, uint64_t stride,
                                                         int d, const uint8_t* __restrict__ queries, uint32_t nq,
                                                         uint32_t k, uint32_t* out_ids, double* out_d) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t qi = blockIdx.x * 8 + warp;
  uint8_t* qs = smem + (size_t)warp * stride;
  double* bd = reinterpret_cast<double*>(smem + 8 * stride) + (size_t)warp * k;
  uint32_t* bi = reinterpret_cast<uint32_t*>(reinterpret_cast<double*>(smem + 8 * stride) + 8 * (size_t)k) + (size_t)warp * k;
  const bool active = qi < nq;
  if (active)
    for (uint64_t c = lane; c < stride / 16; c += 32)
      reinterpret_cast<uint4*>(qs)[c] = reinterpret_cast<const uint4*>(queries + (uint64_t)qi * stride)[c];
  __syncwarp();
  uint32_t cnt = 0;
  double thr = 0.0;
  uint32_t thr_id = 0;
  for (uint64_t b = 0; b < n; b += 32) {
    uint64_t j = b + lane;
    double dj = 0.0;
    bool cand = false;
    if (active && j < n) {
      dj = exact_dist<DT, MT>(points + j * stride, qs, d);
      cand = cnt < k || dless(dj, (uint32_t)j, thr, thr_id);
    }
    unsigned m = __ballot_sync(0xFFFFFFFFu, cand);
    while (m) {
      int src = __ffs(m) - 1;
      m &= m - 1;
      double dv = __shfl_sync(0xFFFFFFFFu, dj, src);
      uint32_t iv = (uint32_t)__shfl_sync(0xFFFFFFFFu, (unsigned)j, src);
      if (!(cnt < k || dless(dv, iv, thr, thr_id))) continue;
      // position = number of entries smaller than (dv, iv)
      uint32_t pos = 0;
      for (uint32_t t = lane; t < cnt; t += 32) pos += dless(bd[t], bi[t], dv, iv) ? 1u : 0u;
      for (int o = 16; o; o >>= 1) pos += __shfl_xor_sync(0xFFFFFFFFu, pos, o);
      uint32_t newcnt = cnt < k ? cnt + 1 : k;
      // shift [pos, newcnt-1) right by one, from the top down in chunks of 32
      for (int top = (int)newcnt - 1; top > (int)pos; top -= 32) {
        int t = top - lane;
        double vd = 0.0;
        uint32_t vi = 0;
        bool mv = t > (int)pos;
        if (mv) { vd = bd[t - 1]; vi = bi[t - 1]; }
        __syncwarp();
        if (mv) { bd[t] = vd; bi[t] = vi; }
        __syncwarp();
      }
      if (lane == 0) { bd[pos] = dv; bi[pos] = iv; }
      __syncwarp();
      cnt = newcnt;
      thr = bd[cnt - 1];
      thr_id = bi[cnt - 1];
    }
  }
  if (active)
    for (uint32_t t = lane; t < k; t += 32) {
      out_ids[(uint64_t)qi * k + t] = t < cnt ? bi[t] : PANN_PAD;
      if (out_d) out_d[(uint64_t)qi * k + t] = t < cnt ? bd[t] : 0.0;
    }
}

// Range groundtruth (compute_range_groundtruth,
// data_tools/compute_range_groundtruth.cpp:14-30): answer i = every base id j
// with Q[i].distance(B[j]) <= radius, in increasing j. A block of 8 warps
// serves 8 queries against one tile of RGT_TILE base rows (the warps read the
// tile's rows in the same order, so L1 serves seven of the eight reads; each
// lane scores two rows at once, opaque_zero keeping products and sums
// unfused as the reference computes them). Pass
// 0 counts each (query, tile)'s answers; pass 1, given the offsets, writes
// them in id order. Distances are the reference's float distances.
constexpr uint32_t RGT_TILE = 8192;

template <int DT, int MT>
__global__ void __launch_bounds__(256) range_gt_kernel(const uint8_t* __restrict__ points, uint64_t n, uint64_t stride,
                                                       int d, int nchunks, const uint8_t* __restrict__ queries,
                                                       uint32_t nq, float radius, uint32_t ntiles, uint32_t* counts,
                                                       const unsigned long long* __restrict__ offs, uint32_t* out,
                                                       uint64_t opaque_zero) {
  extern __shared__ __align__(16) uint8_t smem[];
  const unsigned FULL = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const uint32_t qi = blockIdx.y * 8 + warp;
  if (qi >= nq) return;  // warp-uniform; no block barrier follows
  uint8_t* qs = smem + (size_t)warp * stride;
  stage_query<DT, MT>(qs, queries + (uint64_t)qi * stride, nchunks, lane);
  __syncwarp();
  int32_t qq = 0;
  if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), nchunks);
  const uint64_t t0 = (uint64_t)blockIdx.x * RGT_TILE;
  const uint64_t end = t0 + RGT_TILE < n ? t0 + RGT_TILE : n;
  const uint64_t slot = (uint64_t)qi * ntiles + blockIdx.x;
  const unsigned long long o = offs ? offs[slot] : 0ull;
  uint32_t cnt = 0;
  for (uint64_t j0 = t0; j0 < end; j0 += 64) {  // two rows per lane, their loads interleaved
    const uint64_t ja = j0 + (uint64_t)lane, jb = ja + 32;
    float da = 0.0f, db = 0.0f;
    if (ja < end)
      point_dist2<DT, MT>(points + ja * stride, jb < end ? points + jb * stride : nullptr, qs, nchunks, qq, da, db,
                          opaque_zero);
    const bool ina = ja < end && da <= radius, inb = jb < end && db <= radius;
    const unsigned ma = __ballot_sync(FULL, ina), mb = __ballot_sync(FULL, inb);
    if (offs && ina) out[o + cnt + __popc(ma & lt)] = (uint32_t)ja;
    cnt += __popc(ma);
    if (offs && inb) out[o + cnt + __popc(mb & lt)] = (uint32_t)jb;
    cnt += __popc(mb);
  }
  if (!offs && lane == 0) counts[slot] = cnt;
}

}  // namespace pann

using namespace pann;

extern "C" int pann_range_groundtruth(pann_index* idx, const void* queries, uint32_t nq, float radius,
                                      uint64_t* out_offsets, uint32_t* out_ids, uint64_t ids_cap) {
  if (!idx || !idx->points_set) return fail(PANN_EINVAL, "index has no points");
  idx->range_held = 0;
  if (!out_offsets) return fail(PANN_EINVAL, "out_offsets is NULL");
  if (nq && !queries) return fail(PANN_EINVAL, "queries is NULL");
  out_offsets[0] = 0;
  if (nq == 0) return PANN_OK;
  if ((nq + 7) / 8 > 65535u) return fail(PANN_EINVAL, "at most 524280 queries per call");
  cudaStream_t st = idx->stream;
  const size_t rb = (size_t)idx->d * idx->esize;
  const uint32_t ntiles = (uint32_t)((idx->n + RGT_TILE - 1) / RGT_TILE);
  const uint64_t nslots = (uint64_t)nq * ntiles;
  const size_t smem = 8 * idx->stride;
  if (smem > idx->smem_optin) return fail(PANN_EINVAL, "rows too long for the range groundtruth kernel");
  // the index's resident buffers: staged queries, then per (query, tile) counts and offsets
  PANN_CUDA(idx->q.ensure(idx->stride * (size_t)nq));
  PANN_CUDA(idx->range_meta.ensure(12 * nslots + 8));
  uint8_t* dq = idx->q.as<uint8_t>();
  unsigned long long* doffs = idx->range_meta.as<unsigned long long>();
  uint32_t* dcounts = reinterpret_cast<uint32_t*>(doffs + nslots);
  if (rb != idx->stride) PANN_CUDA(cudaMemsetAsync(dq, 0, idx->stride * (size_t)nq, st));
  PANN_CUDA(cudaMemcpy2DAsync(dq, idx->stride, queries, rb, rb, nq, cudaMemcpyHostToDevice, st));
  const dim3 grid(ntiles, (nq + 7) / 8);
  auto launch = [&](const unsigned long long* o, uint32_t* out) -> cudaError_t {
#define PANN_RGT_CASE(DT, MT)                                                                               \
  if (idx->dtype == DT && idx->metric == MT) {                                                              \
    auto kern = range_gt_kernel<DT, MT>;                                                                    \
    cudaError_t fe = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max()); \
    if (fe != cudaSuccess) return fe;                                                                       \
    kern<<<grid, 256, smem, st>>>(idx->d_points, idx->n, idx->stride, (int)idx->d, (int)idx->nchunks, dq, nq, \
                                  radius, ntiles, dcounts, o, out, 0ull);                                    \
    return cudaGetLastError();                                                                              \
  }
    PANN_RGT_CASE(DT_U8, MT_L2)
    PANN_RGT_CASE(DT_U8, MT_IP)
    PANN_RGT_CASE(DT_I8, MT_L2)
    PANN_RGT_CASE(DT_I8, MT_IP)
    PANN_RGT_CASE(DT_F32, MT_L2)
    PANN_RGT_CASE(DT_F32, MT_IP)
#undef PANN_RGT_CASE
    return cudaErrorInvalidValue;
  };
  // pass 0: counts per (query, tile); offsets in (query, tile) order
  std::vector<uint32_t> counts(nslots);
  std::vector<unsigned long long> offs(nslots);
  PANN_CUDA(launch(nullptr, nullptr));
  PANN_CUDA(cudaMemcpyAsync(counts.data(), dcounts, 4 * nslots, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  uint64_t total = 0;
  for (uint32_t i = 0; i < nq; i++) {
    out_offsets[i] = total;
    for (uint32_t t = 0; t < ntiles; t++) {
      offs[(uint64_t)i * ntiles + t] = total;
      total += counts[(uint64_t)i * ntiles + t];
    }
  }
  out_offsets[nq] = total;
  if (total == 0) return PANN_OK;
  if (total <= ids_cap && !out_ids) return fail(PANN_EINVAL, "out_ids is NULL");
  // pass 1: the ids, in id order per query, into the index's answer buffer
  PANN_CUDA(idx->range_out.ensure(4 * total));
  PANN_CUDA(cudaMemcpyAsync(doffs, offs.data(), 8 * nslots, cudaMemcpyHostToDevice, st));
  PANN_CUDA(launch(doffs, idx->range_out.as<uint32_t>()));
  if (total > ids_cap) {
    PANN_CUDA(cudaStreamSynchronize(st));
    idx->range_held = total;
    return fail(PANN_EOVERFLOW, "range groundtruth needs " + std::to_string(total) + " ids; out_ids holds " +
                                    std::to_string(ids_cap) + " (pann_range_fetch copies them)");
  }
  PANN_CUDA(cudaMemcpyAsync(out_ids, idx->range_out.p, 4 * total, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  return PANN_OK;
}

extern "C" int pann_groundtruth(pann_index* idx, const void* queries, uint32_t nq, uint32_t k, uint32_t* out_ids,
                                double* out_dists) {
  if (!idx || !idx->points_set) return fail(PANN_EINVAL, "index has no points");
  if (!queries || !out_ids) return fail(PANN_EINVAL, "queries or out_ids is NULL");
  if (k == 0 || k > 1024) return fail(PANN_EINVAL, "k must be in [1, 1024]");
  if (nq == 0) return PANN_OK;
  cudaStream_t st = idx->stream;
  size_t rb = (size_t)idx->d * idx->esize;
  uint8_t* dq = nullptr;
  uint32_t* dids = nullptr;
  double* dd = nullptr;
  size_t smem = 8 * idx->stride + 8 * (size_t)k * (sizeof(double) + sizeof(uint32_t));
  if (smem > idx->smem_optin) return fail(PANN_EINVAL, "k too large for the brute-force kernel");
  PANN_CUDA(cudaMalloc(&dq, idx->stride * (size_t)nq));
  PANN_CUDA(cudaMalloc(&dids, 4ull * k * nq));
  PANN_CUDA(cudaMalloc(&dd, 8ull * k * nq));
  PANN_CUDA(cudaMemsetAsync(dq, 0, idx->stride * (size_t)nq, st));
  PANN_CUDA(cudaMemcpy2DAsync(dq, idx->stride, queries, rb, rb, nq, cudaMemcpyHostToDevice, st));
  int blocks = (int)((nq + 7) / 8);
  cudaError_t e = cudaSuccess;
#define PANN_BF_CASE(DT, MT)                                                                                   \
  if (idx->dtype == DT && idx->metric == MT) {                                                                 \
    auto kern = bruteforce_kernel<DT, MT>;                                                                     \
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max());                        \
    kern<<<blocks, 256, smem, st>>>(idx->d_points, idx->n, idx->stride, (int)idx->d, dq, nq, k, dids, dd);     \
    e = cudaGetLastError();                                                                                    \
  }
  PANN_BF_CASE(DT_U8, MT_L2)
  PANN_BF_CASE(DT_U8, MT_IP)
  PANN_BF_CASE(DT_I8, MT_L2)
  PANN_BF_CASE(DT_I8, MT_IP)
  PANN_BF_CASE(DT_F32, MT_L2)
  PANN_BF_CASE(DT_F32, MT_IP)
#undef PANN_BF_CASE
  if (e == cudaSuccess) e = cudaMemcpyAsync(out_ids, dids, 4ull * k * nq, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && out_dists) e = cudaMemcpyAsync(out_dists, dd, 8ull * k * nq, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(dq);
  cudaFree(dids);
  cudaFree(dd);
  if (e != cudaSuccess) return cuda_fail(e, "brute-force top-k");
  return PANN_OK;
}
