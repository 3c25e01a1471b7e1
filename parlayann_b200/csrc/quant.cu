// Quantized search with a float re-rank: the reference's own mixed-precision
// search for float indexes (GraphIndex::search_dispatch,
// python/graph_index.cpp:140-185, which calls beam_search_rerank,
// beamSearch.h:529-597). Euclidian indexes quantize as Euclidian_Point<uint8_t>
// (below); mips indexes as Quantized_Mips_Point<8, true> into an int8 mips
// index (set_quantized_mips).
//
//   pann_index_set_quantized: one-byte scalar quantization of the points as
//     PointRange<Euclidian_Point<uint8_t>>(Points) computes it
//     (generate_parameters and translate_point, euclidian_point.h:186-240):
//     slope and offset from the minimum and maximum value (0 included), each
//     value round(x * slope) - offset clamped to [0, 255]. The quantized rows
//     live in an internal uint8 Euclidean index that shares the graph.
//   pann_search_quantized: the query is translated the same way, the exact
//     uint8 search (the tiers of search.cuh) runs on the quantized rows with
//     k' = min(k * rerank_factor, L) results, and quant_rerank_kernel
//     re-scores those frontier entries with the float distance, orders them
//     by (distance, id) and keeps k. Visited and comparison counts are the
//     quantized search's, as the reference's QueryStats count them.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"
#include "index.cuh"
#include "tiers.cuh"

namespace pann {

// Per block: minimum, maximum and "every value is a non-negative integer" of
// the values (rows of `stride` bytes, d floats each).
__global__ void quant_minmax_kernel(const uint8_t* __restrict__ points, uint64_t n, uint64_t stride, uint32_t d,
                                    float* bmin, float* bmax, uint32_t* bints) {
  __shared__ float smn[8], smx[8];
  __shared__ uint32_t sin_[8];
  float mn = 0.0f, mx = 0.0f;  // generate_parameters starts both at 0 (euclidian_point.h:218-219)
  uint32_t ints = 1;
  const uint64_t total = n * d;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
    const float x = reinterpret_cast<const float*>(points + (e / d) * stride)[e % d];
    mn = fminf(mn, x);
    mx = fmaxf(mx, x);
    ints &= (x >= 0.0f) && (x - (float)(long long)x) == 0.0f;
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    ints &= __shfl_xor_sync(0xFFFFFFFFu, ints, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { smn[w] = mn; smx[w] = mx; sin_[w] = ints; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) { mn = fminf(mn, smn[i]); mx = fmaxf(mx, smx[i]); ints &= sin_[i]; }
    bmin[blockIdx.x] = mn;
    bmax[blockIdx.x] = mx;
    bints[blockIdx.x] = ints;
  }
}

// translate_point (euclidian_point.h:188-212) for n rows of d floats into
// rows of `ostride` bytes (zero padding past d).
__global__ void quant_rows_kernel(const uint8_t* __restrict__ src, uint64_t n, uint64_t sstride, uint32_t d,
                                  float slope, int32_t offset, uint8_t* out, uint64_t ostride) {
  const uint64_t total = n * ostride;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = e / ostride;
    const uint32_t j = (uint32_t)(e % ostride);
    uint8_t v = 0;
    if (j < d) {
      const float x = reinterpret_cast<const float*>(src + i * sstride)[j];
      if (slope == 1.0f && offset == 0) {
        v = (uint8_t)x;
      } else {
        long long r = (long long)roundf(__fmul_rn(x, slope)) - offset;
        r = r < 0 ? 0 : (r > 255 ? 255 : r);
        v = (uint8_t)r;
      }
    }
    out[e] = v;
  }
}

// Quantized_Mips_Point<8, true> (mips_point.h:293-499), the quantizer the
// reference's GraphIndex uses for float mips indexes: per point the minimum
// and maximum of its values (0.0 the starting point of both), ...
__global__ void quant_point_minmax_kernel(const uint8_t* __restrict__ points, uint64_t n, uint64_t stride, uint32_t d,
                                          float* mins, float* maxs) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float* x = reinterpret_cast<const float*>(points + i * stride);
    float mn = 0.0f, mx = 0.0f;
    for (uint32_t j = 0; j < d; j++) {
      mn = fminf(mn, x[j]);
      mx = fmaxf(mx, x[j]);
    }
    mins[i] = mn;
    maxs[i] = mx;
  }
}

// ... and translate_point (:421-436): -127 below -bound, 127 above bound,
// else round(x * scale), stored as int8 (zero padding past d).
__global__ void quant_rows_mips_kernel(const uint8_t* __restrict__ src, uint64_t n, uint64_t sstride, uint32_t d,
                                       float scale, float bound, uint8_t* out, uint64_t ostride) {
  const uint64_t total = n * ostride;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = e / ostride;
    const uint32_t j = (uint32_t)(e % ostride);
    int8_t v = 0;
    if (j < d) {
      const float x = reinterpret_cast<const float*>(src + i * sstride)[j];
      if (x < -bound) v = -127;
      else if (x > bound) v = 127;
      else v = (int8_t)(int32_t)roundf(__fmul_rn(x, scale));
    }
    out[e] = (uint8_t)v;
  }
}

// One warp per query: float distances of the query's kp candidates (a
// PAD-terminated frontier prefix), ranked by (distance, id); the first k are
// written, PAD past the candidates. Shared memory per warp (quant_warp_bytes,
// a multiple of 16 so that every warp's staged query takes 16-byte stores):
// the staged query, kp distances, kp ids.
__host__ __device__ inline uint64_t quant_warp_bytes(uint64_t stride, uint32_t kp) {
  return stride + ((8ull * kp + 15) & ~15ull);
}
template <int MT>
__global__ void __launch_bounds__(128) quant_rerank_kernel(const uint8_t* __restrict__ points, uint64_t stride,
                                                           uint32_t d, uint32_t nchunks,
                                                           const uint8_t* __restrict__ queries, uint32_t nq,
                                                           const uint32_t* __restrict__ cand, uint32_t kp, uint32_t k,
                                                           uint32_t* out_ids, float* out_d, uint32_t* short_count) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint8_t* qs = smem + (size_t)warp * quant_warp_bytes(stride, kp);
  float* cd = reinterpret_cast<float*>(qs + stride);
  uint32_t* ci = reinterpret_cast<uint32_t*>(cd + kp);
  const uint32_t qi = blockIdx.x * (blockDim.x >> 5) + warp;
  if (qi >= nq) return;
  stage_query<DT_F32, MT>(qs, queries + (uint64_t)qi * stride, (int)nchunks, lane);
  const uint32_t* c = cand + (uint64_t)qi * kp;
  uint32_t nv = 0;  // the valid entries are a prefix
  for (uint32_t b = 0; b < kp; b += 32) {
    const bool v = b + lane < kp && c[b + lane] != PANN_PAD;
    nv += __popc(__ballot_sync(0xFFFFFFFFu, v));
  }
  __syncwarp();
  for (uint32_t j = lane; j < nv; j += 32) {
    const uint32_t id = c[j];
    ci[j] = id;
    cd[j] = point_dist<DT_F32, MT>(points + (uint64_t)id * stride, qs, (int)d, (int)nchunks, 0);
  }
  __syncwarp();
  for (uint32_t j = lane; j < nv; j += 32) {
    const float dj = cd[j];
    const uint32_t ij = ci[j];
    uint32_t rank = 0;
    for (uint32_t i = 0; i < nv; i++) rank += cd[i] < dj || (cd[i] == dj && ci[i] < ij);
    if (rank < k) {
      out_ids[(uint64_t)qi * k + rank] = ij;
      out_d[(uint64_t)qi * k + rank] = dj;
    }
  }
  for (uint32_t r = nv + lane; r < k; r += 32) {
    out_ids[(uint64_t)qi * k + r] = PANN_PAD;
    out_d[(uint64_t)qi * k + r] = 0.0f;
  }
  if (lane == 0 && nv < k) atomicAdd(short_count, 1u);
}

}  // namespace pann

using namespace pann;

// The mips quantization (Quantized_Mips_Point<8, true>): trimmed bound from the
// points' minima and maxima, scale = 127 / bound, int8 rows in an internal
// int8 mips index sharing the graph.
static int set_quantized_mips(pann_index* idx) {
  cudaStream_t st = idx->stream;
  const uint64_t n = idx->n;
  PANN_CUDA(idx->tmp.ensure(8ull * std::max<uint64_t>(n, 1)));
  float* mins = idx->tmp.as<float>();
  float* maxs = mins + n;
  quant_point_minmax_kernel<<<(int)std::min<uint64_t>((n + 255) / 256, 65535ull), 256, 0, st>>>(
      idx->d_points, n, idx->stride, idx->d, mins, maxs);
  PANN_CUDA(cudaGetLastError());
  std::vector<float> hmin(n), hmax(n);
  PANN_CUDA(cudaMemcpyAsync(hmin.data(), mins, 4ull * n, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(hmax.data(), maxs, 4ull * n, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  // kth_smallest_copy of the minima at rank cutoff n and of the maxima at (1 - cutoff)(n - 1) (:458-465)
  const double cutoff = .0001;
  const size_t min_rank = (size_t)(cutoff * (double)n);
  const size_t max_rank = (size_t)((1.0 - cutoff) * (double)(n - 1));
  std::nth_element(hmin.begin(), hmin.begin() + min_rank, hmin.end());
  std::nth_element(hmax.begin(), hmax.begin() + max_rank, hmax.end());
  const float min_val = hmin[min_rank], max_val = hmax[max_rank];
  const float bound = std::max(max_val, -min_val);
  const float scale = 127 / bound;  // parameters(max_val, dims): (range / 2) / max_val, :306-307
  if (!idx->quant) {
    pann_index* qi = nullptr;
    int rc = pann_index_create(&qi, PANN_I8, PANN_MIPS, idx->n, idx->d, idx->R);
    if (rc) return rc;
    cudaFree(qi->d_graph);  // the quantized index reads this index's graph
    qi->d_graph = idx->d_graph;
    qi->graph_borrowed = true;
    idx->quant = qi;
  }
  pann_index* qi = idx->quant;
  const uint64_t total = qi->n * qi->stride;
  const int qb = (int)std::min<uint64_t>((total + 255) / 256, 65535ull * 8);
  quant_rows_mips_kernel<<<qb, 256, 0, st>>>(idx->d_points, idx->n, idx->stride, idx->d, scale, bound, qi->d_points,
                                             qi->stride);
  PANN_CUDA(cudaGetLastError());
  PANN_CUDA(cudaStreamSynchronize(st));
  qi->points_set = true;
  idx->q_slope = scale;
  idx->q_offset = 0;
  idx->q_bound = bound;
  return PANN_OK;
}

extern "C" int pann_index_set_quantized(pann_index* idx) {
  if (!idx || !idx->points_set) return fail(PANN_EINVAL, "index has no points");
  if (idx->dtype != PANN_F32) return fail(PANN_EINVAL, "the quantized search covers float indexes");
  if (idx->metric == PANN_MIPS) return set_quantized_mips(idx);
  cudaStream_t st = idx->stream;
  const int blocks = 2 * idx->sm_count;
  PANN_CUDA(idx->tmp.ensure(12ull * blocks));
  float* bmin = idx->tmp.as<float>();
  float* bmax = bmin + blocks;
  uint32_t* bints = reinterpret_cast<uint32_t*>(bmax + blocks);
  quant_minmax_kernel<<<blocks, 256, 0, st>>>(idx->d_points, idx->n, idx->stride, idx->d, bmin, bmax, bints);
  PANN_CUDA(cudaGetLastError());
  std::vector<float> hmin(blocks), hmax(blocks);
  std::vector<uint32_t> hints(blocks);
  PANN_CUDA(cudaMemcpyAsync(hmin.data(), bmin, 4ull * blocks, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(hmax.data(), bmax, 4ull * blocks, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(hints.data(), bints, 4ull * blocks, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  float min_val = 0.0f, max_val = 0.0f;
  bool all_ints = true;
  for (int b = 0; b < blocks; b++) {
    min_val = std::min(min_val, hmin[b]);
    max_val = std::max(max_val, hmax[b]);
    all_ints = all_ints && hints[b] != 0;
  }
  if (all_ints) {  // euclidian_point.h:232-236
    if (max_val < 256) max_val = 255;
    min_val = 0;
  }
  const float slope = 255.0f / (max_val - min_val);  // parameters(min, max, dims), :104-107
  const int32_t offset = (int32_t)std::round(min_val * slope);
  if (!idx->quant) {
    pann_index* qi = nullptr;
    int rc = pann_index_create(&qi, PANN_U8, PANN_L2, idx->n, idx->d, idx->R);
    if (rc) return rc;
    cudaFree(qi->d_graph);  // the quantized index reads this index's graph
    qi->d_graph = idx->d_graph;
    qi->graph_borrowed = true;
    idx->quant = qi;
  }
  pann_index* qi = idx->quant;
  {
    const uint64_t total = qi->n * qi->stride;
    const int qb = (int)std::min<uint64_t>((total + 255) / 256, 65535ull * 8);
    quant_rows_kernel<<<qb, 256, 0, st>>>(idx->d_points, idx->n, idx->stride, idx->d, slope, offset, qi->d_points,
                                          qi->stride);
    PANN_CUDA(cudaGetLastError());
  }
  PANN_CUDA(cudaStreamSynchronize(st));
  qi->points_set = true;
  idx->q_slope = slope;
  idx->q_offset = offset;
  return PANN_OK;
}

extern "C" int pann_index_quant_params(const pann_index* idx, float* slope, int32_t* offset) {
  if (!idx || !idx->quant) return fail(PANN_EINVAL, "index has no quantized points (pann_index_set_quantized)");
  if (slope) *slope = idx->q_slope;
  if (offset) *offset = idx->q_offset;
  return PANN_OK;
}

extern "C" int pann_search_quantized(pann_index* idx, const void* queries, uint32_t nq, const pann_query_params* qp,
                                     double rerank_factor, const uint32_t* starts, uint32_t n_start,
                                     uint32_t* out_ids, float* out_dists, uint32_t* out_visited, uint32_t* out_cmps) {
  if (!idx || !idx->quant) return fail(PANN_EINVAL, "index has no quantized points (pann_index_set_quantized)");
  if (!qp) return fail(PANN_EINVAL, "query params are NULL");
  if (nq && (!queries || !out_ids)) return fail(PANN_EINVAL, "queries or out_ids is NULL");
  pann_index* qi = idx->quant;
  // num_check = min<int>(k * rerank_factor, |frontier|) (beamSearch.h:570)
  const double kr = (double)qp->k * rerank_factor;
  const uint32_t kp = (uint32_t)std::min<double>(std::max(kr, 0.0), (double)qp->beam);
  if (kp < qp->k) return fail(PANN_EINVAL, "k * rerank_factor must be at least k");
  pann_query_params qp2 = *qp;
  qp2.k = kp;
  SearchPlan plan;
  int rc = make_plan(qi, &qp2, n_start, &plan);
  if (rc) return rc;
  if (nq == 0) return PANN_OK;
  const size_t smem = 4 * quant_warp_bytes(idx->stride, kp);
  if (smem > idx->smem_optin) return fail(PANN_EINVAL, "beam too large for the re-rank kernel");
  cudaStream_t st = idx->stream;
  rc = stage_starts(qi, starts, n_start, st);
  if (rc) return rc;
  const size_t rb = 4ull * idx->d;
  PANN_CUDA(idx->q.ensure(idx->stride * (size_t)nq));
  PANN_CUDA(qi->q.ensure(qi->stride * (size_t)nq));
  PANN_CUDA(qi->ids.ensure(4ull * kp * nq));
  PANN_CUDA(qi->dists.ensure(4ull * kp * nq));
  PANN_CUDA(qi->vis.ensure(4ull * nq));
  PANN_CUDA(qi->cmps.ensure(4ull * nq));
  PANN_CUDA(qi->status.ensure(4ull * nq));
  PANN_CUDA(idx->ids.ensure(4ull * qp->k * nq));
  PANN_CUDA(idx->dists.ensure(4ull * qp->k * nq));
  PANN_CUDA(idx->counters.ensure(16));
  if (rb != idx->stride) PANN_CUDA(cudaMemsetAsync(idx->q.p, 0, idx->stride * (size_t)nq, st));
  PANN_CUDA(cudaMemcpy2DAsync(idx->q.p, idx->stride, queries, rb, rb, nq, cudaMemcpyHostToDevice, st));
  {  // the queries, translated as the points were
    const uint64_t total = (uint64_t)nq * qi->stride;
    const int qb = (int)std::min<uint64_t>((total + 255) / 256, 65535ull * 8);
    if (idx->metric == PANN_MIPS)
      quant_rows_mips_kernel<<<qb, 256, 0, st>>>(idx->q.as<uint8_t>(), nq, idx->stride, idx->d, idx->q_slope,
                                                 idx->q_bound, qi->q.as<uint8_t>(), qi->stride);
    else
      quant_rows_kernel<<<qb, 256, 0, st>>>(idx->q.as<uint8_t>(), nq, idx->stride, idx->d, idx->q_slope,
                                            idx->q_offset, qi->q.as<uint8_t>(), qi->stride);
    PANN_CUDA(cudaGetLastError());
  }
  rc = run_search(qi, plan, qi->q.as<uint8_t>(), nullptr, nq, qi->starts.as<uint32_t>(), qi->ids.as<uint32_t>(),
                  qi->dists.as<float>(), qi->vis.as<uint32_t>(), qi->cmps.as<uint32_t>(), qi->status.as<uint32_t>(),
                  nullptr, 0, st);
  if (rc) return rc;
  uint32_t* short_count = idx->counters.as<uint32_t>();
  PANN_CUDA(cudaMemsetAsync(short_count, 0, 4, st));
  {
    auto kern = idx->metric == PANN_MIPS ? quant_rerank_kernel<MT_IP> : quant_rerank_kernel<MT_L2>;
    PANN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max()));
    kern<<<(nq + 3) / 4, 128, smem, st>>>(idx->d_points, idx->stride, idx->d, idx->nchunks, idx->q.as<uint8_t>(), nq,
                                          qi->ids.as<uint32_t>(), kp, qp->k, idx->ids.as<uint32_t>(),
                                          idx->dists.as<float>(), short_count);
    PANN_CUDA(cudaGetLastError());
  }
  std::vector<uint32_t> status(nq);
  uint32_t h_short = 0;
  PANN_CUDA(cudaMemcpyAsync(out_ids, idx->ids.p, 4ull * qp->k * nq, cudaMemcpyDeviceToHost, st));
  if (out_dists) PANN_CUDA(cudaMemcpyAsync(out_dists, idx->dists.p, 4ull * qp->k * nq, cudaMemcpyDeviceToHost, st));
  if (out_visited) PANN_CUDA(cudaMemcpyAsync(out_visited, qi->vis.p, 4ull * nq, cudaMemcpyDeviceToHost, st));
  if (out_cmps) PANN_CUDA(cudaMemcpyAsync(out_cmps, qi->cmps.p, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(status.data(), qi->status.p, 4ull * nq, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaMemcpyAsync(&h_short, short_count, 4, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < nq; i++)
    if (status[i] & (QS_TABLE_FULL | QS_INTERNAL)) return fail(PANN_EOVERFLOW, "a query's seen-set outgrew the largest table");
  if (h_short) return fail(PANN_ESHORT, "beam search returned fewer than k results");
  return PANN_OK;
}
