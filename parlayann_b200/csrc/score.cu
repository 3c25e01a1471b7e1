// pann_score: distances of given (query, point) pairs, at the exact float32 /
// integer arithmetic of Point::distance (euclidian_point.h:54-90,
// mips_point.h:44-66) or at the precision form's approximate bfloat16 / FP8
// scores. Used to state the precision form's scoring error (the scores that
// steer its traversal, before the exact re-rank) against FP64.
//
// One warp per query: the query is staged in shared memory (negated for
// float Euclidean, as the search kernels stage it) and each lane scores the
// pairs j = lane, lane + 32, ... of its query.
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "common.cuh"
#include "index.cuh"
#include "lowprec.cuh"

namespace pann {

template <int DT, int MT, int PREC>
__global__ void __launch_bounds__(128) score_kernel(const uint8_t* __restrict__ points, uint64_t stride, uint32_t d,
                                                    uint32_t nchunks, const uint8_t* __restrict__ lp_rows,
                                                    uint64_t lp_stride, uint32_t lp_chunks,
                                                    const float* __restrict__ scales, const uint8_t* __restrict__ queries,
                                                    uint32_t nq, const uint32_t* __restrict__ ids, uint32_t m,
                                                    float* out) {
  extern __shared__ __align__(16) uint8_t ssm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t qi = blockIdx.x * 4 + warp;
  if (qi >= nq) return;  // warp-uniform, no block barrier below
  uint8_t* qs = ssm + (size_t)warp * stride;
  stage_query<DT, MT>(qs, queries + (uint64_t)qi * stride, (int)nchunks, lane);
  __syncwarp();
  int32_t qq = 0;
  if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), nchunks);
  for (uint32_t j = lane; j < m; j += 32) {
    const uint32_t id = ids[(uint64_t)qi * m + j];
    float dv;
    if (PREC == PREC_F32) {
      dv = point_dist<DT, MT>(points + (uint64_t)id * stride, qs, (int)d, (int)nchunks, qq);
    } else {
      float dummy;
      lp_dist2<MT, PREC>(lp_rows + (uint64_t)id * lp_stride, nullptr, reinterpret_cast<const float*>(qs), scales,
                         (int)d, (int)lp_chunks, dv, dummy);
    }
    out[(uint64_t)qi * m + j] = dv;
  }
}

}  // namespace pann

using namespace pann;

extern "C" int pann_score(pann_index* idx, const void* queries, uint32_t nq, const uint32_t* ids, uint32_t m,
                          int precision, float* out) {
  if (!idx || !idx->points_set) return fail(PANN_EINVAL, "index has no points");
  if (nq == 0 || m == 0) return PANN_OK;
  if (!queries || !ids || !out) return fail(PANN_EINVAL, "queries, ids or out is NULL");
  if (precision != PREC_F32) {
    if (idx->dtype != DT_F32) return fail(PANN_EINVAL, "low-precision scores need a float32 index");
    if (idx->lp_prec != precision) return fail(PANN_EINVAL, "pann_index_set_precision was not called for this precision");
  }
  for (uint64_t i = 0; i < (uint64_t)nq * m; i++)
    if ((uint64_t)ids[i] >= idx->n) return fail(PANN_EINVAL, "point id out of range");
  cudaStream_t st = idx->stream;
  const size_t rb = (size_t)idx->d * idx->esize;
  struct Owned : DevBuf {
    ~Owned() { release(); }
  };
  Owned dq, di, dout;
  PANN_CUDA(dq.ensure(idx->stride * (size_t)nq));
  PANN_CUDA(di.ensure(4ull * nq * m));
  PANN_CUDA(dout.ensure(4ull * nq * m));
  PANN_CUDA(cudaMemsetAsync(dq.p, 0, idx->stride * (size_t)nq, st));
  PANN_CUDA(cudaMemcpy2DAsync(dq.p, idx->stride, queries, rb, rb, nq, cudaMemcpyHostToDevice, st));
  PANN_CUDA(cudaMemcpyAsync(di.p, ids, 4ull * nq * m, cudaMemcpyHostToDevice, st));
  const unsigned blocks = (nq + 3) / 4;
  const size_t smem = 4 * idx->stride;
  cudaError_t e = cudaErrorInvalidValue;
#define PANN_SCORE_CASE(DT, MT, PR)                                                                                 \
  if (idx->dtype == DT && idx->metric == MT && precision == PR) {                                                  \
    score_kernel<DT, MT, PR><<<blocks, 128, smem, st>>>(idx->d_points, idx->stride, idx->d, idx->nchunks,          \
                                                        idx->lp_rows.as<uint8_t>(), idx->lp_stride, idx->lp_chunks, \
                                                        idx->lp_scales.as<float>(), dq.as<uint8_t>(), nq,          \
                                                        di.as<uint32_t>(), m, dout.as<float>());                   \
    e = cudaGetLastError();                                                                                        \
  }
  PANN_SCORE_CASE(DT_U8, MT_L2, PREC_F32)
  PANN_SCORE_CASE(DT_U8, MT_IP, PREC_F32)
  PANN_SCORE_CASE(DT_I8, MT_L2, PREC_F32)
  PANN_SCORE_CASE(DT_I8, MT_IP, PREC_F32)
  PANN_SCORE_CASE(DT_F32, MT_L2, PREC_F32)
  PANN_SCORE_CASE(DT_F32, MT_IP, PREC_F32)
  PANN_SCORE_CASE(DT_F32, MT_L2, PREC_BF16)
  PANN_SCORE_CASE(DT_F32, MT_IP, PREC_BF16)
  PANN_SCORE_CASE(DT_F32, MT_L2, PREC_FP8)
  PANN_SCORE_CASE(DT_F32, MT_IP, PREC_FP8)
#undef PANN_SCORE_CASE
  if (e != cudaSuccess) return cuda_fail(e, "score_kernel");
  PANN_CUDA(cudaMemcpyAsync(out, dout.p, 4ull * nq * m, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  return PANN_OK;
}
