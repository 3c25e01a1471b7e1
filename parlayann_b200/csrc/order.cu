// Job order of the first search tier: the queries farthest from the first
// start point first. Tier 0 runs one query per warp from a shared job
// counter; its last queries decide when it ends, and a query far from the
// start point tends to need more steps, so taking those first shortens the
// tail (the answers do not depend on the order: each query is searched on
// its own). The distance is a plain float32 squared Euclidean distance used
// only to order the jobs.
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <algorithm>

#include "common.cuh"
#include "index.cuh"
#include "tiers.cuh"

namespace pann {

template <int DT>
__global__ void start_dist_kernel(const uint8_t* __restrict__ points, uint64_t stride, uint32_t d,
                                  const uint8_t* __restrict__ queries, const uint32_t* __restrict__ self_ids,
                                  const uint32_t* __restrict__ starts, uint32_t nq, uint32_t* keys, uint32_t* vals) {
  const uint8_t* s = points + (uint64_t)starts[0] * stride;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
    const uint8_t* q = self_ids ? points + (uint64_t)self_ids[i] * stride : queries + (uint64_t)i * stride;
    float acc = 0.0f;
    for (uint32_t t = 0; t < d; t++) {
      float x, y;
      if (DT == DT_F32) {
        x = reinterpret_cast<const float*>(q)[t];
        y = reinterpret_cast<const float*>(s)[t];
      } else if (DT == DT_U8) {
        x = (float)q[t];
        y = (float)s[t];
      } else {
        x = (float)(int8_t)q[t];
        y = (float)(int8_t)s[t];
      }
      const float df = x - y;
      acc = fmaf(df, df, acc);
    }
    keys[i] = __float_as_uint(acc);  // non-negative: the bit pattern orders as the value
    vals[i] = i;
  }
}

int order_far_first(pann_index* idx, const uint8_t* d_queries, const uint32_t* d_self_ids, const uint32_t* d_starts,
                    uint32_t nq, cudaStream_t st, const uint32_t** order) {
  *order = nullptr;
  size_t tmp = 0;
  cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                            (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)nq, 0, 32, st);
  const size_t arrays = (16ull * nq + 255) & ~255ull;  // four arrays of nq words, then CUB's scratch
  PANN_CUDA(idx->order.ensure_grow(arrays + tmp + 256));
  uint32_t* kin = idx->order.as<uint32_t>();
  uint32_t* kout = kin + nq;
  uint32_t* vin = kout + nq;
  uint32_t* vout = vin + nq;
  void* ctmp = idx->order.as<uint8_t>() + arrays;
  const int blocks = (int)std::min<uint64_t>((nq + 255) / 256, 4ull * idx->sm_count);
  if (idx->dtype == DT_F32)
    start_dist_kernel<DT_F32><<<blocks, 256, 0, st>>>(idx->d_points, idx->stride, idx->d, d_queries, d_self_ids,
                                                      d_starts, nq, kin, vin);
  else if (idx->dtype == DT_U8)
    start_dist_kernel<DT_U8><<<blocks, 256, 0, st>>>(idx->d_points, idx->stride, idx->d, d_queries, d_self_ids,
                                                     d_starts, nq, kin, vin);
  else
    start_dist_kernel<DT_I8><<<blocks, 256, 0, st>>>(idx->d_points, idx->stride, idx->d, d_queries, d_self_ids,
                                                     d_starts, nq, kin, vin);
  PANN_CUDA(cudaGetLastError());
  size_t tb = tmp;
  PANN_CUDA(cub::DeviceRadixSort::SortPairsDescending(ctmp, tb, kin, kout, vin, vout, (int)nq, 0, 32, st));
  *order = vout;
  return PANN_OK;
}

}  // namespace pann

namespace pann {

// Batch order keys: (beam << 32 | distance bits) for the nq queries the
// batch holds now (nq read from device memory, so one captured launch
// sequence serves every batch size); slots past nq get key 0 and sort last.
template <int DT>
__global__ void batch_order_keys_kernel(const uint8_t* __restrict__ points, uint64_t stride, uint32_t d,
                                        const uint8_t* __restrict__ queries, const uint32_t* __restrict__ starts,
                                        const uint32_t* __restrict__ qL, const uint32_t* __restrict__ nq_dev,
                                        uint32_t max_q, unsigned long long* keys, uint32_t* vals) {
  const uint32_t nq = *nq_dev;
  const uint8_t* s = points + (uint64_t)starts[0] * stride;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < max_q; i += gridDim.x * blockDim.x) {
    unsigned long long key = 0;
    if (i < nq) {
      const uint8_t* q = queries + (uint64_t)i * stride;
      float acc = 0.0f;
      for (uint32_t t = 0; t < d; t++) {
        float x, y;
        if (DT == DT_F32) {
          x = reinterpret_cast<const float*>(q)[t];
          y = reinterpret_cast<const float*>(s)[t];
        } else if (DT == DT_U8) {
          x = (float)q[t];
          y = (float)s[t];
        } else {
          x = (float)(int8_t)q[t];
          y = (float)(int8_t)s[t];
        }
        const float df = x - y;
        acc = fmaf(df, df, acc);
      }
      key = ((unsigned long long)qL[i] << 32) | __float_as_uint(acc);
    }
    keys[i] = key;
    vals[i] = i;
  }
}

size_t batch_order_scratch_bytes(uint32_t max_q) {
  size_t tmp = 0;
  cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, (const unsigned long long*)nullptr,
                                            (unsigned long long*)nullptr, (const uint32_t*)nullptr,
                                            (uint32_t*)nullptr, (int)max_q, 0, 64);
  return ((16ull * max_q + 4ull * max_q + 255) & ~255ull) + tmp + 256;
}

int order_batch(const pann_index* idx, const uint8_t* d_queries, const uint32_t* d_starts, const uint32_t* d_qL,
                const uint32_t* d_nq, uint32_t max_q, void* scratch, size_t scratch_bytes, uint32_t* d_order,
                cudaStream_t st) {
  unsigned long long* kin = static_cast<unsigned long long*>(scratch);
  unsigned long long* kout = kin + max_q;
  uint32_t* vin = reinterpret_cast<uint32_t*>(kout + max_q);
  const size_t head = (16ull * max_q + 4ull * max_q + 255) & ~255ull;
  void* ctmp = static_cast<uint8_t*>(scratch) + head;
  size_t tb = scratch_bytes - head;
  const int blocks = (int)std::min<uint64_t>((max_q + 255) / 256, 4ull * idx->sm_count);
  if (idx->dtype == DT_F32)
    batch_order_keys_kernel<DT_F32><<<blocks, 256, 0, st>>>(idx->d_points, idx->stride, idx->d, d_queries, d_starts,
                                                            d_qL, d_nq, max_q, kin, vin);
  else if (idx->dtype == DT_U8)
    batch_order_keys_kernel<DT_U8><<<blocks, 256, 0, st>>>(idx->d_points, idx->stride, idx->d, d_queries, d_starts,
                                                           d_qL, d_nq, max_q, kin, vin);
  else
    batch_order_keys_kernel<DT_I8><<<blocks, 256, 0, st>>>(idx->d_points, idx->stride, idx->d, d_queries, d_starts,
                                                           d_qL, d_nq, max_q, kin, vin);
  PANN_CUDA(cudaGetLastError());
  PANN_CUDA(cub::DeviceRadixSort::SortPairsDescending(ctmp, tb, kin, kout, vin, d_order, (int)max_q, 0, 64, st));
  return PANN_OK;
}

}  // namespace pann
