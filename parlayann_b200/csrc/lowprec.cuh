// Low-precision copies of float32 points and their approximate distances
// (the precision form of the search).
//
//   BF16: each value rounded to nearest-even bfloat16; 2 bytes per value.
//   FP8 : E4M3 with one scale per dimension, s_t = max_i |x_it| / 448 (the
//         largest finite E4M3 value); stored value = E4M3(x_it / s_t); 1 byte.
//
// Approximate distances dequantize to float32 and accumulate in float32 with
// fused multiply-adds in any order: they only steer the traversal. The
// search re-ranks its best candidates with the exact float32 distance (the
// reference's sequential sum, common.cuh) before reporting.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include "common.cuh"

namespace pann {

enum Precision { PREC_F32 = 0, PREC_BF16 = 1, PREC_FP8 = 2 };

// bf16 pair (packed in a uint32) -> two floats, exactly
__device__ __forceinline__ float2 bf16x2_to_f2(uint32_t v) {
  return make_float2(__uint_as_float(v << 16), __uint_as_float(v & 0xFFFF0000u));
}
// e4m3 pair (low 16 bits of v) -> two floats, exactly
__device__ __forceinline__ float2 e4m3x2_to_f2(uint32_t v) {
  __half2_raw h = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(v & 0xFFFFu), __NV_E4M3);
  return __half22float2(*reinterpret_cast<__half2*>(&h));
}

// Approximate distances of up to two low-precision rows to the query staged in
// shared memory as float32 (negated for L2, as the exact path stores it).
// FP8 rows are dequantized with the per-dimension scales in shared memory.
template <int MT, int PREC>
__device__ __forceinline__ void lp_dist2(const uint8_t* __restrict__ rowA, const uint8_t* __restrict__ rowB,
                                         const float* qs, const float* scales, int d, int lp_chunks, float& da,
                                         float& db) {
  const bool two = rowB != nullptr;
  const uint4* ra = reinterpret_cast<const uint4*>(rowA);
  const uint4* rb = reinterpret_cast<const uint4*>(two ? rowB : rowA);
  float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
  constexpr int VPC = PREC == PREC_BF16 ? 8 : 16;  // values per 16-byte chunk
  for (int c0 = 0; c0 < lp_chunks; c0 += 8) {
    uint4 ba[8], bb[8];
#pragma unroll
    for (int c = 0; c < 8; c++)
      if (c0 + c < lp_chunks) {
        ba[c] = __ldg(ra + c0 + c);
        bb[c] = two ? __ldg(rb + c0 + c) : make_uint4(0, 0, 0, 0);
      }
#pragma unroll
    for (int c = 0; c < 8; c++) {
      if (c0 + c >= lp_chunks) break;
      const uint32_t wa[4] = {ba[c].x, ba[c].y, ba[c].z, ba[c].w};
      const uint32_t wb[4] = {bb[c].x, bb[c].y, bb[c].z, bb[c].w};
      const int e0 = (c0 + c) * VPC;
#pragma unroll
      for (int w = 0; w < 4; w++) {
#pragma unroll
        for (int h = 0; h < (PREC == PREC_BF16 ? 1 : 2); h++) {
          const int e = e0 + w * (VPC / 4) + 2 * h;
          if (e >= d) break;
          float2 xa, xb;
          if (PREC == PREC_BF16) {
            xa = bf16x2_to_f2(wa[w]);
            xb = bf16x2_to_f2(wb[w]);
          } else {
            xa = e4m3x2_to_f2(wa[w] >> (16 * h));
            xb = e4m3x2_to_f2(wb[w] >> (16 * h));
            xa.x *= scales[e]; xa.y *= scales[e + 1];
            xb.x *= scales[e]; xb.y *= scales[e + 1];
          }
          const float q0 = qs[e], q1 = qs[e + 1];
          if (MT == MT_L2) {
            float t;
            t = xa.x + q0; a0 = fmaf(t, t, a0);
            t = xa.y + q1; a1 = fmaf(t, t, a1);
            t = xb.x + q0; b0 = fmaf(t, t, b0);
            t = xb.y + q1; b1 = fmaf(t, t, b1);
          } else {
            a0 = fmaf(q0, xa.x, a0); a1 = fmaf(q1, xa.y, a1);
            b0 = fmaf(q0, xb.x, b0); b1 = fmaf(q1, xb.y, b1);
          }
        }
      }
    }
  }
  da = MT == MT_L2 ? a0 + a1 : -(a0 + a1);
  if (two) db = MT == MT_L2 ? b0 + b1 : -(b0 + b1);
}

}  // namespace pann
