// Shared device/host definitions for the parlayann_b200 CUDA library.
//
// Data layout in HBM (one index):
//   points : n rows of `stride` bytes (row = d elements of the index dtype,
//            zero-padded to a multiple of 16 bytes so 16-byte vector loads
//            never cross a row), the device copy of PointRange
//            (algorithms/utils/point_range.h:43-141).
//   graph  : n x R uint32, no degree word: the row's live prefix ends at the
//            first PANN_PAD (0xFFFFFFFF). This is the reference's
//            n x (R+1) Graph (algorithms/utils/graph.h:129-255) with slot 0
//            folded into the padding, so every row is R*4 bytes and
//            16-byte aligned (128 B at R=32, 256 B at R=64).
//
// Frontier entries are 64-bit keys: (ordered(dist) << 32) | id. Unsigned key
// order is the reference's (distance, id) order (beamSearch.h:62-64). Bit 31
// of the id word is the "visited" flag; ids are < 2^31, and comparisons mask
// the flag out.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define PANN_PAD 0xFFFFFFFFu
#define PANN_VFLAG 0x80000000ull
#define PANN_KEYMASK (~PANN_VFLAG)

namespace pann {

enum DType { DT_U8 = 0, DT_I8 = 1, DT_F32 = 2 };
enum Metric { MT_L2 = 0, MT_IP = 1 };

// per-query status bits written by the search kernels
enum QueryStatus : uint32_t {
  QS_OK = 0,
  QS_TABLE_FULL = 1,      // the on-chip seen-set filled up; query is re-run with a larger one
  QS_REF_WOULD_GROW = 2,  // the reference's hashset would have grown (hashset.h:25-38)
  QS_SHORT = 4,           // fewer than k results (beamSearch.h:557-562)
  QS_VISIT_OVERFLOW = 8,  // build mode: visited list exceeded its buffer
  QS_INTERNAL = 16,       // a buffer bound the host computed was exceeded (never expected)
};

// Order-preserving map float -> uint32 (as unsigned). -0.0 is folded into +0.0
// because the reference compares distances with float '<', where they are equal.
__host__ __device__ __forceinline__ uint32_t ord_of(float f) {
  uint32_t u;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(f == 0.0f ? 0.0f : f);
#else
  float g = (f == 0.0f) ? 0.0f : f;
  __builtin_memcpy(&u, &g, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float float_of(uint32_t o) {
  uint32_t u = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  __builtin_memcpy(&f, &u, 4);
  return f;
#endif
}
__host__ __device__ __forceinline__ uint64_t make_key(float d, uint32_t id) {
  return ((uint64_t)ord_of(d) << 32) | (uint64_t)id;
}
__host__ __device__ __forceinline__ uint32_t key_id(uint64_t k) { return (uint32_t)(k & 0x7FFFFFFFull); }
__host__ __device__ __forceinline__ float key_dist(uint64_t k) { return float_of((uint32_t)(k >> 32)); }

// ------------------------------------------------------------ distances
// Exact restatements of euclidian_point.h:54-90 and mips_point.h:44-66.
// Integer types: exact int32 sums (any order), converted to float with
// round-to-nearest as the reference's (float) cast. float32: one sequential
// sum in dimension order, each subtract / multiply / add rounded separately
// (no FMA), which is what the reference computes under -ffp-contract=off.
// `row` is the base point (the reference's `this`), `q` the other operand.

// 4-way byte dot products with int32 accumulation (unsigned / signed bytes)
__device__ __forceinline__ int32_t dp4u(uint32_t a, uint32_t b, int32_t c) {
  return (int32_t)__dp4a(a, b, (uint32_t)c);
}
__device__ __forceinline__ int32_t dp4s(uint32_t a, uint32_t b, int32_t c) { return __dp4a((int)a, (int)b, c); }

// uint8/int8 rows as 16-byte chunks; q staged in shared memory.
template <int DT, int MT>
__device__ __forceinline__ float dist_int_row(const uint4* __restrict__ row, const uint4* q, int nchunks,
                                              int32_t qq) {
  int32_t pq = 0, pp = 0;
#pragma unroll 4
  for (int c = 0; c < nchunks; c++) {
    uint4 a = __ldg(row + c);
    uint4 b = q[c];
    if (DT == DT_U8) {
      pq = dp4u(a.x, b.x, pq); pq = dp4u(a.y, b.y, pq); pq = dp4u(a.z, b.z, pq); pq = dp4u(a.w, b.w, pq);
      if (MT == MT_L2) { pp = dp4u(a.x, a.x, pp); pp = dp4u(a.y, a.y, pp); pp = dp4u(a.z, a.z, pp); pp = dp4u(a.w, a.w, pp); }
    } else {
      pq = dp4s(a.x, b.x, pq); pq = dp4s(a.y, b.y, pq); pq = dp4s(a.z, b.z, pq); pq = dp4s(a.w, b.w, pq);
      if (MT == MT_L2) { pp = dp4s(a.x, a.x, pp); pp = dp4s(a.y, a.y, pp); pp = dp4s(a.z, a.z, pp); pp = dp4s(a.w, a.w, pp); }
    }
  }
  if (MT == MT_L2) return __int2float_rn(qq + pp - 2 * pq);
  return -__int2float_rn(pq);
}

// float rows: sequential sum over exactly d elements.
template <int MT>
__device__ __forceinline__ float dist_f32_row(const float4* __restrict__ row, const float* q, int d) {
  float r = 0.0f;
  int nfull = d >> 2;
#pragma unroll 4
  for (int c = 0; c < nfull; c++) {
    float4 a = __ldg(row + c);
    const float* qc = q + 4 * c;
    if (MT == MT_L2) {
      float t;
      t = __fsub_rn(qc[0], a.x); r = __fadd_rn(r, __fmul_rn(t, t));
      t = __fsub_rn(qc[1], a.y); r = __fadd_rn(r, __fmul_rn(t, t));
      t = __fsub_rn(qc[2], a.z); r = __fadd_rn(r, __fmul_rn(t, t));
      t = __fsub_rn(qc[3], a.w); r = __fadd_rn(r, __fmul_rn(t, t));
    } else {
      r = __fadd_rn(r, __fmul_rn(qc[0], a.x));
      r = __fadd_rn(r, __fmul_rn(qc[1], a.y));
      r = __fadd_rn(r, __fmul_rn(qc[2], a.z));
      r = __fadd_rn(r, __fmul_rn(qc[3], a.w));
    }
  }
  int rem = d & 3;
  if (rem) {
    float4 a = __ldg(row + nfull);
    const float* qc = q + 4 * nfull;
    float av[4] = {a.x, a.y, a.z, a.w};
    for (int e = 0; e < rem; e++) {
      if (MT == MT_L2) { float t = __fsub_rn(qc[e], av[e]); r = __fadd_rn(r, __fmul_rn(t, t)); }
      else r = __fadd_rn(r, __fmul_rn(qc[e], av[e]));
    }
  }
  return MT == MT_L2 ? r : -r;
}

// query-side constant for integer L2 (sum of squares of q)
template <int DT>
__device__ __forceinline__ int32_t sq_norm_int(const uint4* q, int nchunks) {
  int32_t s = 0;
  for (int c = 0; c < nchunks; c++) {
    uint4 b = q[c];
    if (DT == DT_U8) { s = dp4u(b.x, b.x, s); s = dp4u(b.y, b.y, s); s = dp4u(b.z, b.z, s); s = dp4u(b.w, b.w, s); }
    else { s = dp4s(b.x, b.x, s); s = dp4s(b.y, b.y, s); s = dp4s(b.z, b.z, s); s = dp4s(b.w, b.w, s); }
  }
  return s;
}

// Distance between the point stored at `row` and the query staged in shared
// memory at `qs` (as bytes). qq is sq_norm_int of the query (integer L2 only).
template <int DT, int MT>
__device__ __forceinline__ float point_dist(const uint8_t* __restrict__ row, const uint8_t* qs, int d,
                                            int nchunks, int32_t qq) {
  if (DT == DT_F32) return dist_f32_row<MT>(reinterpret_cast<const float4*>(row), reinterpret_cast<const float*>(qs), d);
  return dist_int_row<DT, MT>(reinterpret_cast<const uint4*>(row), reinterpret_cast<const uint4*>(qs), nchunks, qq);
}

__device__ __forceinline__ uint32_t hash_slot(uint32_t id, uint32_t mask) {
  return (id * 0x9E3779B1u) >> 7 & mask;
}

}  // namespace pann
