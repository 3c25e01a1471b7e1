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

// Rows are read as 16-byte chunks in batches of one 128-byte line. Before the
// first batch, the row's other lines are prefetched into L2, so all lines of a
// row are in flight together and a row costs about one memory round trip
// instead of one per line.
constexpr int ROW_CHUNKS = 8;

__device__ __forceinline__ void prefetch_row_l2(const void* row, int nchunks) {
  const char* p = static_cast<const char*>(row);
  for (int c = ROW_CHUNKS; c < nchunks; c += ROW_CHUNKS) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + 16 * c));
}

// uint8/int8 rows; q (16-byte chunks) staged in shared memory.
template <int DT, int MT>
__device__ __forceinline__ void int_chunk(uint4 a, uint4 b, int32_t& pq, int32_t& pp) {
  if (DT == DT_U8) {
    pq = dp4u(a.x, b.x, pq); pq = dp4u(a.y, b.y, pq); pq = dp4u(a.z, b.z, pq); pq = dp4u(a.w, b.w, pq);
    if (MT == MT_L2) { pp = dp4u(a.x, a.x, pp); pp = dp4u(a.y, a.y, pp); pp = dp4u(a.z, a.z, pp); pp = dp4u(a.w, a.w, pp); }
  } else {
    pq = dp4s(a.x, b.x, pq); pq = dp4s(a.y, b.y, pq); pq = dp4s(a.z, b.z, pq); pq = dp4s(a.w, b.w, pq);
    if (MT == MT_L2) { pp = dp4s(a.x, a.x, pp); pp = dp4s(a.y, a.y, pp); pp = dp4s(a.z, a.z, pp); pp = dp4s(a.w, a.w, pp); }
  }
}
template <int MT>
__device__ __forceinline__ float int_result(int32_t qq, int32_t pq, int32_t pp) {
  if (MT == MT_L2) return __int2float_rn(qq + pp - 2 * pq);
  return -__int2float_rn(pq);
}

template <int DT, int MT>
__device__ __forceinline__ float dist_int_row(const uint4* __restrict__ row, const uint4* q, int nchunks,
                                              int32_t qq) {
  int32_t pq = 0, pp = 0;
  prefetch_row_l2(row, nchunks);
  for (int c0 = 0; c0 < nchunks; c0 += ROW_CHUNKS) {
    uint4 buf[ROW_CHUNKS];
#pragma unroll
    for (int c = 0; c < ROW_CHUNKS; c++)
      if (c0 + c < nchunks) buf[c] = __ldg(row + c0 + c);
#pragma unroll
    for (int c = 0; c < ROW_CHUNKS; c++)
      if (c0 + c < nchunks) int_chunk<DT, MT>(buf[c], q[c0 + c], pq, pp);
  }
  return int_result<MT>(qq, pq, pp);
}

// float32 terms. For Euclidean distance the staged query holds -q, so the
// difference is formed as x + (-q) = x - q (exact negation, same rounding as
// q - x) and (x - q)^2 == (q - x)^2 bit for bit; for mips the query holds q.
template <int MT>
__device__ __forceinline__ float f32_chunk(float r, float4 a, float4 qc) {
  if (MT == MT_L2) {
    float t;
    t = __fadd_rn(a.x, qc.x); r = __fadd_rn(r, __fmul_rn(t, t));
    t = __fadd_rn(a.y, qc.y); r = __fadd_rn(r, __fmul_rn(t, t));
    t = __fadd_rn(a.z, qc.z); r = __fadd_rn(r, __fmul_rn(t, t));
    t = __fadd_rn(a.w, qc.w); r = __fadd_rn(r, __fmul_rn(t, t));
  } else {
    r = __fadd_rn(r, __fmul_rn(qc.x, a.x));
    r = __fadd_rn(r, __fmul_rn(qc.y, a.y));
    r = __fadd_rn(r, __fmul_rn(qc.z, a.z));
    r = __fadd_rn(r, __fmul_rn(qc.w, a.w));
  }
  return r;
}

// Two rows in one packed f32x2 chain (sm_100 paired FP32): add.rn.f32x2 and
// mul.rn.f32x2 round every component to nearest like the scalar operations.
// The backend nevertheless fuses a paired multiply feeding a paired add into
// one fused multiply-add (measured on sm_100a), which rounds the product
// away. Each product is therefore OR-ed with `opq`, a zero the compiler cannot
// see (it arrives as a kernel argument), so the add's operand is no longer a
// multiply result and the two roundings of the reference stay separate.
__device__ __forceinline__ uint64_t pk2(float lo, float hi) {
  return (uint64_t)__float_as_uint(lo) | ((uint64_t)__float_as_uint(hi) << 32);
}
__device__ __forceinline__ uint64_t add2_rn(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t mul2_rn(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
template <int MT>
__device__ __forceinline__ uint64_t f32_chunk2(uint64_t r, float4 a, float4 b, float4 qc, uint64_t opq) {
  if (MT == MT_L2) {
    uint64_t t;
    t = add2_rn(pk2(a.x, b.x), pk2(qc.x, qc.x)); r = add2_rn(r, mul2_rn(t, t) | opq);
    t = add2_rn(pk2(a.y, b.y), pk2(qc.y, qc.y)); r = add2_rn(r, mul2_rn(t, t) | opq);
    t = add2_rn(pk2(a.z, b.z), pk2(qc.z, qc.z)); r = add2_rn(r, mul2_rn(t, t) | opq);
    t = add2_rn(pk2(a.w, b.w), pk2(qc.w, qc.w)); r = add2_rn(r, mul2_rn(t, t) | opq);
  } else {
    r = add2_rn(r, mul2_rn(pk2(qc.x, qc.x), pk2(a.x, b.x)) | opq);
    r = add2_rn(r, mul2_rn(pk2(qc.y, qc.y), pk2(a.y, b.y)) | opq);
    r = add2_rn(r, mul2_rn(pk2(qc.z, qc.z), pk2(a.z, b.z)) | opq);
    r = add2_rn(r, mul2_rn(pk2(qc.w, qc.w), pk2(a.w, b.w)) | opq);
  }
  return r;
}

// float rows: one sequential sum in dimension order. Rows and the staged
// query are zero-padded to whole 16-byte chunks; a padded term adds +0.0,
// which leaves the running sum unchanged bit for bit (it starts at +0.0 and
// can never be -0.0), so whole chunks are summed without per-element tests.
// 16-byte chunks of a float row in flight at once: 12 of a 96-d row's 24
// (the rest prefetched to L2) took the 1M x 96 build from 8.94 s to 8.12 s
// (its prune steps score candidate rows this way), with the same graph; 24
// slowed its searches (registers); the exact search itself was unchanged.
#ifndef PANN_F32_ROW_CHUNKS
#define PANN_F32_ROW_CHUNKS 12
#endif
template <int MT>
__device__ __forceinline__ float dist_f32_row(const float4* __restrict__ row, const float4* q, int nvec) {
  constexpr int CH = PANN_F32_ROW_CHUNKS;
  float r = 0.0f;
  prefetch_row_l2(row, nvec);
  for (int c0 = 0; c0 < nvec; c0 += CH) {
    float4 buf[CH];
#pragma unroll
    for (int c = 0; c < CH; c++)
      if (c0 + c < nvec) buf[c] = __ldg(row + c0 + c);
#pragma unroll
    for (int c = 0; c < CH; c++)
      if (c0 + c < nvec) r = f32_chunk<MT>(r, buf[c], q[c0 + c]);
  }
  return MT == MT_L2 ? r : -r;
}

// Two rows against the same query, their loads and sums interleaved so the
// two dependency chains overlap. rowB may be null (then db is not written).
// Loads go in batches of PAIR_CHUNKS 16-byte chunks per row (the rows' other
// lines are prefetched into L2 first), which keeps the register footprint
// within the 168-register budget of three resident 128-thread blocks per SM
// (the shared-memory seen tables allow three anyway); measured faster than
// 4-chunk batches at four blocks and than 12- or 24-chunk batches, which spill.
constexpr int PAIR_CHUNKS = 8;
template <int DT, int MT, int CH = PAIR_CHUNKS>
__device__ __forceinline__ void point_dist2(const uint8_t* __restrict__ rowA, const uint8_t* __restrict__ rowB,
                                            const uint8_t* qs, int nchunks, int32_t qq, float& da, float& db,
                                            uint64_t opq) {
  const bool two = rowB != nullptr;
  const uint4* ra = reinterpret_cast<const uint4*>(rowA);
  const uint4* rb = reinterpret_cast<const uint4*>(two ? rowB : rowA);
  prefetch_row_l2(ra, nchunks);
  if (two) prefetch_row_l2(rb, nchunks);
  if (DT == DT_F32) {
    const float4* q = reinterpret_cast<const float4*>(qs);
    uint64_t r = 0;  // two +0.0f
    for (int c0 = 0; c0 < nchunks; c0 += CH) {
      float4 ba[CH], bb[CH];
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (c0 + c < nchunks) {
          ba[c] = __ldg(reinterpret_cast<const float4*>(ra) + c0 + c);
          bb[c] = two ? __ldg(reinterpret_cast<const float4*>(rb) + c0 + c) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (c0 + c < nchunks) r = f32_chunk2<MT>(r, ba[c], bb[c], q[c0 + c], opq);
    }
    const float rx = __uint_as_float((uint32_t)r), ry = __uint_as_float((uint32_t)(r >> 32));
    da = MT == MT_L2 ? rx : -rx;
    if (two) db = MT == MT_L2 ? ry : -ry;
  } else {
    const uint4* q = reinterpret_cast<const uint4*>(qs);
    int32_t pa = 0, qa = 0, pb = 0, qb = 0;
    for (int c0 = 0; c0 < nchunks; c0 += CH) {
      uint4 ba[CH], bb[CH];
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (c0 + c < nchunks) {
          ba[c] = __ldg(ra + c0 + c);
          if (two) bb[c] = __ldg(rb + c0 + c);
        }
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (c0 + c < nchunks) {
          uint4 qc = q[c0 + c];
          int_chunk<DT, MT>(ba[c], qc, qa, pa);
          if (two) int_chunk<DT, MT>(bb[c], qc, qb, pb);
        }
    }
    da = int_result<MT>(qq, qa, pa);
    if (two) db = int_result<MT>(qq, qb, pb);
  }
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
  (void)d;
  if (DT == DT_F32)
    return dist_f32_row<MT>(reinterpret_cast<const float4*>(row), reinterpret_cast<const float4*>(qs), nchunks);
  return dist_int_row<DT, MT>(reinterpret_cast<const uint4*>(row), reinterpret_cast<const uint4*>(qs), nchunks, qq);
}

// Stage a query row (nchunks 16-byte chunks) into shared memory, warp-wide.
// float32 Euclidean rows are stored negated (see f32_chunk).
template <int DT, int MT>
__device__ __forceinline__ void stage_query(uint8_t* qs, const uint8_t* __restrict__ src, int nchunks, int lane) {
  for (int c = lane; c < nchunks; c += 32) {
    uint4 v = __ldg(reinterpret_cast<const uint4*>(src) + c);
    if (DT == DT_F32 && MT == MT_L2) v = make_uint4(v.x ^ 0x80000000u, v.y ^ 0x80000000u, v.z ^ 0x80000000u, v.w ^ 0x80000000u);
    reinterpret_cast<uint4*>(qs)[c] = v;
  }
}

__device__ __forceinline__ uint32_t hash_slot(uint32_t id, uint32_t mask) {
  return (id * 0x9E3779B1u) >> 7 & mask;
}

}  // namespace pann
