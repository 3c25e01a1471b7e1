// Exact brute-force top-k (compute_groundtruth, data_tools/compute_groundtruth.cpp:22-60).
// Integer types: exact integer distance. float32: FP64 arithmetic (the FP64
// oracle recall is measured against). Results ordered by (distance, id).
//
// A block of 8 warps serves 8 queries; the warps sweep the base points in the
// same order, one point per lane, so each 32-row tile is read from HBM once
// and served to the other warps from L1. Each warp keeps its query's top-k
// as a sorted list in shared memory.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
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

// ---------------------------------------------------------------------------
// Exact top-k for float32 points, fast: a float32 candidate pass, then FP64
// distances of the candidates only.
//
// Pass 1 (gt_cand_kernel): a block scores GT_QT queries against the points of
// one slice of the base in tiles of GT_PT rows (queries and rows staged
// transposed in shared memory; each thread accumulates a 4 x 8 register tile
// of dot products with float32 FMAs), as D32 = |b|^2 - 2 q.b for Euclidean
// distance (|q|^2 is the same for every point of a query and is left out) or
// -q.b for mips. A point whose D32 is below the query's current threshold is
// appended to the (query, slice) buffer; a buffer that could overflow on the
// next tile is cut to its C best keys, whose C-th distance becomes the
// threshold. At the end of the slice every buffer holds its slice's C best
// (by D32, then id) and the slice's threshold.
//
// Pass 2 (gt_final_kernel, a warp per query): s_k = the k-th smallest D32 of
// the union (which holds the global top C by D32). Every D32 is within
// `bound` of the exact value |b|^2 - 2 q.b (or -q.b): the float32 dot
// product's error is at most (d + 1) u |q||b| and |b|^2 and the final FMA add
// at most u each (u = 2^-24), so with B = max |b|,
//   bound = 2 (2 u B^2 + (2d + 4) u |q| B)   (Euclidean),
//   bound = 2 (d + 2) u |q| B                 (mips),
// twice the first-order bound. A true top-k point x has D32(x) <= s_k +
// 2 bound; if every slice's threshold is above that, no slice cut such a
// point, and the FP64 distances (exact_dist, the same arithmetic as
// bruteforce_kernel) of the candidates with D32 <= s_k + 2 bound decide the
// answer, ties by id. A query that fails the test is recomputed by
// bruteforce_kernel.
constexpr int GT_QT = 64, GT_PT = 128;

struct GtArgs {
  const float* points;  // n rows of spf floats (rows zero-padded)
  const float* pnorm;   // |b|^2 rounded to float (Euclidean)
  uint64_t n;
  uint32_t spf;         // floats per row
  uint32_t dpad;        // dimensions rounded up to 4
  const float* queries; // nq rows of spf floats
  uint32_t nq;
  uint32_t slices;
  uint64_t slice_len;
  uint32_t C, CB;
  uint64_t* cand;       // per (query, slice): CB keys
  uint32_t* count;      // per (query, slice)
  float* thr;           // per (query, slice): the slice's C-th D32 (+inf: fewer than C points)
};

// Sort the cnt keys of buf (cnt <= CB) and keep the best `keep` in place;
// warp-cooperative rank placement through the warp's scratch row.
__device__ __forceinline__ void gt_cut(uint64_t* buf, uint32_t cnt, uint32_t keep, uint64_t* scr, int lane) {
  for (uint32_t i = lane; i < cnt; i += 32) scr[i] = buf[i];
  __syncwarp();
  for (uint32_t i = lane; i < cnt; i += 32) {
    const uint64_t ki = scr[i];
    uint32_t r = 0;
    for (uint32_t j = 0; j < cnt; j++) r += scr[j] < ki;
    if (r < keep) buf[r] = ki;
  }
  __syncwarp();
}

template <int MT>
__global__ void __launch_bounds__(256, 2) gt_cand_kernel(GtArgs g) {
  extern __shared__ __align__(16) float gsm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tq = tid & 15, tp = tid >> 4;
  const uint32_t dp = g.dpad;
  float* qT = gsm;                    // dp x GT_QT
  float* pT = qT + (size_t)dp * GT_QT;  // dp x GT_PT
  float* thr_s = pT + (size_t)dp * GT_PT;
  uint32_t* cnt_s = reinterpret_cast<uint32_t*>(thr_s + GT_QT);
  uint64_t* scr = reinterpret_cast<uint64_t*>(cnt_s + GT_QT) + (size_t)warp * g.CB;
  const uint32_t q0 = blockIdx.x * GT_QT;
  const uint32_t slice = blockIdx.y;
  const uint64_t p_begin = (uint64_t)slice * g.slice_len;
  const uint64_t p_end = p_begin + g.slice_len < g.n ? p_begin + g.slice_len : g.n;
  for (uint32_t e = tid; e < dp * GT_QT; e += 256) {
    const uint32_t i = e % GT_QT, t = e / GT_QT;
    qT[(size_t)t * GT_QT + i] = q0 + i < g.nq ? g.queries[(uint64_t)(q0 + i) * g.spf + t] : 0.0f;
  }
  if (tid < GT_QT) {
    thr_s[tid] = __int_as_float(0x7f800000);
    cnt_s[tid] = 0;
  }
  __syncthreads();
  const uint32_t dq4 = dp / 4;
  for (uint64_t p0 = p_begin; p0 < p_end; p0 += GT_PT) {
    // stage the tile transposed: lanes take consecutive rows at one 16-byte chunk
    for (uint32_t e = tid; e < dq4 * GT_PT; e += 256) {
      const uint32_t j = e % GT_PT, c = e / GT_PT;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (p0 + j < p_end) v = __ldg(reinterpret_cast<const float4*>(g.points + (p0 + j) * g.spf) + c);
      pT[(size_t)(4 * c + 0) * GT_PT + j] = v.x;
      pT[(size_t)(4 * c + 1) * GT_PT + j] = v.y;
      pT[(size_t)(4 * c + 2) * GT_PT + j] = v.z;
      pT[(size_t)(4 * c + 3) * GT_PT + j] = v.w;
    }
    __syncthreads();
    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;
    for (uint32_t t = 0; t < dp; t++) {
      const float4 a = reinterpret_cast<const float4*>(qT + (size_t)t * GT_QT)[tq];
      const float4 b0 = reinterpret_cast<const float4*>(pT + (size_t)t * GT_PT)[2 * tp];
      const float4 b1 = reinterpret_cast<const float4*>(pT + (size_t)t * GT_PT)[2 * tp + 1];
      const float av[4] = {a.x, a.y, a.z, a.w};
      const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = __fmaf_rn(av[i], bv[j], acc[i][j]);
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const uint64_t pj = p0 + 8 * tp + j;
      if (pj >= p_end) continue;
      const float pn = MT == MT_L2 ? __ldg(g.pnorm + pj) : 0.0f;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const uint32_t ql = 4 * tq + i;
        if (q0 + ql >= g.nq) continue;
        const float dv = MT == MT_L2 ? __fmaf_rn(-2.0f, acc[i][j], pn) : -acc[i][j];
        if (dv < thr_s[ql]) {
          const uint32_t pos = atomicAdd(cnt_s + ql, 1u);
          if (pos < g.CB)
            g.cand[((uint64_t)(q0 + ql) * g.slices + slice) * g.CB + pos] = make_key(dv, (uint32_t)pj);
        }
      }
    }
    __syncthreads();
    // cut the buffers that the next tile could overflow (a tile adds at most GT_PT per query)
    const bool last = p0 + GT_PT >= p_end;
    for (uint32_t ql = warp; ql < GT_QT; ql += 8) {
      const uint32_t c = cnt_s[ql];
      if (q0 + ql >= g.nq || !(c > g.CB - GT_PT || (last && c > 0))) continue;
      uint64_t* buf = g.cand + ((uint64_t)(q0 + ql) * g.slices + slice) * g.CB;
      const uint32_t keep = c < g.C ? c : g.C;
      gt_cut(buf, c, keep, scr, lane);
      if (lane == 0) {
        cnt_s[ql] = keep;
        if (keep == g.C) thr_s[ql] = key_dist(buf[g.C - 1]);
      }
      __syncwarp();
    }
    __syncthreads();
  }
  if (tid < GT_QT && q0 + tid < g.nq) {
    g.count[(uint64_t)(q0 + tid) * g.slices + slice] = cnt_s[tid];
    g.thr[(uint64_t)(q0 + tid) * g.slices + slice] = cnt_s[tid] == g.C ? thr_s[tid] : __int_as_float(0x7f800000);
  }
}

template <int MT>
__global__ void __launch_bounds__(256) gt_final_kernel(GtArgs g, const uint8_t* __restrict__ pts_bytes, uint64_t stride,
                                                       int d, const uint8_t* __restrict__ q_bytes, float bmax, uint32_t k,
                                                       uint32_t* out_ids, double* out_d, uint32_t* fallback,
                                                       uint32_t* nfallback) {
  extern __shared__ __align__(16) uint8_t fsm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t qi = blockIdx.x * 8 + warp;
  if (qi >= g.nq) return;  // warp-uniform, no block barrier below
  const uint32_t U = g.slices * g.C;
  uint64_t* keys = reinterpret_cast<uint64_t*>(fsm) + (size_t)warp * U;
  // gather the union of the slices' candidates (slots past a slice's count are padding)
  uint32_t m = 0;
  float tmin = __int_as_float(0x7f800000);
  for (uint32_t s = 0; s < g.slices; s++) {
    const uint64_t slot = (uint64_t)qi * g.slices + s;
    const uint32_t c = g.count[slot];
    tmin = fminf(tmin, g.thr[slot]);
    for (uint32_t i = lane; i < c; i += 32) keys[m + i] = g.cand[slot * g.CB + i];
    m += c;
  }
  __syncwarp();
  // s_k: the k-th smallest key of the union
  uint64_t sk = ~0ull;
  for (uint32_t i = lane; i < m; i += 32) {
    const uint64_t ki = keys[i];
    uint32_t r = 0;
    for (uint32_t j = 0; j < m; j++) r += keys[j] < ki;
    if (r == (k <= m ? k - 1 : m - 1)) sk = ki;
  }
  for (int o = 16; o; o >>= 1) {
    const uint64_t t = __shfl_xor_sync(0xFFFFFFFFu, sk, o);
    sk = t < sk ? t : sk;
  }
  const float* qf = reinterpret_cast<const float*>(q_bytes + (uint64_t)qi * stride);
  double qn2 = 0.0;
  for (int t = lane; t < d; t += 32) qn2 += (double)qf[t] * (double)qf[t];
  for (int o = 16; o; o >>= 1) qn2 += __shfl_xor_sync(0xFFFFFFFFu, qn2, o);
  const double u = 5.9604644775390625e-08;  // 2^-24
  const double qn = sqrt(qn2), B = (double)bmax;
  const double bound = MT == MT_L2 ? 2.0 * (2.0 * u * B * B + (2.0 * d + 4.0) * u * qn * B) + 1e-12
                                   : 2.0 * ((double)d + 2.0) * u * qn * B + 1e-12;
  const double lim = (double)key_dist(sk) + 2.0 * bound;
  if (m < k || !((double)tmin > lim)) {
    if (lane == 0) fallback[atomicAdd(nfallback, 1u)] = qi;
    return;
  }
  // FP64 distances of the candidates within the margin, compacted in place
  uint32_t nc = 0;
  for (uint32_t b = 0; b < m; b += 32) {
    const uint32_t i = b + lane;
    const bool in = i < m && (double)key_dist(keys[i]) <= lim;
    const uint64_t ki = in ? keys[i] : 0ull;
    const unsigned msk = __ballot_sync(0xFFFFFFFFu, in);
    __syncwarp();
    if (in) keys[nc + __popc(msk & ((1u << lane) - 1))] = ki;
    nc += __popc(msk);
    __syncwarp();
  }
  // each lane scores its candidates, then rank by (FP64 distance, id)
  double* d64 = reinterpret_cast<double*>(fsm + (size_t)64 * U) + (size_t)warp * U;
  uint32_t* idv = reinterpret_cast<uint32_t*>(fsm + (size_t)128 * U) + (size_t)warp * U;
  for (uint32_t i = lane; i < nc; i += 32) {
    const uint32_t id = key_id(keys[i]);
    idv[i] = id;
    d64[i] = exact_dist<DT_F32, MT>(pts_bytes + (uint64_t)id * stride, q_bytes + (uint64_t)qi * stride, d);
  }
  __syncwarp();
  for (uint32_t i = lane; i < nc; i += 32) {
    uint32_t r = 0;
    for (uint32_t j = 0; j < nc; j++) r += dless(d64[j], idv[j], d64[i], idv[i]);
    if (r < k) {
      out_ids[(uint64_t)qi * k + r] = idv[i];
      if (out_d) out_d[(uint64_t)qi * k + r] = d64[i];
    }
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

// |b|^2 of every row in FP64, stored rounded to float, and the largest |b|
// (as the bits of a non-negative double, whose order is the integer order).
__global__ void gt_norms_kernel(const float* __restrict__ pts, uint64_t n, uint32_t spf, int d, float* pnorm,
                                unsigned long long* bmax_bits) {
  double mx = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float* r = pts + i * spf;
    double s = 0.0;
    for (int t = 0; t < d; t++) s += (double)r[t] * (double)r[t];
    pnorm[i] = (float)s;
    mx = fmax(mx, sqrt(s));
  }
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(bmax_bits, (unsigned long long)__double_as_longlong(mx));
}

// The float32 fast path of pann_groundtruth (see gt_cand_kernel); dq holds
// the queries in device rows of idx->stride bytes. Queries that fail the
// margin test are recomputed with bruteforce_kernel.
static int groundtruth_f32_fast(pann_index* idx, const uint8_t* dq, uint32_t nq, uint32_t k, uint32_t* dids,
                                double* dd, cudaStream_t st) {
  const uint32_t C = std::max<uint32_t>(64, (2 * k + 31) / 32 * 32);
  const uint32_t CB = C + GT_PT;
  const uint32_t qtiles = (nq + GT_QT - 1) / GT_QT;
  uint64_t slices = std::max<uint64_t>(1, (4ull * idx->sm_count + qtiles - 1) / qtiles);
  slices = std::min<uint64_t>(slices, std::max<uint64_t>(1, idx->n / 4096));
  slices = std::min<uint64_t>(slices, std::max<uint32_t>(1, 1024 / C));
  const uint64_t slice_len = (idx->n + slices - 1) / slices;
  const uint32_t U = (uint32_t)slices * C;
  const uint32_t dpad = (idx->d + 3) & ~3u;
  const size_t smem1 = 4ull * dpad * (GT_QT + GT_PT) + 8ull * GT_QT + 8ull * 8 * CB;
  const size_t smem2 = 20ull * 8 * U;
  if (smem1 > idx->smem_optin || smem2 > idx->smem_optin) return PANN_EINVAL;  // caller takes the plain kernel
  struct Owned : DevBuf {
    ~Owned() { release(); }
  };
  Owned cand, cnt, thr, pn, misc;
  PANN_CUDA(cand.ensure(8ull * nq * slices * CB));
  PANN_CUDA(cnt.ensure(4ull * nq * slices));
  PANN_CUDA(thr.ensure(4ull * nq * slices));
  PANN_CUDA(pn.ensure(4ull * idx->n));
  PANN_CUDA(misc.ensure(64 + 4ull * nq));
  unsigned long long* bmax_bits = misc.as<unsigned long long>();
  uint32_t* nfall = reinterpret_cast<uint32_t*>(misc.as<uint8_t>() + 8);
  uint32_t* fall = reinterpret_cast<uint32_t*>(misc.as<uint8_t>() + 64);
  PANN_CUDA(cudaMemsetAsync(misc.p, 0, 64, st));
  gt_norms_kernel<<<4 * idx->sm_count, 256, 0, st>>>(reinterpret_cast<const float*>(idx->d_points), idx->n,
                                                     (uint32_t)(idx->stride / 4), (int)idx->d, pn.as<float>(), bmax_bits);
  PANN_CUDA(cudaGetLastError());
  GtArgs g{};
  g.points = reinterpret_cast<const float*>(idx->d_points);
  g.pnorm = pn.as<float>();
  g.n = idx->n;
  g.spf = (uint32_t)(idx->stride / 4);
  g.dpad = dpad;
  g.queries = reinterpret_cast<const float*>(dq);
  g.nq = nq;
  g.slices = (uint32_t)slices;
  g.slice_len = slice_len;
  g.C = C;
  g.CB = CB;
  g.cand = cand.as<uint64_t>();
  g.count = cnt.as<uint32_t>();
  g.thr = thr.as<float>();
  dim3 grid1(qtiles, (unsigned)slices);
  if (idx->metric == MT_L2) {
    PANN_CUDA(cudaFuncSetAttribute(gt_cand_kernel<MT_L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max()));
    gt_cand_kernel<MT_L2><<<grid1, 256, smem1, st>>>(g);
  } else {
    PANN_CUDA(cudaFuncSetAttribute(gt_cand_kernel<MT_IP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max()));
    gt_cand_kernel<MT_IP><<<grid1, 256, smem1, st>>>(g);
  }
  PANN_CUDA(cudaGetLastError());
  unsigned long long bm = 0;
  PANN_CUDA(cudaMemcpyAsync(&bm, bmax_bits, 8, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  double bmax_d;
  std::memcpy(&bmax_d, &bm, 8);
  const float bmax = (float)(bmax_d * (1.0 + 1e-6));
  const unsigned blocks2 = (nq + 7) / 8;
  if (idx->metric == MT_L2) {
    PANN_CUDA(cudaFuncSetAttribute(gt_final_kernel<MT_L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max()));
    gt_final_kernel<MT_L2><<<blocks2, 256, smem2, st>>>(g, idx->d_points, idx->stride, (int)idx->d, dq, bmax, k, dids,
                                                        dd, fall, nfall);
  } else {
    PANN_CUDA(cudaFuncSetAttribute(gt_final_kernel<MT_IP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max()));
    gt_final_kernel<MT_IP><<<blocks2, 256, smem2, st>>>(g, idx->d_points, idx->stride, (int)idx->d, dq, bmax, k, dids,
                                                        dd, fall, nfall);
  }
  PANN_CUDA(cudaGetLastError());
  uint32_t nf = 0;
  PANN_CUDA(cudaMemcpyAsync(&nf, nfall, 4, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  idx->gt_fallbacks = nf;
  if (nf == 0) return PANN_OK;
  // recompute the queries that failed the margin test with the plain FP64 kernel
  std::vector<uint32_t> fl(nf);
  PANN_CUDA(cudaMemcpyAsync(fl.data(), fall, 4ull * nf, cudaMemcpyDeviceToHost, st));
  PANN_CUDA(cudaStreamSynchronize(st));
  Owned fq, fids, fd;
  PANN_CUDA(fq.ensure(idx->stride * (size_t)nf));
  PANN_CUDA(fids.ensure(4ull * k * nf));
  PANN_CUDA(fd.ensure(8ull * k * nf));
  for (uint32_t i = 0; i < nf; i++)
    PANN_CUDA(cudaMemcpyAsync(fq.as<uint8_t>() + (size_t)i * idx->stride, dq + (size_t)fl[i] * idx->stride, idx->stride,
                              cudaMemcpyDeviceToDevice, st));
  const size_t smem = 8 * idx->stride + 8 * (size_t)k * (sizeof(double) + sizeof(uint32_t));
  auto kern = idx->metric == MT_L2 ? bruteforce_kernel<DT_F32, MT_L2> : bruteforce_kernel<DT_F32, MT_IP>;
  PANN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max()));
  kern<<<(nf + 7) / 8, 256, smem, st>>>(idx->d_points, idx->n, idx->stride, (int)idx->d, fq.as<uint8_t>(), nf, k,
                                        fids.as<uint32_t>(), fd.as<double>());
  PANN_CUDA(cudaGetLastError());
  for (uint32_t i = 0; i < nf; i++) {
    PANN_CUDA(cudaMemcpyAsync(dids + (size_t)fl[i] * k, fids.as<uint32_t>() + (size_t)i * k, 4ull * k,
                              cudaMemcpyDeviceToDevice, st));
    if (dd)
      PANN_CUDA(cudaMemcpyAsync(dd + (size_t)fl[i] * k, fd.as<double>() + (size_t)i * k, 8ull * k,
                                cudaMemcpyDeviceToDevice, st));
  }
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
  bool done = false;
  if (idx->dtype == DT_F32 && k <= 256 && !std::getenv("PANN_GT_PLAIN")) {
    int rc = groundtruth_f32_fast(idx, dq, nq, k, dids, dd, st);
    if (rc != PANN_OK && rc != PANN_EINVAL) {
      cudaFree(dq);
      cudaFree(dids);
      cudaFree(dd);
      return rc;
    }
    done = rc == PANN_OK;
  }
#define PANN_BF_CASE(DT, MT)                                                                                   \
  if (!done && idx->dtype == DT && idx->metric == MT) {                                                        \
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
