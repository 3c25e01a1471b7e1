// Multi-parent tile search: the throughput variant of the precision form
// (pann_search_options::parents > 0).
//
// The exact search expands one frontier node per step, as filtered_beam_search
// does (beamSearch.h:116-222); every step is a chain of dependent memory round
// trips (adjacency row, then the neighbours' rows) for one warp. This kernel
// gives each query a CTA and expands the `parents` best unvisited frontier
// entries per step: their adjacency rows are read together, the new
// neighbours (an exact shared-memory seen set) form one candidate tile whose
// low-precision rows are staged into shared memory with cp.async, one round
// trip per CWs rows (CWs picked at launch for occupancy), all 128 threads
// score the tile (bfloat16, or FP8 E4M3 with
// per-dimension scales, float32 accumulation), and the survivors are merged
// into the sorted frontier by rank. The best `rerank` (default 4k) frontier
// entries are re-scored with the exact float32 distance before the top k are
// written. The visiting order differs from the reference's (several parents
// per step), so this is a search of its own with its own recall curve,
// measured against FP64 brute force; it is not a parity path.
#include <cuda_runtime.h>
#include <algorithm>
#include <string>

#include "common.cuh"
#include "index.cuh"
#include "lowprec.cuh"
#include "tiers.cuh"
#include "umma.cuh"

namespace pann {

enum : uint32_t { QS_TRUNCATED = 32u };  // the seen table filled: the search stopped early

struct TileLayout {
  size_t q, sc, fr, fr2, cand, cid, table, stage, misc, qb, nrm, tcw, total;
  uint32_t sstride;  // staged row stride (bytes; CUDA-core scoring)
};

// Rows a tensor-core scoring round takes: the MMA's M.
constexpr uint32_t TC_ROWS = 128;

// CW: candidates a step can produce (parents x degree); CWs: rows staged at
// once (a step with more candidates stages and scores them in rounds). With
// tensor-core scoring (tc) the rows are staged TC_ROWS at a time in the
// core-matrix layout (umma.cuh), beside the query operand (16 rows: the
// query's split terms, the rest zero), the staged rows' squared norms and the
// MMA barrier and tensor-memory address.
__host__ __device__ inline TileLayout tile_layout(uint32_t d, uint32_t L, uint32_t CW, uint32_t S,
                                                  uint64_t lp_stride, uint32_t CWs, bool tc = false) {
  TileLayout t{};
  size_t o = 0;
  const size_t dpad = (d + 3) & ~3u;
  // rows at an odd multiple of 16 bytes apart: conflict-free 16-byte reads
  t.sstride = (uint32_t)(((lp_stride / 16) % 2 == 0) ? lp_stride + 16 : lp_stride);
  // every region starts on a 16-byte boundary (cp.async destinations and MMA operands need it)
#define PANN_TILE_TAKE(field, bytes) \
  t.field = o;                        \
  o += ((size_t)(bytes) + 15) & ~(size_t)15;
  PANN_TILE_TAKE(q, 4 * dpad)
  PANN_TILE_TAKE(sc, 4 * dpad)
  PANN_TILE_TAKE(fr, 8ull * L)
  PANN_TILE_TAKE(fr2, 8ull * L)
  PANN_TILE_TAKE(cand, 8ull * (CW > L ? CW : L))
  PANN_TILE_TAKE(cid, 4ull * CW)
  PANN_TILE_TAKE(table, 4ull * S)
  if (tc) {
    PANN_TILE_TAKE(stage, (size_t)TC_ROWS * lp_stride)
    PANN_TILE_TAKE(qb, 16 * lp_stride)
    PANN_TILE_TAKE(nrm, 4ull * TC_ROWS)
    PANN_TILE_TAKE(tcw, 16)
  } else {
    PANN_TILE_TAKE(stage, (size_t)CWs * t.sstride)
  }
  PANN_TILE_TAKE(misc, 64)
#undef PANN_TILE_TAKE
  t.total = o;
  return t;
}

// Exact float32 distance in the reference's order (euclidian_point.h:83-90,
// mips_point.h:60-66): sequential sum, every product and sum rounded on its own.
template <int MT>
__device__ __forceinline__ float exact_f32_dist(const float* __restrict__ row, const float* q, uint32_t d) {
  float r = 0.0f;
  for (uint32_t i = 0; i < d; i++) {
    if (MT == MT_L2) {
      const float t = __fsub_rn(__ldg(row + i), q[i]);
      r = __fadd_rn(r, __fmul_rn(t, t));
    } else {
      r = __fadd_rn(r, __fmul_rn(__ldg(row + i), q[i]));
    }
  }
  return MT == MT_L2 ? r : -r;
}

// Approximate distance of one staged low-precision row (16-byte reads).
template <int MT, int PREC>
__device__ __forceinline__ float tile_row_dist(const uint8_t* row, const float* q, const float* sc, uint32_t d,
                                               uint32_t chunks) {
  float a0 = 0.f, a1 = 0.f;
  constexpr uint32_t VPC = PREC == PREC_BF16 ? 8 : 16;
  for (uint32_t c = 0; c < chunks; c++) {
    const uint4 v = reinterpret_cast<const uint4*>(row)[c];
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
      for (int h = 0; h < (PREC == PREC_BF16 ? 1 : 2); h++) {
        const uint32_t e = c * VPC + j * (VPC / 4) + 2 * h;
        if (e >= d) break;
        float2 x;
        if (PREC == PREC_BF16) {
          x = bf16x2_to_f2(w[j]);
        } else {
          x = e4m3x2_to_f2(w[j] >> (16 * h));
          x.x *= sc[e];
          x.y *= sc[e + 1];
        }
        if (MT == MT_L2) {
          const float t0 = x.x - q[e], t1 = x.y - q[e + 1];
          a0 = fmaf(t0, t0, a0);
          a1 = fmaf(t1, t1, a1);
        } else {
          a0 = fmaf(x.x, q[e], a0);
          a1 = fmaf(x.y, q[e + 1], a1);
        }
      }
    }
  }
  return MT == MT_L2 ? a0 + a1 : -(a0 + a1);
}

// Seen-set slots of a query with beam L: (L + 16) * nel * 1.35 rounded up to
// a multiple of 32, within [4 (R + 1), 16384] (not a power of two: slots are
// chosen by multiplicative range reduction); a query stops early (flagged) when
// its set reaches 15/16 of that. Per query, so a batch answers each query as a
// search with that query's beam alone would.
__host__ __device__ inline uint32_t tile_seen_slots(uint32_t L, uint32_t nel, uint32_t R) {
  uint64_t s = ((uint64_t)(L + 16) * nel * 135 / 100 + 31) & ~31ull;
  const uint64_t lo = 4ull * (R + 1);
  if (s < lo) s = (lo + 31) & ~31ull;
  if (s > 16384) s = 16384;
  return (uint32_t)s;
}

// Home slot in [0, S) of an id (Fibonacci hashing, then range reduction).
__device__ __forceinline__ uint32_t tile_slot(uint32_t id, uint32_t S) { return __umulhi(id * 0x9E3779B1u, S); }

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(gmem_src) : "memory");
}

// Time the MMA barrier is waited for before a round is given up (one second,
// far beyond any MMA's latency; the query is then marked QS_INTERNAL).
constexpr uint64_t TC_WAIT_LIMIT = 1000000000ull;

// TC: score each staged round on the tensor cores (tcgen05.mma, M = 128 rows,
// N = 16, float32 accumulator in tensor memory) instead of one row per thread
// on the CUDA cores. The A operand is the staged rows as stored (bfloat16, or
// E4M3 of x / s_t); the B operand is the query split into terms that the
// operand format holds exactly: bfloat16 hi + lo, or for FP8 three E4M3 terms
// of s_t q_t, each scaled by a power of two into the format's range. The MMA
// gives each row's dot product with every term; their sum is b.q to about
// float32 accuracy, and the Euclidean score is |b|^2 - 2 b.q + |q|^2 with the
// row's squared norm precomputed (SearchArgs::lp_norms). The traversal, the
// cutoff, the merge and the exact re-rank are those of the CUDA-core scoring.
template <int MT, int PREC, bool TC>
__global__ void __launch_bounds__(128) search_tile_kernel(SearchArgs a, uint32_t W, uint32_t S, uint32_t CW,
                                                          uint32_t CWs) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const unsigned FULL = 0xFFFFFFFFu;
  const TileLayout ly = tile_layout(a.d, a.L, CW, S, a.lp_stride, CWs, TC);
  float* qf = reinterpret_cast<float*>(smem + ly.q);
  float* sc = reinterpret_cast<float*>(smem + ly.sc);
  uint64_t* frA = reinterpret_cast<uint64_t*>(smem + ly.fr);
  uint64_t* frB = reinterpret_cast<uint64_t*>(smem + ly.fr2);
  uint64_t* cand = reinterpret_cast<uint64_t*>(smem + ly.cand);
  uint32_t* cid = reinterpret_cast<uint32_t*>(smem + ly.cid);
  uint32_t* table = reinterpret_cast<uint32_t*>(smem + ly.table);
  uint8_t* stage = smem + ly.stage;
  uint32_t* misc = reinterpret_cast<uint32_t*>(smem + ly.misc);
  // misc: [0] job  [1] new ids  [2] kept candidates  [3] parents  [4] table entries  [5..8] parent ids
  //       [9] truncated
  uint32_t* par = misc + 5;
  const uint32_t nel = a.dl < a.R ? a.dl : a.R;
  if (PREC == PREC_FP8)
    for (uint32_t i = tid; i < a.d; i += blockDim.x) sc[i] = a.lp_scales[i];
  const uint32_t njobs = a.njobs_dev ? *a.njobs_dev : a.nq;
  // tensor-core state: the MMA barrier, the tensor-memory columns (32, of
  // which the 16 of N are used), the barrier's phase
  uint32_t bar = 0, tmem = 0, phase = 0;
  bool tc_ok = true;
  if (TC) {
    bar = smem_u32(smem + ly.tcw);
    if (warp == 0) tmem_alloc(smem_u32(smem + ly.tcw + 8), 32);
    if (tid == 0) mbar_init(bar, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    tmem = *reinterpret_cast<volatile uint32_t*>(smem + ly.tcw + 8);
  }

  for (;;) {
    __syncthreads();
    if (tid == 0) misc[0] = atomicAdd(a.job_counter, 1u);
    __syncthreads();
    const uint32_t job = misc[0];
    if (job >= njobs) break;
    const uint32_t qi = a.job_list ? a.job_list[job] : job;
    const uint32_t L = a.qL ? a.qL[qi] : a.L;
    const uint32_t kq = a.qk ? a.qk[qi] : a.k;
    const uint32_t Sq = a.qL ? tile_seen_slots(L, nel, a.R) : S;  // <= S
    const uint32_t fill_limit = Sq - Sq / 16;
    const float* qsrc = reinterpret_cast<const float*>(a.queries + (uint64_t)qi * a.stride);
    for (uint32_t i = tid; i < a.d; i += blockDim.x) qf[i] = qsrc[i];
    for (uint32_t i = tid; i < Sq; i += blockDim.x) table[i] = PANN_PAD;
    if (tid < 15) misc[1 + tid] = 0;
    __syncthreads();
    float tc_qn = 0.0f, tc_unscale = 1.0f;
    if (TC) {
      // the query operand: 16 rows of lp_chunks chunks, rows past the split terms zero
      uint8_t* qb = smem + ly.qb;
      for (uint32_t i = tid; i < 16 * a.lp_chunks * 4; i += blockDim.x) reinterpret_cast<uint32_t*>(qb)[i] = 0u;
      // |q|^2 (Euclidean) and, for FP8, max |s_t q_t| (float bits; non-negative floats order as integers)
      float part = 0.0f, mx = 0.0f;
      for (uint32_t t = tid; t < a.d; t += blockDim.x) {
        part += qf[t] * qf[t];
        if (PREC == PREC_FP8) mx = fmaxf(mx, fabsf(sc[t] * qf[t]));
      }
      for (int o = 16; o; o >>= 1) {
        part += __shfl_xor_sync(FULL, part, o);
        mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
      }
      if (lane == 0) {
        atomicAdd(reinterpret_cast<float*>(misc + 10), part);
        atomicMax(misc + 11, __float_as_uint(mx));
      }
      __syncthreads();
      tc_qn = __uint_as_float(misc[10]);
      // FP8 terms: v = s_t q_t 2^e0 with max |v| in [128, 256); three E4M3 terms of 4 bits each
      int e0 = 0;
      if (PREC == PREC_FP8) {
        const float m = __uint_as_float(misc[11]);
        int ex = 0;
        if (m > 0.0f) frexpf(m, &ex);
        e0 = 8 - ex;
        tc_unscale = ldexpf(1.0f, -e0);
      }
      for (uint32_t t = tid; t < a.d; t += blockDim.x) {
        if (PREC == PREC_BF16) {
          const __nv_bfloat16 hi = __float2bfloat16_rn(qf[t]);
          const __nv_bfloat16 lo = __float2bfloat16_rn(qf[t] - __bfloat162float(hi));
          const uint32_t c = (2 * t) / 16, b = (2 * t) % 16;
          *reinterpret_cast<__nv_bfloat16*>(qb + cm_offset(0, c, a.lp_chunks) + b) = hi;
          *reinterpret_cast<__nv_bfloat16*>(qb + cm_offset(1, c, a.lp_chunks) + b) = lo;
        } else {
          float v = ldexpf(sc[t] * qf[t], e0);
          const uint32_t c = t / 16, b = t % 16;
#pragma unroll
          for (uint32_t j = 0; j < 3; j++) {
            const __nv_fp8_e4m3 f(v);
            qb[cm_offset(j, c, a.lp_chunks) + b] = *reinterpret_cast<const uint8_t*>(&f);
            v = (v - float(f)) * 16.0f;
          }
        }
      }
      fence_async_smem();
      __syncthreads();
    }
    // start points: approximate distances from global rows, all in the seen set
    for (uint32_t s = tid; s < a.n_start; s += blockDim.x) {
      const uint32_t id = a.starts[s];
      const float dd = tile_row_dist<MT, PREC>(a.lp_rows + (uint64_t)id * a.lp_stride, qf, sc, a.d, a.lp_chunks);
      cand[s] = make_key(dd, id);
      uint32_t h = tile_slot(id, Sq);
      for (uint32_t p = 0; p < Sq; p++) {
        const uint32_t old = atomicCAS(table + h, PANN_PAD, id);
        if (old == PANN_PAD || old == id) break;
        h = h + 1 == Sq ? 0 : h + 1;
      }
    }
    __syncthreads();
    for (uint32_t s = tid; s < a.n_start; s += blockDim.x) {
      uint32_t r = 0;
      for (uint32_t j = 0; j < a.n_start; j++) r += cand[j] < cand[s];
      frA[r] = cand[s];
    }
    if (tid == 0) misc[4] = a.n_start;
    uint64_t* fr = frA;
    uint64_t* fr2 = frB;
    uint32_t fn = a.n_start;
    uint64_t nvis = 0;
    uint32_t cmps = a.n_start;
    __syncthreads();

    for (;;) {
      // ---- the best `parents` unvisited frontier entries (warp 0)
      const uint64_t room = a.limit > nvis ? a.limit - nvis : 0;
      const uint32_t wlim = (uint32_t)(room < W ? room : W);
      if (warp == 0) {
        uint32_t np = 0, npre = 0;
        for (uint32_t b = 0; b < fn && npre < W; b += 32) {
          const uint32_t i = b + lane;
          unsigned m = __ballot_sync(FULL, i < fn && !(fr[i] & PANN_VFLAG));
          while (m && np < wlim) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            if (lane == 0) {
              par[np] = key_id(fr[b + j]);
              fr[b + j] |= PANN_VFLAG;
            }
            np++;
          }
          // the next best unvisited entries are the likely parents of the
          // next step: start their adjacency rows on their way to L2
          while (m && npre < W) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            if (lane == (int)npre)
              asm volatile("prefetch.global.L2 [%0];" ::"l"(a.graph + (uint64_t)key_id(fr[b + j]) * a.R));
            npre++;
          }
        }
        if (lane == 0) {
          misc[3] = misc[9] ? 0u : np;
          misc[1] = 0;
          misc[2] = 0;
        }
      }
      __syncthreads();
      const uint32_t np = misc[3];
      if (np == 0) break;
      nvis += np;
      // ---- adjacency rows of the parents; new neighbours into the tile
      for (uint32_t x = tid; x < np * nel; x += blockDim.x) {
        const uint32_t p = x / nel, j = x - p * nel;
        const uint32_t id = a.graph[(uint64_t)par[p] * a.R + j];
        if (id == PANN_PAD) continue;
        uint32_t h = tile_slot(id, Sq);
        for (uint32_t probe = 0; probe < Sq; probe++) {
          const uint32_t old = atomicCAS(table + h, PANN_PAD, id);
          if (old == id) break;
          if (old == PANN_PAD) {
            const uint32_t e = atomicAdd(misc + 4, 1u);
            if (e >= fill_limit) misc[9] = 1;  // stop after this step: the table is nearly full
            cid[atomicAdd(misc + 1, 1u)] = id;
            break;
          }
          h = h + 1 == Sq ? 0 : h + 1;
        }
      }
      __syncthreads();
      const uint32_t ncand = misc[1];
      const float cutoff = fn == L ? key_dist(fr[L - 1]) : 3.40282346638528859812e+38F;
      for (uint32_t c0 = 0; c0 < ncand && tc_ok; c0 += CWs) {
        const uint32_t nr = ncand - c0 < CWs ? ncand - c0 : CWs;
        // ---- stage the tile's rows (one round trip per CWs rows)
        for (uint32_t x = tid; x < nr * a.lp_chunks; x += blockDim.x) {
          const uint32_t r = x / a.lp_chunks, c = x - r * a.lp_chunks;
          const uint32_t off = TC ? cm_offset(r, c, a.lp_chunks) : r * ly.sstride + 16 * c;
          cp_async16(stage + off, a.lp_rows + (uint64_t)cid[c0 + r] * a.lp_stride + 16 * c);
        }
        if (TC)
          for (uint32_t r = tid; r < nr; r += blockDim.x)
            reinterpret_cast<float*>(smem + ly.nrm)[r] = __ldg(a.lp_norms + cid[c0 + r]);
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        if (TC) {
          fence_async_smem();
          __syncthreads();
          if (tid == 0) {
            tc_fence_after();
            const uint32_t sbo = a.lp_chunks * 128u;
            const uint32_t sa = smem_u32(stage), sq = smem_u32(smem + ly.qb);
            for (uint32_t kb = 0; kb < a.lp_chunks / 2; kb++) {
              const uint64_t ad = umma_desc(sa + kb * 256u, 128u, sbo), bd = umma_desc(sq + kb * 256u, 128u, sbo);
              if (PREC == PREC_BF16) umma_bf16(tmem, ad, bd, umma_idesc(1, TC_ROWS, 16), kb > 0);
              else umma_fp8(tmem, ad, bd, umma_idesc(0, TC_ROWS, 16), kb > 0);
            }
            umma_commit(bar);
          }
          const bool done = mbar_wait(bar, phase, TC_WAIT_LIMIT);
          phase ^= 1u;
          if (__syncthreads_or(!done)) {
            tc_ok = false;  // the query is marked QS_INTERNAL; its MMA may still run: stop using the stage
            break;
          }
          tc_fence_after();
          float v[4];
          tmem_ld4(tmem + ((uint32_t)(warp * 32) << 16), v);
          const uint32_t r = tid;  // TMEM lane = staged row
          if (r < nr) {
            const float dot = PREC == PREC_BF16 ? v[0] + v[1] : (v[0] + v[1] * 0.0625f + v[2] * 0.00390625f) * tc_unscale;
            const float dd = MT == MT_L2 ? reinterpret_cast<const float*>(smem + ly.nrm)[r] + tc_qn - 2.0f * dot : -dot;
            if (dd < cutoff) cand[atomicAdd(misc + 2, 1u)] = make_key(dd, cid[c0 + r]);
          }
          tc_fence_before();
        } else {
          __syncthreads();
          // ---- score; keep those below the cutoff of a full frontier (beamSearch.h:173-182)
          for (uint32_t r = tid; r < nr; r += blockDim.x) {
            const float dd = tile_row_dist<MT, PREC>(stage + (size_t)r * ly.sstride, qf, sc, a.d, a.lp_chunks);
            if (dd < cutoff) cand[atomicAdd(misc + 2, 1u)] = make_key(dd, cid[c0 + r]);
          }
        }
        __syncthreads();  // the next round overwrites the staged rows (and the accumulator)
      }
      if (!tc_ok) break;
      cmps += ncand;
      const uint32_t nc = misc[2];
      if (nc > 0) {
        // ---- merge by rank: keys are distinct (ids are), visited flags ignored in the order
        for (uint32_t i = tid; i < fn; i += blockDim.x) {
          const uint64_t key = fr[i], mk = key & PANN_KEYMASK;
          uint32_t r = i;
          for (uint32_t j = 0; j < nc; j++) r += cand[j] < mk;
          if (r < L) fr2[r] = key;
        }
        for (uint32_t j = tid; j < nc; j += blockDim.x) {
          const uint64_t ck = cand[j];
          uint32_t lo = 0, hi = fn;
          while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if ((fr[mid] & PANN_KEYMASK) < ck) lo = mid + 1; else hi = mid;
          }
          uint32_t r = lo;
          for (uint32_t t = 0; t < nc; t++) r += cand[t] < ck;
          if (r < L) fr2[r] = ck;
        }
        fn = fn + nc < L ? fn + nc : L;
        uint64_t* t = fr; fr = fr2; fr2 = t;
      }
      __syncthreads();
    }

    // ---- exact float32 re-rank of the best entries, then the top k
    const uint32_t rr = a.rerank ? a.rerank : 4 * kq;
    const uint32_t nr = fn < (rr > kq ? rr : kq) ? fn : (rr > kq ? rr : kq);
    for (uint32_t i = tid; i < nr; i += blockDim.x) {
      const uint32_t id = key_id(fr[i]);
      const float dd = exact_f32_dist<MT>(reinterpret_cast<const float*>(a.points + (uint64_t)id * a.stride), qf, a.d);
      cand[i] = make_key(dd, id);
    }
    __syncthreads();
    uint32_t* const oid = a.out_ids + (uint64_t)qi * a.kstride;
    float* const odist = a.out_dists ? a.out_dists + (uint64_t)qi * a.kstride : nullptr;
    for (uint32_t i = tid; i < nr; i += blockDim.x) {
      const uint64_t key = cand[i];
      uint32_t r = 0;
      for (uint32_t j = 0; j < nr; j++) r += cand[j] < key;
      if (r < kq) {
        oid[r] = key_id(key);
        if (odist) odist[r] = key_dist(key);
      }
    }
    for (uint32_t j = (nr < kq ? nr : kq) + tid; j < a.kstride; j += blockDim.x) {
      oid[j] = PANN_PAD;
      if (odist) odist[j] = 0.0f;
    }
    if (tid == 0) {
      uint32_t status = 0;
      if (fn < kq) status |= QS_SHORT;
      if (misc[9]) status |= QS_TRUNCATED;
      if (!tc_ok) status |= QS_INTERNAL;
      if (a.out_visited) a.out_visited[qi] = (uint32_t)nvis;
      if (a.out_cmps) a.out_cmps[qi] = cmps;
      if (a.out_status) a.out_status[qi] = status;
    }
    if (!tc_ok) break;  // this block takes no more queries (the others do)
  }
  if (TC) {
    if (!tc_ok) mbar_wait(bar, phase ^ 1u, TC_WAIT_LIMIT);  // the round that did not finish in time
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 32);
  }
}

// Blocks of `threads` threads with `smem` bytes of dynamic shared memory that
// one multiprocessor holds, from the kernel's registers and static shared
// memory and the device's per-multiprocessor limits.
static int resident_blocks(const void* k, int threads, size_t smem) {
  cudaFuncAttributes fa{};
  int dev = 0, smem_sm = 0, regs_sm = 0, thr_sm = 0, reserved = 0;
  if (cudaFuncGetAttributes(&fa, k) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess) return 1;
  if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess)
    return 1;
  cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  const size_t per_block_smem = smem + fa.sharedSizeBytes + (size_t)reserved;
  const int warps = (threads + 31) / 32;
  const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;  // allocated per warp in units of 256
  int by_smem = per_block_smem ? (int)((size_t)smem_sm / per_block_smem) : 32;
  int by_regs = regs_warp ? regs_sm / (warps * regs_warp) : 32;
  int by_thr = thr_sm / threads;
  return std::max(1, std::min({by_smem, by_regs, by_thr}));
}

// Rows staged at once: the most that still gives the best occupancy among
// CW, 3/4 CW and 1/2 CW (steps with more new candidates stage in rounds);
// with tensor-core scoring, rounds of TC_ROWS rows.
template <int MT, int PREC, bool TC>
static int launch_tile_t(const pann_index* idx, const SearchArgs& a, uint32_t W, uint32_t S, uint32_t CW,
                         cudaStream_t st, uint32_t tile_rows) {
  auto k = search_tile_kernel<MT, PREC, TC>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max());
  if (e != cudaSuccess) return cuda_fail(e, "tile kernel attribute");
  uint32_t CWs = TC ? TC_ROWS : CW;
  size_t smem = tile_layout(idx->d, a.L, CW, S, idx->lp_stride, CWs, TC).total;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 128, smem) != cudaSuccess || occ <= 0) occ = 1;
  if (!TC && tile_rows > 0) {
    CWs = std::min<uint32_t>(CW, std::max<uint32_t>(16, (tile_rows + 15) & ~15u));
    smem = tile_layout(idx->d, a.L, CW, S, idx->lp_stride, CWs).total;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 128, smem) != cudaSuccess || occ <= 0) occ = 1;
  }
  for (uint32_t f = 3; f >= 2 && !TC && tile_rows == 0; f--) {
    const uint32_t cws = std::max<uint32_t>(32, (CW * f / 4 + 15) & ~15u);
    const size_t sm2 = tile_layout(idx->d, a.L, CW, S, idx->lp_stride, cws).total;
    int occ2 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k, 128, sm2) == cudaSuccess && occ2 > occ) {
      occ = occ2;
      CWs = cws;
      smem = sm2;
    }
  }
  if (TC) {
    // the occupancy query has answered 1 block per SM for this kernel even
    // where 5 fit (measured); the blocks a multiprocessor holds by its shared
    // memory, registers and threads, capped by tensor memory: 32 columns a
    // block, 512 an SM
    occ = std::min(std::max(occ, resident_blocks(reinterpret_cast<const void*>(k), 128, smem)), 16);
  }
  const uint64_t want = a.nq;
  const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)occ * idx->sm_count));
  k<<<blocks, 128, smem, st>>>(a, W, S, CW, CWs);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "tile kernel launch");
  return PANN_OK;
}

// Sizes and launches the tile kernel; returns PANN_EINVAL (and does nothing)
// when its state does not fit in shared memory, so the caller can take the
// single-parent path. scorer 1 scores on the tensor cores (rows of an even
// number of 16-byte chunks; otherwise a clear error).
int enqueue_tile(const pann_index* idx, const SearchPlan& plan, SearchArgs a, uint32_t parents, uint32_t* job_counter,
                 int precision, uint32_t rerank, cudaStream_t st, uint32_t scorer, uint32_t tile_rows) {
  const bool tc = scorer == PANN_SCORER_TENSOR;
  if (tc && (idx->lp_chunks % 2 != 0 || !idx->lp_norms.p))
    return fail(PANN_EDEVICE, "tensor-core scoring needs low-precision rows of an even number of 16-byte chunks "
                              "(bfloat16: d a multiple of 16; FP8: of 32)");
  const uint32_t nel = std::min(plan.dl, idx->R);
  uint32_t W = std::max<uint32_t>(1, std::min<uint32_t>(parents, 4));
  const uint32_t S = tile_seen_slots(plan.L, nel, idx->R);
  TileLayout ly = tile_layout(idx->d, plan.L, W * nel, S, idx->lp_stride, tc ? TC_ROWS : W * nel, tc);
  while (ly.total > idx->smem_optin && W > 1) {
    W--;
    ly = tile_layout(idx->d, plan.L, W * nel, S, idx->lp_stride, tc ? TC_ROWS : W * nel, tc);
  }
  if (ly.total > idx->smem_optin) return fail(PANN_EINVAL, "tile search state does not fit in shared memory");
  a.lp_rows = idx->lp_rows.as<uint8_t>();
  a.lp_stride = idx->lp_stride;
  a.lp_chunks = idx->lp_chunks;
  a.lp_scales = idx->lp_scales.as<float>();
  a.lp_norms = idx->lp_norms.as<float>();
  a.rerank = rerank;
  a.job_counter = job_counter;
  PANN_CUDA(cudaMemsetAsync(job_counter, 0, 4, st));
  const int mt = idx->metric;
#define PANN_TILE_CASE(MTV, PRV)                                                          \
  if (mt == MTV && precision == PRV)                                                    \
    return tc ? launch_tile_t<MTV, PRV, true>(idx, a, W, S, W * nel, st, 0)             \
              : launch_tile_t<MTV, PRV, false>(idx, a, W, S, W * nel, st, tile_rows);
  PANN_TILE_CASE(MT_L2, PREC_BF16)
  PANN_TILE_CASE(MT_IP, PREC_BF16)
  PANN_TILE_CASE(MT_L2, PREC_FP8)
  PANN_TILE_CASE(MT_IP, PREC_FP8)
#undef PANN_TILE_CASE
  return fail(PANN_EINVAL, "the tile search needs a bfloat16 or FP8 precision");
}

}  // namespace pann
