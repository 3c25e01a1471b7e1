// Vamana batch-insertion build on the device: knn_index::build_index and
// batch_insert (algorithms/vamana/index.h:150-319).
//
// Per batch [floor, ceiling) of the insertion order, against the pre-batch graph:
//   1. search      beam search from point 0 for every inserted point (build
//                  mode of the search kernel: the query is the point itself,
//                  which is skipped as a neighbour; the visited list is kept)
//                                                        (index.h:247-264)
//   2. prune       candidates = visited list + current out-neighbours with
//                  their distances, sorted by (dist, id) with a segmented
//                  radix sort, then the greedy alpha-pruning of robustPrune
//                  (index.h:63-120), written straight into the graph rows
//                                                        (index.h:265-273)
//   3. reverse     (new neighbour, inserted point) pairs, stable radix sort by
//                  neighbour = group_by_key (index.h:281-285); per target,
//                  append without repeats when it fits, else robustPrune of
//                  the grouped candidates + current neighbours (index.h:292-303)
// The batch schedule is the reference's prefix doubling (index.h:206-240).
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "index.cuh"

namespace pann {

// Insertion order: indices sorted by splitmix64(seed + i) (the same keys the
// oracle's ParlayLib shim uses for parlay::random_permutation, index.h:212).
__host__ __device__ inline uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

__global__ void perm_keys_kernel(uint64_t* keys, uint32_t* idx, uint64_t n, uint64_t seed) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    keys[i] = splitmix64(seed + i);
    idx[i] = (uint32_t)i;
  }
}

// Job i assembles candidate keys for point pts[i] into keys[begin[i] ..):
//   provided (dist,id) keys (src_keys, src_n) or ids (src_ids, src_n) whose
//   distance to the point is computed here, then the point's current
//   out-neighbours with their distances (robustPrune add = true, index.h:72-77).
template <int DT, int MT>
__global__ void __launch_bounds__(128) assemble_kernel(const uint8_t* __restrict__ points, uint64_t stride, int d,
                                                       int nchunks, const uint32_t* __restrict__ graph, uint32_t R,
                                                       uint32_t njobs, const uint32_t* __restrict__ pts,
                                                       const uint64_t* __restrict__ src_keys, uint32_t src_keys_stride,
                                                       const uint32_t* __restrict__ src_ids,
                                                       const uint32_t* __restrict__ src_off,
                                                       const uint32_t* __restrict__ src_n,
                                                       const uint32_t* __restrict__ seg_begin, uint32_t* seg_end,
                                                       uint64_t* keys, unsigned long long* dist_cmps) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  uint8_t* qs = smem + (size_t)warp * stride;
  for (uint32_t job = blockIdx.x * wpb + warp; job < njobs; job += gridDim.x * wpb) {
    const uint32_t p = pts[job];
    stage_query<DT, MT>(qs, points + (uint64_t)p * stride, nchunks, lane);
    __syncwarp();
    int32_t qq = 0;
    if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), nchunks);
    uint64_t* out = keys + seg_begin[job];
    uint32_t m = src_n[job];
    uint32_t cmps = 0;
    if (src_keys) {
      const uint64_t* sk = src_keys + (uint64_t)job * src_keys_stride;
      for (uint32_t t = lane; t < m; t += 32) out[t] = sk[t];
    } else {
      const uint32_t* si = src_ids + src_off[job];
      for (uint32_t t = lane; t < m; t += 32) {
        uint32_t c = si[t];
        float dd = point_dist<DT, MT>(points + (uint64_t)c * stride, qs, d, nchunks, qq);
        out[t] = make_key(dd, c);
      }
      cmps += m;  // robustPrune id overload (index.h:131-134)
    }
    const uint32_t* g = graph + (uint64_t)p * R;
    uint32_t deg = 0;
    for (uint32_t b = 0; b < R; b += 32) {
      uint32_t j = b + lane;
      uint32_t v = j < R ? __ldg(g + j) : PANN_PAD;
      bool ok = v != PANN_PAD;
      unsigned msk = __ballot_sync(0xFFFFFFFFu, ok);
      if (ok) {
        float dd = point_dist<DT, MT>(points + (uint64_t)v * stride, qs, d, nchunks, qq);
        out[m + b + __popc(msk & ((1u << lane) - 1))] = make_key(dd, v);
      }
      deg += __popc(msk);
    }
    cmps += deg;
    if (lane == 0) {
      seg_end[job] = seg_begin[job] + m + deg;
      atomicAdd(dist_cmps, (unsigned long long)cmps);
    }
    __syncwarp();
  }
}

// Greedy part of robustPrune (index.h:85-116) on a (dist,id)-sorted segment:
// drop repeated ids, then repeatedly take the first live candidate p* (skipping
// the point itself) and kill every later p' with alpha * d(p*, p') <= d(p, p')
// (compared in double). Killed entries get the flag bit; the selection is
// written to the point's graph row, padded.
template <int DT, int MT>
__global__ void __launch_bounds__(128) greedy_prune_kernel(const uint8_t* __restrict__ points, uint64_t stride, int d,
                                                           int nchunks, uint32_t* graph, uint32_t R, uint32_t njobs,
                                                           const uint32_t* __restrict__ pts,
                                                           const uint32_t* __restrict__ seg_begin,
                                                           const uint32_t* __restrict__ seg_end, uint64_t* keys,
                                                           double alpha, unsigned long long* dist_cmps) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const unsigned FULL = 0xFFFFFFFFu;
  uint8_t* qs = smem + (size_t)warp * stride;
  for (uint32_t job = blockIdx.x * wpb + warp; job < njobs; job += gridDim.x * wpb) {
    const uint32_t p = pts[job];
    uint64_t* K = keys + seg_begin[job];
    const uint32_t m = seg_end[job] - seg_begin[job];
    // unique by id (:86-88): equal ids carry equal distances, so repeats are adjacent
    for (uint32_t b = 0; b < m; b += 32) {
      uint32_t i = b + lane;
      bool dup = false;
      if (i < m && i > 0) dup = key_id(K[i]) == key_id(K[i - 1]);
      __syncwarp();
      if (dup) K[i] |= PANN_VFLAG;
    }
    __syncwarp();
    uint32_t nsel = 0, idx = 0;
    unsigned long long cmps = 0;
    uint32_t* row = graph + (uint64_t)p * R;
    while (nsel < R && idx < m) {
      // next live candidate at or after idx
      int found = -1;
      for (uint32_t b = idx; b < m && found < 0; b += 32) {
        uint32_t i = b + lane;
        bool live = i < m && !(K[i] & PANN_VFLAG);
        unsigned msk = __ballot_sync(FULL, live);
        if (msk) found = (int)(b + __ffs(msk) - 1);
      }
      if (found < 0) break;
      const uint32_t pstar = key_id(K[found]);
      idx = (uint32_t)found + 1;
      if (pstar == p) continue;  // :99-101
      if (lane == 0) row[nsel] = pstar;
      nsel++;
      stage_query<DT, MT>(qs, points + (uint64_t)pstar * stride, nchunks, lane);
      __syncwarp();
      int32_t qq = 0;
      if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), nchunks);
      for (uint32_t b = idx; b < m; b += 32) {
        uint32_t i = b + lane;
        bool live = false;
        uint64_t k = 0;
        if (i < m) {
          k = K[i];
          live = !(k & PANN_VFLAG);
        }
        cmps += __popc(__ballot_sync(FULL, live));
        if (live) {
          float dsp = point_dist<DT, MT>(points + (uint64_t)key_id(k) * stride, qs, d, nchunks, qq);
          double dpp = (double)key_dist(k);
          if (__dmul_rn(alpha, (double)dsp) <= dpp) K[i] = k | PANN_VFLAG;
        }
      }
      __syncwarp();
    }
    for (uint32_t j = nsel + lane; j < R; j += 32) row[j] = PANN_PAD;
    if (lane == 0) atomicAdd(dist_cmps, cmps);
    __syncwarp();
  }
}

// Distance of the row at `row` (shared or global memory: generic loads) to the
// point staged at qs, with point_dist's arithmetic (common.cuh).
template <int DT, int MT>
__device__ __forceinline__ float row_dist_generic(const uint8_t* row, const uint8_t* qs, int nchunks, int32_t qq) {
  if (DT == DT_F32) {
    const float4* r = reinterpret_cast<const float4*>(row);
    const float4* q = reinterpret_cast<const float4*>(qs);
    float acc = 0.0f;
    for (int c0 = 0; c0 < nchunks; c0 += ROW_CHUNKS) {
      float4 b[ROW_CHUNKS];
#pragma unroll
      for (int c = 0; c < ROW_CHUNKS; c++)
        if (c0 + c < nchunks) b[c] = r[c0 + c];
#pragma unroll
      for (int c = 0; c < ROW_CHUNKS; c++)
        if (c0 + c < nchunks) acc = f32_chunk<MT>(acc, b[c], q[c0 + c]);
    }
    return MT == MT_L2 ? acc : -acc;
  } else {
    const uint4* r = reinterpret_cast<const uint4*>(row);
    const uint4* q = reinterpret_cast<const uint4*>(qs);
    int32_t pq = 0, pp = 0;
    for (int c = 0; c < nchunks; c++) int_chunk<DT, MT>(r[c], q[c], pq, pp);
    return int_result<MT>(qq, pq, pp);
  }
}

// The greedy part of robustPrune as greedy_prune_kernel computes it, with one
// block of 128 threads per job and the candidates' rows staged in shared
// memory (the first `cap_rows` of the segment; later ones are read from
// global memory): each selection is one pass of the block over the live
// candidates after it, every distance from shared memory, instead of a
// warp's dependent global loads. Same answers: the same candidates, the same
// order of selections, the same float / integer distance and the alpha test
// in double.
template <int DT, int MT>
__global__ void __launch_bounds__(128) greedy_prune_block_kernel(const uint8_t* __restrict__ points, uint64_t stride,
                                                                 int nchunks, uint32_t* graph, uint32_t R,
                                                                 uint32_t njobs, const uint32_t* __restrict__ pts,
                                                                 const uint32_t* __restrict__ seg_begin,
                                                                 const uint32_t* __restrict__ seg_end, uint64_t* keys,
                                                                 double alpha, uint32_t cap_rows,
                                                                 unsigned long long* dist_cmps) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint8_t* qs = smem;                     // p*
  uint8_t* rows = smem + stride;          // cap_rows staged candidate rows
  __shared__ int s_found;
  __shared__ unsigned long long s_cmps;
  for (uint32_t job = blockIdx.x; job < njobs; job += gridDim.x) {
    const uint32_t p = pts[job];
    uint64_t* K = keys + seg_begin[job];
    const uint32_t m = seg_end[job] - seg_begin[job];
    const uint32_t staged = m < cap_rows ? m : cap_rows;
    // unique by id (index.h:86-88), and the rows of the first `staged` candidates
    for (uint32_t i = tid; i < m; i += 128)
      if (i > 0 && key_id(K[i]) == key_id(K[i - 1])) K[i] |= PANN_VFLAG;
    for (uint32_t x = tid; x < staged * (uint32_t)nchunks; x += 128) {
      const uint32_t r = x / nchunks, c = x - r * nchunks;
      reinterpret_cast<uint4*>(rows + (size_t)r * stride)[c] =
          __ldg(reinterpret_cast<const uint4*>(points + (uint64_t)key_id(K[r]) * stride) + c);
    }
    if (tid == 0) s_cmps = 0;
    __syncthreads();
    uint32_t nsel = 0, idx = 0;
    uint32_t* row = graph + (uint64_t)p * R;
    while (nsel < R && idx < m) {
      if (warp == 0) {
        int found = -1;
        for (uint32_t b = idx; b < m && found < 0; b += 32) {
          const uint32_t i = b + lane;
          const bool live = i < m && !(K[i] & PANN_VFLAG);
          const unsigned msk = __ballot_sync(0xFFFFFFFFu, live);
          if (msk) found = (int)(b + __ffs(msk) - 1);
        }
        if (lane == 0) s_found = found;
      }
      __syncthreads();
      const int found = s_found;
      if (found < 0) break;
      const uint32_t pstar = key_id(K[found]);
      idx = (uint32_t)found + 1;
      if (pstar == p) {  // :99-101
        __syncthreads();
        continue;
      }
      if (tid == 0) row[nsel] = pstar;
      nsel++;
      const uint8_t* src = (uint32_t)found < staged ? rows + (size_t)found * stride : points + (uint64_t)pstar * stride;
      for (int c = tid; c < nchunks; c += 128) {
        uint4 v = reinterpret_cast<const uint4*>(src)[c];
        // staged as stage_query stages it: float32 Euclidean rows negated (f32_chunk forms x + (-q))
        if (DT == DT_F32 && MT == MT_L2) v = make_uint4(v.x ^ 0x80000000u, v.y ^ 0x80000000u, v.z ^ 0x80000000u, v.w ^ 0x80000000u);
        reinterpret_cast<uint4*>(qs)[c] = v;
      }
      __syncthreads();
      int32_t qq = 0;
      if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), nchunks);
      uint32_t my_cmps = 0;
      for (uint32_t i = idx + tid; i < m; i += 128) {
        const uint64_t k = K[i];
        if (k & PANN_VFLAG) continue;
        my_cmps++;
        const uint8_t* r = i < staged ? rows + (size_t)i * stride : points + (uint64_t)key_id(k) * stride;
        const float dsp = row_dist_generic<DT, MT>(r, qs, nchunks, qq);
        if (__dmul_rn(alpha, (double)dsp) <= (double)key_dist(k)) K[i] = k | PANN_VFLAG;
      }
      for (int o = 16; o; o >>= 1) my_cmps += __shfl_xor_sync(0xFFFFFFFFu, my_cmps, o);
      if (lane == 0 && my_cmps) atomicAdd(&s_cmps, (unsigned long long)my_cmps);
      __syncthreads();
    }
    for (uint32_t j = nsel + tid; j < R; j += 128) row[j] = PANN_PAD;
    __syncthreads();
    if (tid == 0) atomicAdd(dist_cmps, s_cmps);
  }
}

// Reverse-edge pairs: key = new neighbour (PAD for empty slots), value = inserted point.
__global__ void reverse_pairs_kernel(const uint32_t* __restrict__ graph, uint32_t R, const uint32_t* __restrict__ pts,
                                     uint32_t B, uint32_t* kout, uint32_t* vout) {
  uint64_t total = (uint64_t)B * R;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t i = (uint32_t)(t / R), j = (uint32_t)(t - (uint64_t)i * R);
    uint32_t p = pts[i];
    kout[t] = graph[(uint64_t)p * R + j];
    vout[t] = p;
  }
}

// Per group (target j with m new in-edges): append without repeats when
// m + deg(j) <= R (add_neighbors_without_repeats, index.h:140-146,294-297),
// else record a robustPrune job (index.h:298-301). One warp per group.
__global__ void reverse_classify_kernel(uint32_t* graph, uint32_t R, const uint32_t* __restrict__ uniq,
                                        const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offs,
                                        const uint32_t* __restrict__ num_runs, const uint32_t* __restrict__ vals,
                                        uint32_t* job_pts, uint32_t* job_off, uint32_t* job_n, uint32_t* job_begin,
                                        uint32_t* njobs, unsigned long long* seg_total) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  const uint32_t runs = *num_runs;
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < runs; r += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t tgt = uniq[r];
    if (tgt == PANN_PAD) continue;
    const uint32_t m = counts[r], off = offs[r];
    uint32_t* row = graph + (uint64_t)tgt * R;
    uint32_t deg = 0;
    for (uint32_t b = 0; b < R; b += 32) {
      uint32_t j = b + lane;
      deg += __popc(__ballot_sync(FULL, j < R && row[j] != PANN_PAD));
    }
    if (m + deg <= R) {
      // old neighbours not among the new candidates, in order
      uint32_t keep_cnt = 0;
      uint32_t oldv[32];  // up to 1024 / 32 per lane
      bool keepv[32];
      int nslot = (int)((R + 31) / 32);
      for (int s = 0; s < nslot; s++) {
        uint32_t j = s * 32 + lane;
        uint32_t v = (j < deg) ? row[j] : PANN_PAD;
        bool keep = v != PANN_PAD;
        if (keep)
          for (uint32_t t = 0; t < m; t++)
            if (vals[off + t] == v) { keep = false; break; }
        oldv[s] = v;
        keepv[s] = keep;
      }
      __syncwarp();
      for (uint32_t t = lane; t < m; t += 32) row[t] = vals[off + t];
      for (int s = 0; s < nslot; s++) {
        unsigned msk = __ballot_sync(FULL, keepv[s]);
        if (keepv[s]) row[m + keep_cnt + __popc(msk & ((1u << lane) - 1))] = oldv[s];
        keep_cnt += __popc(msk);
      }
      for (uint32_t j = m + keep_cnt + lane; j < R; j += 32) row[j] = PANN_PAD;
      __syncwarp();
    } else if (lane == 0) {
      // a segment of exactly m candidates + deg current neighbours, packed by an atomic cursor
      uint32_t t = atomicAdd(njobs, 1u);
      job_pts[t] = tgt;
      job_off[t] = off;
      job_n[t] = m;
      job_begin[t] = (uint32_t)atomicAdd(seg_total, (unsigned long long)(m + deg));
    }
  }
}

// Final per-vertex sort by distance (index.h:180-185); ties by id.
template <int DT, int MT>
__global__ void __launch_bounds__(128) sort_neighbors_kernel(const uint8_t* __restrict__ points, uint64_t stride, int d,
                                                             int nchunks, uint32_t* graph, uint32_t R, uint64_t n) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  uint8_t* qs = smem + (size_t)warp * (stride + 16ull * R);
  uint64_t* kin = reinterpret_cast<uint64_t*>(qs + stride);
  uint64_t* kout = kin + R;
  for (uint64_t v = (uint64_t)blockIdx.x * wpb + warp; v < n; v += (uint64_t)gridDim.x * wpb) {
    stage_query<DT, MT>(qs, points + v * stride, nchunks, lane);
    __syncwarp();
    int32_t qq = 0;
    if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), nchunks);
    uint32_t* row = graph + v * R;
    uint32_t deg = 0;
    for (uint32_t b = 0; b < R; b += 32) {
      uint32_t j = b + lane;
      uint32_t u = j < R ? row[j] : PANN_PAD;
      bool ok = u != PANN_PAD;
      unsigned msk = __ballot_sync(0xFFFFFFFFu, ok);
      // Points[i].distance(Points[j]): row i is `this`
      if (ok) {
        // distance(row v, point u): the query operand is u, the row operand is v
        float dd = point_dist<DT, MT>(points + (uint64_t)u * stride, qs, d, nchunks, qq);
        kin[b + __popc(msk & ((1u << lane) - 1))] = make_key(dd, u);
      }
      deg += __popc(msk);
    }
    __syncwarp();
    for (uint32_t i = lane; i < deg; i += 32) {
      uint64_t ki = kin[i];
      uint32_t r = 0;
      for (uint32_t j = 0; j < deg; j++) r += kin[j] < ki;
      kout[r] = ki;
    }
    __syncwarp();
    for (uint32_t i = lane; i < deg; i += 32) row[i] = key_id(kout[i]);
    __syncwarp();
  }
}

// ------------------------------------------------------------ host side

// Batch schedule of batch_insert (index.h:206-240), same double arithmetic.
static void batch_schedule(uint64_t n, uint64_t m, std::vector<uint64_t>& fl, std::vector<uint64_t>& ce) {
  const double base = 2.0, max_fraction = 0.02;
  uint64_t max_batch = std::min<uint64_t>((uint64_t)(max_fraction * (double)(float)n), 1000000ull);
  if (max_batch == 0) max_batch = n;
  uint64_t count = 0, inc = 0;
  while (count < m) {
    uint64_t f, c;
    if (std::pow(base, (double)inc) <= (double)max_batch) {
      f = (uint64_t)std::pow(base, (double)inc) - 1;
      c = std::min<uint64_t>((uint64_t)std::pow(base, (double)(inc + 1)) - 1, m);
      count = c;
    } else {
      f = count;
      c = std::min<uint64_t>(count + max_batch, m);
      count += max_batch;
    }
    fl.push_back(f);
    ce.push_back(c);
    inc++;
  }
}

// Which greedy kernel a prune step runs: one warp per job (the default), or
// one block per job with the candidates' rows staged in shared memory
// (PANN_PRUNE_KERNEL=block). Measured on the 1M x 96 float build (R 64, L 128,
// two passes), the block kernel is slower in both steps: 0.91 s against
// 0.69 s for the insertion prunes, whose lists are the visited nodes, and
// more for the re-prunes, whose lists are a full row plus its new reverse
// edges; with 64 KB of staged rows a block, far fewer jobs are resident at
// once. Both give the same graph.
static bool prune_block_kernel(bool reprune) {
  (void)reprune;
  static const bool block = [] {
    const char* e = std::getenv("PANN_PRUNE_KERNEL");
    return e && !std::strcmp(e, "block");
  }();
  return block;
}

// robustPrune's greedy part for njobs segments: the block kernel with up to
// 64 KB of staged candidate rows per block, or the warp-per-job kernel.
template <int DT, int MT>
static cudaError_t launch_greedy(const pann_index* idx, uint32_t njobs, const uint32_t* pts, const uint32_t* sb,
                                 const uint32_t* se, uint64_t* keys, double alpha, unsigned long long* cmps,
                                 bool reprune, cudaStream_t st) {
  if (njobs == 0) return cudaSuccess;
  if (!prune_block_kernel(reprune)) {
    const int wpb = 4;
    const int blocks = (int)std::min<uint32_t>((njobs + wpb - 1) / wpb, 65535);
    greedy_prune_kernel<DT, MT><<<blocks, 32 * wpb, wpb * idx->stride, st>>>(
        idx->d_points, idx->stride, (int)idx->d, (int)idx->nchunks, idx->d_graph, idx->R, njobs, pts, sb, se, keys,
        alpha, cmps);
    return cudaGetLastError();
  }
  auto k = greedy_prune_block_kernel<DT, MT>;
  // dynamic + static shared memory must stay within the opt-in limit; rows
  // past the staged ones are read from global memory (cap_rows may be 0)
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, k);
  if (e != cudaSuccess) return e;
  const uint64_t limit = (uint64_t)smem_attr_max() - fa.sharedSizeBytes;
  if (idx->stride > limit) return cudaErrorInvalidValue;
  const uint32_t cap_rows =
      (uint32_t)std::min<uint64_t>((64ull << 10) / idx->stride, (limit - idx->stride) / idx->stride);
  const size_t smem = idx->stride * (1 + (size_t)cap_rows);
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int blocks = (int)std::min<uint32_t>(njobs, 2u * 65535u);
  k<<<blocks, 128, smem, st>>>(idx->d_points, idx->stride, (int)idx->nchunks, idx->d_graph, idx->R, njobs, pts, sb, se,
                               keys, alpha, cap_rows, cmps);
  return cudaGetLastError();
}

template <typename F>
static cudaError_t dispatch_dm(int dtype, int metric, F&& f) {
  if (dtype == DT_U8 && metric == MT_L2) return f(std::integral_constant<int, DT_U8>(), std::integral_constant<int, MT_L2>());
  if (dtype == DT_U8 && metric == MT_IP) return f(std::integral_constant<int, DT_U8>(), std::integral_constant<int, MT_IP>());
  if (dtype == DT_I8 && metric == MT_L2) return f(std::integral_constant<int, DT_I8>(), std::integral_constant<int, MT_L2>());
  if (dtype == DT_I8 && metric == MT_IP) return f(std::integral_constant<int, DT_I8>(), std::integral_constant<int, MT_IP>());
  if (dtype == DT_F32 && metric == MT_L2) return f(std::integral_constant<int, DT_F32>(), std::integral_constant<int, MT_L2>());
  if (dtype == DT_F32 && metric == MT_IP) return f(std::integral_constant<int, DT_F32>(), std::integral_constant<int, MT_IP>());
  return cudaErrorInvalidValue;
}

struct BuildBufs {
  DevBuf perm, vis_keys, vis_n, cmps, status, seg_a, seg_b, seg_begin, seg_end, pk_a, pk_b, pv_a, pv_b, uniq, counts,
      offs, nruns, jobs, job_off, job_n, cub_tmp, counters, start;
  void release() {
    for (DevBuf* b : {&perm, &vis_keys, &vis_n, &cmps, &status, &seg_a, &seg_b, &seg_begin, &seg_end, &pk_a, &pk_b,
                      &pv_a, &pv_b, &uniq, &counts, &offs, &nruns, &jobs, &job_off, &job_n, &cub_tmp, &counters,
                      &start})
      b->release();
  }
};

__global__ void iota_begin_kernel(uint32_t* begin, uint32_t n, uint32_t cap) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) begin[i] = i * cap;
}

__global__ void status_or_kernel(const uint32_t* status, uint32_t n, uint32_t* out) {
  uint32_t acc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc |= status[i];
  for (int o = 16; o; o >>= 1) acc |= __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicOr(out, acc);
}
__global__ void count_flag_kernel(const uint32_t* status, uint32_t n, uint32_t flag, uint32_t* out) {
  uint32_t acc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc += (status[i] & flag) ? 1u : 0u;
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}
// Sum of end[i] - begin[i] (segment lengths) and of the live degrees of the rows rows[i].
__global__ void seg_len_sum_kernel(const uint32_t* begin, const uint32_t* end, uint32_t n, unsigned long long* out) {
  unsigned long long acc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += end[i] - begin[i];
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}
__global__ void degree_sum_kernel(const uint32_t* graph, uint32_t R, const uint32_t* rows, uint32_t n,
                                  unsigned long long* out) {
  unsigned long long acc = 0;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < (uint64_t)n * R;
       e += (uint64_t)gridDim.x * blockDim.x)
    acc += graph[(uint64_t)rows[e / R] * R + e % R] != PANN_PAD;
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

__global__ void sum_kernel(const uint32_t* v, uint32_t n, unsigned long long* out) {
  unsigned long long acc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += v[i];
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

}  // namespace pann

using namespace pann;

extern "C" int pann_build(pann_index* idx, const pann_build_params* bp, const uint32_t* perm, pann_build_stats* stats) {
  if (!idx || !bp) return fail(PANN_EINVAL, "index or build params is NULL");
  if (!idx->points_set) return fail(PANN_EINVAL, "index has no points");
  if (bp->R != idx->R) return fail(PANN_EINVAL, "build R must equal the index's max degree");
  if (bp->L == 0 || bp->num_passes < 1 || !(bp->alpha > 0.0))
    return fail(PANN_EINVAL, "build needs L > 0, num_passes >= 1, alpha > 0");
  const uint64_t n = idx->n;
  const uint32_t R = idx->R;
  cudaStream_t st = idx->stream;
  if (perm)
    for (uint64_t i = 0; i < n; i++)
      if ((uint64_t)perm[i] >= n)
        return fail(PANN_EINVAL, "ERROR: invalid point " + std::to_string(perm[i]) + " given to batch_insert");

  BuildBufs bb;
  auto cleanup = [&]() { bb.release(); };
  auto cu = [&](cudaError_t e, const char* what) -> int {
    if (e == cudaSuccess) return PANN_OK;
    cleanup();
    return cuda_fail(e, what);
  };
#define BCUDA(call) do { int _rc = cu((call), #call); if (_rc) return _rc; } while (0)

  cudaEvent_t ev0, ev1, ea, eb, ec, ed;
  cudaEventCreate(&ev0); cudaEventCreate(&ev1);
  cudaEventCreate(&ea); cudaEventCreate(&eb); cudaEventCreate(&ec); cudaEventCreate(&ed);
  double t_search = 0, t_prune = 0, t_rev = 0;
  BCUDA(cudaEventRecord(ev0, st));

  // empty graph (Graph(maxDeg, n) is zeroed: every degree 0)
  BCUDA(cudaMemsetAsync(idx->d_graph, 0xFF, sizeof(uint32_t) * R * n, st));
  // insertion order
  BCUDA(bb.perm.ensure(4 * n));
  uint32_t* d_perm = bb.perm.as<uint32_t>();
  if (perm) {
    BCUDA(cudaMemcpyAsync(d_perm, perm, 4 * n, cudaMemcpyHostToDevice, st));
  } else {
    DevBuf k1, k2, i1;
    BCUDA(k1.ensure(8 * n)); BCUDA(k2.ensure(8 * n)); BCUDA(i1.ensure(4 * n));
    perm_keys_kernel<<<(int)std::min<uint64_t>((n + 255) / 256, 65535), 256, 0, st>>>(k1.as<uint64_t>(),
                                                                                      i1.as<uint32_t>(), n, bp->perm_seed);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, k1.as<uint64_t>(), k2.as<uint64_t>(), i1.as<uint32_t>(), d_perm,
                                    (int)n, 0, 64, st);
    DevBuf tmp;
    BCUDA(tmp.ensure(tb + 16));
    BCUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, k1.as<uint64_t>(), k2.as<uint64_t>(), i1.as<uint32_t>(), d_perm,
                                          (int)n, 0, 64, st));
    BCUDA(cudaStreamSynchronize(st));
    k1.release(); k2.release(); i1.release(); tmp.release();
  }

  std::vector<uint64_t> fl, ce;
  batch_schedule(n, n, fl, ce);
  uint64_t maxB = 0;
  for (size_t b = 0; b < fl.size(); b++) maxB = std::max(maxB, ce[b] - fl[b]);

  uint32_t vis_cap = std::max<uint32_t>(2 * bp->L + 64, 128);
  const uint32_t start0 = 0;
  BCUDA(bb.start.ensure(16));
  BCUDA(cudaMemcpyAsync(bb.start.p, &start0, 4, cudaMemcpyHostToDevice, st));
  BCUDA(bb.counters.ensure(256));
  uint32_t* c32 = bb.counters.as<uint32_t>();  // [0] status or, [1] njobs, [2] flagged count
  // [0] dist cmps, [1] visited, [2] reverse prune segment cursor, [3] search cmps,
  // [4] insertion prune candidates, [5] reverse-edge pairs
  unsigned long long* c64 = reinterpret_cast<unsigned long long*>(c32 + 8);
  BCUDA(cudaMemsetAsync(bb.counters.p, 0, 256, st));

  const uint64_t pairs_cap = maxB * R;
  auto alloc_batch = [&](uint32_t vcap) -> int {
    uint64_t segcap = vcap + R;
    uint64_t seg_items = maxB * segcap;
    BCUDA(bb.vis_keys.ensure(8 * maxB * vcap));
    BCUDA(bb.vis_n.ensure(4 * maxB));
    BCUDA(bb.cmps.ensure(4 * maxB));
    BCUDA(bb.status.ensure(4 * maxB));
    BCUDA(bb.seg_a.ensure(8 * seg_items));
    BCUDA(bb.seg_b.ensure(8 * seg_items));
    BCUDA(bb.seg_begin.ensure(4 * std::max<uint64_t>(maxB, pairs_cap)));
    BCUDA(bb.seg_end.ensure(4 * std::max<uint64_t>(maxB, pairs_cap)));
    BCUDA(bb.pk_a.ensure(4 * pairs_cap)); BCUDA(bb.pk_b.ensure(4 * pairs_cap));
    BCUDA(bb.pv_a.ensure(4 * pairs_cap)); BCUDA(bb.pv_b.ensure(4 * pairs_cap));
    BCUDA(bb.uniq.ensure(4 * pairs_cap)); BCUDA(bb.counts.ensure(4 * pairs_cap)); BCUDA(bb.offs.ensure(4 * pairs_cap));
    BCUDA(bb.nruns.ensure(16));
    BCUDA(bb.jobs.ensure(4 * pairs_cap)); BCUDA(bb.job_off.ensure(4 * pairs_cap)); BCUDA(bb.job_n.ensure(4 * pairs_cap));
    // CUB temporary storage: the largest of the three uses
    size_t t1 = 0, t2 = 0, t3 = 0, t4 = 0;
    cub::DeviceSegmentedSort::SortKeys(nullptr, t1, bb.seg_a.as<uint64_t>(), bb.seg_b.as<uint64_t>(), (int)seg_items,
                                       (int)std::max<uint64_t>(maxB, pairs_cap), bb.seg_begin.as<uint32_t>(),
                                       bb.seg_end.as<uint32_t>(), st);
    cub::DeviceRadixSort::SortPairs(nullptr, t2, bb.pk_a.as<uint32_t>(), bb.pk_b.as<uint32_t>(), bb.pv_a.as<uint32_t>(),
                                    bb.pv_b.as<uint32_t>(), (int)pairs_cap, 0, 32, st);
    cub::DeviceRunLengthEncode::Encode(nullptr, t3, bb.pk_b.as<uint32_t>(), bb.uniq.as<uint32_t>(),
                                       bb.counts.as<uint32_t>(), bb.nruns.as<uint32_t>(), (int)pairs_cap, st);
    cub::DeviceScan::ExclusiveSum(nullptr, t4, bb.counts.as<uint32_t>(), bb.offs.as<uint32_t>(), (int)pairs_cap, st);
    BCUDA(bb.cub_tmp.ensure(std::max(std::max(t1, t2), std::max(t3, t4)) + 256));
    return PANN_OK;
  };
  {
    int rc = alloc_batch(vis_cap);
    if (rc) return rc;
  }

  const int dtype = idx->dtype, metric = idx->metric;
  const uint64_t stride = idx->stride;
  const int d = (int)idx->d, nch = (int)idx->nchunks;
  const int wpb = 4;
  const size_t warp_smem = stride;
  uint32_t batches = 0;
  uint64_t reprunes = 0, prune_cands = 0, inserted = 0;

  for (int pass = 0; pass < bp->num_passes; pass++) {
    const double alpha = (pass == bp->num_passes - 1) ? bp->alpha : 1.0;  // index.h:173-178
    for (size_t b = 0; b < fl.size(); b++) {
      const uint32_t B = (uint32_t)(ce[b] - fl[b]);
      const uint32_t* pts = d_perm + fl[b];
      batches++;
      // ---- 1. search (QueryParams(0, L, n, maxDeg, rerank, batch_factor), index.h:251-252)
      pann_query_params qp{0, bp->L, n, R, bp->batch_factor};
      SearchPlan plan;
      {
        int rc = make_plan(idx, &qp, 1, &plan);
        if (rc) { cleanup(); return rc; }
      }
      uint32_t sor = 0;
      for (;;) {
        BCUDA(cudaEventRecord(ea, st));
        BCUDA(cudaMemsetAsync(c32, 0, 4, st));
        int rc = run_search(idx, plan, nullptr, pts, B, bb.start.as<uint32_t>(), nullptr, nullptr,
                            bb.vis_n.as<uint32_t>(), bb.cmps.as<uint32_t>(), bb.status.as<uint32_t>(),
                            bb.vis_keys.as<uint64_t>(), vis_cap, st);
        if (rc) { cleanup(); return rc; }
        status_or_kernel<<<64, 256, 0, st>>>(bb.status.as<uint32_t>(), B, c32);
        BCUDA(cudaMemcpyAsync(&sor, c32, 4, cudaMemcpyDeviceToHost, st));
        BCUDA(cudaEventRecord(eb, st));
        BCUDA(cudaStreamSynchronize(st));
        if (sor & (QS_TABLE_FULL | QS_INTERNAL)) {
          cleanup();
          return fail(PANN_EOVERFLOW, "build search: a seen-set outgrew the largest table");
        }
        if (sor & QS_VISIT_OVERFLOW) {
          vis_cap *= 2;
          int rc2 = alloc_batch(vis_cap);
          if (rc2) return rc2;
          continue;
        }
        break;
      }
      {
        float ms = 0;
        cudaEventElapsedTime(&ms, ea, eb);
        t_search += ms * 1e-3;
      }
      count_flag_kernel<<<64, 256, 0, st>>>(bb.status.as<uint32_t>(), B, QS_REF_WOULD_GROW, c32 + 2);
      sum_kernel<<<64, 256, 0, st>>>(bb.cmps.as<uint32_t>(), B, c64);
      sum_kernel<<<64, 256, 0, st>>>(bb.cmps.as<uint32_t>(), B, c64 + 3);
      sum_kernel<<<64, 256, 0, st>>>(bb.vis_n.as<uint32_t>(), B, c64 + 1);
      // ---- 2. robustPrune of the inserted points
      BCUDA(cudaEventRecord(ea, st));
      const uint32_t segcap = vis_cap + R;
      iota_begin_kernel<<<(B + 255) / 256, 256, 0, st>>>(bb.seg_begin.as<uint32_t>(), B, segcap);
      BCUDA(dispatch_dm(dtype, metric, [&](auto DTc, auto MTc) {
        constexpr int DT = decltype(DTc)::value, MT = decltype(MTc)::value;
        int blocks = (int)std::min<uint32_t>((B + wpb - 1) / wpb, 65535);
        assemble_kernel<DT, MT><<<blocks, 32 * wpb, wpb * warp_smem, st>>>(
            idx->d_points, stride, d, nch, idx->d_graph, R, B, pts, bb.vis_keys.as<uint64_t>(), vis_cap, nullptr,
            nullptr, bb.vis_n.as<uint32_t>(), bb.seg_begin.as<uint32_t>(), bb.seg_end.as<uint32_t>(),
            bb.seg_a.as<uint64_t>(), c64);
        return cudaGetLastError();
      }));
      {
        size_t tb = bb.cub_tmp.bytes;
        BCUDA(cub::DeviceSegmentedSort::SortKeys(bb.cub_tmp.p, tb, bb.seg_a.as<uint64_t>(), bb.seg_b.as<uint64_t>(),
                                                 (int)((uint64_t)B * segcap), (int)B, bb.seg_begin.as<uint32_t>(),
                                                 bb.seg_end.as<uint32_t>(), st));
      }
      BCUDA(dispatch_dm(dtype, metric, [&](auto DTc, auto MTc) {
        constexpr int DT = decltype(DTc)::value, MT = decltype(MTc)::value;
        return launch_greedy<DT, MT>(idx, B, pts, bb.seg_begin.as<uint32_t>(), bb.seg_end.as<uint32_t>(),
                                     bb.seg_b.as<uint64_t>(), alpha, c64, false, st);
      }));
      BCUDA(cudaEventRecord(eb, st));
      seg_len_sum_kernel<<<64, 256, 0, st>>>(bb.seg_begin.as<uint32_t>(), bb.seg_end.as<uint32_t>(), B, c64 + 4);
      degree_sum_kernel<<<128, 256, 0, st>>>(idx->d_graph, R, pts, B, c64 + 5);
      // ---- 3. reverse edges
      const uint64_t np = (uint64_t)B * R;
      reverse_pairs_kernel<<<(int)std::min<uint64_t>((np + 255) / 256, 65535), 256, 0, st>>>(
          idx->d_graph, R, pts, B, bb.pk_a.as<uint32_t>(), bb.pv_a.as<uint32_t>());
      {
        size_t tb = bb.cub_tmp.bytes;
        int bits = 1;
        while (bits < 32 && (1ull << bits) <= n) bits++;
        // PAD (all ones) must still sort last: sort all 32 bits when n needs fewer
        BCUDA(cub::DeviceRadixSort::SortPairs(bb.cub_tmp.p, tb, bb.pk_a.as<uint32_t>(), bb.pk_b.as<uint32_t>(),
                                              bb.pv_a.as<uint32_t>(), bb.pv_b.as<uint32_t>(), (int)np, 0, 32, st));
        tb = bb.cub_tmp.bytes;
        BCUDA(cub::DeviceRunLengthEncode::Encode(bb.cub_tmp.p, tb, bb.pk_b.as<uint32_t>(), bb.uniq.as<uint32_t>(),
                                                 bb.counts.as<uint32_t>(), bb.nruns.as<uint32_t>(), (int)np, st));
        tb = bb.cub_tmp.bytes;
        BCUDA(cub::DeviceScan::ExclusiveSum(bb.cub_tmp.p, tb, bb.counts.as<uint32_t>(), bb.offs.as<uint32_t>(),
                                            (int)np, st));
      }
      BCUDA(cudaMemsetAsync(c32 + 1, 0, 4, st));
      BCUDA(cudaMemsetAsync(c64 + 2, 0, 8, st));
      {
        int blocks = (int)std::min<uint64_t>((np * 32 + 255) / 256, 65535);
        reverse_classify_kernel<<<blocks, 256, 0, st>>>(idx->d_graph, R, bb.uniq.as<uint32_t>(),
                                                        bb.counts.as<uint32_t>(), bb.offs.as<uint32_t>(),
                                                        bb.nruns.as<uint32_t>(), bb.pv_b.as<uint32_t>(),
                                                        bb.jobs.as<uint32_t>(), bb.job_off.as<uint32_t>(),
                                                        bb.job_n.as<uint32_t>(), bb.seg_begin.as<uint32_t>(), c32 + 1,
                                                        c64 + 2);
        BCUDA(cudaGetLastError());
      }
      uint32_t njobs = 0;
      unsigned long long seg_total = 0;
      BCUDA(cudaMemcpyAsync(&njobs, c32 + 1, 4, cudaMemcpyDeviceToHost, st));
      BCUDA(cudaMemcpyAsync(&seg_total, c64 + 2, 8, cudaMemcpyDeviceToHost, st));
      BCUDA(cudaStreamSynchronize(st));
      reprunes += njobs;
      prune_cands += seg_total;
      inserted += B;
      if (njobs) {
        if (seg_total >= 0x7FFFFFFFull) {
          cleanup();
          return fail(PANN_ENOMEM, "reverse-edge prune segments exceed 2^31 keys");
        }
        // scratch for exactly seg_total keys (grown if this batch needs more)
        BCUDA(bb.seg_a.ensure_grow(8 * seg_total + 8));
        BCUDA(bb.seg_b.ensure_grow(8 * seg_total + 8));
        {
          size_t need = 0;
          cub::DeviceSegmentedSort::SortKeys(nullptr, need, bb.seg_a.as<uint64_t>(), bb.seg_b.as<uint64_t>(),
                                             (int)seg_total, (int)njobs, bb.seg_begin.as<uint32_t>(),
                                             bb.seg_end.as<uint32_t>(), st);
          BCUDA(bb.cub_tmp.ensure_grow(need + 256));
        }
        BCUDA(dispatch_dm(dtype, metric, [&](auto DTc, auto MTc) {
          constexpr int DT = decltype(DTc)::value, MT = decltype(MTc)::value;
          int blocks = (int)std::min<uint32_t>((njobs + wpb - 1) / wpb, 65535);
          assemble_kernel<DT, MT><<<blocks, 32 * wpb, wpb * warp_smem, st>>>(
              idx->d_points, stride, d, nch, idx->d_graph, R, njobs, bb.jobs.as<uint32_t>(), nullptr, 0,
              bb.pv_b.as<uint32_t>(), bb.job_off.as<uint32_t>(), bb.job_n.as<uint32_t>(), bb.seg_begin.as<uint32_t>(),
              bb.seg_end.as<uint32_t>(), bb.seg_a.as<uint64_t>(), c64);
          return cudaGetLastError();
        }));
        {
          size_t tb = bb.cub_tmp.bytes;
          BCUDA(cub::DeviceSegmentedSort::SortKeys(bb.cub_tmp.p, tb, bb.seg_a.as<uint64_t>(), bb.seg_b.as<uint64_t>(),
                                                   (int)seg_total, (int)njobs, bb.seg_begin.as<uint32_t>(),
                                                   bb.seg_end.as<uint32_t>(), st));
        }
        BCUDA(dispatch_dm(dtype, metric, [&](auto DTc, auto MTc) {
          constexpr int DT = decltype(DTc)::value, MT = decltype(MTc)::value;
          return launch_greedy<DT, MT>(idx, njobs, bb.jobs.as<uint32_t>(), bb.seg_begin.as<uint32_t>(),
                                       bb.seg_end.as<uint32_t>(), bb.seg_b.as<uint64_t>(), alpha, c64, true, st);
        }));
      }
      BCUDA(cudaEventRecord(ec, st));
      BCUDA(cudaEventSynchronize(ec));
      {
        float ms = 0;
        cudaEventElapsedTime(&ms, ea, eb);
        t_prune += ms * 1e-3;
        cudaEventElapsedTime(&ms, eb, ec);
        t_rev += ms * 1e-3;
      }
    }
  }
  if (bp->sort_neighbors) {
    BCUDA(dispatch_dm(dtype, metric, [&](auto DTc, auto MTc) {
      constexpr int DT = decltype(DTc)::value, MT = decltype(MTc)::value;
      size_t sm = wpb * (stride + 16ull * R);
      auto kern = sort_neighbors_kernel<DT, MT>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr_max());
      int blocks = (int)std::min<uint64_t>((n + wpb - 1) / wpb, 65535ull * 8);
      kern<<<blocks, 32 * wpb, sm, st>>>(idx->d_points, stride, d, nch, idx->d_graph, R, n);
      return cudaGetLastError();
    }));
  }
  BCUDA(cudaEventRecord(ev1, st));
  BCUDA(cudaEventSynchronize(ev1));
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    std::memset(stats, 0, sizeof(*stats));
    stats->seconds = ms * 1e-3;
    stats->search_seconds = t_search;
    stats->prune_seconds = t_prune;
    stats->reverse_seconds = t_rev;
    unsigned long long h64[6] = {0, 0, 0, 0, 0, 0};
    uint32_t h32[4] = {0, 0, 0, 0};
    cudaMemcpy(h64, c64, 48, cudaMemcpyDeviceToHost);
    cudaMemcpy(h32, c32, 16, cudaMemcpyDeviceToHost);
    stats->dist_cmps = h64[0];
    stats->visited_total = h64[1];
    stats->batches = batches;
    stats->flagged = h32[2];
    stats->search_cmps = h64[3];
    stats->prune_candidates = h64[4] + prune_cands;
    stats->edge_pairs = h64[5];
    stats->reprunes = reprunes;
    stats->inserted = inserted;
  }
  cudaEventDestroy(ev0); cudaEventDestroy(ev1);
  cudaEventDestroy(ea); cudaEventDestroy(eb); cudaEventDestroy(ec); cudaEventDestroy(ed);
  cleanup();
  return PANN_OK;
#undef BCUDA
}
