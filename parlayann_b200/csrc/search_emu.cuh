// Exact-emulation tier of the beam search, for queries on which the
// reference's seen-set would grow (hashset.h:25-38).
//
// The reference's hashset is exact until it grows. When it grows, the key
// that triggered the growth is placed by probing from its slot under the OLD
// mask, so a later lookup of that key from its slot under the new mask can
// miss it: the id is then scored again (full_dist_cmps counts it again), may
// re-enter the candidate list, and is deduplicated by std::unique
// (beamSearch.h:198-199), by set_union against the frontier (:202-205), or
// excluded from the unvisited frontier by set_difference against the visited
// list (:217-222). Because those duplicates change counters and can change the
// deferral test (:185-192), this tier reproduces them exactly:
//   * the hashset is emulated as written: the reference's hash
//     (k * 0xbf58476d1ce4e5b9) & mask, linear probing, growth when
//     num_entries > size/2 with the re-inserted keys added to num_entries,
//     re-insertion in old-slot order, the triggering key probed from its
//     old-mask slot, inserts in adjacency order (lane 0, sequentially);
//   * candidates are sorted, repeated ids dropped, ids already in the
//     frontier dropped (set_union keeps the frontier copy), and candidates
//     whose id was visited before enter the frontier already marked visited.
// The emulated table ping-pongs between two regions A (sizes S0, 4 S0, ...)
// and B (2 S0, 8 S0, ...), in shared memory when they fit (SMEM = true) or in
// global memory per resident block. Queries reach this tier only when the fast
// tiers flagged them.
#pragma once
#include "search.cuh"

namespace pann {

struct EmuArgs {
  uint32_t* gA;      // global regions (SMEM = false): capA / capB slots per block
  uint32_t* gB;
  uint32_t capA, capB;
  uint32_t bits0;    // initial capacity 2^bits0 (beamSearch.h:66, hashset.h:50-54)
  uint32_t vs_slots; // exact visited-id set, in shared memory (power of two)
  uint32_t base_bytes;  // search state bytes before the visited set
  uint32_t* overflow_list;  // queries whose emulated table outgrew this tier
  uint32_t* overflow_count;
};

__device__ __forceinline__ uint32_t ref_slot(uint32_t k, uint32_t mask) {
  return (uint32_t)(((uint64_t)k * 0xbf58476d1ce4e5b9ull) & (uint64_t)mask);
}

// State of the emulated hashset; meaningful in lane 0 only.
struct EmuHash {
  uint32_t* cur;
  uint32_t* other;
  uint32_t cur_cap, other_cap;
  uint32_t bits;
  long long num_entries;
};

// Lane 0: process keys[j0..n) in order (hashset.h:22-48) until one needs the
// table to grow. Writes each key reported unseen (and != self) to out[*nout].
// Returns the index of the key that needs growth, or -1 when all are done.
__device__ int emu_run(EmuHash& h, const uint32_t* keys, int j0, int n, bool stop_at_pad, uint32_t self,
                       uint32_t* out, int* nout) {
  for (int j = j0; j < n; j++) {
    uint32_t a = keys[j];
    if (stop_at_pad && a == PANN_PAD) return -1;
    uint32_t size = 1u << h.bits, mask = size - 1;
    uint32_t loc = ref_slot(a, mask);
    if (h.cur[loc] == a) continue;
    if (h.num_entries > (long long)(size / 2)) return j;
    bool hit = false;
    if (h.cur[loc] != PANN_PAD) {
      loc = (loc + 1) & mask;
      while (h.cur[loc] != PANN_PAD && h.cur[loc] != a) loc = (loc + 1) & mask;
      hit = h.cur[loc] == a;
    }
    if (hit) continue;
    h.cur[loc] = a;
    h.num_entries++;
    if (out && a != self) out[(*nout)++] = a;
  }
  return -1;
}

// Warp: grow the table (re-insert in old-slot order), then lane 0 finishes the
// call for key a from its old-mask slot. Returns false if the new table does
// not fit this tier's capacity.
__device__ bool emu_grow_and_insert(EmuHash& h, uint32_t a, uint32_t self, uint32_t* out, int* nout, int lane) {
  const unsigned FULL = 0xFFFFFFFFu;
  uint32_t size = 0, other_cap = 0;
  uint32_t* other = nullptr;
  if (lane == 0) { size = 1u << h.bits; other_cap = h.other_cap; other = h.other; }
  size = __shfl_sync(FULL, size, 0);
  other_cap = __shfl_sync(FULL, other_cap, 0);
  other = reinterpret_cast<uint32_t*>(__shfl_sync(FULL, reinterpret_cast<unsigned long long>(other), 0));
  const uint32_t nsize = size * 2;
  if (nsize > other_cap) return false;
  for (uint32_t i = lane; i < nsize; i += 32) other[i] = PANN_PAD;
  __syncwarp();
  __threadfence_block();
  if (lane == 0) {
    const uint32_t oldmask = size - 1, nmask = nsize - 1;
    long long added = 0;
    for (uint32_t i = 0; i < size; i++) {
      uint32_t k = h.cur[i];
      if (k != PANN_PAD) {
        uint32_t l2 = ref_slot(k, nmask);
        while (other[l2] != PANN_PAD && other[l2] != k) l2 = (l2 + 1) & nmask;
        other[l2] = k;
        added++;
      }
    }
    h.num_entries += added;
    uint32_t* t = h.cur; h.cur = h.other; h.other = t;
    uint32_t c = h.cur_cap; h.cur_cap = h.other_cap; h.other_cap = c;
    h.bits += 1;
    // the call that grew the table continues with its old-mask slot (hashset.h:23,39-45)
    uint32_t loc = ref_slot(a, oldmask);
    bool hit = false;
    if (h.cur[loc] != PANN_PAD) {
      loc = (loc + 1) & nmask;
      while (h.cur[loc] != PANN_PAD && h.cur[loc] != a) loc = (loc + 1) & nmask;
      hit = h.cur[loc] == a;
    }
    if (!hit) {
      h.cur[loc] = a;
      h.num_entries++;
      if (out && a != self) out[(*nout)++] = a;
    }
  }
  __syncwarp();
  return true;
}

// Run the emulated hashset over keys[0..n) (warp-uniform call). Returns false
// on capacity overflow. *nout (lane 0) counts keys reported unseen.
__device__ bool emu_lookup_all(EmuHash& h, const uint32_t* keys, int n, bool stop_at_pad, uint32_t self,
                               uint32_t* out, int* nout, int lane) {
  const unsigned FULL = 0xFFFFFFFFu;
  int j = 0;
  for (;;) {
    int g = -1;
    if (lane == 0) g = emu_run(h, keys, j, n, stop_at_pad, self, out, nout);
    g = __shfl_sync(FULL, g, 0);
    __syncwarp();
    if (g < 0) return true;
    uint32_t a = 0;
    if (lane == 0) a = keys[g];
    a = __shfl_sync(FULL, a, 0);
    if (!emu_grow_and_insert(h, a, self, out, nout, lane)) return false;
    j = g + 1;
  }
}

__device__ __forceinline__ void vset_insert(uint32_t* t, uint32_t mask, uint32_t id) {
  uint32_t h = hash_slot(id, mask);
  for (uint32_t p = 0; p <= mask; p++) {
    uint32_t old = atomicCAS(t + h, PANN_PAD, id);
    if (old == PANN_PAD || old == id) return;
    h = (h + 1) & mask;
  }
}
__device__ __forceinline__ bool vset_has(const uint32_t* t, uint32_t mask, uint32_t id) {
  uint32_t h = hash_slot(id, mask);
  for (uint32_t p = 0; p <= mask; p++) {
    uint32_t v = t[h];
    if (v == id) return true;
    if (v == PANN_PAD) return false;
    h = (h + 1) & mask;
  }
  return false;
}

// True if the masked key k is in the sorted frontier fr[0..fn).
__device__ __forceinline__ bool frontier_has(const uint64_t* fr, int fn, uint64_t k) {
  int lo = 0, hi = fn;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if ((fr[mid] & PANN_KEYMASK) < k) lo = mid + 1; else hi = mid;
  }
  return lo < fn && (fr[lo] & PANN_KEYMASK) == k;
}

__host__ __device__ inline size_t emu_smem_bytes(uint32_t base_bytes, uint32_t vs_slots, uint32_t capA, uint32_t capB,
                                                 bool smem_tables) {
  size_t b = base_bytes + 4ull * vs_slots;
  if (smem_tables) b += 4ull * capA + 4ull * capB;
  return b;
}

// One warp per flagged query.
template <int DT, int MT, bool SMEM>
__global__ void __launch_bounds__(32) search_emulate_kernel(SearchArgs a, EmuArgs e) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  uint8_t* qs = smem;
  uint64_t* frA = reinterpret_cast<uint64_t*>(smem + a.stride);
  uint64_t* frB = frA + a.L;
  uint64_t* cand = frB + a.L;
  uint64_t* cand2 = cand + a.Ccap;
  uint32_t* nbuf = reinterpret_cast<uint32_t*>(cand2 + a.Ccap);
  uint32_t* vset = reinterpret_cast<uint32_t*>(smem + e.base_bytes);
  uint32_t* tabA;
  uint32_t* tabB;
  if (SMEM) {
    tabA = vset + e.vs_slots;
    tabB = tabA + e.capA;
  } else {
    tabA = e.gA + (size_t)blockIdx.x * e.capA;
    tabB = e.gB + (size_t)blockIdx.x * e.capB;
  }
  const uint32_t vmask = e.vs_slots - 1;
  const uint32_t njobs = a.njobs_dev ? *a.njobs_dev : a.nq;
  const uint32_t L = a.L;

  for (;;) {
    uint32_t job = 0;
    if (lane == 0) job = atomicAdd(a.job_counter, 1u);
    job = __shfl_sync(FULL, job, 0);
    if (job >= njobs) break;
    const uint32_t qi = a.job_list ? a.job_list[job] : job;
    const uint32_t self = a.self_ids ? a.self_ids[qi] : PANN_PAD;
    const uint8_t* qsrc = a.self_ids ? a.points + (uint64_t)self * a.stride : a.queries + (uint64_t)qi * a.stride;
    for (uint32_t c = lane; c < a.nchunks; c += 32)
      reinterpret_cast<uint4*>(qs)[c] = __ldg(reinterpret_cast<const uint4*>(qsrc) + c);
    for (uint32_t i = lane; i < (1u << e.bits0); i += 32) tabA[i] = PANN_PAD;
    for (uint32_t i = lane; i < e.vs_slots; i += 32) vset[i] = PANN_PAD;
    __syncwarp();
    __threadfence_block();
    EmuHash h;
    h.cur = tabA; h.other = tabB; h.cur_cap = e.capA; h.other_cap = e.capB;
    h.bits = e.bits0; h.num_entries = 0;
    bool ok = true;
    int32_t qq = 0;
    if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), a.nchunks);

    // starting points, inserted in the given order (:73-76)
    for (uint32_t s = lane; s < a.n_start; s += 32) {
      uint32_t id = a.starts[s];
      float dd = point_dist<DT, MT>(a.points + (uint64_t)id * a.stride, qs, a.d, a.nchunks, qq);
      frB[s] = make_key(dd, id);
    }
    {
      int dummy = 0;
      ok = emu_lookup_all(h, a.starts, (int)a.n_start, false, PANN_PAD, nullptr, &dummy, lane);
    }
    __syncwarp();
    uint64_t* fr = frA;
    uint64_t* fr2 = frB;
    warp_rank_sort(frB, fr, (int)a.n_start, lane);
    __syncwarp();
    int fn = (int)a.n_start;
    int cn = 0;
    uint32_t cmps = a.n_start;
    uint64_t nvis = 0;
    uint32_t status = QS_REF_WOULD_GROW;
    if (!ok) status |= QS_TABLE_FULL;

    while (ok) {
      __syncwarp();
      int first = -1, cnt = 0;
      for (int b = 0; b < fn; b += 32) {
        int i = b + lane;
        bool unv = (i < fn) && !(fr[i] & PANN_VFLAG);
        unsigned m = __ballot_sync(FULL, unv);
        if (first < 0 && m) first = b + __ffs(m) - 1;
        cnt += __popc(m);
      }
      if (first < 0 || nvis >= a.limit) break;
      const uint64_t cur_key = fr[first];
      __syncwarp();
      if (lane == 0) fr[first] = cur_key | PANN_VFLAG;
      nvis++;
      if (a.vis_keys && lane == 0 && nvis <= a.vis_cap) a.vis_keys[(uint64_t)qi * a.vis_cap + (nvis - 1)] = cur_key & PANN_KEYMASK;
      if (nvis > a.vis_cap && a.vis_keys) status |= QS_VISIT_OVERFLOW;
      if (nvis > (uint64_t)(vmask / 4 * 3)) { status |= QS_INTERNAL; break; }
      if (lane == 0) vset_insert(vset, vmask, key_id(cur_key));
      const bool full = (fn == (int)L);
      const float cutoff = full ? key_dist(fr[fn - 1]) : 3.40282346638528859812e+38F;
      const uint32_t cid = key_id(cur_key);
      const uint32_t nel = a.dl < a.R ? a.dl : a.R;
      // adjacency ids, staged in shared memory (cand2 is free until the merge),
      // then looked up in order (:153-159)
      uint32_t* row = reinterpret_cast<uint32_t*>(cand2);
      for (uint32_t j = lane; j < nel; j += 32) row[j] = __ldg(a.graph + (uint64_t)cid * a.R + j);
      __syncwarp();
      int nnew = 0;
      if (!emu_lookup_all(h, row, (int)nel, true, self, nbuf, &nnew, lane)) {
        status |= QS_TABLE_FULL;
        break;
      }
      nnew = __shfl_sync(FULL, nnew, 0);
      __syncwarp();
      cmps += (uint32_t)nnew;
      if ((uint32_t)(cn + nnew) > a.Ccap) { status |= QS_INTERNAL; break; }
      for (int b = 0; b < nnew; b += 32) {
        int i = b + lane;
        bool keep = false;
        uint64_t key = 0;
        if (i < nnew) {
          uint32_t v = nbuf[i];
          float dd = point_dist<DT, MT>(a.points + (uint64_t)v * a.stride, qs, a.d, a.nchunks, qq);
          keep = !(dd >= cutoff);
          key = make_key(dd, v);
        }
        unsigned mk = __ballot_sync(FULL, keep);
        if (keep) cand[cn + __popc(mk & ((1u << lane) - 1))] = key;
        cn += __popc(mk);
      }
      if (cn == 0 || (a.limit >= 2ull * L && (double)cn < a.batch_factor * (double)L && cnt - 1 >= 1)) continue;
      __syncwarp();
      warp_rank_sort(cand, cand2, cn, lane);
      __syncwarp();
      // unique by id, drop ids already in the frontier, mark ids visited before
      int un = 0;
      for (int b = 0; b < cn; b += 32) {
        int i = b + lane;
        bool keepc = false;
        uint64_t k = 0;
        if (i < cn) {
          k = cand2[i];
          keepc = !(i > 0 && key_id(cand2[i - 1]) == key_id(k)) && !frontier_has(fr, fn, k);
          if (keepc && vset_has(vset, vmask, key_id(k))) k |= PANN_VFLAG;
        }
        unsigned mk = __ballot_sync(FULL, keepc);
        if (keepc) cand[un + __popc(mk & ((1u << lane) - 1))] = k;
        un += __popc(mk);
      }
      __syncwarp();
      fn = warp_merge(fr, fn, cand, un, fr2, (int)L, lane);
      uint64_t* t = fr; fr = fr2; fr2 = t;
      cn = 0;
      __syncwarp();
    }

    if (status & QS_TABLE_FULL) {
      // the emulated table outgrew this tier: the next tier (larger, global) re-runs it
      if (lane == 0) {
        if (e.overflow_list) e.overflow_list[atomicAdd(e.overflow_count, 1u)] = qi;
        if (a.out_status) a.out_status[qi] = status;
      }
      __syncwarp();
      continue;
    }
    if (status & QS_INTERNAL) {
      if (lane == 0 && a.out_status) a.out_status[qi] = status;
      __syncwarp();
      continue;
    }
    if ((uint32_t)fn < a.k) status |= QS_SHORT;
    for (uint32_t j = lane; j < a.k; j += 32) {
      bool okk = j < (uint32_t)fn;
      a.out_ids[(uint64_t)qi * a.k + j] = okk ? key_id(fr[j]) : PANN_PAD;
      if (a.out_dists) a.out_dists[(uint64_t)qi * a.k + j] = okk ? key_dist(fr[j]) : 0.0f;
    }
    if (lane == 0) {
      if (a.out_visited) a.out_visited[qi] = (uint32_t)nvis;
      if (a.out_cmps) a.out_cmps[qi] = cmps;
      if (a.out_status) a.out_status[qi] = status;
    }
    __syncwarp();
  }
}

}  // namespace pann
