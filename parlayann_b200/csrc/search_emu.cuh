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
  uint32_t* overflow_rec;
  uint32_t* overflow_count;
  const uint32_t* job_rec;  // per job: resume record (tier 0's saved state) or PAD
  // 1: a pass that runs beside the search tiers still publishing hand-offs
  // (see emu_claim); 0: every job is published
  uint32_t early;
};

// job_rec value of a hand-off slot taken but not yet written
constexpr uint32_t EMU_NOT_READY = 0xFEFEFEFEu;

// The next job of an emulation pass, or PANN_PAD when there is none (one
// thread). With early set the pass runs while tier 0 and tier 2 still hand
// queries over: it takes the next job only if that slot is published (its
// record index written after the record itself, behind a fence) and
// otherwise ends; it never waits. A pass after the search tiers takes every
// job left. Passes take jobs from one counter, so each job runs once.
__device__ __forceinline__ uint32_t emu_claim(uint32_t* counter, const uint32_t* njobs_dev, uint32_t nq,
                                              const uint32_t* job_rec, bool early) {
  if (!early) {
    const uint32_t njobs = njobs_dev ? *njobs_dev : nq;
    const uint32_t j = atomicAdd(counter, 1u);
    return j < njobs ? j : PANN_PAD;
  }
  uint32_t c = *reinterpret_cast<volatile uint32_t*>(counter);
  for (uint32_t guard = 0; guard < (1u << 20); guard++) {
    const uint32_t n = *reinterpret_cast<const volatile uint32_t*>(njobs_dev);
    if (c >= n) break;
    if (reinterpret_cast<const volatile uint32_t*>(job_rec)[c] == EMU_NOT_READY) break;
    const uint32_t prev = atomicCAS(counter, c, c + 1);
    if (prev == c) {
      __threadfence();
      return c;
    }
    c = prev;
  }
  return PANN_PAD;
}

// (k * 0xbf58476d1ce4e5b9) & mask for mask < 2^32: the product's low 32 bits
// depend only on the multiplier's low 32 bits, so 32-bit arithmetic suffices.
__device__ __forceinline__ uint32_t ref_slot(uint32_t k, uint32_t mask) { return (k * 0x1ce4e5b9u) & mask; }

// State of the emulated hashset, identical in every lane of the warp.
struct EmuHash {
  uint32_t* cur;
  uint32_t* other;
  uint32_t cur_cap, other_cap;
  uint32_t bits;
  long long num_entries;
};

// Order-preserving parallel linear probing. Lanes in `act` each hold a key;
// the result equals processing them in lane order one at a time ("find the
// key or the first empty slot from pos, insert there"). Rounds: every
// unfinished lane scans the current table to its key or its first empty slot.
// Lanes that stop at different empty slots do not interact, except through a
// lane that lost a shared slot to a lower lane: in lane order it continues
// past that slot and may take a slot that a higher lane found empty. So in a
// round the lowest lane of each shared slot inserts only if it is below the
// lowest losing lane; every other unfinished lane scans again in the next
// round (the lowest unfinished lane always inserts, so rounds end). Returns,
// per lane, whether it inserted (*ins) and the slot where it stopped (*pos).
__device__ __forceinline__ void emu_probe_rounds(uint32_t* tab, uint32_t mask, uint32_t key, bool act, uint32_t start,
                                                 int lane, bool* ins, uint32_t* pos) {
  const unsigned FULL = 0xFFFFFFFFu;
  uint32_t p = start;
  bool done = !act;
  bool inserted = false;
  for (;;) {
    if (!done) {
      uint32_t v = tab[p];
      while (v != PANN_PAD && v != key) { p = (p + 1) & mask; v = tab[p]; }
      if (v == key) done = true;
    }
    unsigned want = __ballot_sync(FULL, !done);
    if (!want) break;
    unsigned grp = __match_any_sync(FULL, done ? (0x80000000u | (uint32_t)lane) : p);
    const bool lowest = !done && (__ffs(grp & want) - 1) == lane;
    const unsigned losers = want & ~__ballot_sync(FULL, lowest);
    const unsigned below = losers ? ((1u << (__ffs(losers) - 1)) - 1u) : FULL;
    const bool win = lowest && ((below >> lane) & 1u);
    if (win) {
      tab[p] = key;
      inserted = true;
      done = true;
    }
    const unsigned won = __ballot_sync(FULL, win);
    __syncwarp();
    if (won == want) break;  // nobody lost a slot: every call is finished
  }
  *ins = inserted;
  *pos = p;
}

// Longest cluster the ranked placement replays; a longer one (or more long
// clusters than the scratch lists) sends it to the plain sequential pass.
constexpr uint32_t EMU_LONG_CLUSTER = 256;

// Warp: place the keys keys[0..cnt) into the empty table `other` (mask
// nmask) exactly as inserting them one at a time in rank order would
// (hashset.h:39-47: probe from the key's slot to its first empty slot; a key
// already there is not inserted again). With linear probing the set of
// occupied slots does not depend on the insertion order; only which key sits
// where inside a cluster (a maximal run of occupied slots) does, and a key
// only ever lands in the cluster that holds its home. So: (A) the keys'
// ranks are placed in any order (lanes take ranks far apart, so they seldom
// share slots), which fixes the clusters; (B) the lane whose key starts a
// cluster of up to 8 keys replays it in rank order, each key at the first
// free slot from its home, and the warp replays each longer cluster
// together. A cluster longer than EMU_LONG_CLUSTER sends the placement to a
// plain sequential pass instead. `tail` (tail_words words after the keys,
// which may alias the keys' own buffer past cnt) holds the owner bits and
// the list of long clusters.
__device__ __forceinline__ void emu_place_ranked(uint32_t* keys, uint32_t cnt, uint32_t* other, uint32_t nmask,
                                                 uint32_t tail_words, int lane) {
  const unsigned FULL = 0xFFFFFFFFu;
  const uint32_t nsize = nmask + 1;
  const uint4 e4 = make_uint4(PANN_PAD, PANN_PAD, PANN_PAD, PANN_PAD);
  // (A) ranks into the new table, lane l taking rank l * nb + b in batch b; a
  // key the old table holds twice keeps the smaller rank (its first copy in
  // old-slot order, the one the reference inserts; the other copy finds it)
  const uint32_t nb = (cnt + 31) / 32;
  const uint32_t stride = nb | 1u;  // odd: the 32 lanes' ranks fall in 32 different banks
  for (uint32_t b = 0; b < stride; b++) {
    const uint32_t r = (uint32_t)lane * stride + b;
    bool done = r >= cnt;
    const uint32_t k = done ? PANN_PAD : keys[r];
    uint32_t p = ref_slot(k, nmask);
    for (;;) {
      if (!done) {
        uint32_t w = other[p];
        while (w != PANN_PAD && keys[w] != k) { p = (p + 1) & nmask; w = other[p]; }
        if (w != PANN_PAD) {
          done = true;
          if (r < w) atomicMin(other + p, r);
        }
      }
      const unsigned want = __ballot_sync(FULL, !done);
      if (!want) break;
      const unsigned grp = __match_any_sync(FULL, done ? (0x80000000u | (uint32_t)lane) : p);
      if (!done && (__ffs(grp & want) - 1) == lane) {
        other[p] = r;
        done = true;
      }
      __syncwarp();
    }
  }
  __syncwarp();
  __threadfence_block();
  bool fallback = false;
  // (B) owners: keys that start a cluster, one bit per rank in the old table's
  // free tail; then each owner replays its cluster of up to 8 keys in
  // registers, and the warp each longer one (listed in the free tail)
  const uint32_t words = nb;
  uint32_t* owner = keys + ((cnt + 3) & ~3u);
  uint32_t* scratch = owner + ((words + 3) & ~3u);
  const bool scratch_ok = (size_t)(scratch - keys) + 32ull * 64 <= (size_t)tail_words;
  if (!fallback) {
    // the rank at each cluster's first slot (occupied, the slot before it
    // empty), found by one pass over the slots
    for (uint32_t b = lane; b < nb; b += 32) owner[b] = 0;
    __syncwarp();
    for (uint32_t base = 0; base < nsize; base += 32) {
      const uint32_t p = base + (uint32_t)lane;
      const uint32_t w = p < nsize ? other[p] : PANN_PAD;
      if (w != PANN_PAD && other[(p - 1) & nmask] == PANN_PAD) atomicOr(owner + (w >> 5), 1u << (w & 31));
    }
    __syncwarp();
    __threadfence_block();
    // clusters of up to 8 keys are replayed by their owner lane in registers;
    // longer ones are listed (start, length) in the scratch rows and replayed
    // by the whole warp afterwards, so one long cluster does not hold 31 idle
    // lanes for the square of its length
    uint32_t* longs = scratch;
    const uint32_t long_cap = scratch_ok ? 1024u : 0u;  // (start, length) pairs in 2048 words
    uint32_t nlong = 0;
    for (uint32_t b = 0; b < nb; b++) {
      const uint32_t r = b * 32 + lane;
      bool is_long = false;
      uint32_t s0 = 0, m = 0;
      if (r < cnt && ((owner[b] >> lane) & 1u)) {
        s0 = ref_slot(keys[r], nmask);
        while (other[s0] != r) s0 = (s0 + 1) & nmask;
        m = 1;
        while (m <= 8 && other[(s0 + m) & nmask] != PANN_PAD) m++;
        if (m == 1) {
          other[s0] = keys[r];
        } else if (m <= 8) {
          uint32_t ix[8], kx[8], ox[8];
#pragma unroll
          for (int j = 0; j < 8; j++) ix[j] = (uint32_t)j < m ? other[(s0 + j) & nmask] : 0xFFFFFFFFu;
#pragma unroll
          for (int j = 0; j < 8; j++) {
            kx[j] = (uint32_t)j < m ? keys[ix[j]] : 0u;
            ox[j] = (ref_slot(kx[j], nmask) - s0) & nmask;  // home offset inside the cluster
          }
          uint32_t taken = 0, used = 0;
          for (uint32_t t = 0; t < m; t++) {
            uint32_t best = 0xFFFFFFFFu, bj = 0;
#pragma unroll
            for (int j = 0; j < 8; j++)
              if (!((used >> j) & 1u) && ix[j] < best) { best = ix[j]; bj = (uint32_t)j; }
            used |= 1u << bj;
            uint32_t key = 0, o = 0;
#pragma unroll
            for (int j = 0; j < 8; j++)
              if ((uint32_t)j == bj) { key = kx[j]; o = ox[j]; }
            const uint32_t pos = (uint32_t)(__ffs(~taken & (~0u << o)) - 1);
            taken |= 1u << pos;
            other[(s0 + pos) & nmask] = key;
          }
        } else {
          is_long = true;  // its length is measured by the warp below
        }
      }
      const unsigned lm = __ballot_sync(FULL, is_long);
      if (is_long) {
        const uint32_t at = nlong + __popc(lm & ((1u << lane) - 1));
        if (at < long_cap) {
          longs[2 * at] = s0;
          longs[2 * at + 1] = m;
        }
      }
      nlong += __popc(lm);
      __syncwarp();
    }
    fallback = nlong > long_cap;
    // Long clusters, one at a time over the warp. Inserting a cluster's keys
    // in rank order with linear probing leaves at each slot, left to right,
    // the smallest-rank key whose home is at or before that slot among those
    // not yet placed (a key of smaller rank that could reach the slot was
    // inserted first and found every slot before it taken by smaller ranks),
    // so each slot is one warp minimum over the eligible ranks.
    for (uint32_t c = 0; c < nlong && !fallback; c++) {
      const uint32_t s0 = longs[2 * c];
      uint32_t m = 9;  // longer than 8: count 32 slots at a time up to its first empty slot
      for (;;) {
        const unsigned emp = __ballot_sync(FULL, other[(s0 + m + (uint32_t)lane) & nmask] == PANN_PAD);
        if (emp) {
          m += (uint32_t)(__ffs(emp) - 1);
          break;
        }
        m += 32;
        if (m > EMU_LONG_CLUSTER) break;
      }
      if (m > EMU_LONG_CLUSTER) {
        fallback = true;
        break;
      }
      uint32_t rk[EMU_LONG_CLUSTER / 32], ky[EMU_LONG_CLUSTER / 32], of[EMU_LONG_CLUSTER / 32];
#pragma unroll
      for (int j = 0; j < EMU_LONG_CLUSTER / 32; j++) {
        const uint32_t i = (uint32_t)j * 32 + (uint32_t)lane;
        rk[j] = 0xFFFFFFFFu;
        of[j] = 0xFFFFFFFFu;
        ky[j] = 0;
        if (i < m) {
          rk[j] = other[(s0 + i) & nmask];
          ky[j] = keys[rk[j]];
          of[j] = (ref_slot(ky[j], nmask) - s0) & nmask;
        }
      }
      __syncwarp();
      for (uint32_t t = 0; t < m; t++) {
        uint32_t best = 0xFFFFFFFFu, bkey = 0;
        int bj = -1;
#pragma unroll
        for (int j = 0; j < EMU_LONG_CLUSTER / 32; j++)
          if (of[j] <= t && rk[j] < best) { best = rk[j]; bkey = ky[j]; bj = j; }
        const uint32_t wmin = __reduce_min_sync(FULL, best);
        if (bj >= 0 && best == wmin) {
#pragma unroll
          for (int j = 0; j < EMU_LONG_CLUSTER / 32; j++)
            if (j == bj) { rk[j] = 0xFFFFFFFFu; of[j] = 0xFFFFFFFFu; }
          other[(s0 + t) & nmask] = bkey;
        }
      }
      __syncwarp();
    }
  }
  if (fallback) {
    // the plain sequential re-insertion
    for (uint32_t i = lane; i < (nsize >> 2); i += 32) reinterpret_cast<uint4*>(other)[i] = e4;
    __syncwarp();
    if (lane == 0) {
      for (uint32_t i = 0; i < cnt; i++) {
        const uint32_t k = keys[i];
        uint32_t p = ref_slot(k, nmask);
        while (other[p] != PANN_PAD && other[p] != k) p = (p + 1) & nmask;
        other[p] = k;
      }
    }
    __syncwarp();
  }
}

// Warp: grow the table (hashset.h:25-38): every key of the old table is
// re-inserted in old-slot order (num_entries counts each re-insertion), then
// the key that triggered the growth continues from its old-mask slot
// (:39-47). Returns false if the grown table does not fit this tier. The
// re-insertion is emu_place_ranked with the keys' ranks in old-slot order.
__device__ __forceinline__ bool emu_grow(EmuHash& h, uint32_t a, int lane, bool* a_seen) {
  const unsigned FULL = 0xFFFFFFFFu;
  const uint32_t size = 1u << h.bits, nsize = size * 2;
  if (nsize > h.other_cap) return false;
  uint32_t* other = h.other;
  const uint4 e4 = make_uint4(PANN_PAD, PANN_PAD, PANN_PAD, PANN_PAD);
  for (uint32_t i = lane; i < (nsize >> 2); i += 32) reinterpret_cast<uint4*>(other)[i] = e4;
  __syncwarp();
  const uint32_t oldmask = size - 1, nmask = nsize - 1;
  // the old table's keys compacted to its front in slot order (writes never
  // pass the chunk being read): keys[r] is the key of rank r
  uint32_t cnt = 0;
  for (uint32_t base = 0; base < size; base += 128) {  // 4 slots per lane per step
    uint32_t k4[4];
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint32_t i = base + 4 * (uint32_t)lane + (uint32_t)j;
      k4[j] = i < size ? h.cur[i] : PANN_PAD;
      c += k4[j] != PANN_PAD;
    }
    uint32_t pre = c;  // inclusive prefix over lanes
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, pre, d);
      if (lane >= d) pre += t;
    }
    const uint32_t total = __shfl_sync(FULL, pre, 31);
    __syncwarp();
    uint32_t at = cnt + pre - c;
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (k4[j] != PANN_PAD) h.cur[at++] = k4[j];
    cnt += total;
    __syncwarp();
  }
  emu_place_ranked(h.cur, cnt, other, nmask, size, lane);
  __threadfence_block();
  const long long added = cnt;
  h.num_entries += added;
  uint32_t* t = h.cur; h.cur = h.other; h.other = t;
  uint32_t c = h.cur_cap; h.cur_cap = h.other_cap; h.other_cap = c;
  h.bits += 1;
  // the call that grew the table: probe from the old-mask slot
  int hit = 0;
  if (lane == 0) {
    uint32_t loc = ref_slot(a, oldmask);
    if (h.cur[loc] != PANN_PAD) {
      loc = (loc + 1) & nmask;
      while (h.cur[loc] != PANN_PAD && h.cur[loc] != a) loc = (loc + 1) & nmask;
      hit = h.cur[loc] == a;
    }
    if (!hit) h.cur[loc] = a;
  }
  hit = __shfl_sync(FULL, hit, 0);
  __syncwarp();
  __threadfence_block();
  if (!hit) h.num_entries++;
  *a_seen = hit != 0;
  return true;
}

// hashset::operator() (hashset.h:22-48) for up to 32 keys, lane i holding the
// i-th key in call order (valid lanes form a prefix). *seen gets each call's
// result. Returns false if the table would outgrow this tier.
__device__ __forceinline__ bool emu_batch(EmuHash& h, uint32_t key, bool valid, int lane, bool* seen) {
  const unsigned FULL = 0xFFFFFFFFu;
  unsigned todo = __ballot_sync(FULL, valid);
  bool my_seen = false;
  while (todo) {
    const bool act = (todo >> lane) & 1u;
    const uint32_t size = 1u << h.bits, mask = size - 1;
    const uint32_t home = ref_slot(key, mask);
    const bool home_hit0 = act && h.cur[home] == key;  // present at its home before this batch
    __syncwarp();
    bool ins;
    uint32_t pos;
    emu_probe_rounds(h.cur, mask, key, act, home, lane, &ins, &pos);
    // a repeated key whose first copy in this batch was inserted at that home
    unsigned kgrp = __match_any_sync(FULL, act ? key : (0x80000000u | (uint32_t)lane));
    int first = __ffs(kgrp & todo) - 1;
    bool f_ins = __shfl_sync(FULL, ins, first < 0 ? lane : first);
    uint32_t f_pos = __shfl_sync(FULL, pos, first < 0 ? lane : first);
    bool home_hit = home_hit0 || (act && first >= 0 && first < lane && f_ins && f_pos == home);
    // calls that miss their home slot check for growth against num_entries so far
    unsigned insm = __ballot_sync(FULL, act && ins);
    long long before = h.num_entries + __popc(insm & ((1u << lane) - 1));
    bool grows = act && !home_hit && before > (long long)(size / 2);
    unsigned gm = __ballot_sync(FULL, grows);
    if (!gm) {
      if (act) my_seen = !ins;
      h.num_entries += __popc(insm);
      break;
    }
    const int g = __ffs(gm) - 1;
    // undo the tentative inserts of calls at or after g, keep the earlier ones
    if (act && ins && lane >= g) h.cur[pos] = PANN_PAD;
    __syncwarp();
    __threadfence_block();
    if (act && lane < g) my_seen = !ins;
    h.num_entries += __popc(insm & ((1u << g) - 1));
    uint32_t ag = __shfl_sync(FULL, key, g);
    bool gseen = false;
    if (!emu_grow(h, ag, lane, &gseen)) return false;
    if (lane == g) my_seen = gseen;
    todo &= ~((2u << g) - 1u);  // calls after g run against the grown table
  }
  *seen = my_seen;
  return true;
}

// As emu_batch, but stops at the first call that grows the table: the calls
// before it take effect (their results in *seen) and *grow_lane gets the
// growing call's lane, -1 if none. The caller grows the table for that key
// (emu_grow_block) and continues with the lanes after it.
__device__ __forceinline__ void emu_batch_part(EmuHash& h, uint32_t key, bool act, int lane, bool* seen,
                                               int* grow_lane) {
  const unsigned FULL = 0xFFFFFFFFu;
  const unsigned todo = __ballot_sync(FULL, act);
  const uint32_t size = 1u << h.bits, mask = size - 1;
  const uint32_t home = ref_slot(key, mask);
  const bool home_hit0 = act && h.cur[home] == key;
  __syncwarp();
  bool ins;
  uint32_t pos;
  emu_probe_rounds(h.cur, mask, key, act, home, lane, &ins, &pos);
  const unsigned kgrp = __match_any_sync(FULL, act ? key : (0x80000000u | (uint32_t)lane));
  const int first = __ffs(kgrp & todo) - 1;
  const bool f_ins = __shfl_sync(FULL, ins, first < 0 ? lane : first);
  const uint32_t f_pos = __shfl_sync(FULL, pos, first < 0 ? lane : first);
  const bool home_hit = home_hit0 || (act && first >= 0 && first < lane && f_ins && f_pos == home);
  const unsigned insm = __ballot_sync(FULL, act && ins);
  const long long before = h.num_entries + __popc(insm & ((1u << lane) - 1));
  const bool grows = act && !home_hit && before > (long long)(size / 2);
  const unsigned gm = __ballot_sync(FULL, grows);
  if (!gm) {
    if (act) *seen = !ins;
    h.num_entries += __popc(insm);
    *grow_lane = -1;
    return;
  }
  const int g = __ffs(gm) - 1;
  if (act && ins && lane >= g) h.cur[pos] = PANN_PAD;  // undo the calls at and after g
  __syncwarp();
  __threadfence_block();
  if (act && lane < g) *seen = !ins;
  h.num_entries += __popc(insm & ((1u << g) - 1));
  *grow_lane = g;
}

// Block: emu_place_ranked with every thread of the block (nth threads, NW
// warps). (A) ranks claim slots with compare-and-swap in any order (the set
// of occupied slots does not depend on it; a repeated key keeps its smaller
// rank); (B) cluster owners from one pass over the slots, clusters of up to
// 8 keys replayed by their owner thread, longer ones by one warp each;
// beyond EMU_LONG_CLUSTER keys, or more long clusters than the free tail
// lists, a sequential pass by thread 0. ctl: 4 words of shared scratch.
__device__ __forceinline__ void emu_place_ranked_block(uint32_t* keys, uint32_t cnt, uint32_t* other, uint32_t nmask,
                                                       uint32_t tail_words, int tid, int nth, volatile uint32_t* ctl) {
  const unsigned FULL = 0xFFFFFFFFu;
  const int lane = tid & 31, warp = tid >> 5, nw = nth >> 5;
  const uint32_t nsize = nmask + 1;
  volatile uint32_t* vo = other;
  for (uint32_t r = (uint32_t)tid; r < cnt; r += (uint32_t)nth) {
    const uint32_t k = keys[r];
    uint32_t p = ref_slot(k, nmask);
    for (;;) {
      uint32_t w = vo[p];
      if (w == PANN_PAD) {
        w = atomicCAS(other + p, PANN_PAD, r);
        if (w == PANN_PAD) break;
      }
      if (keys[w] == k) {
        atomicMin(other + p, r);
        break;
      }
      p = (p + 1) & nmask;
    }
  }
  const uint32_t nb = (cnt + 31) / 32;
  uint32_t* owner = keys + ((cnt + 3) & ~3u);
  uint32_t* longs = owner + ((nb + 3) & ~3u);
  const uint32_t room = (size_t)(longs - keys) < (size_t)tail_words ? tail_words - (uint32_t)(longs - keys) : 0u;
  const uint32_t long_cap = room < 1024u ? room : 1024u;
  if (tid == 0) { ctl[0] = 0; ctl[1] = 0; }
  for (uint32_t b = (uint32_t)tid; b < nb; b += (uint32_t)nth) owner[b] = 0;
  __syncthreads();
  for (uint32_t p = (uint32_t)tid; p < nsize; p += (uint32_t)nth) {
    const uint32_t w = vo[p];
    if (w != PANN_PAD && vo[(p - 1) & nmask] == PANN_PAD) atomicOr(owner + (w >> 5), 1u << (w & 31));
  }
  __syncthreads();
  for (uint32_t r = (uint32_t)tid; r < cnt; r += (uint32_t)nth) {
    if (!((owner[r >> 5] >> (r & 31)) & 1u)) continue;
    const uint32_t s0 = ref_slot(keys[r], nmask);  // an owner sits at its home
    uint32_t m = 1;
    while (m <= 8 && vo[(s0 + m) & nmask] != PANN_PAD) m++;
    if (m == 1) {
      other[s0] = keys[r];
    } else if (m <= 8) {
      uint32_t ix[8], kx[8], ox[8];
#pragma unroll
      for (int j = 0; j < 8; j++) ix[j] = (uint32_t)j < m ? vo[(s0 + j) & nmask] : 0xFFFFFFFFu;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        kx[j] = (uint32_t)j < m ? keys[ix[j]] : 0u;
        ox[j] = (ref_slot(kx[j], nmask) - s0) & nmask;
      }
      uint32_t taken = 0, used = 0;
      for (uint32_t t = 0; t < m; t++) {
        uint32_t best = 0xFFFFFFFFu, bj = 0;
#pragma unroll
        for (int j = 0; j < 8; j++)
          if (!((used >> j) & 1u) && ix[j] < best) { best = ix[j]; bj = (uint32_t)j; }
        used |= 1u << bj;
        uint32_t key = 0, o = 0;
#pragma unroll
        for (int j = 0; j < 8; j++)
          if ((uint32_t)j == bj) { key = kx[j]; o = ox[j]; }
        const uint32_t pos = (uint32_t)(__ffs(~taken & (~0u << o)) - 1);
        taken |= 1u << pos;
        other[(s0 + pos) & nmask] = key;
      }
    } else {
      const uint32_t at = atomicAdd((uint32_t*)ctl, 1u);
      if (at < long_cap) longs[at] = s0;
    }
  }
  __syncthreads();
  const uint32_t nlong = ctl[0];
  bool fallback = nlong > long_cap;
  for (uint32_t c = (uint32_t)warp; c < nlong && !fallback; c += (uint32_t)nw) {
    const uint32_t s0 = longs[c];
    uint32_t m = 9;
    for (;;) {
      const unsigned emp = __ballot_sync(FULL, vo[(s0 + m + (uint32_t)lane) & nmask] == PANN_PAD);
      if (emp) {
        m += (uint32_t)(__ffs(emp) - 1);
        break;
      }
      m += 32;
      if (m > EMU_LONG_CLUSTER) break;
    }
    if (m > EMU_LONG_CLUSTER) {
      if (lane == 0) ctl[1] = 1;
      break;
    }
    uint32_t rk[EMU_LONG_CLUSTER / 32], ky[EMU_LONG_CLUSTER / 32], of[EMU_LONG_CLUSTER / 32];
#pragma unroll
    for (int j = 0; j < EMU_LONG_CLUSTER / 32; j++) {
      const uint32_t i = (uint32_t)j * 32 + (uint32_t)lane;
      rk[j] = 0xFFFFFFFFu;
      of[j] = 0xFFFFFFFFu;
      ky[j] = 0;
      if (i < m) {
        rk[j] = vo[(s0 + i) & nmask];
        ky[j] = keys[rk[j]];
        of[j] = (ref_slot(ky[j], nmask) - s0) & nmask;
      }
    }
    __syncwarp();
    for (uint32_t t = 0; t < m; t++) {
      uint32_t best = 0xFFFFFFFFu, bkey = 0;
      int bj = -1;
#pragma unroll
      for (int j = 0; j < EMU_LONG_CLUSTER / 32; j++)
        if (of[j] <= t && rk[j] < best) { best = rk[j]; bkey = ky[j]; bj = j; }
      const uint32_t wmin = __reduce_min_sync(FULL, best);
      if (bj >= 0 && best == wmin) {
#pragma unroll
        for (int j = 0; j < EMU_LONG_CLUSTER / 32; j++)
          if (j == bj) { rk[j] = 0xFFFFFFFFu; of[j] = 0xFFFFFFFFu; }
        other[(s0 + t) & nmask] = bkey;
      }
    }
    __syncwarp();
  }
  __syncthreads();
  if (fallback || ctl[1]) {
    const uint4 e4 = make_uint4(PANN_PAD, PANN_PAD, PANN_PAD, PANN_PAD);
    for (uint32_t i = (uint32_t)tid; i < (nsize >> 2); i += (uint32_t)nth) reinterpret_cast<uint4*>(other)[i] = e4;
    __syncthreads();
    if (tid == 0) {
      for (uint32_t i = 0; i < cnt; i++) {
        const uint32_t k = keys[i];
        uint32_t p = ref_slot(k, nmask);
        while (vo[p] != PANN_PAD && vo[p] != k) p = (p + 1) & nmask;
        vo[p] = k;
      }
    }
  }
  __syncthreads();
}

// Block: emu_grow with every thread (the table state passed in, the
// triggering key a). Returns false (every thread alike) if the grown table
// does not fit `other_cap`; else *added = re-inserted keys and *a_seen =
// whether a was found. ctl: 8 words of shared scratch.
__device__ __forceinline__ bool emu_grow_block(uint32_t* cur, uint32_t* other, uint32_t bits, uint32_t other_cap,
                                               uint32_t a, int tid, int nth, volatile uint32_t* ctl, uint32_t* added,
                                               bool* a_seen) {
  const unsigned FULL = 0xFFFFFFFFu;
  const int lane = tid & 31, warp = tid >> 5, nw = nth >> 5;
  const uint32_t size = 1u << bits, nsize = size * 2;
  if (nsize > other_cap) return false;
  const uint4 e4 = make_uint4(PANN_PAD, PANN_PAD, PANN_PAD, PANN_PAD);
  for (uint32_t i = (uint32_t)tid; i < (nsize >> 2); i += (uint32_t)nth) reinterpret_cast<uint4*>(other)[i] = e4;
  // the old table's keys compacted to its front in slot order
  uint32_t cnt = 0;
  for (uint32_t base = 0; base < size; base += 4u * (uint32_t)nth) {
    uint32_t k4[4];
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint32_t i = base + 4 * (uint32_t)tid + (uint32_t)j;
      k4[j] = i < size ? cur[i] : PANN_PAD;
      c += k4[j] != PANN_PAD;
    }
    uint32_t pre = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, pre, d);
      if (lane >= d) pre += t;
    }
    if (lane == 31) ctl[4 + warp] = pre;
    __syncthreads();
    uint32_t woff = 0, total = 0;
    for (int w = 0; w < nw; w++) {
      const uint32_t t = ctl[4 + w];
      woff += w < warp ? t : 0u;
      total += t;
    }
    __syncthreads();
    uint32_t at = cnt + woff + pre - c;
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (k4[j] != PANN_PAD) cur[at++] = k4[j];
    cnt += total;
    __syncthreads();
  }
  emu_place_ranked_block(cur, cnt, other, nsize - 1, size, tid, nth, ctl);
  // the call that grew the table: probe from the old-mask slot in the new table
  if (tid == 0) {
    uint32_t loc = ref_slot(a, size - 1);
    uint32_t hit = 0;
    if (other[loc] != PANN_PAD) {
      loc = (loc + 1) & (nsize - 1);
      while (other[loc] != PANN_PAD && other[loc] != a) loc = (loc + 1) & (nsize - 1);
      hit = other[loc] == a;
    }
    if (!hit) other[loc] = a;
    ctl[0] = hit;
  }
  __syncthreads();
  *added = cnt;
  *a_seen = ctl[0] != 0;
  __syncthreads();
  return true;
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

  for (;;) {
    uint32_t job = 0;
    if (lane == 0) job = atomicAdd(a.job_counter, 1u);
    job = __shfl_sync(FULL, job, 0);
    if (job >= njobs) break;
    const uint32_t qi = a.job_list ? a.job_list[job] : job;
    const uint32_t rec_id = e.job_rec ? e.job_rec[job] : PANN_PAD;
    const uint32_t L = a.qL ? a.qL[qi] : a.L;  // this query's beam
    const uint32_t kq = a.qk ? a.qk[qi] : a.k;
    const uint32_t bits0 = a.qL ? ref_bits(L, a.dl) : e.bits0;
    const uint32_t self = a.self_ids ? a.self_ids[qi] : PANN_PAD;
    const uint8_t* qsrc = a.self_ids ? a.points + (uint64_t)self * a.stride : a.queries + (uint64_t)qi * a.stride;
    stage_query<DT, MT>(qs, qsrc, (int)a.nchunks, lane);
    for (uint32_t i = lane; i < (1u << bits0); i += 32) tabA[i] = PANN_PAD;
    for (uint32_t i = lane; i < e.vs_slots; i += 32) vset[i] = PANN_PAD;
    __syncwarp();
    __threadfence_block();
    EmuHash h;
    h.cur = tabA; h.other = tabB; h.cur_cap = e.capA; h.other_cap = e.capB;
    h.bits = bits0; h.num_entries = 0;
    bool ok = true;
    bool sdummy;
    int32_t qq = 0;
    if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), a.nchunks);

    uint64_t* fr = frA;
    uint64_t* fr2 = frB;
    int fn, cn;
    uint32_t cmps;
    uint64_t nvis;
    float u0 = 0.0f;  // distance of unvisited_frontier[0] at the last merge (early stopping)
    bool u0_fresh = true;
    if (rec_id != PANN_PAD) {
      // resume tier 0's query: its state before the visit that could cross the
      // growth threshold, and the reference's table rebuilt from the insertion
      // log (no growth can have happened before that visit)
      const ResumeLayout ly = resume_layout(a.L, a.Ccap, a.logcap, a.viscap);
      const uint32_t* rec = a.rec_pool + (size_t)rec_id * a.rec_words;
      fn = (int)rec[1];
      cn = (int)rec[2];
      nvis = rec[3];
      cmps = rec[4];
      const uint32_t entries = rec[5];
      u0 = __uint_as_float(rec[6]);  // taken by tier 0 before it handed over
      u0_fresh = false;
      const uint64_t* rfr = reinterpret_cast<const uint64_t*>(rec + ly.fr);
      const uint64_t* rcand = reinterpret_cast<const uint64_t*>(rec + ly.cand);
      for (int i = lane; i < fn; i += 32) fr[i] = rfr[i];
      for (int i = lane; i < cn; i += 32) cand[i] = rcand[i];
      // the logged ids, inserted in log order (staged in table B, unused until a growth)
      for (uint32_t i = lane; i < entries; i += 32) h.other[i] = rec[ly.log + i];
      __syncwarp();
      emu_place_ranked(h.other, entries, h.cur, (1u << h.bits) - 1, h.other_cap, lane);
      __syncwarp();
      h.num_entries = entries;
      for (uint32_t i = lane; i < (uint32_t)nvis; i += 32) vset_insert(vset, vmask, rec[ly.vis + i]);
    } else {
      // starting points, inserted in the given order (:73-76)
      for (uint32_t s = lane; s < a.n_start; s += 32) {
        uint32_t id = a.starts[s];
        float dd = point_dist<DT, MT>(a.points + (uint64_t)id * a.stride, qs, a.d, a.nchunks, qq);
        frB[s] = make_key(dd, id);
      }
      for (uint32_t s0 = 0; s0 < a.n_start && ok; s0 += 32)
        ok = emu_batch(h, s0 + lane < a.n_start ? a.starts[s0 + lane] : PANN_PAD, s0 + lane < a.n_start, lane, &sdummy);
      __syncwarp();
      warp_rank_sort(frB, fr, (int)a.n_start, lane);
      fn = (int)a.n_start;
      cn = 0;
      cmps = a.n_start;
      nvis = 0;
    }
    __syncwarp();
    uint32_t status = QS_REF_WOULD_GROW;
    if (!ok) status |= QS_TABLE_FULL;

    while (ok) {
      __syncwarp();
      int first = -1, second = -1, cnt = 0;
      for (int b = 0; b < fn; b += 32) {
        int i = b + lane;
        bool unv = (i < fn) && !(fr[i] & PANN_VFLAG);
        unsigned m = __ballot_sync(FULL, unv);
        cnt += __popc(m);
        if (first < 0 && m) {
          first = b + __ffs(m) - 1;
          m &= m - 1;
        }
        if (first >= 0 && second < 0 && m) second = b + __ffs(m) - 1;
      }
      if (first < 0 || nvis >= a.limit) break;
      // the next node to expand is most often the following unvisited entry:
      // its adjacency row goes to L2 while this visit runs
      if (second >= 0 && (uint32_t)lane * 32 < a.R)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a.graph + (uint64_t)key_id(fr[second]) * a.R + 32 * lane));
      if (u0_fresh) {
        u0 = key_dist(fr[first]);
        u0_fresh = false;
      }
      if (a.es_count > 0.0 && (double)nvis >= a.es_count && !((double)key_dist(fr[0]) <= a.es_radius) &&
          !((double)u0 <= a.es_esr))
        break;  // early_stopping (earlyStopping.h:19-29)
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
      // adjacency ids looked up in order, 32 calls per batch (:153-159)
      int nnew = 0;
      bool full_tab = false;
      const uint32_t* grow = a.graph + (uint64_t)cid * a.R;
      uint32_t vnext = (uint32_t)lane < nel ? __ldg(grow + lane) : PANN_PAD;  // one chunk ahead
      for (uint32_t b = 0; b < nel; b += 32) {
        const uint32_t v = vnext;
        vnext = (b + 32 + lane < nel) ? __ldg(grow + b + 32 + lane) : PANN_PAD;
        bool seen = false;
        if (!emu_batch(h, v, v != PANN_PAD, lane, &seen)) { full_tab = true; break; }
        bool isnew = v != PANN_PAD && !seen && v != self;
        unsigned mn = __ballot_sync(FULL, isnew);
        if (isnew) nbuf[nnew + __popc(mn & ((1u << lane) - 1))] = v;
        nnew += __popc(mn);
      }
      if (full_tab) {
        status |= QS_TABLE_FULL;
        break;
      }
      __syncwarp();
      cmps += (uint32_t)nnew;
      if ((uint32_t)(cn + nnew) > a.Ccap) { status |= QS_INTERNAL; break; }
      // two rows per lane per round: rows b+lane and b+32+lane
      for (int b = 0; b < nnew; b += 64) {
        const int i0 = b + lane, i1 = b + 32 + lane;
        float d0 = 0.0f, d1 = 0.0f;
        uint32_t v0 = 0, v1 = 0;
        if (i0 < nnew) {
          v0 = nbuf[i0];
          v1 = i1 < nnew ? nbuf[i1] : 0u;
          // one warp per SM here: registers are plentiful, load whole rows at once
          point_dist2<DT, MT, 12>(a.points + (uint64_t)v0 * a.stride,
                              i1 < nnew ? a.points + (uint64_t)v1 * a.stride : nullptr, qs, a.nchunks, qq, d0, d1,
                              a.opaque_zero);
        }
        bool keep0 = i0 < nnew && !(d0 >= cutoff);
        unsigned m0 = __ballot_sync(FULL, keep0);
        if (keep0) cand[cn + __popc(m0 & ((1u << lane) - 1))] = make_key(d0, v0);
        cn += __popc(m0);
        bool keep1 = i1 < nnew && !(d1 >= cutoff);
        unsigned m1 = __ballot_sync(FULL, keep1);
        if (keep1) cand[cn + __popc(m1 & ((1u << lane) - 1))] = make_key(d1, v1);
        cn += __popc(m1);
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
      u0_fresh = true;
      uint64_t* t = fr; fr = fr2; fr2 = t;
      cn = 0;
      __syncwarp();
    }

    if (status & QS_TABLE_FULL) {
      // the emulated table outgrew this tier: the next tier (larger, global) re-runs it
      if (lane == 0) {
        if (e.overflow_list) {
          uint32_t pos = atomicAdd(e.overflow_count, 1u);
          e.overflow_list[pos] = qi;
          e.overflow_rec[pos] = rec_id;
        }
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
    // a query handed over before its table could cross the growth threshold
    // may finish without the reference's hashset ever growing
    if (h.bits == bits0) status &= ~(uint32_t)QS_REF_WOULD_GROW;
    if ((uint32_t)fn < kq) status |= QS_SHORT;
    for (uint32_t j = lane; j < a.kstride; j += 32) {
      bool okk = j < (uint32_t)fn && j < kq;
      a.out_ids[(uint64_t)qi * a.kstride + j] = okk ? key_id(fr[j]) : PANN_PAD;
      if (a.out_dists) a.out_dists[(uint64_t)qi * a.kstride + j] = okk ? key_dist(fr[j]) : 0.0f;
    }
    if (lane == 0) {
      if (a.out_visited) a.out_visited[qi] = (uint32_t)nvis;
      if (a.out_cmps) a.out_cmps[qi] = cmps;
      if (a.out_status) a.out_status[qi] = status;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// The same emulation with one block of NW warps per query (shared-memory
// tables only). The per-visit work that does not touch the reference's table
// runs beside it: warp 0 makes the hashset calls in order, while warps
// 1..NW-1 score every neighbour of the visited node (each thread one whole
// row, all its loads in flight at once), so the rows arrive while the table
// is probed; the distances of the ids the table reports new are then taken
// from that set. Sorting, de-duplication and the merge run on all threads.
// Per query the results, counters and status bits equal the single-warp
// kernel's (the same calls on the same table in the same order; candidates
// are a set until sorted, and every order-sensitive step keeps its order).
//
// Shared memory: the query, the two frontiers, the two candidate buffers, the
// new ids with their positions in the adjacency row, the distances of the
// whole row, control words, the visited-id set and the tables A and B.
struct EmuBlockLayout {
  uint32_t fr, cand, nbuf, npos, dall, ctrl, vset, tabA, tabB, bytes;
};
__host__ __device__ inline EmuBlockLayout emu_block_layout(uint64_t stride, uint32_t L, uint32_t Ccap, uint32_t R,
                                                           uint32_t vs, uint32_t capA, uint32_t capB) {
  EmuBlockLayout y;
  const uint32_t R4 = (R + 3) & ~3u;
  uint64_t o = (stride + 15) & ~15ull;
  y.fr = (uint32_t)o;   o += 16ull * L;
  y.cand = (uint32_t)o; o += 16ull * Ccap;
  y.nbuf = (uint32_t)o; o += 4ull * R4;
  y.npos = (uint32_t)o; o += 4ull * R4;
  y.dall = (uint32_t)o; o += 4ull * R4;
  y.ctrl = (uint32_t)o; o += 128;
  y.vset = (uint32_t)o; o += 4ull * vs;
  y.tabA = (uint32_t)o; o += 4ull * capA;
  y.tabB = (uint32_t)o; o += 4ull * capB;
  y.bytes = (uint32_t)((o + 15) & ~15ull);
  return y;
}

// Distance of one whole row, all of its 16-byte chunks loaded before the sum
// (CH >= the row's chunk count keeps every load of the row in flight at once).
template <int DT, int MT, int CH>
__device__ __forceinline__ float row_dist_whole(const uint8_t* __restrict__ row, const uint8_t* qs, int nchunks,
                                                int32_t qq) {
  if (DT == DT_F32) {
    const float4* r = reinterpret_cast<const float4*>(row);
    const float4* q = reinterpret_cast<const float4*>(qs);
    float acc = 0.0f;
    for (int c0 = 0; c0 < nchunks; c0 += CH) {
      float4 b[CH];
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (c0 + c < nchunks) b[c] = __ldg(r + c0 + c);
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (c0 + c < nchunks) acc = f32_chunk<MT>(acc, b[c], q[c0 + c]);
    }
    return MT == MT_L2 ? acc : -acc;
  } else {
    const uint4* r = reinterpret_cast<const uint4*>(row);
    const uint4* q = reinterpret_cast<const uint4*>(qs);
    int32_t pq = 0, pp = 0;
    for (int c0 = 0; c0 < nchunks; c0 += CH) {
      uint4 b[CH];
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (c0 + c < nchunks) b[c] = __ldg(r + c0 + c);
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (c0 + c < nchunks) int_chunk<DT, MT>(b[c], q[c0 + c], pq, pp);
    }
    return int_result<MT>(qq, pq, pp);
  }
}

// Rank sort of n keys from `in` into `out` over all threads of the block
// (ties by index, as warp_rank_sort).
__device__ __forceinline__ void block_rank_sort(const uint64_t* in, uint64_t* out, int n, int tid, int nth) {
  for (int i = tid; i < n; i += nth) {
    const uint64_t ki = in[i] & PANN_KEYMASK;
    int r = 0;
    for (int j = 0; j < n; j++) {
      const uint64_t kj = in[j] & PANN_KEYMASK;
      r += (kj < ki) | ((kj == ki) & (j < i));
    }
    out[r] = in[i];
  }
}

// set_union + trim (as warp_merge) over all threads of the block.
__device__ __forceinline__ int block_merge(const uint64_t* fr, int fn, const uint64_t* c, int cn, uint64_t* out,
                                           int L, int tid, int nth) {
  for (int i = tid; i < fn; i += nth) {
    const uint64_t k = fr[i] & PANN_KEYMASK;
    int lo = 0, hi = cn;
    while (lo < hi) { int mid = (lo + hi) >> 1; if ((c[mid] & PANN_KEYMASK) < k) lo = mid + 1; else hi = mid; }
    if (i + lo < L) out[i + lo] = fr[i];
  }
  for (int j = tid; j < cn; j += nth) {
    const uint64_t k = c[j] & PANN_KEYMASK;
    int lo = 0, hi = fn;
    while (lo < hi) { int mid = (lo + hi) >> 1; if ((fr[mid] & PANN_KEYMASK) < k) lo = mid + 1; else hi = mid; }
    if (j + lo < L) out[j + lo] = c[j];
  }
  const int t = fn + cn;
  return t < L ? t : L;
}

template <int DT, int MT, int NW, int CH>
__global__ void __launch_bounds__(NW * 32, 1) search_emulate_block_kernel(SearchArgs a, EmuArgs e) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nth = NW * 32;
  const unsigned FULL = 0xFFFFFFFFu;
  const EmuBlockLayout y = emu_block_layout(a.stride, a.L, a.Ccap, a.R, e.vs_slots, e.capA, e.capB);
  uint8_t* qs = smem;
  uint64_t* frA = reinterpret_cast<uint64_t*>(smem + y.fr);
  uint64_t* frB = frA + a.L;
  uint64_t* cand = reinterpret_cast<uint64_t*>(smem + y.cand);
  uint64_t* cand2 = cand + a.Ccap;
  uint32_t* nbuf = reinterpret_cast<uint32_t*>(smem + y.nbuf);
  uint32_t* npos = reinterpret_cast<uint32_t*>(smem + y.npos);
  float* dall = reinterpret_cast<float*>(smem + y.dall);
  volatile uint32_t* ctrl = reinterpret_cast<volatile uint32_t*>(smem + y.ctrl);
  uint32_t* vset = reinterpret_cast<uint32_t*>(smem + y.vset);
  uint32_t* tabA = reinterpret_cast<uint32_t*>(smem + y.tabA);
  uint32_t* tabB = reinterpret_cast<uint32_t*>(smem + y.tabB);
  const uint32_t vmask = e.vs_slots - 1;
  const uint32_t nel = a.dl < a.R ? a.dl : a.R;

  for (;;) {
    __syncthreads();
    if (tid == 0) ctrl[0] = emu_claim(a.job_counter, a.njobs_dev, a.nq, e.job_rec, e.early != 0);
    __syncthreads();
    const uint32_t job = ctrl[0];
    if (job == PANN_PAD) break;
    if (e.early) __threadfence();  // the record was published behind a fence
    const uint32_t qi = a.job_list ? a.job_list[job] : job;
    const uint32_t rec_id = e.job_rec ? e.job_rec[job] : PANN_PAD;
    const uint32_t L = a.qL ? a.qL[qi] : a.L;
    const uint32_t kq = a.qk ? a.qk[qi] : a.k;
    const uint32_t bits0 = a.qL ? ref_bits(L, a.dl) : e.bits0;
    const uint32_t self = a.self_ids ? a.self_ids[qi] : PANN_PAD;
    const uint8_t* qsrc = a.self_ids ? a.points + (uint64_t)self * a.stride : a.queries + (uint64_t)qi * a.stride;
    for (int c = tid; c < (int)a.nchunks; c += nth) {
      uint4 v = __ldg(reinterpret_cast<const uint4*>(qsrc) + c);
      if (DT == DT_F32 && MT == MT_L2) v = make_uint4(v.x ^ 0x80000000u, v.y ^ 0x80000000u, v.z ^ 0x80000000u, v.w ^ 0x80000000u);
      reinterpret_cast<uint4*>(qs)[c] = v;
    }
    for (uint32_t i = tid; i < (1u << bits0); i += nth) tabA[i] = PANN_PAD;
    for (uint32_t i = tid; i < e.vs_slots; i += nth) vset[i] = PANN_PAD;
    __syncthreads();
    EmuHash h;  // used by warp 0 only
    h.cur = tabA; h.other = tabB; h.cur_cap = e.capA; h.other_cap = e.capB;
    h.bits = bits0; h.num_entries = 0;
    int32_t qq = 0;
    if (DT != DT_F32 && MT == MT_L2) qq = sq_norm_int<DT>(reinterpret_cast<const uint4*>(qs), a.nchunks);

    uint64_t* fr = frA;
    uint64_t* fr2 = frB;
    int fn, cn;
    uint32_t cmps;
    uint64_t nvis;
    float u0 = 0.0f;
    bool u0_fresh = true;
    bool ok = true;
    if (rec_id != PANN_PAD) {
      const ResumeLayout ly = resume_layout(a.L, a.Ccap, a.logcap, a.viscap);
      const uint32_t* rec = a.rec_pool + (size_t)rec_id * a.rec_words;
      fn = (int)rec[1];
      cn = (int)rec[2];
      nvis = rec[3];
      cmps = rec[4];
      const uint32_t entries = rec[5];
      u0 = __uint_as_float(rec[6]);
      u0_fresh = false;
      const uint64_t* rfr = reinterpret_cast<const uint64_t*>(rec + ly.fr);
      const uint64_t* rcand = reinterpret_cast<const uint64_t*>(rec + ly.cand);
      for (int i = tid; i < fn; i += nth) fr[i] = rfr[i];
      for (int i = tid; i < cn; i += nth) cand[i] = rcand[i];
      // the logged ids, inserted in log order (staged in table B, unused until a growth)
      for (uint32_t i = tid; i < entries; i += nth) tabB[i] = rec[ly.log + i];
      __syncthreads();
      emu_place_ranked_block(tabB, entries, tabA, (1u << bits0) - 1, e.capB, tid, nth, ctrl + 20);
      h.num_entries = entries;
      for (uint32_t i = tid; i < (uint32_t)nvis; i += nth) vset_insert(vset, vmask, rec[ly.vis + i]);
    } else {
      for (uint32_t s = tid; s < a.n_start; s += nth) {
        const uint32_t id = a.starts[s];
        frB[s] = make_key(point_dist<DT, MT>(a.points + (uint64_t)id * a.stride, qs, a.d, a.nchunks, qq), id);
      }
      if (warp == 0) {
        bool sdummy;
        for (uint32_t s0 = 0; s0 < a.n_start && ok; s0 += 32)
          ok = emu_batch(h, s0 + lane < a.n_start ? a.starts[s0 + lane] : PANN_PAD, s0 + lane < a.n_start, lane,
                         &sdummy);
        if (lane == 0) ctrl[1] = ok;
      }
      __syncthreads();
      ok = ctrl[1] != 0;
      block_rank_sort(frB, fr, (int)a.n_start, tid, nth);
      fn = (int)a.n_start;
      cn = 0;
      cmps = a.n_start;
      nvis = 0;
    }
    __syncthreads();
    uint32_t status = QS_REF_WOULD_GROW;
    if (!ok) status |= QS_TABLE_FULL;

    while (ok) {
      // first and second unvisited frontier entries, the number unvisited (every warp alike)
      int first = -1, second = -1, cnt = 0;
      for (int b = 0; b < fn; b += 32) {
        const int i = b + lane;
        const bool unv = (i < fn) && !(fr[i] & PANN_VFLAG);
        unsigned m = __ballot_sync(FULL, unv);
        cnt += __popc(m);
        if (first < 0 && m) {
          first = b + __ffs(m) - 1;
          m &= m - 1;
        }
        if (first >= 0 && second < 0 && m) second = b + __ffs(m) - 1;
      }
      if (first < 0 || nvis >= a.limit) break;
      if (warp == 1 && second >= 0 && (uint32_t)lane * 32 < a.R)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a.graph + (uint64_t)key_id(fr[second]) * a.R + 32 * lane));
      if (u0_fresh) {
        u0 = key_dist(fr[first]);
        u0_fresh = false;
      }
      if (a.es_count > 0.0 && (double)nvis >= a.es_count && !((double)key_dist(fr[0]) <= a.es_radius) &&
          !((double)u0 <= a.es_esr))
        break;  // early_stopping (earlyStopping.h:19-29)
      const uint64_t cur_key = fr[first];
      const bool full = (fn == (int)L);
      const float cutoff = full ? key_dist(fr[fn - 1]) : 3.40282346638528859812e+38F;
      __syncthreads();  // every thread has read the frontier before it changes
      nvis++;
      if (tid == 0) {
        fr[first] = cur_key | PANN_VFLAG;
        if (a.vis_keys && nvis <= a.vis_cap) a.vis_keys[(uint64_t)qi * a.vis_cap + (nvis - 1)] = cur_key & PANN_KEYMASK;
        vset_insert(vset, vmask, key_id(cur_key));
      }
      if (nvis > a.vis_cap && a.vis_keys) status |= QS_VISIT_OVERFLOW;
      if (nvis > (uint64_t)(vmask / 4 * 3)) { status |= QS_INTERNAL; break; }
      const uint32_t cid = key_id(cur_key);
      const uint32_t* grow = a.graph + (uint64_t)cid * a.R;
      {
        // warp 0 makes the hashset calls in adjacency order (:153-159) while
        // warps 1..NW-1 score every neighbour; a call that grows the table
        // stops the calls, the whole block grows it (emu_grow_block), and
        // warp 0 goes on with the calls after it
        int nnew = 0;            // warp 0's state from here on
        bool full_tab = false;
        uint32_t b = 0, v = PANN_PAD;
        unsigned pend = 0;
        bool open = false, seen = false;
        int g = -1;
        bool first_round = true;
        for (;;) {
          if (warp == 0) {
            g = -1;
            while (!full_tab) {
              if (!open) {
                if (b >= nel) break;
                v = b + lane < nel ? __ldg(grow + b + lane) : PANN_PAD;
                pend = __ballot_sync(FULL, v != PANN_PAD);
                seen = false;
                open = true;
              }
              if (pend) {
                emu_batch_part(h, v, (pend >> lane) & 1u, lane, &seen, &g);
                if (g >= 0) {
                  pend &= ~((2u << g) - 1u);
                  break;
                }
                pend = 0;
              }
              const bool isnew = v != PANN_PAD && !seen && v != self;
              const unsigned mn = __ballot_sync(FULL, isnew);
              if (isnew) {
                const int at = nnew + __popc(mn & ((1u << lane) - 1));
                nbuf[at] = v;
                npos[at] = b + lane;
              }
              nnew += __popc(mn);
              b += 32;
              open = false;
            }
            const uint32_t gkey = __shfl_sync(FULL, v, g < 0 ? 0 : g);
            if (lane == 0) {
              ctrl[2] = (uint32_t)nnew;
              ctrl[3] = full_tab;
              ctrl[16] = g >= 0 && !full_tab ? gkey : PANN_PAD;
              ctrl[18] = h.cur == tabB;
              ctrl[19] = h.bits;
              ctrl[28] = h.other_cap;
            }
          } else if (first_round) {
            // every neighbour scored while warp 0 probes the table
            for (uint32_t j = tid - 32; j < nel; j += nth - 32) {
              const uint32_t u = __ldg(grow + j);
              if (u != PANN_PAD)
                dall[j] = row_dist_whole<DT, MT, CH>(a.points + (uint64_t)u * a.stride, qs, a.nchunks, qq);
            }
          }
          __syncthreads();
          first_round = false;
          const uint32_t gk = ctrl[16];
          if (gk == PANN_PAD) break;
          uint32_t* gcur = ctrl[18] ? tabB : tabA;
          uint32_t* goth = ctrl[18] ? tabA : tabB;
          uint32_t added = 0;
          bool aseen = false;
          const bool grew = emu_grow_block(gcur, goth, ctrl[19], ctrl[28], gk, tid, nth, ctrl + 20, &added, &aseen);
          if (warp == 0) {
            if (!grew) {
              full_tab = true;
            } else {
              h.num_entries += added;
              uint32_t* t = h.cur; h.cur = h.other; h.other = t;
              const uint32_t c = h.cur_cap; h.cur_cap = h.other_cap; h.other_cap = c;
              h.bits += 1;
              if (!aseen) h.num_entries++;
              if (lane == g) seen = aseen;
            }
          }
          __syncthreads();
        }
      }
      const int nnew = (int)ctrl[2];
      if (ctrl[3]) {
        status |= QS_TABLE_FULL;
        break;
      }
      cmps += (uint32_t)nnew;
      if ((uint32_t)(cn + nnew) > a.Ccap) { status |= QS_INTERNAL; break; }
      if (warp == 0) {
        for (int b = 0; b < nnew; b += 32) {
          const int i = b + lane;
          float dv = 0.0f;
          uint32_t v = 0;
          if (i < nnew) {
            v = nbuf[i];
            dv = dall[npos[i]];
          }
          const bool keep = i < nnew && !(dv >= cutoff);
          const unsigned m = __ballot_sync(FULL, keep);
          if (keep) cand[cn + __popc(m & ((1u << lane) - 1))] = make_key(dv, v);
          cn += __popc(m);
        }
        if (lane == 0) ctrl[4] = (uint32_t)cn;
      }
      __syncthreads();
      cn = (int)ctrl[4];
      if (cn == 0 || (a.limit >= 2ull * L && (double)cn < a.batch_factor * (double)L && cnt - 1 >= 1)) continue;
      block_rank_sort(cand, cand2, cn, tid, nth);
      __syncthreads();
      // unique by id, drop ids already in the frontier, mark ids visited before (order kept)
      int un = 0;
      for (int b = 0; b < cn; b += nth) {
        const int i = b + tid;
        bool keepc = false;
        uint64_t k = 0;
        if (i < cn) {
          k = cand2[i];
          keepc = !(i > 0 && key_id(cand2[i - 1]) == key_id(k)) && !frontier_has(fr, fn, k);
          if (keepc && vset_has(vset, vmask, key_id(k))) k |= PANN_VFLAG;
        }
        const unsigned mk = __ballot_sync(FULL, keepc);
        if (lane == 0) ctrl[8 + warp] = __popc(mk);
        __syncthreads();
        int before = 0, tot = 0;
        for (int w = 0; w < NW; w++) {
          const int c = (int)ctrl[8 + w];
          before += w < warp ? c : 0;
          tot += c;
        }
        if (keepc) cand[un + before + __popc(mk & ((1u << lane) - 1))] = k;
        un += tot;
        __syncthreads();
      }
      fn = block_merge(fr, fn, cand, un, fr2, (int)L, tid, nth);
      u0_fresh = true;
      uint64_t* t = fr; fr = fr2; fr2 = t;
      cn = 0;
      __syncthreads();
    }
    __syncthreads();

    if (status & QS_TABLE_FULL) {
      if (tid == 0) {
        if (e.overflow_list) {
          const uint32_t pos = atomicAdd(e.overflow_count, 1u);
          e.overflow_list[pos] = qi;
          e.overflow_rec[pos] = rec_id;
        }
        if (a.out_status) a.out_status[qi] = status;
      }
      continue;
    }
    if (status & QS_INTERNAL) {
      if (tid == 0 && a.out_status) a.out_status[qi] = status;
      continue;
    }
    if (warp == 0 && h.bits == bits0) status &= ~(uint32_t)QS_REF_WOULD_GROW;
    if ((uint32_t)fn < kq) status |= QS_SHORT;
    for (uint32_t j = tid; j < a.kstride; j += nth) {
      const bool okk = j < (uint32_t)fn && j < kq;
      a.out_ids[(uint64_t)qi * a.kstride + j] = okk ? key_id(fr[j]) : PANN_PAD;
      if (a.out_dists) a.out_dists[(uint64_t)qi * a.kstride + j] = okk ? key_dist(fr[j]) : 0.0f;
    }
    if (tid == 0) {
      if (a.out_visited) a.out_visited[qi] = (uint32_t)nvis;
      if (a.out_cmps) a.out_cmps[qi] = cmps;
      if (a.out_status) a.out_status[qi] = status;
    }
  }
}

}  // namespace pann
