"""CPU checks of the placement rules the exact-emulation kernels rely on.

The emulation tier (parlayann_b200/csrc/search_emu.cuh) reproduces the
reference's seen-set (algorithms/utils/hashset.h:13-55: slot
(k * 0xbf58476d1ce4e5b9) & mask, linear probing, growth re-inserting every key
in old-slot order) with parallel algorithms whose results must equal the
reference's one-at-a-time insertion. These tests restate those algorithms in
Python, step for step as the kernels run them, and compare them with
sequential insertion on random tables:

* emu_probe_rounds: up to 32 keys in call order, inserted in rounds;
* emu_place_ranked_block: placement of ranked keys into an empty table
  (compare-and-swap rank placement, owners from one pass over the slots,
  clusters of up to 8 keys replayed per thread, longer ones by the
  slot-by-slot minimum rule).

They need no GPU; the GPU parity tests check the kernels themselves.
"""
import random

import pytest

PAD = 0xFFFFFFFF


def ref_slot(k, mask):
    """hashset.h:17-20 restated: the product's low bits depend only on the
    multiplier's low 32 bits (the kernels' ref_slot)."""
    return ((k * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF) & mask


def seq_insert(tab, mask, key, start=None):
    """hashset::operator() (hashset.h:39-47): probe to the key or the first
    empty slot; insert there. Returns (inserted, slot)."""
    p = ref_slot(key, mask) if start is None else start
    while tab[p] != PAD and tab[p] != key:
        p = (p + 1) & mask
    if tab[p] == key:
        return False, p
    tab[p] = key
    return True, p


def probe_rounds(tab, mask, keys, active):
    """emu_probe_rounds as the warp runs it: lanes in call order."""
    n = len(keys)
    pos = [ref_slot(k, mask) for k in keys]
    done = [not a for a in active]
    ins = [False] * n
    while True:
        for i in range(n):
            if not done[i]:
                p = pos[i]
                while tab[p] != PAD and tab[p] != keys[i]:
                    p = (p + 1) & mask
                pos[i] = p
                if tab[p] == keys[i]:
                    done[i] = True
        want = [i for i in range(n) if not done[i]]
        if not want:
            break
        lowest = {}
        for i in want:  # the lowest unfinished lane of each slot
            lowest.setdefault(pos[i], i)
        is_lowest = {i for i in lowest.values()}
        losers = [i for i in want if i not in is_lowest]
        bound = min(losers) if losers else n
        won = [i for i in want if i in is_lowest and i < bound]
        for i in won:
            tab[pos[i]] = keys[i]
            ins[i] = True
            done[i] = True
        if len(won) == len(want):
            break
    return ins


def place_ranked(keys, nmask, order):
    """emu_place_ranked_block: returns the table the kernel writes for keys
    placed in rank order (rank = index in keys); `order` is the order in which
    threads happen to claim slots in phase A."""
    nsize = nmask + 1
    slot_rank = [PAD] * nsize
    for r in order:  # (A) compare-and-swap placement; a repeated key keeps its smaller rank
        k = keys[r]
        p = ref_slot(k, nmask)
        while True:
            w = slot_rank[p]
            if w == PAD:
                slot_rank[p] = r
                break
            if keys[w] == k:
                slot_rank[p] = min(w, r)
                break
            p = (p + 1) & nmask
    out = [PAD] * nsize
    owners = [slot_rank[p] for p in range(nsize) if slot_rank[p] != PAD and slot_rank[(p - 1) & nmask] == PAD]
    for r in owners:
        s0 = ref_slot(keys[r], nmask)  # an owner sits at its home
        m = 1
        while slot_rank[(s0 + m) & nmask] != PAD:
            m += 1
        ranks = [slot_rank[(s0 + j) & nmask] for j in range(m)]
        offs = {rk: (ref_slot(keys[rk], nmask) - s0) & nmask for rk in ranks}
        if m <= 8:
            # (B) short cluster: ranks in order, each at the first free offset from its home
            taken = set()
            for rk in sorted(ranks):
                o = offs[rk]
                while o in taken:
                    o += 1
                taken.add(o)
                out[(s0 + o) & nmask] = keys[rk]
        else:
            # long cluster: each slot, left to right, takes the smallest rank not
            # yet placed whose home is at or before it
            left = set(ranks)
            for j in range(m):
                rk = min(x for x in left if offs[x] <= j)
                left.remove(rk)
                out[(s0 + j) & nmask] = keys[rk]
    return out


def test_probe_rounds_equal_sequential_calls():
    rng = random.Random(7)
    for trial in range(400):
        bits = rng.randint(5, 10)
        mask = (1 << bits) - 1
        tab = [PAD] * (mask + 1)
        for k in rng.sample(range(1 << 20), rng.randint(0, (mask + 1) // 3)):
            seq_insert(tab, mask, k)
        # call order with repeats and keys already present
        pool = [k for k in tab if k != PAD][:8] + [rng.randrange(1 << 20) for _ in range(40)]
        n = rng.randint(1, 32)
        keys = [rng.choice(pool) for _ in range(n)]
        active = [rng.random() < 0.9 for _ in range(n)]
        ref = list(tab)
        want = [seq_insert(ref, mask, k)[0] if a else False for k, a in zip(keys, active)]
        got_tab = list(tab)
        got = probe_rounds(got_tab, mask, keys, active)
        assert got == want, trial
        assert got_tab == ref, trial


@pytest.mark.parametrize("cluster_heavy", [False, True])
def test_ranked_placement_equals_rank_order_insertion(cluster_heavy):
    rng = random.Random(11 + cluster_heavy)
    long_seen = 0
    for trial in range(300):
        bits = rng.randint(4, 11)
        nmask = (1 << bits) - 1
        cnt = rng.randint(1, (nmask + 1) // 2)
        if cluster_heavy:
            # keys sharing few homes make long clusters (the long-cluster rule)
            homes = {}
            keys = []
            cand = 0
            nh = max(1, cnt // 24)
            while len(keys) < cnt:
                cand += 1
                h = ref_slot(cand, nmask)
                if h in homes or len(homes) < nh:
                    homes[h] = True
                    keys.append(cand)
        else:
            keys = [rng.randrange(1 << 24) for _ in range(cnt)]
        for _ in range(rng.randint(0, 4)):  # repeated keys: the smaller rank counts
            keys.insert(rng.randrange(len(keys) + 1), rng.choice(keys))
        ref = [PAD] * (nmask + 1)
        for k in keys:
            seq_insert(ref, nmask, k)
        if sum(1 for x in ref if x != PAD) > (nmask + 1) // 2 + 4:
            continue
        order = list(range(len(keys)))
        rng.shuffle(order)
        got = place_ranked(keys, nmask, order)
        assert got == ref, trial
        run = best = 0
        for x in ref + ref:
            run = run + 1 if x != PAD else 0
            best = max(best, run)
        long_seen += best > 8
    if cluster_heavy:
        assert long_seen > 50  # the long-cluster rule was exercised
