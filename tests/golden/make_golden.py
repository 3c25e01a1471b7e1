"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own code.

The reference (ParlayANN) ships no golden vectors or known-answer tests, so
these fixtures are outputs of its beam search, robustPrune and Vamana build,
compiled in place from the checkout by oracle/Makefile (oracle/_ref). Inputs
are small seeded arrays, stored in the fixture next to the outputs.

    python tests/golden/make_golden.py      (needs oracle/_ref/libpann_ref.so)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402


def pts(dtype, n, d, seed):
    rng = np.random.default_rng(seed)
    if dtype == np.float32:
        return rng.standard_normal((n, d)).astype(np.float32)
    if dtype == np.uint8:
        return rng.integers(0, 256, (n, d)).astype(np.uint8)
    return rng.integers(-128, 128, (n, d)).astype(np.int8)


def main():
    assert O.have_ref(), "build oracle/_ref first (make -C oracle)"
    cases = []
    # search on seeded random graphs: every dtype x metric, with deferral, limit and degree_limit variants
    for ci, (dtype, metric) in enumerate([(np.uint8, 0), (np.uint8, 1), (np.int8, 0), (np.int8, 1),
                                          (np.float32, 0), (np.float32, 1)]):
        base = pts(dtype, 600, 24, 100 + ci)
        q = pts(dtype, 24, 24, 200 + ci)
        g = O.random_graph(600, 10, 300 + ci)
        for vi, (k, L, lim, dl, bf, starts) in enumerate([(10, 20, None, None, 0.125, (0,)),
                                                           (5, 12, 20, None, 0.125, (0, 7, 9)),
                                                           (8, 40, None, 6, 1.0, (3,)),
                                                           (1, 8, 5, None, 0.5, (0,))]):
            r = O.search("ref", base, q, g, k, L, limit=lim, degree_limit=dl, batch_factor=bf, starts=starts,
                         metric=metric, full=True, visited_cap=256)
            name = f"search_{np.dtype(dtype).name}_{'l2' if metric == 0 else 'mips'}_{vi}"
            np.savez_compressed(os.path.join(HERE, name + ".npz"), base=base, queries=q, graph=g, k=k, L=L,
                                limit=-1 if lim is None else lim, degree_limit=-1 if dl is None else dl,
                                batch_factor=bf, starts=np.asarray(starts, np.uint32), metric=metric,
                                **{x: r[x] for x in ["ids", "dists", "visited", "cmps", "frontier_n", "frontier_ids",
                                                     "frontier_d", "visited_ids", "visited_d"]})
            cases.append(name)
    # robustPrune known answers
    base = pts(np.uint8, 300, 16, 7)
    g = O.random_graph(300, 8, 8)
    rng = np.random.default_rng(9)
    for t in range(4):
        p = int(rng.integers(0, 300))
        cand = rng.choice(300, size=40, replace=False).astype(np.uint32)
        cd = np.array([O.olib().oracle_distance(0, 0, 16, base[c].ctypes.data, base[p].ctypes.data) for c in cand],
                      np.float32)
        alpha = [1.0, 1.2, 1.5, 2.0][t]
        nb, cm = O.robust_prune("ref", base, g, p, cand, cd, alpha, add=bool(t % 2 == 0))
        np.savez_compressed(os.path.join(HERE, f"prune_u8_{t}.npz"), base=base, graph=g, p=p, cand_ids=cand,
                            cand_d=cd, alpha=alpha, add=int(t % 2 == 0), out=nb, cmps=cm)
        cases.append(f"prune_u8_{t}")
    # Vamana build (two passes, R=10, L=20, alpha 1.2)
    for dtype, metric, nm in [(np.uint8, 0, "u8_l2"), (np.float32, 0, "f32_l2"), (np.float32, 1, "f32_mips")]:
        base = pts(dtype, 800, 12, 11)
        gr, tot = O.build_graph("ref", base, 10, 20, 1.2, 2, metric=metric)
        np.savez_compressed(os.path.join(HERE, f"build_{nm}.npz"), base=base, R=10, L=20, alpha=1.2, passes=2,
                            metric=metric, graph=gr, dist_total=tot, perm=O.permutation(800))
        cases.append(f"build_{nm}")
    # range search (RangeSearch / DoubleBeamRangeSearch): greedy expansions
    # large enough for the seen-set to grow, early stopping, all three types
    for ci, (dtype, metric, quant) in enumerate([(np.uint8, 0, 0.2), (np.float32, 0, 0.3), (np.float32, 1, 0.1)]):
        base = pts(dtype, 3000, 8, 500 + ci)
        q = pts(dtype, 16, 8, 600 + ci)
        g = O.random_graph(3000, 24, 700 + ci)
        rng = np.random.default_rng(800 + ci)
        for i in range(0, 3000, 5):                     # repeated ids inside some rows
            deg = g[i, 0]
            g[i, 1 + rng.integers(0, deg, 3)] = g[i, 1 + rng.integers(0, deg, 3)]
        samp = [O.olib().oracle_distance(O._DT[base.dtype], metric, 8, q[i].ctypes.data, base[j].ctypes.data)
                for i in range(4) for j in range(0, 3000, 7)]
        radius = float(np.quantile(samp, quant))
        runs = [(1, 10, 0, 0.0), (1, 24, 10, 2 * radius), (2, 12, 0, 0.0), (3, 16, 6, radius)]
        out = dict(base=base, queries=q, graph=g, radius=radius, metric=metric,
                   runs=np.array([(t, b, c, e) for t, b, c, e in runs], np.float64))
        for j, (rtype, beam, esc, esr) in enumerate(runs):
            r = O.range_search("ref", base, q, g, beam, radius, rtype, esr=esr, esc=esc, metric=metric)
            out[f"counts{j}"] = np.array([len(x) for x in r["ids"]], np.int64)
            out[f"ids{j}"] = np.concatenate(r["ids"]).astype(np.uint32)
            out[f"visited{j}"] = r["visited"]
            out[f"cmps{j}"] = r["cmps"]
        name = f"range_{np.dtype(dtype).name}_{'l2' if metric == 0 else 'mips'}"
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        cases.append(name)
    cases += range_groundtruth_fixtures()
    cases += quantized_fixtures()
    print("\n".join(cases))


def range_groundtruth_fixtures():
    """compute_range_groundtruth (data_tools/compute_range_groundtruth.cpp:14-30), the tool's own code:
    every base id within the radius, in id order."""
    cases = []
    for ci, (dtype, metric, quant) in enumerate([(np.uint8, 0, 0.02), (np.int8, 1, 0.01), (np.float32, 0, 0.03),
                                                 (np.float32, 1, 0.02)]):
        base = pts(dtype, 2000, 11, 900 + ci)
        q = pts(dtype, 12, 11, 950 + ci)
        samp = [O.olib().oracle_distance(O._DT[base.dtype], metric, 11, q[i].ctypes.data, base[j].ctypes.data)
                for i in range(4) for j in range(0, 2000, 7)]
        radius = np.float32(np.quantile(samp, quant))
        offs, ids = O.range_groundtruth("ref", base, q, float(radius), metric=metric)
        name = f"rangegt_{np.dtype(dtype).name}_{'l2' if metric == 0 else 'mips'}"
        np.savez_compressed(os.path.join(HERE, name + ".npz"), base=base, queries=q, radius=radius, metric=metric,
                            offsets=offs, ids=ids)
        cases.append(name)
    return cases


def quantized_fixtures():
    """beam_search_rerank over one-byte scalar-quantized float points (beamSearch.h:529-597,
    euclidian_point.h:186-240), as GraphIndex::search_dispatch calls it."""
    cases = []
    for ci, (n, d, R, L, k, rf) in enumerate([(1200, 16, 12, 30, 10, 100.0), (1000, 12, 10, 20, 5, 2.0)]):
        base = pts(np.float32, n, d, 1000 + ci)
        q = pts(np.float32, 30, d, 1100 + ci)
        g = O.random_graph(n, R, 1200 + ci)
        r = O.search_quantized("ref", base, q, g, k, L, rerank_factor=rf)
        name = f"quant_f32_{ci}"
        np.savez_compressed(os.path.join(HERE, name + ".npz"), base=base, queries=q, graph=g, k=k, L=L,
                            rerank_factor=rf, ids=r["ids"], dists=r["dists"], visited=r["visited"], cmps=r["cmps"],
                            slope=np.float32(r["slope"]), offset=np.int32(r["offset"]))
        cases.append(name)
    return cases


if __name__ == "__main__":
    main()
