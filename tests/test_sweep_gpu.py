"""Seeded random parameter sweeps of the CUDA search (through the C ABI)
against the oracle, in the same parameter space as the oracle's own sweeps
against the in-place reference (tests/test_oracle_pin.py): every dtype and
metric, beams 1-79, k, visit and degree limits, batch factors up to 1,
several start points, rows with repeated neighbours, small and odd
dimensions and degrees. Bar: bit-exact ids, distances, visited counts and
distance-comparison counts.

Opt-in (PANN_GPU_SWEEP=1) until the sweep has run on a B200; the fixed-case
parity tests in test_search_gpu.py and test_range_gpu.py run by default.
"""
import os

import numpy as np
import pytest

import parlayann_b200 as P
from conftest import random_points
from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("PANN_GPU_SWEEP") != "1", reason="opt-in: PANN_GPU_SWEEP=1")]


def _search_cases(count, seed):
    rng = np.random.default_rng(seed)
    dts = [np.uint8, np.int8, np.float32]
    for case in range(count):
        dtype = dts[case % 3]
        metric = [P.L2, P.MIPS][(case // 3) % 2]
        n = int(rng.integers(200, 900))
        d = int(rng.integers(3, 40))
        R = int(rng.integers(4, 33))
        L = int(rng.integers(1, 80))
        k = int(rng.integers(1, L + 1))
        lim = None if rng.random() < 0.6 else int(rng.integers(1, 3 * L + 2))
        dl = None if rng.random() < 0.6 else int(rng.integers(1, R + 1))
        bf = float(rng.choice([0.0, 0.125, 0.5, 1.0]))
        ns = int(rng.integers(1, min(L, 4) + 1))
        yield case, dtype, metric, n, d, R, L, k, lim, dl, bf, ns


def test_search_random_sweep_matches_oracle(lib_built):
    for case, dtype, metric, n, d, R, L, k, lim, dl, bf, ns in _search_cases(36, 4242):
        base = random_points(dtype, n, d, 100 + case)
        q = random_points(dtype, 16, d, 200 + case)
        g = O.random_graph(n, R, 300 + case)
        if case % 4 == 0:  # a repeated neighbour in some rows
            for i in range(0, n, 7):
                if g[i, 0] >= 2:
                    g[i, 2] = g[i, 1]
        st = tuple(int(x) for x in np.random.default_rng(400 + case).choice(n, size=ns, replace=False))
        idx = P.Index(base, R, metric)
        idx.set_graph(g)
        # a small visit limit on a sparse graph can leave fewer than k results:
        # both sides then pad with 0xFFFFFFFF and 0.0
        r = idx.search(q, k, L, limit=lim, degree_limit=dl, batch_factor=bf, starts=st, allow_short=True)
        o = O.search("oracle", base, q, g, k, L, limit=lim, degree_limit=dl, batch_factor=bf, starts=st,
                     metric=metric)
        msg = f"case {case}: {np.dtype(dtype).name} metric {metric} n {n} d {d} R {R} L {L} k {k} " \
              f"limit {lim} dl {dl} bf {bf} starts {st}"
        np.testing.assert_array_equal(r.ids, o["ids"], err_msg=msg)
        np.testing.assert_array_equal(r.dists.view(np.uint32), o["dists"].view(np.uint32), err_msg=msg)
        np.testing.assert_array_equal(r.visited, o["visited"], err_msg=msg)
        np.testing.assert_array_equal(r.cmps, o["cmps"], err_msg=msg)
        idx.close()


def test_range_random_sweep_matches_oracle(lib_built):
    rng = np.random.default_rng(7777)
    dts = [np.uint8, np.int8, np.float32]
    for case in range(24):
        dtype = dts[case % 3]
        metric = [P.L2, P.MIPS][(case // 3) % 2]
        n = int(rng.integers(300, 1500))
        d = int(rng.integers(3, 24))
        R = int(rng.integers(4, 25))
        base = random_points(dtype, n, d, 500 + case)
        q = random_points(dtype, 6, d, 600 + case)
        g = O.random_graph(n, R, 700 + case)
        quant = float(rng.choice([0.002, 0.01, 0.05, 0.2]))
        beam = int(rng.integers(1, 41))
        rtype = int(rng.choice([O.RANGE_GREEDY, O.RANGE_DOUBLING, O.RANGE_BEAM]))
        start = int(rng.integers(0, n))
        esc = 0 if rng.random() < 0.5 else int(rng.integers(1, 30))
        esr_f = float(rng.choice([0.0, 1.0, 1.5, 3.0]))
        dt = O._DT[base.dtype]
        samp = [O.olib().oracle_distance(dt, metric, d, np.ascontiguousarray(q[i]).ctypes.data,
                                         np.ascontiguousarray(base[j]).ctypes.data)
                for i in range(len(q)) for j in range(0, n, 7)]
        radius = float(np.quantile(samp, quant))
        o = O.range_search("oracle", base, q, g, beam, radius, rtype, start=start, esr=esr_f * radius, esc=esc,
                           metric=metric)
        idx = P.Index(base, R, metric)
        idx.set_graph(g)
        r = idx.range_search(q, beam, radius, rtype, start=start, early_stopping_radius=esr_f * radius,
                             early_stopping_count=esc)
        msg = f"case {case}: beam {beam} type {rtype} quant {quant} esc {esc} esr {esr_f}"
        for x, y in zip(r["ids"], o["ids"]):
            np.testing.assert_array_equal(x, y, err_msg=msg)
        np.testing.assert_array_equal(r["visited"], o["visited"], err_msg=msg)
        np.testing.assert_array_equal(r["cmps"], o["cmps"], err_msg=msg)
        idx.close()


def test_build_random_sweep_matches_oracle(lib_built):
    """Seeded random Vamana builds (every dtype and metric, R 3-24, L from R to
    80, alpha 1.0-1.5, one or two passes, search batch factors up to 1): the
    GPU graph equals the oracle's (the oracle is pinned to the reference's
    build by the same sweep in tests/test_oracle_pin.py)."""
    rng = np.random.default_rng(91)
    dts = [np.uint8, np.int8, np.float32]
    for case in range(12):
        dtype = dts[case % 3]
        metric = [P.L2, P.MIPS][(case // 3) % 2]
        n = int(rng.integers(200, 1500))
        d = int(rng.integers(2, 24))
        R = int(rng.integers(3, 25))
        L = int(rng.integers(R, 81))
        alpha = float(rng.choice([1.0, 1.1, 1.2, 1.5]))
        passes = int(rng.integers(1, 3))
        bf = float(rng.choice([0.125, 0.5, 1.0]))
        base = random_points(dtype, n, d, 800 + case)
        idx = P.Index(base, R, metric)
        st = idx.build(L, alpha, num_passes=passes, batch_factor=bf)
        o, tot = O.build_graph("oracle", base, R, L, alpha, passes, batch_factor=bf, metric=metric)
        g = idx.get_graph()
        assert [tuple(r[1:1 + r[0]].tolist()) for r in g] == [tuple(r[1:1 + r[0]].tolist()) for r in o], case
        assert st.dist_cmps == tot, case
        idx.close()
