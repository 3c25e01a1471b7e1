"""Pin the C oracle (oracle/pann_oracle.c) to the reference.

1. Against the golden fixtures in tests/golden/, which are outputs of the
   reference's own beam search / robustPrune / Vamana build compiled in place
   (tests/golden/make_golden.py).
2. Where the in-place reference library is present (oracle/_ref), against it
   directly on further seeded cases.
CPU only.
"""
import glob
import os

import numpy as np
import pytest

from conftest import random_points
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _opt(v):
    v = int(v)
    return None if v < 0 else v


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "search_*.npz"))), ids=os.path.basename)
def test_oracle_search_matches_golden(path, lib_built):
    z = np.load(path)
    r = O.search("oracle", z["base"], z["queries"], z["graph"], int(z["k"]), int(z["L"]), limit=_opt(z["limit"]),
                 degree_limit=_opt(z["degree_limit"]), batch_factor=float(z["batch_factor"]),
                 starts=z["starts"].tolist(), metric=int(z["metric"]), full=True, visited_cap=256)
    for key in ["ids", "dists", "visited", "cmps", "frontier_n", "frontier_ids", "frontier_d", "visited_ids",
                "visited_d"]:
        np.testing.assert_array_equal(r[key], z[key], err_msg=key)
    assert r["hash_grew"].sum() == 0


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "prune_*.npz"))), ids=os.path.basename)
def test_oracle_prune_matches_golden(path, lib_built):
    z = np.load(path)
    nb, cm = O.robust_prune("oracle", z["base"], z["graph"], int(z["p"]), z["cand_ids"], z["cand_d"],
                            float(z["alpha"]), add=bool(int(z["add"])))
    np.testing.assert_array_equal(nb, z["out"])
    assert cm == int(z["cmps"])


def _live_rows(g):
    return [tuple(r[1:1 + r[0]].tolist()) for r in g]


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "build_*.npz"))), ids=os.path.basename)
def test_oracle_build_matches_golden(path, lib_built):
    z = np.load(path)
    g, tot = O.build_graph("oracle", z["base"], int(z["R"]), int(z["L"]), float(z["alpha"]), int(z["passes"]),
                           metric=int(z["metric"]), perm=z["perm"])
    assert tot == int(z["dist_total"])
    # neighbour order after the final sort may differ only inside groups of equal distance
    ga, gb = _live_rows(g), _live_rows(z["graph"])
    for a, b in zip(ga, gb):
        assert sorted(a) == sorted(b)
    same_order = sum(a == b for a, b in zip(ga, gb))
    assert same_order >= 0.95 * len(ga)


def test_golden_permutation_is_the_shim_order(lib_built):
    z = np.load(os.path.join(GOLD, "build_u8_l2.npz"))
    np.testing.assert_array_equal(O.permutation(len(z["perm"])), z["perm"])


needs_ref = pytest.mark.skipif(not O.have_ref(), reason="in-place reference library not built here")


@needs_ref
@pytest.mark.parametrize("dtype", [np.uint8, np.int8, np.float32])
@pytest.mark.parametrize("metric", [0, 1])
def test_oracle_search_matches_reference(dtype, metric, lib_built):
    base = random_points(dtype, 1500, 20, 5)
    q = random_points(dtype, 40, 20, 6)
    g = O.random_graph(1500, 14, 7)
    for k, L, lim, dl, bf, st in [(10, 30, None, None, 0.125, (0,)), (10, 10, None, None, 0.125, (1,)),
                                  (4, 16, 12, 5, 0.25, (0, 2)), (2, 64, None, None, 0.125, (5,)),
                                  (3, 6, 2, None, 0.125, (0,))]:
        a = O.search("oracle", base, q, g, k, L, limit=lim, degree_limit=dl, batch_factor=bf, starts=st,
                     metric=metric, full=True)
        b = O.search("ref", base, q, g, k, L, limit=lim, degree_limit=dl, batch_factor=bf, starts=st, metric=metric,
                     full=True)
        for key in ["ids", "dists", "visited", "cmps", "frontier_n", "frontier_ids", "frontier_d", "visited_ids",
                    "visited_d"]:
            np.testing.assert_array_equal(a[key], b[key], err_msg=f"{key} k={k} L={L}")


@needs_ref
def test_oracle_search_matches_reference_random_sweep(lib_built):
    """Seeded random QueryParams over every dtype and metric on small random
    graphs (repeated neighbours included, as the reference's graph allows):
    the restatement and the in-place reference agree on everything they
    return."""
    rng = np.random.default_rng(2024)
    dts = [np.uint8, np.int8, np.float32]
    for case in range(36):
        dtype = dts[case % 3]
        metric = (case // 3) % 2
        n = int(rng.integers(200, 900))
        d = int(rng.integers(3, 40))
        R = int(rng.integers(4, 33))
        base = random_points(dtype, n, d, 100 + case)
        q = random_points(dtype, 8, d, 200 + case)
        g = O.random_graph(n, R, 300 + case)
        if case % 4 == 0:  # a repeated neighbour in some rows
            for i in range(0, n, 7):
                if g[i, 0] >= 2:
                    g[i, 2] = g[i, 1]
        L = int(rng.integers(1, 80))
        k = int(rng.integers(1, L + 1))
        lim = None if rng.random() < 0.6 else int(rng.integers(1, 3 * L + 2))
        dl = None if rng.random() < 0.6 else int(rng.integers(1, R + 1))
        # batch_factor <= 1: above it the reference's set_union can write past
        # new_frontier (sized 2·max(L, starts) + max degree, beamSearch.h:95-96)
        bf = float(rng.choice([0.0, 0.125, 0.5, 1.0]))
        ns = int(rng.integers(1, min(L, 4) + 1))
        st = tuple(int(x) for x in rng.choice(n, size=ns, replace=False))
        args = dict(limit=lim, degree_limit=dl, batch_factor=bf, starts=st, metric=metric, full=True)
        a = O.search("oracle", base, q, g, k, L, **args)
        b = O.search("ref", base, q, g, k, L, **args)
        for key in ["ids", "dists", "visited", "cmps", "frontier_n", "frontier_ids", "frontier_d", "visited_ids",
                    "visited_d"]:
            np.testing.assert_array_equal(a[key], b[key], err_msg=f"case {case} {key}")


@needs_ref
def test_oracle_hashset_growth_regime(lib_built):
    """A tiny beam with a dense graph pushes the reference's seen-set past its
    growth threshold; the restatement reproduces the reference's results there
    too (its hashset growth, hashset.h:25-38, is restated as written)."""
    base = random_points(np.uint8, 20000, 8, 1)
    q = random_points(np.uint8, 20, 8, 2)
    g = O.random_graph(20000, 64, 3, min_deg=60)
    a = O.search("oracle", base, q, g, 10, 40, degree_limit=64, batch_factor=1.0, full=True)
    b = O.search("ref", base, q, g, 10, 40, degree_limit=64, batch_factor=1.0, full=True)
    for key in ["ids", "dists", "visited", "cmps"]:
        np.testing.assert_array_equal(a[key], b[key])
    assert a["hash_grew"].sum() > 0


@needs_ref
@pytest.mark.parametrize("dtype,metric", [(np.uint8, 0), (np.int8, 1), (np.float32, 0)])
def test_oracle_build_matches_reference(dtype, metric, lib_built):
    base = random_points(dtype, 1200, 16, 9)
    ga, ta = O.build_graph("oracle", base, 12, 24, 1.2, 2, metric=metric)
    gb, tb = O.build_graph("ref", base, 12, 24, 1.2, 2, metric=metric)
    assert ta == tb
    for a, b in zip(_live_rows(ga), _live_rows(gb)):
        assert sorted(a) == sorted(b)


@needs_ref
def test_oracle_build_matches_reference_random_sweep(lib_built):
    """Seeded random Vamana builds (every dtype and metric, R 3-24, L from R
    to 80, alpha 1.0-1.5, one or two passes, search batch factors up to 1):
    the restatement and the in-place reference give the same neighbour set
    per vertex and the same distance-comparison total."""
    rng = np.random.default_rng(91)
    dts = [np.uint8, np.int8, np.float32]
    for case in range(12):
        dtype = dts[case % 3]
        metric = (case // 3) % 2
        n = int(rng.integers(200, 1500))
        d = int(rng.integers(2, 24))
        R = int(rng.integers(3, 25))
        L = int(rng.integers(R, 81))
        alpha = float(rng.choice([1.0, 1.1, 1.2, 1.5]))
        passes = int(rng.integers(1, 3))
        bf = float(rng.choice([0.125, 0.5, 1.0]))
        base = random_points(dtype, n, d, 800 + case)
        ga, ta = O.build_graph("oracle", base, R, L, alpha, passes, batch_factor=bf, metric=metric)
        gb, tb = O.build_graph("ref", base, R, L, alpha, passes, batch_factor=bf, metric=metric)
        assert ta == tb, case
        for a, b in zip(_live_rows(ga), _live_rows(gb)):
            assert sorted(a) == sorted(b), case


@needs_ref
def test_oracle_prune_matches_reference(lib_built):
    base = random_points(np.float32, 400, 12, 3)
    g = O.random_graph(400, 9, 4)
    rng = np.random.default_rng(5)
    for t in range(10):
        p = int(rng.integers(0, 400))
        cand = rng.choice(400, size=int(rng.integers(1, 60)), replace=False).astype(np.uint32)
        cd = np.array([O.olib().oracle_distance(2, 0, 12, base[c].ctypes.data, base[p].ctypes.data) for c in cand],
                      np.float32)
        for alpha in (1.0, 1.2):
            for add in (True, False):
                a = O.robust_prune("oracle", base, g, p, cand, cd, alpha, add)
                b = O.robust_prune("ref", base, g, p, cand, cd, alpha, add)
                np.testing.assert_array_equal(a[0], b[0])
                assert a[1] == b[1]


@needs_ref
def test_oracle_prune_matches_reference_random_sweep(lib_built):
    """Seeded random robustPrune calls (every dtype and metric, R 2-32, up to
    120 candidates with repeated ids and the point itself among them in a
    third of the cases, alpha 1.0-2.0, with and without the point's current
    neighbours): same neighbours in the same order, same comparison count."""
    rng = np.random.default_rng(31)
    dts = [np.uint8, np.int8, np.float32]
    for case in range(60):
        dtype = dts[case % 3]
        metric = (case // 3) % 2
        n = int(rng.integers(50, 600))
        d = int(rng.integers(2, 30))
        R = int(rng.integers(2, 33))
        base = random_points(dtype, n, d, 1000 + case)
        g = O.random_graph(n, R, 1100 + case)
        p = int(rng.integers(0, n))
        m = int(rng.integers(1, min(n, 120)))
        cand = rng.choice(n, size=m, replace=False).astype(np.uint32)
        if case % 3 == 0:
            cand = np.concatenate([cand, cand[: m // 3], [p]]).astype(np.uint32)
        dt = O._DT[base.dtype]
        cd = np.array([O.olib().oracle_distance(dt, metric, d, base[c].ctypes.data, base[p].ctypes.data)
                       for c in cand], np.float32)
        alpha = float(rng.choice([1.0, 1.1, 1.2, 1.5, 2.0]))
        add = bool(rng.random() < 0.5)
        a = O.robust_prune("oracle", base, g, p, cand, cd, alpha, add, metric=metric)
        b = O.robust_prune("ref", base, g, p, cand, cd, alpha, add, metric=metric)
        np.testing.assert_array_equal(a[0], b[0], err_msg=f"case {case}")
        assert a[1] == b[1], case


def sample_radius(base, q, metric, quant):
    d = q.shape[1]
    dt = O._DT[base.dtype]
    samp = [O.olib().oracle_distance(dt, metric, d, np.ascontiguousarray(q[i]).ctypes.data,
                                     np.ascontiguousarray(base[j]).ctypes.data)
            for i in range(min(4, len(q))) for j in range(0, len(base), 7)]
    return float(np.quantile(samp, quant))


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "range_*.npz"))), ids=os.path.basename)
def test_oracle_range_search_matches_golden(path, lib_built):
    """RangeSearch / DoubleBeamRangeSearch (rangeSearch.h:183-276,
    doublingSearch.h:50-157): answers in the reference's order (duplicates the
    reference's growing hashset lets through included), visited and
    comparison counts."""
    z = np.load(path)
    for j, (rtype, beam, esc, esr) in enumerate(z["runs"]):
        r = O.range_search("oracle", z["base"], z["queries"], z["graph"], int(beam), float(z["radius"]), int(rtype),
                           esr=float(esr), esc=int(esc), metric=int(z["metric"]))
        np.testing.assert_array_equal([len(x) for x in r["ids"]], z[f"counts{j}"], err_msg=f"counts run {j}")
        np.testing.assert_array_equal(np.concatenate(r["ids"]), z[f"ids{j}"], err_msg=f"ids run {j}")
        np.testing.assert_array_equal(r["visited"], z[f"visited{j}"], err_msg=f"visited run {j}")
        np.testing.assert_array_equal(r["cmps"], z[f"cmps{j}"], err_msg=f"cmps run {j}")


@needs_ref
@pytest.mark.parametrize("dtype,metric", [(np.uint8, 0), (np.int8, 1), (np.float32, 0), (np.float32, 1)])
def test_oracle_range_search_matches_reference(dtype, metric, lib_built):
    base = random_points(dtype, 5000, 8, 61)
    q = random_points(dtype, 24, 8, 62)
    g = O.random_graph(5000, 20, 63)
    grew = 0
    for quant in (0.01, 0.15):
        radius = sample_radius(base, q, metric, quant)
        for rtype in (O.RANGE_GREEDY, O.RANGE_DOUBLING, O.RANGE_BEAM):
            for beam, esc, esr in [(10, 0, 0.0), (20, 10, 1.5 * radius)]:
                a = O.range_search("oracle", base, q, g, beam, radius, rtype, esr=esr, esc=esc, metric=metric)
                b = O.range_search("ref", base, q, g, beam, radius, rtype, esr=esr, esc=esc, metric=metric)
                for x, y in zip(a["ids"], b["ids"]):
                    np.testing.assert_array_equal(x, y)
                np.testing.assert_array_equal(a["visited"], b["visited"])
                np.testing.assert_array_equal(a["cmps"], b["cmps"])
                grew += int(a["hash_grew"].sum())
    assert grew > 0   # the greedy expansion's seen-set grew somewhere


@needs_ref
def test_oracle_range_search_matches_reference_random_sweep(lib_built):
    """Seeded random range searches (every dtype and metric, Greedy / Doubling
    / Beam, beams 1-40, radii from the 0.2 % to the 20 % quantile, random
    start points, early stopping on and off): the restatement and the
    in-place reference return the same answers in the same order and the
    same counters."""
    rng = np.random.default_rng(77)
    dts = [np.uint8, np.int8, np.float32]
    answers = 0
    for case in range(24):
        dtype = dts[case % 3]
        metric = (case // 3) % 2
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
        radius = sample_radius(base, q, metric, quant)
        kw = dict(start=start, esr=esr_f * radius, esc=esc, metric=metric)
        a = O.range_search("oracle", base, q, g, beam, radius, rtype, **kw)
        b = O.range_search("ref", base, q, g, beam, radius, rtype, **kw)
        for x, y in zip(a["ids"], b["ids"]):
            np.testing.assert_array_equal(x, y, err_msg=f"case {case}")
        np.testing.assert_array_equal(a["visited"], b["visited"], err_msg=f"case {case}")
        np.testing.assert_array_equal(a["cmps"], b["cmps"], err_msg=f"case {case}")
        answers += sum(len(x) for x in a["ids"])
    assert answers > 1000


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "rangegt_*.npz"))), ids=os.path.basename)
def test_oracle_range_groundtruth_matches_golden(path, lib_built):
    """compute_range_groundtruth (data_tools/compute_range_groundtruth.cpp:14-30): every base id within the
    radius, in id order, as the tool itself computed it."""
    z = np.load(path)
    offs, ids = O.range_groundtruth("oracle", z["base"], z["queries"], float(z["radius"]), metric=int(z["metric"]))
    np.testing.assert_array_equal(offs, z["offsets"])
    np.testing.assert_array_equal(ids, z["ids"])
    assert len(ids) > 0


@needs_ref
@pytest.mark.parametrize("dtype,metric", [(np.uint8, 0), (np.int8, 1), (np.float32, 0), (np.float32, 1)])
def test_oracle_range_groundtruth_matches_reference(dtype, metric, lib_built):
    base = random_points(dtype, 3000, 9, 131)
    q = random_points(dtype, 16, 9, 132)
    for quant in (0.001, 0.05):
        radius = sample_radius(base, q, metric, quant)
        a = O.range_groundtruth("oracle", base, q, radius, metric=metric)
        b = O.range_groundtruth("ref", base, q, radius, metric=metric)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])


@needs_ref
def test_oracle_range_groundtruth_matches_reference_random_sweep(lib_built):
    """Seeded random range groundtruth runs (every dtype and metric, radii
    from the 0.1 % to the 30 % quantile): every base id within the radius in
    id order, as compute_range_groundtruth.cpp gives it."""
    rng = np.random.default_rng(57)
    dts = [np.uint8, np.int8, np.float32]
    for case in range(12):
        dtype = dts[case % 3]
        metric = (case // 3) % 2
        n = int(rng.integers(200, 3000))
        d = int(rng.integers(2, 40))
        base = random_points(dtype, n, d, 1200 + case)
        q = random_points(dtype, 8, d, 1300 + case)
        radius = sample_radius(base, q, metric, float(rng.choice([0.001, 0.01, 0.1, 0.3])))
        a = O.range_groundtruth("oracle", base, q, radius, metric=metric)
        b = O.range_groundtruth("ref", base, q, radius, metric=metric)
        np.testing.assert_array_equal(a[0], b[0], err_msg=f"case {case}")
        np.testing.assert_array_equal(a[1], b[1], err_msg=f"case {case}")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "quant_*.npz"))), ids=os.path.basename)
def test_oracle_quantized_search_matches_golden(path, lib_built):
    """beam_search_rerank over one-byte scalar-quantized points (beamSearch.h:529-597, euclidian_point.h:186-240):
    quantization parameters, re-ranked ids and float distances, visited and comparison counts."""
    z = np.load(path)
    r = O.search_quantized("oracle", z["base"], z["queries"], z["graph"], int(z["k"]), int(z["L"]),
                           rerank_factor=float(z["rerank_factor"]))
    assert r["slope"] == float(z["slope"]) and r["offset"] == int(z["offset"])
    np.testing.assert_array_equal(r["ids"], z["ids"])
    np.testing.assert_array_equal(r["dists"].view(np.uint32), z["dists"].view(np.uint32))
    np.testing.assert_array_equal(r["visited"], z["visited"])
    np.testing.assert_array_equal(r["cmps"], z["cmps"])


@needs_ref
@pytest.mark.parametrize("seed,n,d,R,L,k,rf", [(0, 3000, 16, 20, 40, 10, 100.0), (1, 3000, 24, 24, 30, 5, 2.0),
                                               (2, 20000, 32, 24, 40, 10, 100.0)])
def test_oracle_mips_quantized_search_matches_reference(seed, n, d, R, L, k, rf, lib_built):
    """The mips quantizer GraphIndex uses for float mips indexes (Quantized_Mips_Point<8, true>,
    mips_point.h:293-499; python/graph_index.cpp:69,167-185) on L2-normalised points: trimmed bound,
    scale, int8 rows, the quantized search and the float re-rank."""
    rng = np.random.default_rng(170 + seed)
    base = rng.standard_normal((n, d)).astype(np.float32)
    base /= np.linalg.norm(base, axis=1, keepdims=True).astype(np.float32)
    q = rng.standard_normal((40, d)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True).astype(np.float32)
    g = O.random_graph(n, R, 180 + seed)
    a = O.search_quantized("oracle", base, q, g, k, L, rerank_factor=rf, metric=1)
    b = O.search_quantized("ref", base, q, g, k, L, rerank_factor=rf, metric=1)
    assert a["slope"] == b["slope"] and b["offset"] == 0
    for key in ("ids", "visited", "cmps"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    np.testing.assert_array_equal(a["dists"].view(np.uint32), b["dists"].view(np.uint32))


@needs_ref
def test_oracle_quantized_search_matches_reference_random_sweep(lib_built):
    """Seeded random beam_search_rerank cases over one-byte points (Euclidean
    scalar quantization and the mips quantizer; value scales 0.01-37 so slope
    and offset vary; k, beam, rerank factor, visit and degree limits, batch
    factor and start point random): the restatement and the in-place
    reference agree on parameters, ids, distance bits and counters."""
    rng = np.random.default_rng(123)
    for case in range(16):
        metric = case % 2
        n = int(rng.integers(300, 2500))
        d = int(rng.integers(2, 40))
        R = int(rng.integers(4, 25))
        L = int(rng.integers(2, 70))
        k = int(rng.integers(1, L + 1))
        rf = float(rng.choice([1.0, 1.5, 2.0, 100.0]))
        lim = None if rng.random() < 0.7 else int(rng.integers(k, 3 * L + 2))
        dl = None if rng.random() < 0.7 else int(rng.integers(1, R + 1))
        bf = float(rng.choice([0.0, 0.125, 0.5, 1.0]))
        start = int(rng.integers(0, n))
        scale = float(rng.choice([1.0, 0.01, 37.0]))
        base = (rng.standard_normal((n, d)) * scale).astype(np.float32)
        q = (rng.standard_normal((8, d)) * scale).astype(np.float32)
        if metric == 1:
            base /= np.linalg.norm(base, axis=1, keepdims=True).astype(np.float32)
            q /= np.linalg.norm(q, axis=1, keepdims=True).astype(np.float32)
        g = O.random_graph(n, R, 900 + case)
        kw = dict(rerank_factor=rf, limit=lim, degree_limit=dl, batch_factor=bf, start=start, metric=metric)
        a = O.search_quantized("oracle", base, q, g, k, L, **kw)
        b = O.search_quantized("ref", base, q, g, k, L, **kw)
        assert a["slope"] == b["slope"] and (metric == 1 or a["offset"] == b["offset"]), case
        for key in ("ids", "visited", "cmps"):
            np.testing.assert_array_equal(a[key], b[key], err_msg=f"case {case} {key}")
        np.testing.assert_array_equal(a["dists"].view(np.uint32), b["dists"].view(np.uint32), err_msg=f"case {case}")


@needs_ref
def test_oracle_quantized_search_matches_reference(lib_built):
    for seed, (n, d, R, L, k, rf) in enumerate([(3000, 16, 20, 40, 10, 100.0), (3000, 24, 24, 30, 5, 2.0)]):
        base = random_points(np.float32, n, d, 140 + seed)
        q = random_points(np.float32, 40, d, 150 + seed)
        g = O.random_graph(n, R, 160 + seed)
        a = O.search_quantized("oracle", base, q, g, k, L, rerank_factor=rf)
        b = O.search_quantized("ref", base, q, g, k, L, rerank_factor=rf)
        assert (a["slope"], a["offset"]) == (b["slope"], b["offset"])
        for key in ("ids", "visited", "cmps"):
            np.testing.assert_array_equal(a[key], b[key])
        np.testing.assert_array_equal(a["dists"].view(np.uint32), b["dists"].view(np.uint32))
    # every value a non-negative integer: the quantization is the identity
    base = np.random.default_rng(1).integers(0, 200, (2000, 12)).astype(np.float32)
    q = np.random.default_rng(2).integers(0, 200, (30, 12)).astype(np.float32)
    g = O.random_graph(2000, 16, 5)
    a = O.search_quantized("oracle", base, q, g, 5, 20)
    b = O.search_quantized("ref", base, q, g, 5, 20)
    assert (a["slope"], a["offset"]) == (b["slope"], b["offset"]) == (1.0, 0)
    np.testing.assert_array_equal(a["ids"], b["ids"])
