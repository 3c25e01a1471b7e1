"""Parity of the CUDA beam search (through the C ABI) with the oracle.

Bar: bit-exact for every dtype and metric -- identical top-k ids, distances,
visited counts and distance-comparison counts. Float32 distances are computed
in the reference's sequential order without FMA, so they are bit-identical
too (the required bar for float is 1e-5 relative distance error and >= 99.9%
identical top-k lists; the tests assert the stronger exact equality, and
FLOAT_RTOL documents the required one).
"""
import glob
import os

import numpy as np
import pytest

import parlayann_b200 as P
from conftest import random_points
from oracle import oracle as O

pytestmark = pytest.mark.gpu
FLOAT_RTOL = 1e-5
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def check_same(g, o, msg="", allow_flagged=False):
    ok = np.ones(len(g.visited), bool)
    if allow_flagged:
        ok = g.flags == 0
    np.testing.assert_array_equal(g.ids[ok], o["ids"][ok], err_msg=f"ids {msg}")
    np.testing.assert_array_equal(g.visited[ok], o["visited"][ok], err_msg=f"visited {msg}")
    np.testing.assert_array_equal(g.cmps[ok], o["cmps"][ok], err_msg=f"cmps {msg}")
    np.testing.assert_allclose(g.dists[ok], o["dists"][ok], rtol=FLOAT_RTOL, err_msg=f"dists {msg}")
    np.testing.assert_array_equal(g.dists[ok], o["dists"][ok], err_msg=f"dists bits {msg}")


CASES = [  # k, L, limit, degree_limit, batch_factor, starts
    (10, 20, None, None, 0.125, (0,)),
    (10, 10, None, None, 0.125, (3,)),
    (5, 12, 20, None, 0.125, (0, 7, 9)),
    (8, 40, None, 6, 1.0, (3,)),
    (1, 8, 5, None, 0.5, (0,)),
    (3, 6, 1, None, 0.125, (0,)),
    (16, 64, None, None, 0.125, (0, 1, 2, 3)),
    (4, 4, None, None, 0.0, (11,)),
]


@pytest.mark.parametrize("dtype", [np.uint8, np.int8, np.float32], ids=["u8", "i8", "f32"])
@pytest.mark.parametrize("metric", [P.L2, P.MIPS], ids=["l2", "mips"])
def test_search_random_graph_matches_oracle(dtype, metric, lib_built):
    base = random_points(dtype, 3000, 40, 11)
    q = random_points(dtype, 200, 40, 12)
    g = O.random_graph(3000, 16, 13)
    idx = P.Index(base, 16, metric)
    idx.set_graph(g)
    for (k, L, lim, dl, bf, st) in CASES:
        r = idx.search(q, k, L, limit=lim, degree_limit=dl, batch_factor=bf, starts=st)
        o = O.search("oracle", base, q, g, k, L, limit=lim, degree_limit=dl, batch_factor=bf, starts=st,
                     metric=metric)
        check_same(r, o, f"k={k} L={L} limit={lim} dl={dl} bf={bf}")
    idx.close()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "search_*.npz"))), ids=os.path.basename)
def test_search_matches_golden(path, lib_built):
    z = np.load(path)
    lim = int(z["limit"])
    dl = int(z["degree_limit"])
    idx = P.Index(z["base"], z["graph"].shape[1] - 1, int(z["metric"]))
    idx.set_graph(z["graph"])
    r = idx.search(z["queries"], int(z["k"]), int(z["L"]), limit=None if lim < 0 else lim,
                   degree_limit=None if dl < 0 else dl, batch_factor=float(z["batch_factor"]),
                   starts=z["starts"].tolist())
    np.testing.assert_array_equal(r.ids, z["ids"])
    np.testing.assert_array_equal(r.dists, z["dists"])
    np.testing.assert_array_equal(r.visited, z["visited"])
    np.testing.assert_array_equal(r.cmps, z["cmps"])
    idx.close()


@pytest.mark.parametrize("dtype,metric", [(np.uint8, P.L2), (np.float32, P.MIPS), (np.int8, P.L2)])
def test_search_lists_match_oracle(dtype, metric, lib_built):
    """Full beam_search output (frontier and sorted visited list), as
    filtered_beam_search returns it (beamSearch.h:225-227)."""
    base = random_points(dtype, 2000, 24, 91)
    q = random_points(dtype, 60, 24, 92)
    g = O.random_graph(2000, 12, 93)
    idx = P.Index(base, 12, metric)
    idx.set_graph(g)
    for (L, lim, bf, st) in [(20, None, 0.125, (0,)), (8, 12, 0.5, (1, 2)), (40, None, 1.0, (5,))]:
        r = idx.search_lists(q, L, limit=lim, batch_factor=bf, starts=st, visited_cap=512)
        o = O.search("oracle", base, q, g, 1, L, limit=lim, batch_factor=bf, starts=st, metric=metric, full=True,
                     visited_cap=512)
        np.testing.assert_array_equal(r["frontier_n"], o["frontier_n"])
        np.testing.assert_array_equal(r["visited"], o["visited"])
        np.testing.assert_array_equal(r["cmps"], o["cmps"])
        for i in range(q.shape[0]):
            f = int(o["frontier_n"][i])
            np.testing.assert_array_equal(r["frontier_ids"][i, :f], o["frontier_ids"][i, :f])
            np.testing.assert_array_equal(r["frontier_d"][i, :f], o["frontier_d"][i, :f])
            v = int(o["visited"][i])
            np.testing.assert_array_equal(r["visited_ids"][i, :v], o["visited_ids"][i, :v])
            np.testing.assert_array_equal(r["visited_d"][i, :v], o["visited_d"][i, :v])
    idx.close()


def test_search_vamana_graph_u8(lib_built):
    """A Vamana graph on a seeded uint8 mixture (the reference's own build
    restated by the oracle), queried across beams."""
    base = P.synth_mixture(P.U8, 4000, 128, 16, 0, 0)
    q = P.synth_mixture(P.U8, 300, 128, 16, 0, 1)
    g, _ = O.build_graph("oracle", base, 24, 48, 1.2, 2)
    idx = P.Index(base, 24)
    idx.set_graph(g)
    for L in (10, 20, 50, 100):
        r = idx.search(q, 10, L)
        o = O.search("oracle", base, q, g, 10, L)
        check_same(r, o, f"L={L}")
    idx.close()


def test_search_float_mixture_mips(lib_built):
    base = P.synth_mixture(P.F32, 3000, 96, 32, 1, 0, sigma=0.3, normalize=True)
    q = P.synth_mixture(P.F32, 200, 96, 32, 1, 1, sigma=0.3, normalize=True)
    g, _ = O.build_graph("oracle", base, 32, 64, 1.2, 1, metric=1)
    idx = P.Index(base, 32, P.MIPS)
    idx.set_graph(g)
    for L in (10, 40, 128):
        check_same(idx.search(q, 10, L), O.search("oracle", base, q, g, 10, L, metric=1), f"L={L}")
    idx.close()


@pytest.mark.parametrize("slots", ["512", "1024"])
def test_seen_table_tiers_are_exact(slots, lib_built, monkeypatch):
    """Force the first-tier seen table to overflow so queries re-run in the
    larger tiers (shared-memory, then global); results must not change."""
    base = random_points(np.uint8, 20000, 16, 21)
    q = random_points(np.uint8, 64, 16, 22)
    g = O.random_graph(20000, 64, 23, min_deg=48)
    idx = P.Index(base, 64)
    idx.set_graph(g)
    monkeypatch.setenv("PANN_SEEN_SLOTS", slots)
    for L in (16, 64, 200):
        r = idx.search(q, 10, L)
        o = O.search("oracle", base, q, g, 10, L)
        check_same(r, o, f"slots={slots} L={L}")
    idx.close()


@pytest.mark.parametrize("L,bf", [(40, 1.0), (100, 1.0), (12, 0.125)])
def test_hashset_growth_is_reproduced(L, bf, lib_built):
    """Where the reference's hashset grows (hashset.h:25-38) the query is
    flagged and re-run by the exact-emulation tier: results, visited and
    comparison counts still equal the reference's, duplicates included."""
    base = random_points(np.uint8, 20000, 8, 1)
    q = random_points(np.uint8, 64, 8, 2)
    g = O.random_graph(20000, 64, 3, min_deg=60)
    idx = P.Index(base, 64)
    idx.set_graph(g)
    r = idx.search(q, 10, L, batch_factor=bf)
    o = O.search("oracle", base, q, g, 10, L, batch_factor=bf)
    np.testing.assert_array_equal(r.flags == 1, o["hash_grew"] > 0)  # flagged exactly where it grows
    check_same(r, o)
    idx.close()


@pytest.mark.parametrize("L", [40, 50])
def test_hashset_growth_with_repeated_neighbours(L, lib_built):
    """Adjacency lists with repeated ids under hashset growth: the emulation
    must reproduce the reference's duplicate handling (std::unique, set_union,
    set_difference) exactly."""
    base = random_points(np.uint8, 20000, 8, 5)
    q = random_points(np.uint8, 48, 8, 6)
    g = O.random_graph(20000, 64, 7, min_deg=60)
    rng = np.random.default_rng(8)
    for i in range(0, 20000, 3):          # repeat some ids inside a row
        deg = g[i, 0]
        g[i, 1 + rng.integers(0, deg, 4)] = g[i, 1 + rng.integers(0, deg, 4)]
    idx = P.Index(base, 64)
    idx.set_graph(g)
    r = idx.search(q, 10, L, batch_factor=1.0)
    o = O.search("oracle", base, q, g, 10, L, batch_factor=1.0)
    assert (o["hash_grew"] > 0).sum() > 0
    check_same(r, o)
    idx.close()


def test_search_edge_cases(lib_built):
    base = random_points(np.float32, 500, 7, 31)   # odd dimension: padded rows
    g = O.random_graph(500, 5, 32)
    g[10, 0] = 0                                  # an isolated vertex
    idx = P.Index(base, 5)
    idx.set_graph(g)
    q = np.concatenate([base[:20], random_points(np.float32, 20, 7, 33)])  # queries equal to base points
    for (k, L, st) in [(1, 1, (0,)), (5, 5, (1, 2, 3, 4, 5)), (2, 3, (10,)), (7, 9, (10, 11))]:
        r = idx.search(q, k, L, starts=st, allow_short=True)
        o = O.search("oracle", base, q, g, k, L, starts=st)
        check_same(r, o, f"k={k} L={L}")
    # errors the reference abort()s on come back as status codes
    with pytest.raises(P.PannError) as e:
        idx.search(q, 10, 5)                      # k > L (beamSearch.h:612-616)
    assert e.value.code == P.PANN_EINVAL
    with pytest.raises(P.PannError):
        idx.search(q, 2, 4, starts=())            # no start point (beamSearch.h:51-53)
    with pytest.raises(P.PannError):
        idx.search(q, 2, 2, starts=(0, 1, 2))     # more start points than beam (:54-56)
    with pytest.raises(P.PannError):
        idx.search(q, 2, 4, starts=(600,))        # start id out of range
    # an isolated start returns fewer than k results (beamSearch.h:557-562)
    with pytest.raises(P.PannError) as e:
        idx.search(q, 3, 4, starts=(10,))
    assert e.value.code == P.PANN_ESHORT
    idx.close()


def test_empty_batch_and_large_batch(lib_built):
    base = random_points(np.uint8, 5000, 32, 41)
    g = O.random_graph(5000, 12, 42)
    idx = P.Index(base, 12)
    idx.set_graph(g)
    r = idx.search(np.zeros((0, 32), np.uint8), 5, 10)
    assert r.ids.shape == (0, 5)
    q = random_points(np.uint8, 20000, 32, 43)
    r = idx.search(q, 5, 10)
    o = O.search("oracle", base, q[:500], g, 5, 10)
    np.testing.assert_array_equal(r.ids[:500], o["ids"])
    idx.close()


def test_graph_roundtrip_and_file_format(tmp_path, lib_built):
    base = random_points(np.uint8, 1000, 16, 51)
    g = O.random_graph(1000, 9, 52)
    idx = P.Index(base, 9)
    idx.set_graph(g)
    np.testing.assert_array_equal(idx.get_graph(), g)
    path = str(tmp_path / "g.bin")
    idx.save_graph(path)
    raw = np.fromfile(path, dtype=np.uint32)      # graph.h:210-237 layout
    assert raw[0] == 1000 and raw[1] == 9
    np.testing.assert_array_equal(raw[2:1002], g[:, 0])
    edges = np.concatenate([g[i, 1:1 + g[i, 0]] for i in range(1000)])
    np.testing.assert_array_equal(raw[1002:], edges)
    idx2 = P.Index(base, 9)
    idx2.load_graph(path)
    np.testing.assert_array_equal(idx2.get_graph(), g)
    idx.close()
    idx2.close()


@pytest.mark.parametrize("dtype,metric", [(np.uint8, P.L2), (np.int8, P.MIPS), (np.float32, P.L2),
                                          (np.float32, P.MIPS)])
def test_groundtruth_matches_oracle(dtype, metric, lib_built):
    base = random_points(dtype, 3000, 24, 61)
    q = random_points(dtype, 50, 24, 62)
    idx = P.Index(base, 8, metric)
    ids, dd = idx.groundtruth(q, 20)
    oi, od = O.groundtruth(base, q, 20, metric=metric)
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(dd, od)
    idx.close()


@pytest.mark.parametrize("metric", [P.L2, P.MIPS])
@pytest.mark.parametrize("k", [10, 20, 100])
def test_groundtruth_float_fast_path_equals_plain_kernel(metric, k, lib_built, monkeypatch):
    """The float32 candidate pass + FP64 re-rank gives the plain FP64 kernel's answers exactly."""
    base = P.synth_mixture(P.F32, 200_000, 96, 64, 5, 0, sigma=0.3, normalize=True)
    q = P.synth_mixture(P.F32, 300, 96, 64, 5, 1, sigma=0.3, normalize=True)
    idx = P.Index(base, 8, metric)
    ids, dd = idx.groundtruth(q, k)
    monkeypatch.setenv("PANN_GT_PLAIN", "1")
    pi, pd = idx.groundtruth(q, k)
    np.testing.assert_array_equal(ids, pi)
    np.testing.assert_array_equal(dd, pd)
    idx.close()


def test_groundtruth_float_fast_path_with_duplicates(lib_built):
    """Thousands of copies of one point: equal distances defeat the margin test for the queries
    near it, which the plain kernel then answers (ties by id)."""
    rng = np.random.default_rng(8)
    base = rng.standard_normal((60_000, 32)).astype(np.float32)
    base[10_000:14_000] = base[5]
    q = np.concatenate([base[5:6] + 1e-3 * rng.standard_normal((4, 32)).astype(np.float32),
                        rng.standard_normal((40, 32)).astype(np.float32)])
    idx = P.Index(base, 8)
    ids, dd = idx.groundtruth(q, 20)
    oi, od = O.groundtruth(base, q, 20)
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(dd, od)
    idx.close()


def test_many_queries_far_first_order_and_overlapped_emulation(lib_built):
    """More queries than tier 0 has warps, so the jobs are taken farthest from the start point first,
    and enough hashset growth that the emulation pass beside tier 0 takes hand-offs while tier 0
    still runs: every answer, counter and growth flag still equals the oracle's."""
    base = random_points(np.uint8, 20000, 8, 11)
    q = random_points(np.uint8, 3000, 8, 12)
    g = O.random_graph(20000, 64, 13, min_deg=60)
    idx = P.Index(base, 64)
    idx.set_graph(g)
    r = idx.search(q, 10, 40, batch_factor=1.0)
    o = O.search("oracle", base, q, g, 10, 40, batch_factor=1.0)
    assert (o["hash_grew"] > 0).sum() > 10
    np.testing.assert_array_equal(r.flags == 1, o["hash_grew"] > 0)
    check_same(r, o)
    idx.close()
