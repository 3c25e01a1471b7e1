"""Range search on the GPU (pann_range_search) against the oracle and the
reference's own outputs (golden fixtures from RangeSearch /
DoubleBeamRangeSearch compiled in place). Bar: identical answers in the
reference's order (duplicates included), visited and comparison counts."""
import glob
import os

import numpy as np
import pytest

import parlayann_b200 as P
from conftest import random_points
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def sample_radius(base, q, metric, quant):
    d = q.shape[1]
    dt = O._DT[base.dtype]
    samp = [O.olib().oracle_distance(dt, metric, d, np.ascontiguousarray(q[i]).ctypes.data,
                                     np.ascontiguousarray(base[j]).ctypes.data)
            for i in range(min(4, len(q))) for j in range(0, len(base), max(1, len(base) // 2000))]
    return float(np.quantile(samp, quant))


def check(r, o, msg=""):
    assert len(r["ids"]) == len(o["ids"])
    for i, (x, y) in enumerate(zip(r["ids"], o["ids"])):
        np.testing.assert_array_equal(x, y, err_msg=f"answer {i} {msg}")
    np.testing.assert_array_equal(r["visited"], o["visited"], err_msg=f"visited {msg}")
    np.testing.assert_array_equal(r["cmps"], o["cmps"], err_msg=f"cmps {msg}")
    if "hash_grew" in o:
        np.testing.assert_array_equal(r["flags"] != 0, o["hash_grew"] > 0, err_msg=f"growth flags {msg}")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "range_*.npz"))), ids=os.path.basename)
def test_range_search_matches_golden(path, lib_built):
    z = np.load(path)
    metric = int(z["metric"])
    idx = P.Index(z["base"], z["graph"].shape[1] - 1, metric)
    idx.set_graph(z["graph"])
    for j, (rtype, beam, esc, esr) in enumerate(z["runs"]):
        r = idx.range_search(z["queries"], int(beam), float(z["radius"]), int(rtype), early_stopping_radius=float(esr),
                             early_stopping_count=int(esc))
        np.testing.assert_array_equal([len(x) for x in r["ids"]], z[f"counts{j}"], err_msg=f"counts run {j}")
        np.testing.assert_array_equal(np.concatenate(r["ids"]), z[f"ids{j}"], err_msg=f"ids run {j}")
        np.testing.assert_array_equal(r["visited"], z[f"visited{j}"], err_msg=f"visited run {j}")
        np.testing.assert_array_equal(r["cmps"], z[f"cmps{j}"], err_msg=f"cmps run {j}")
    idx.close()


@pytest.mark.parametrize("dtype,metric", [(np.uint8, P.L2), (np.int8, P.MIPS), (np.float32, P.L2),
                                          (np.float32, P.MIPS)], ids=["u8-l2", "i8-mips", "f32-l2", "f32-mips"])
def test_range_search_matches_oracle(dtype, metric, lib_built):
    base = random_points(dtype, 8000, 12, 71)
    q = random_points(dtype, 64, 12, 72)
    g = O.random_graph(8000, 24, 73)
    rng = np.random.default_rng(74)
    for i in range(0, 8000, 5):                     # repeated ids inside some rows
        deg = g[i, 0]
        g[i, 1 + rng.integers(0, deg, 3)] = g[i, 1 + rng.integers(0, deg, 3)]
    idx = P.Index(base, 24, metric)
    idx.set_graph(g)
    for quant in (0.005, 0.05, 0.25):
        radius = sample_radius(base, q, metric, quant)
        for rtype in (P.RANGE_GREEDY, P.RANGE_DOUBLING, P.RANGE_BEAM):
            for beam, esc, esr in [(10, 0, 0.0), (32, 12, 1.5 * radius)]:
                r = idx.range_search(q, beam, radius, rtype, early_stopping_radius=esr, early_stopping_count=esc)
                o = O.range_search("oracle", base, q, g, beam, radius, rtype, esr=esr, esc=esc, metric=metric)
                check(r, o, f"quant={quant} type={rtype} beam={beam} esc={esc}")
    idx.close()


def test_range_search_large_expansions_and_beam_growth(lib_built):
    """Expansions of tens of thousands of points per query (several growths of
    the expansion's hashset, answers past the first tier's queue), and a dense
    graph on which the beam's own hashset grows."""
    base = random_points(np.uint8, 100000, 6, 81)
    q = random_points(np.uint8, 6, 6, 82)
    g = O.random_graph(100000, 32, 83)
    idx = P.Index(base, 32)
    idx.set_graph(g)
    radius = sample_radius(base, q, P.L2, 0.7)
    r = idx.range_search(q, 16, radius, P.RANGE_GREEDY)
    o = O.range_search("oracle", base, q, g, 16, radius, O.RANGE_GREEDY)
    assert max(len(x) for x in o["ids"]) > 65536
    check(r, o, "large")
    idx.close()

    base = random_points(np.uint8, 20000, 8, 1)
    q = random_points(np.uint8, 48, 8, 2)
    g = O.random_graph(20000, 64, 3, min_deg=60)
    idx = P.Index(base, 64)
    idx.set_graph(g)
    for quant, esc in [(0.002, 0), (0.002, 15), (0.02, 0)]:
        radius = sample_radius(base, q, P.L2, quant)
        r = idx.range_search(q, 40, radius, P.RANGE_GREEDY, early_stopping_radius=2 * radius,
                             early_stopping_count=esc)
        o = O.range_search("oracle", base, q, g, 40, radius, O.RANGE_GREEDY, esr=2 * radius, esc=esc)
        check(r, o, f"growth quant={quant} esc={esc}")
    idx.close()


def test_range_search_edge_cases(lib_built):
    base = random_points(np.float32, 500, 7, 91)    # odd dimension: padded rows
    g = O.random_graph(500, 6, 92)
    g[10, 0] = 0                                   # an isolated vertex
    idx = P.Index(base, 6)
    idx.set_graph(g)
    q = np.concatenate([base[:5], random_points(np.float32, 5, 7, 93)])
    for start in (0, 10):
        for radius in (0.0, 1e30, -1.0):
            r = idx.range_search(q, 4, radius, P.RANGE_GREEDY, start=start)
            o = O.range_search("oracle", base, q, g, 4, radius, O.RANGE_GREEDY, start=start)
            check(r, o, f"start={start} radius={radius}")
    r = idx.range_search(q[:0], 4, 1.0)
    assert r["ids"] == [] and r["offsets"].tolist() == [0]
    with pytest.raises(P.PannError):
        idx.range_search(q, 4, 1.0, rtype=7)
    with pytest.raises(P.PannError):
        idx.range_search(q, 4, 1.0, start=600)
    idx.close()


def test_range_fetch_returns_the_held_answers(lib_built):
    """A call with no room for the answers (or out_ids NULL, cap 0) fills the
    offsets and counts and leaves the answers on the device; pann_range_fetch
    copies them, equal to a call given enough room."""
    import ctypes

    base = random_points(np.uint8, 20000, 8, 1)
    q = random_points(np.uint8, 24, 8, 2)
    g = O.random_graph(20000, 32, 3)
    idx = P.Index(base, 32)
    idx.set_graph(g)
    radius = sample_radius(base, q, P.L2, 0.05)
    want = idx.range_search(q, 16, radius, P.RANGE_GREEDY)
    total = int(want["offsets"][-1])
    assert total > len(q) * 16 * 4            # the wrapper itself went through the fetch
    lib = P.lib()
    rp = P.RangeParams(16, P.RANGE_GREEDY, radius, 0.0, 0)
    offs = np.zeros(len(q) + 1, np.uint64)
    vis = np.zeros(len(q), np.uint32)
    ptr = lambda a: ctypes.c_void_p(a.ctypes.data)   # noqa: E731
    rc = lib.pann_range_search(idx.handle, ptr(q), len(q), ctypes.byref(rp), 0, ptr(offs), None, 0, ptr(vis),
                               None, None)
    assert rc == P.PANN_EOVERFLOW
    np.testing.assert_array_equal(offs, want["offsets"])
    np.testing.assert_array_equal(vis, want["visited"])
    small = np.zeros(total - 1, np.uint32)
    assert lib.pann_range_fetch(idx.handle, ptr(small), len(small)) == P.PANN_EOVERFLOW
    ids = np.zeros(total, np.uint32)
    assert lib.pann_range_fetch(idx.handle, ptr(ids), total) == 0
    np.testing.assert_array_equal(ids, np.concatenate(want["ids"]))
    assert lib.pann_range_fetch(idx.handle, ptr(ids), total) == P.PANN_EINVAL   # taken: nothing held
    idx.close()


@pytest.mark.parametrize("dtype,metric", [(np.uint8, P.L2), (np.int8, P.MIPS), (np.float32, P.L2),
                                          (np.float32, P.MIPS)], ids=["u8-l2", "i8-mips", "f32-l2", "f32-mips"])
def test_range_groundtruth_matches_oracle(dtype, metric, lib_built):
    """pann_range_groundtruth against the oracle's compute_range_groundtruth
    (pinned to the tool itself in test_oracle_pin): the same ids in id order,
    over several tiles of base rows and an odd dimension."""
    base = random_points(dtype, 20000, 9, 121)
    q = random_points(dtype, 37, 9, 122)
    idx = P.Index(base, 8, metric)
    for quant in (0.0005, 0.02):
        radius = sample_radius(base, q, metric, quant)
        offs, ids = idx.range_groundtruth(q, radius)
        o_offs, o_ids = O.range_groundtruth("oracle", base, q, radius, metric=metric)
        np.testing.assert_array_equal(offs, o_offs, err_msg=f"offsets quant={quant}")
        np.testing.assert_array_equal(ids, o_ids, err_msg=f"ids quant={quant}")
        assert len(ids) > 0
    offs, ids = idx.range_groundtruth(q, -1e30)      # nothing in range
    assert int(offs[-1]) == 0 and len(ids) == 0
    offs, ids = idx.range_groundtruth(q[:0], 1.0)
    assert offs.tolist() == [0]
    idx.close()


def test_range_groundtruth_radius_boundary(lib_built):
    """A point at exactly the radius is in the answer (dist <= r, compute_range_groundtruth.cpp:24)."""
    base = random_points(np.uint8, 5000, 8, 131)
    q = random_points(np.uint8, 4, 8, 132)
    idx = P.Index(base, 8)
    d = np.array([O.olib().oracle_distance(0, 0, 8, q[0].ctypes.data, base[j].ctypes.data) for j in range(5000)],
                 np.float32)
    radius = float(np.sort(d)[40])                         # an exact distance value
    offs, ids = idx.range_groundtruth(q, radius)
    o_offs, o_ids = O.range_groundtruth("oracle", base, q, radius)
    np.testing.assert_array_equal(offs, o_offs)
    np.testing.assert_array_equal(ids, o_ids)
    assert int((d <= radius).sum()) == int(offs[1] - offs[0])
    # a range search with nothing held afterwards: fetch refuses
    idx.range_search(q[:0], 4, radius)
    with pytest.raises(P.PannError):
        P._check(P.lib().pann_range_fetch(idx.handle, None, 0))
    idx.close()
