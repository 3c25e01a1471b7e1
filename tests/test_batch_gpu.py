"""Batched form (pann_batch_*): queries with their own k and beam in one
launch sequence must give, per query, exactly what the oracle's beam search
gives with that query's QueryParams (beamSearch.h:492-526 runs the same mix as
independent beam_search calls). Bar: bit-exact ids, distances, visited and
comparison counts on every dtype, with CUDA-graph replay and autotuning on."""
import numpy as np
import pytest

import parlayann_b200 as P
from conftest import random_points
from oracle import oracle as O

pytestmark = pytest.mark.gpu
PAD = 0xFFFFFFFF


def per_query_oracle(base, q, g, k, beam, metric=0, batch_factor=0.125, starts=(0,)):
    """Oracle results for each query with its own (k, beam), grouped by shape."""
    nq = len(q)
    kmax = int(k.max())
    ids = np.full((nq, kmax), PAD, np.uint32)
    dists = np.zeros((nq, kmax), np.float32)
    vis = np.zeros(nq, np.uint32)
    cmps = np.zeros(nq, np.uint32)
    grew = np.zeros(nq, np.int32)
    for kk, LL in sorted(set(zip(k.tolist(), beam.tolist()))):
        sel = np.where((k == kk) & (beam == LL))[0]
        o = O.search("oracle", base, q[sel], g, kk, LL, metric=metric, batch_factor=batch_factor, starts=starts)
        ids[sel, :kk] = o["ids"]
        dists[sel, :kk] = o["dists"]
        vis[sel] = o["visited"]
        cmps[sel] = o["cmps"]
        grew[sel] = o["hash_grew"]
    return dict(ids=ids, dists=dists, visited=vis, cmps=cmps, hash_grew=grew)


def check(r, o, msg=""):
    np.testing.assert_array_equal(r.ids, o["ids"], err_msg=f"ids {msg}")
    np.testing.assert_array_equal(r.dists.view(np.uint32), o["dists"].view(np.uint32), err_msg=f"dists {msg}")
    np.testing.assert_array_equal(r.visited, o["visited"], err_msg=f"visited {msg}")
    np.testing.assert_array_equal(r.cmps, o["cmps"], err_msg=f"cmps {msg}")
    np.testing.assert_array_equal(r.flags == 1, o["hash_grew"] > 0, err_msg=f"growth flags {msg}")


def uneven_shapes(nq, seed, ks=(1, 10, 25)):
    """Per-query k uniform in ks and beam uniform in [k, 4k] (hop counts uneven)."""
    rng = np.random.default_rng(seed)
    k = rng.choice(np.asarray(ks, np.uint32), nq).astype(np.uint32)
    beam = np.array([rng.integers(kk, 4 * kk + 1) for kk in k], np.uint32)
    return k, np.maximum(beam, 1).astype(np.uint32)


@pytest.mark.parametrize("dtype,metric", [(np.uint8, P.L2), (np.int8, P.MIPS), (np.float32, P.L2),
                                          (np.float32, P.MIPS)], ids=["u8-l2", "i8-mips", "f32-l2", "f32-mips"])
def test_batch_uneven_k_and_beam_match_oracle(dtype, metric, lib_built):
    base = random_points(dtype, 8000, 24, 11)
    g = O.random_graph(8000, 32, 12)
    idx = P.Index(base, 32, metric)
    idx.set_graph(g)
    q = random_points(dtype, 600, 24, 13)
    k, beam = uneven_shapes(len(q), 14)
    b = idx.batch(len(q), int(k.max()), int(beam.max()))
    r = b.run(q, k, beam)
    o = per_query_oracle(base, q, g, k, beam, metric=metric)
    check(r, o, "first run")
    # second run replays the captured graph, on a smaller batch with other shapes
    k2, beam2 = uneven_shapes(300, 15)
    r2 = b.run(q[:300], k2, beam2)
    assert b.config()["graph"]
    o2 = per_query_oracle(base, q[:300], g, k2, beam2, metric=metric)
    check(r2, o2, "graph replay")
    b.close()
    idx.close()


def test_batch_hashset_growth_per_query(lib_built):
    """Queries whose beam makes the reference's hashset grow sit beside ones
    whose beam does not; each is reproduced exactly (emulation with the
    query's own initial capacity)."""
    base = random_points(np.uint8, 20000, 8, 1)
    g = O.random_graph(20000, 64, 3, min_deg=60)
    idx = P.Index(base, 64)
    idx.set_graph(g)
    q = random_points(np.uint8, 200, 8, 2)
    rng = np.random.default_rng(3)
    beam = rng.choice(np.array([12, 24, 40, 50, 64], np.uint32), len(q)).astype(np.uint32)
    k = np.minimum(beam, 10).astype(np.uint32)
    b = idx.batch(len(q), 10, 64, batch_factor=1.0)
    r = b.run(q, k, beam)
    o = per_query_oracle(base, q, g, k, beam, batch_factor=1.0)
    assert (o["hash_grew"] > 0).sum() > 0
    check(r, o)
    r = b.run(q, k, beam)   # replayed
    check(r, o, "replay")
    b.close()
    idx.close()


def test_batch_autotune_and_fixed_shapes(lib_built):
    base = random_points(np.uint8, 20000, 32, 21)
    g = O.random_graph(20000, 48, 22)
    idx = P.Index(base, 48)
    idx.set_graph(g)
    q = random_points(np.uint8, 2000, 32, 23)
    k, beam = uneven_shapes(len(q), 24, ks=(1, 10, 40))
    o = per_query_oracle(base, q, g, k, beam)
    for opts in (dict(autotune=True), dict(seen_slots=512, warps_per_block=2), dict(use_graph=False)):
        b = idx.batch(len(q), int(k.max()), int(beam.max()), **opts)
        check(b.run(q, k, beam), o, str(opts))
        cfg = b.config()
        if "seen_slots" in opts:
            assert cfg["seen_slots"] == 512 and cfg["warps_per_block"] == 2
        assert cfg["cta_per_query"] == opts.get("cta_per_query", cfg["cta_per_query"])
        assert cfg["register_blocks"] in (3, 4)
        assert cfg["graph"] == opts.get("use_graph", True)
        b.close()
    idx.close()


def test_batch_equals_plain_search_at_uniform_shape(lib_built):
    base = random_points(np.float32, 20000, 48, 31)
    g = O.random_graph(20000, 32, 32)
    idx = P.Index(base, 32)
    idx.set_graph(g)
    q = random_points(np.float32, 1000, 48, 33)
    plain = idx.search(q, 10, 45)
    b = idx.batch(len(q), 10, 45)
    r = b.run(q, 10, 45)
    for key in ("ids", "visited", "cmps"):
        np.testing.assert_array_equal(getattr(r, key), getattr(plain, key), err_msg=key)
    np.testing.assert_array_equal(r.dists.view(np.uint32), plain.dists.view(np.uint32))
    b.close()
    # the precision form, batched, equals the precision form, plain, query by query
    idx.set_precision(P.PREC_BF16)
    k, beam = uneven_shapes(len(q), 34)
    b = idx.batch(len(q), int(k.max()), int(beam.max()), precision=P.PREC_BF16)
    r = b.run(q, k, beam)
    for kk, LL in sorted(set(zip(k.tolist(), beam.tolist()))):
        sel = np.where((k == kk) & (beam == LL))[0]
        p = idx.search(q[sel], kk, LL, precision=P.PREC_BF16)
        np.testing.assert_array_equal(r.ids[sel, :kk], p.ids)
        np.testing.assert_array_equal(r.dists[sel, :kk].view(np.uint32), p.dists.view(np.uint32))
        np.testing.assert_array_equal(r.visited[sel], p.visited)
    b.close()
    idx.close()


def test_batch_argument_errors(lib_built):
    base = random_points(np.uint8, 1000, 16, 41)
    g = O.random_graph(1000, 8, 42)
    idx = P.Index(base, 8)
    idx.set_graph(g)
    q = random_points(np.uint8, 10, 16, 43)
    b = idx.batch(10, 5, 20, starts=(0, 1))
    for k, beam in [(6, 20), (5, 21), (5, 4), (0, 4), (1, 1)]:   # k > bound, beam > bound, k > beam, k = 0, beam < starts
        with pytest.raises(P.PannError) as e:
            b.run(q, k, beam)
        assert e.value.code == P.PANN_EINVAL
    with pytest.raises(P.PannError):
        b.run(np.concatenate([q, q]), 5, 10)                   # more queries than max_queries
    r = b.run(q[:0], 5, 10)                                    # empty run
    assert r.ids.shape == (0, 5)
    b.close()
    idx.close()


def test_batch_cta_per_query_with_hashset_growth(lib_built):
    """CTA per query (every query on one block of the exact-emulation kernel) gives the oracle's
    answers, the queries whose hashset grows included, and again on graph replay."""
    base = random_points(np.uint8, 20000, 8, 1)
    g = O.random_graph(20000, 64, 3, min_deg=60)
    idx = P.Index(base, 64)
    idx.set_graph(g)
    q = random_points(np.uint8, 300, 8, 2)
    rng = np.random.default_rng(5)
    # beams up to 50: the emulated tables (4 + 2 times 2^ceil(log2(2 (10 + 50) 64)) slots) fit in shared memory
    beam = rng.choice(np.array([12, 24, 40, 50], np.uint32), len(q)).astype(np.uint32)
    k = np.minimum(beam, 10).astype(np.uint32)
    b = idx.batch(len(q), 10, 50, batch_factor=1.0, cta_per_query=True)
    o = per_query_oracle(base, q, g, k, beam, batch_factor=1.0)
    assert (o["hash_grew"] > 0).sum() > 0
    check(b.run(q, k, beam), o, "cta")
    check(b.run(q, k, beam), o, "cta replay")
    assert b.config()["cta_per_query"]
    b.close()
    idx.close()


def test_batch_tile_autotune_keeps_answers(lib_built):
    """The tile search's rows per round, picked by the autotuner, do not change its answers."""
    base = P.synth_mixture(P.F32, 20000, 64, 32, 2, 0, sigma=0.3, normalize=True)
    q = P.synth_mixture(P.F32, 1000, 64, 32, 2, 1, sigma=0.3, normalize=True)
    idx = P.Index(base, 32)
    idx.build(48, 1.2)
    idx.set_precision(P.PREC_FP8)
    plain = idx.search(q, 10, 40, precision=P.PREC_FP8, parents=3)
    b = idx.batch(len(q), 10, 40, precision=P.PREC_FP8, parents=3, autotune=True)
    r = b.run(q, 10, 40)
    np.testing.assert_array_equal(r.ids[:, :10], plain.ids)
    np.testing.assert_array_equal(r.dists[:, :10].view(np.uint32), plain.dists.view(np.uint32))
    assert b.config()["tile_rows"] > 0
    b.close()
    idx.close()


def test_batch_cta_per_query_refused_when_tables_do_not_fit(lib_built):
    base = random_points(np.uint8, 4000, 8, 6)
    idx = P.Index(base, 64)
    idx.set_graph(O.random_graph(4000, 64, 7, min_deg=60))
    with pytest.raises(P.PannError) as e:
        idx.batch(10, 10, 200, cta_per_query=True)
    assert "CTA per query" in str(e.value)
    idx.close()
