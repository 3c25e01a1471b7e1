"""The precision form (float32 indexes): traversal scored from a bfloat16 or
FP8-E4M3 (per-dimension scales) copy of the points, best 4k re-ranked with the
exact float32 distance. Results are not bit-exact with the reference (the
traversal differs by design); the tests bound the recall loss against FP64
brute force and check that every reported distance is the exact float32
distance of its id (the re-rank), and that results are reproducible."""
import numpy as np
import pytest

import parlayann_b200 as P
from conftest import random_points
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RECALL_LOSS = {P.PREC_BF16: 0.01, P.PREC_FP8: 0.03}  # allowed recall@10 loss vs the exact search


@pytest.fixture(scope="module")
def mix_index(lib_built):
    base = P.synth_mixture(P.F32, 30000, 96, 64, 1, 0, sigma=0.3, normalize=True)
    q = P.synth_mixture(P.F32, 500, 96, 64, 1, 1, sigma=0.3, normalize=True)
    out = {}
    for metric in (P.L2, P.MIPS):
        idx = P.Index(base, 32, metric)
        idx.build(64, 1.2, num_passes=1)
        gt, _ = idx.groundtruth(q, 10)
        out[metric] = (idx, gt)
    yield base, q, out
    for idx, _ in out.values():
        idx.close()


@pytest.mark.parametrize("metric", [P.L2, P.MIPS], ids=["l2", "mips"])
@pytest.mark.parametrize("prec", [P.PREC_BF16, P.PREC_FP8], ids=["bf16", "fp8"])
def test_precision_recall_and_exact_rerank(mix_index, metric, prec):
    base, q, out = mix_index
    idx, gt = out[metric]
    exact = idx.search(q, 10, 40)
    idx.set_precision(prec)
    r = idx.search(q, 10, 40, precision=prec)
    r2 = idx.search(q, 10, 40, precision=prec)
    np.testing.assert_array_equal(r.ids, r2.ids)          # deterministic
    rec_exact = P.recall_at_k(exact.ids, gt, 10)
    rec = P.recall_at_k(r.ids, gt, 10)
    assert rec >= rec_exact - RECALL_LOSS[prec], (rec, rec_exact)
    # every reported distance is the exact float32 distance (sequential sum)
    for i in range(0, q.shape[0], 25):
        for j in range(10):
            v = int(r.ids[i, j])
            dd = O.olib().oracle_distance(2, metric, 96, base[v].ctypes.data, q[i].ctypes.data)
            assert r.dists[i, j] == np.float32(dd)
        assert np.all(np.diff(r.dists[i]) >= 0)
    idx.set_precision(P.PREC_F32)


def test_precision_requires_float_points(lib_built):
    idx = P.Index(np.zeros((100, 8), np.uint8), 4)
    with pytest.raises(P.PannError):
        idx.set_precision(P.PREC_BF16)
    idx.close()


@pytest.mark.parametrize("metric", [P.L2, P.MIPS], ids=["l2", "mips"])
@pytest.mark.parametrize("prec", [P.PREC_BF16, P.PREC_FP8], ids=["bf16", "fp8"])
@pytest.mark.parametrize("parents", [1, 2, 4])
def test_tile_search_recall_and_exact_rerank(mix_index, metric, prec, parents):
    """The multi-parent tile search (one CTA per query, `parents` nodes
    expanded per step): recall against FP64 brute force within the same
    bound as the single-parent precision form, exact float32 distances in the
    answer, deterministic, and the batched form gives the same answers."""
    base, q, out = mix_index
    idx, gt = out[metric]
    exact = idx.search(q, 10, 40)
    idx.set_precision(prec)
    r = idx.search(q, 10, 40, precision=prec, parents=parents)
    r2 = idx.search(q, 10, 40, precision=prec, parents=parents)
    np.testing.assert_array_equal(r.ids, r2.ids)
    rec_exact = P.recall_at_k(exact.ids, gt, 10)
    rec = P.recall_at_k(r.ids, gt, 10)
    # a different visiting order (several parents a step, no deferral): a looser bound
    assert rec >= rec_exact - RECALL_LOSS[prec] - 0.03, (rec, rec_exact)
    assert (r.visited > 0).all() and (r.cmps > 0).all()
    for i in range(0, q.shape[0], 25):
        assert len(set(r.ids[i].tolist())) == 10
        for j in range(10):
            v = int(r.ids[i, j])
            dd = O.olib().oracle_distance(2, metric, 96, base[v].ctypes.data, q[i].ctypes.data)
            assert r.dists[i, j] == np.float32(dd)
        assert np.all(np.diff(r.dists[i]) >= 0)
    # batched with per-query k and beam: each query as its own plain tile search
    rng = np.random.default_rng(9)
    ks = rng.choice(np.array([1, 10], np.uint32), len(q)).astype(np.uint32)
    Ls = np.array([rng.integers(max(10, kk), 4 * max(10, kk) + 1) for kk in ks], np.uint32)
    b = idx.batch(len(q), 10, int(Ls.max()), precision=prec, parents=parents)
    rb = b.run(q, ks, Ls)
    for kk, LL in sorted(set(zip(ks.tolist(), Ls.tolist()))):
        sel = np.where((ks == kk) & (Ls == LL))[0]
        p = idx.search(q[sel], kk, LL, precision=prec, parents=parents)
        np.testing.assert_array_equal(rb.ids[sel, :kk], p.ids)
        np.testing.assert_array_equal(rb.visited[sel], p.visited)
    b.close()
    idx.set_precision(P.PREC_F32)


@pytest.mark.parametrize("rf,k,L", [(100.0, 10, 40), (100.0, 10, 45), (2.0, 5, 30), (1.0, 8, 8), (3.0, 3, 9)])
def test_quantized_search_matches_oracle(rf, k, L, lib_built):
    """pann_search_quantized against the oracle's beam_search_rerank restatement (pinned to the reference):
    the same quantization parameters, re-ranked ids, float distances bit for bit, visited and comparison
    counts."""
    base = random_points(np.float32, 12000, 20, 301)
    q = random_points(np.float32, 400, 20, 302)
    g = O.random_graph(12000, 24, 303)
    idx = P.Index(base, 24)
    idx.set_graph(g)
    idx.set_quantized()
    r = idx.search_quantized(q, k, L, rerank_factor=rf)
    o = O.search_quantized("oracle", base, q, g, k, L, rerank_factor=rf)
    assert idx.quant_params() == (o["slope"], o["offset"])
    np.testing.assert_array_equal(r.ids, o["ids"])
    np.testing.assert_array_equal(r.dists.view(np.uint32), o["dists"].view(np.uint32))
    np.testing.assert_array_equal(r.visited, o["visited"])
    np.testing.assert_array_equal(r.cmps, o["cmps"])
    idx.close()


@pytest.mark.parametrize("rf,k,L", [(100.0, 10, 40), (2.0, 5, 30), (1.0, 8, 8)])
def test_mips_quantized_search_matches_oracle(rf, k, L, lib_built):
    """The mips quantized search (Quantized_Mips_Point<8, true> rows in an int8 mips index, float
    re-rank) against the oracle restatement pinned to the reference: the scale, ids, float distances
    bit for bit, visited and comparison counts, on L2-normalised points and queries."""
    rng = np.random.default_rng(321)
    base = rng.standard_normal((12000, 20)).astype(np.float32)
    base /= np.linalg.norm(base, axis=1, keepdims=True).astype(np.float32)
    q = rng.standard_normal((400, 20)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True).astype(np.float32)
    g = O.random_graph(12000, 24, 323)
    idx = P.Index(base, 24, P.MIPS)
    idx.set_graph(g)
    idx.set_quantized()
    r = idx.search_quantized(q, k, L, rerank_factor=rf)
    o = O.search_quantized("oracle", base, q, g, k, L, rerank_factor=rf, metric=1)
    assert idx.quant_params() == (o["slope"], 0)
    np.testing.assert_array_equal(r.ids, o["ids"])
    np.testing.assert_array_equal(r.dists.view(np.uint32), o["dists"].view(np.uint32))
    np.testing.assert_array_equal(r.visited, o["visited"])
    np.testing.assert_array_equal(r.cmps, o["cmps"])
    idx.close()


def test_quantized_search_integer_valued_points_and_errors(lib_built):
    rng = np.random.default_rng(311)
    base = rng.integers(0, 256, (5000, 16)).astype(np.float32)
    q = rng.integers(0, 256, (100, 16)).astype(np.float32)
    g = O.random_graph(5000, 16, 312)
    idx = P.Index(base, 16)
    idx.set_graph(g)
    with pytest.raises(P.PannError):
        idx.search_quantized(q, 5, 20)                      # no quantized copy yet
    idx.set_quantized()
    assert idx.quant_params() == (1.0, 0)                   # the quantization is the identity
    r = idx.search_quantized(q, 5, 20)
    o = O.search_quantized("oracle", base, q, g, 5, 20)
    np.testing.assert_array_equal(r.ids, o["ids"])
    with pytest.raises(P.PannError):
        idx.search_quantized(q, 5, 20, rerank_factor=0.5)   # fewer re-ranked entries than k
    idx.close()
    u8 = P.Index(base.astype(np.uint8), 16)
    with pytest.raises(P.PannError):
        u8.set_quantized()                                  # float indexes only
    u8.close()


def test_quantized_search_edge_cases(lib_built):
    """Empty batches, several start points, a visit limit and a degree limit go through the quantized search as
    they do through beam_search_rerank."""
    base = random_points(np.float32, 3000, 12, 321)
    q = random_points(np.float32, 50, 12, 322)
    g = O.random_graph(3000, 16, 323)
    idx = P.Index(base, 16)
    idx.set_graph(g)
    idx.set_quantized()
    r = idx.search_quantized(q[:0], 5, 20)
    assert r.ids.shape == (0, 5)
    # limit and degree limit, as QueryParams carries them into the quantized beam search
    r = idx.search_quantized(q, 5, 20, limit=12, degree_limit=10)
    o = O.search_quantized("oracle", base, q, g, 5, 20, limit=12, degree_limit=10)
    np.testing.assert_array_equal(r.ids, o["ids"])
    np.testing.assert_array_equal(r.visited, o["visited"])
    np.testing.assert_array_equal(r.cmps, o["cmps"])
    with pytest.raises(P.PannError):
        idx.search_quantized(q, 21, 20)                     # k > beam
    idx.close()


@pytest.mark.parametrize("metric", [P.L2, P.MIPS], ids=["l2", "mips"])
def test_score_pairs_exact_and_low_precision(mix_index, metric):
    """pann_score: the exact scores are Point::distance bit for bit; the bfloat16 / FP8 scores stay
    within their precision's error of the FP64 distance."""
    base, q, out = mix_index
    idx, gt = out[metric]
    rng = np.random.default_rng(4)
    ids = np.concatenate([gt, rng.integers(0, base.shape[0], (q.shape[0], 6))], axis=1).astype(np.uint32)
    ex = idx.score(q, ids)
    np.testing.assert_array_equal(ex.view(np.uint32), P.point_distances(q, base, ids, metric).view(np.uint32))
    rows = base[ids.ravel().astype(np.int64)].reshape(ids.shape + (base.shape[1],)).astype(np.float64)
    q64 = q.astype(np.float64)[:, None, :]
    d64 = ((rows - q64) ** 2).sum(-1) if metric == P.L2 else -(rows * q64).sum(-1)
    for prec, tol in ((P.PREC_BF16, 0.02), (P.PREC_FP8, 0.2)):
        idx.set_precision(prec)
        lp = idx.score(q, ids, prec).astype(np.float64)
        # absolute error relative to the scale of the distances (|q||b| = 1 here)
        assert np.abs(lp - d64).max() < tol, (prec, np.abs(lp - d64).max())
    idx.set_precision(P.PREC_F32)


@pytest.mark.parametrize("metric", [P.L2, P.MIPS], ids=["l2", "mips"])
@pytest.mark.parametrize("prec", [P.PREC_BF16, P.PREC_FP8], ids=["bf16", "fp8"])
@pytest.mark.parametrize("parents", [2, 3])
def test_tile_search_tensor_core_scoring(mix_index, metric, prec, parents):
    """Tile scoring on the tensor cores (tcgen05.mma, 128 staged rows against the query's split
    terms): the same recall as scoring on the CUDA cores within 0.02, the bound of the CUDA-core
    tile search against the exact search, exact float32 distances in the answer, deterministic, and
    the batched form gives the same answers."""
    base, q, out = mix_index
    idx, gt = out[metric]
    exact = idx.search(q, 10, 40)
    idx.set_precision(prec)
    tc = idx.search(q, 10, 40, precision=prec, parents=parents, scorer=P.SCORER_TENSOR)
    tc2 = idx.search(q, 10, 40, precision=prec, parents=parents, scorer=P.SCORER_TENSOR)
    cu = idx.search(q, 10, 40, precision=prec, parents=parents)
    np.testing.assert_array_equal(tc.ids, tc2.ids)
    assert (tc.flags & 16).sum() == 0
    rec_tc, rec_cu = P.recall_at_k(tc.ids, gt, 10), P.recall_at_k(cu.ids, gt, 10)
    rec_exact = P.recall_at_k(exact.ids, gt, 10)
    assert abs(rec_tc - rec_cu) <= 0.02, (rec_tc, rec_cu)
    assert rec_tc >= rec_exact - 2 * RECALL_LOSS[prec], (rec_tc, rec_exact)
    np.testing.assert_array_equal(tc.dists.view(np.uint32), idx.score(q, tc.ids).view(np.uint32))
    b = idx.batch(len(q), 10, 40, precision=prec, parents=parents, scorer=P.SCORER_TENSOR)
    br = b.run(q, 10, 40)
    np.testing.assert_array_equal(br.ids[:, :10], tc.ids)
    b.close()
    idx.set_precision(P.PREC_F32)


def test_tensor_core_scoring_needs_whole_mma_steps(lib_built):
    base = P.synth_mixture(P.F32, 2000, 40, 8, 1, 0, sigma=0.3, normalize=True)   # 80-byte bf16 rows
    idx = P.Index(base, 16)
    idx.build(32, 1.2)
    idx.set_precision(P.PREC_BF16)
    with pytest.raises(P.PannError) as e:
        idx.search(base[:8], 5, 20, precision=P.PREC_BF16, parents=2, scorer=P.SCORER_TENSOR)
    assert "tensor-core" in str(e.value)
    idx.close()
