"""Pins, on the CPU, the pieces the benchmark measures recall and makes its
data with, against the reference compiled in place (oracle/_ref):

* recall_with_ties equals the reference's checkRecall (check_nn_recall.h:86-112:
  the groundtruth's ties at the k-th distance, recomputed with the reference's
  own float distance) on the reference's own answers;
* the host groundtruth used by the reference arm of bench.py
  (oracle.groundtruth_fast: float32 candidates, FP64 re-rank) equals the C
  oracle's FP64 brute force;
* the reference library's data generator produces the same rows as the
  product's pann_synth_mixture.
"""
import os
import tempfile

import numpy as np
import pytest

import parlayann_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (reference checkout absent)")


@pytest.mark.parametrize("dtype,metric,L", [(np.uint8, P.L2, 12), (np.uint8, P.L2, 30), (np.float32, P.L2, 16),
                                            (np.float32, P.MIPS, 20), (np.int8, P.MIPS, 14)])
def test_recall_with_ties_matches_check_recall(dtype, metric, L, lib_built):
    rng = np.random.default_rng(11 + L)
    n, d, nq, k = 3000, 24, 300, 10
    if dtype == np.uint8:
        base = rng.integers(0, 4, (n, d)).astype(np.uint8)     # few values: many tied distances
        q = rng.integers(0, 4, (nq, d)).astype(np.uint8)
    elif dtype == np.int8:
        base = rng.integers(-3, 4, (n, d)).astype(np.int8)
        q = rng.integers(-3, 4, (nq, d)).astype(np.int8)
    else:
        base = rng.standard_normal((n, d)).astype(np.float32)
        q = rng.standard_normal((nq, d)).astype(np.float32)
    g, _ = O.build_graph("oracle", base, 16, 32, 1.2, 1, metric=metric)
    gt, gd = O.groundtruth(base, q, 40, metric=metric)
    r = O.search("ref", base, q, g, k, L, metric=metric)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "gt.ibin")
        O.write_ibin(path, gt, gd)
        ref = O.check_recall(base, q, g, path, k, L, metric=metric)
    ours = P.recall_with_ties(r["ids"], gt, k, q, base, metric)
    assert ours == pytest.approx(ref["recall"], abs=0.0, rel=1e-7)
    if dtype == np.uint8:
        # the tie rule matters here: without it the count is lower
        assert P.recall_at_k(r["ids"], gt, k) <= ours


def test_point_distances_match_oracle(lib_built):
    rng = np.random.default_rng(3)
    for dtype in (np.uint8, np.int8, np.float32):
        for metric in (P.L2, P.MIPS):
            base = (rng.standard_normal((200, 33)).astype(np.float32) if dtype == np.float32 else
                    rng.integers(-128 if dtype == np.int8 else 0, 128 if dtype == np.int8 else 256,
                                 (200, 33)).astype(dtype))
            q = base[:7].copy()
            ids = rng.integers(0, 200, (7, 5))
            got = P.point_distances(q, base, ids, metric)
            for i in range(7):
                for j in range(5):
                    a = np.ascontiguousarray(base[ids[i, j]])
                    b = np.ascontiguousarray(q[i])
                    want = np.float32(O.olib().oracle_distance(O._DT[base.dtype], metric, 33, O._p(a), O._p(b)))
                    assert want.view(np.uint32) == got[i, j].view(np.uint32)


@pytest.mark.parametrize("metric", [P.L2, P.MIPS])
def test_groundtruth_fast_is_exact(metric, lib_built):
    base = P.synth_mixture(P.F32, 20000, 32, 16, 3, 0, sigma=0.3, normalize=True)
    q = P.synth_mixture(P.F32, 64, 32, 16, 3, 1, sigma=0.3, normalize=True)
    ids, dd = O.groundtruth_fast(base, q, 20, metric=metric, cand=48, chunk=20)
    gi, gdd = O.groundtruth(base, q, 20, metric=metric)
    np.testing.assert_array_equal(ids, gi)
    np.testing.assert_allclose(dd, gdd, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("dtype,d,comps,seed,stream,norm", [(P.U8, 128, 64, 0, 0, False), (P.U8, 128, 64, 0, 1, False),
                                                            (P.F32, 96, 256, 1, 0, True), (P.F32, 96, 256, 1, 1, True),
                                                            (P.F32, 17, 5, 9, 3, False)])
def test_reference_generator_matches_product(dtype, d, comps, seed, stream, norm, lib_built):
    kw = dict(sigma=0.3, normalize=norm) if dtype == P.F32 else {}
    a = P.synth_mixture(dtype, 3000, d, comps, seed, stream, **kw)
    b = O.synth_mixture(dtype, 3000, d, comps, seed, stream, **kw)
    assert a.dtype == b.dtype
    np.testing.assert_array_equal(a.view(np.uint8), b.view(np.uint8))
