"""Parity at the full size of the small uint8 configuration: 100,000 base +
1,000 query vectors, 128-d uint8, 64-component Gaussian mixture (centres
uniform in [32, 224], sigma 20, seed 0), Vamana R=32, L=64, alpha=1.2, two
passes; beam search k=10 at beams 10, 20, 50 and 100.

Against the reference compiled in place (oracle/_ref), on the host cores:
* the GPU build (pann_build) and the reference's knn_index::build_index with
  the same insertion order give the same graph: the same neighbours per
  vertex, in the same order up to the order of equal distances (the
  reference's final per-vertex std::sort compares distances only), and the
  same total of distance comparisons;
* on that graph the GPU search (pann_search, every tier) and the reference's
  beam_search give bit-identical answers: ids, distances, visited counts and
  distance-comparison counts, for every query and beam.
"""
import numpy as np
import pytest

import parlayann_b200 as P
from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (reference checkout absent)")]

N, NQ, D, R, LB, ALPHA = 100_000, 1_000, 128, 32, 64, 1.2


@pytest.fixture(scope="module")
def c0(lib_built):
    base = P.synth_mixture(P.U8, N, D, 64, 0, 0)
    q = P.synth_mixture(P.U8, NQ, D, 64, 0, 1)
    idx = P.Index(base, R)
    st = idx.build(LB, ALPHA, num_passes=2, batch_factor=0.125)
    g_gpu = idx.get_graph()
    g_ref, tot_ref = O.build_graph("ref", base, R, LB, ALPHA, 2, batch_factor=0.125)
    yield base, q, idx, st, g_gpu, g_ref, tot_ref
    idx.close()


def _row_dists(base, g, i):
    nb = g[i, 1:1 + g[i, 0]].astype(np.int64)
    diff = base[nb].astype(np.int64) - base[i].astype(np.int64)
    return (diff * diff).sum(1)


def test_c0_build_matches_reference(c0):
    base, q, idx, st, g_gpu, g_ref, tot_ref = c0
    assert st.dist_cmps == tot_ref
    np.testing.assert_array_equal(g_gpu[:, 0], g_ref[:, 0])
    for i in range(N):
        a = g_gpu[i, 1:1 + g_gpu[i, 0]]
        b = g_ref[i, 1:1 + g_ref[i, 0]]
        if not np.array_equal(a, b):
            assert sorted(a.tolist()) == sorted(b.tolist()), f"vertex {i}: different neighbours"
            np.testing.assert_array_equal(_row_dists(base, g_gpu, i), _row_dists(base, g_ref, i),
                                          err_msg=f"vertex {i}: order differs beyond equal distances")


@pytest.mark.parametrize("which", ["reference_graph", "gpu_graph"])
@pytest.mark.parametrize("L", [10, 20, 50, 100])
def test_c0_search_matches_reference(c0, which, L):
    base, q, idx, st, g_gpu, g_ref, tot_ref = c0
    g = g_ref if which == "reference_graph" else g_gpu
    idx.set_graph(g)
    r = idx.search(q, 10, L, batch_factor=0.125)
    o = O.search("ref", base, q, g, 10, L, batch_factor=0.125)
    np.testing.assert_array_equal(r.ids, o["ids"])
    np.testing.assert_array_equal(r.dists.view(np.uint32), o["dists"].view(np.uint32))
    np.testing.assert_array_equal(r.visited, o["visited"])
    np.testing.assert_array_equal(r.cmps, o["cmps"])
    idx.set_graph(g_gpu)
