"""Serving form (pann_server_*): continuous batching of concurrent requests.

Each request's answer must be the same alone and in the mix (bit-exact: ids
and distances for k-NN, ids in order for range requests), whatever other
requests share its batch or run beside it on the device."""
import threading

import numpy as np
import pytest

import parlayann_b200 as P
from conftest import random_points
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make_requests(q, nreq, seed, kinds=(0, 0, 0, 1)):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(nreq):
        kind = int(rng.choice(kinds))
        nq = int(rng.integers(1, 65))
        row = int(rng.integers(0, len(q) - nq))
        if kind == 0:
            k = int(rng.choice([5, 20]))
            beam = int(rng.integers(k, 4 * k + 1))
            reqs.append(("knn", row, nq, k, beam))
        else:
            reqs.append(("range", row, min(nq, 8), 12, 0))
    return reqs


@pytest.mark.parametrize("dtype,metric", [(np.uint8, P.L2), (np.float32, P.MIPS)], ids=["u8-l2", "f32-mips"])
def test_server_mix_equals_alone(dtype, metric, lib_built):
    base = random_points(dtype, 20000, 16, 101)
    g = O.random_graph(20000, 32, 102)
    q = random_points(dtype, 4000, 16, 103)
    idx = P.Index(base, 32, metric)
    idx.set_graph(g)
    samp = np.array([O.olib().oracle_distance(O._DT[base.dtype], metric, 16, q[i].ctypes.data, base[j].ctypes.data)
                     for i in range(4) for j in range(0, 20000, 10)])
    radius = float(np.quantile(samp, 0.02))
    reqs = make_requests(q, 240, 104)
    # every request alone first (the server must be the index's only user while it runs)
    alone = []
    for kind, row, nq, k, beam in reqs:
        if kind == "knn":
            r = idx.search(q[row:row + nq], k, beam)
            alone.append((r.ids, r.dists))
        else:
            alone.append(idx.range_search(q[row:row + nq], k, radius, P.RANGE_GREEDY)["ids"])
    srv = P.Server(idx, max_batch_queries=256, inflight=3, max_k=20, max_beam=80)
    tickets = [None] * len(reqs)

    def submitter(part):
        for i in range(part, len(reqs), 4):
            kind, row, nq, k, beam = reqs[i]
            if kind == "knn":
                tickets[i] = srv.submit_knn(q[row:row + nq], k, beam)
            else:
                tickets[i] = srv.submit_range(q[row:row + nq], k, radius, P.RANGE_GREEDY)

    threads = [threading.Thread(target=submitter, args=(p,)) for p in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for i, (kind, row, nq, k, beam) in enumerate(reqs):
        out = srv.wait(tickets[i])
        if kind == "knn":
            ids, dists, lat = out
            np.testing.assert_array_equal(ids, alone[i][0], err_msg=f"request {i} ids")
            np.testing.assert_array_equal(dists.view(np.uint32), alone[i][1].view(np.uint32),
                                          err_msg=f"request {i} dists")
        else:
            lists, lat = out
            for a, b in zip(lists, alone[i]):
                np.testing.assert_array_equal(a, b, err_msg=f"range request {i}")
        assert lat > 0
    st = srv.stats()
    assert st["requests"] == len(reqs)
    assert st["queries"] == sum(r[2] for r in reqs)
    assert 0 < st["p50_s"] <= st["p99_s"]
    srv.close()
    idx.close()


def test_server_replay_and_errors(lib_built):
    base = random_points(np.uint8, 20000, 16, 111)
    g = O.random_graph(20000, 32, 112)
    q = random_points(np.uint8, 2000, 16, 113)
    idx = P.Index(base, 32)
    idx.set_graph(g)
    srv = P.Server(idx, max_batch_queries=128, inflight=2, max_k=10, max_beam=40)
    n = 300
    rng = np.random.default_rng(114)
    arrival = np.cumsum(rng.exponential(1e-4, n))
    nq = rng.integers(1, 33, n)
    rows = rng.integers(0, 2000 - 33, n)
    lat, wall = srv.replay(arrival, np.zeros(n), nq, np.full(n, 10), np.full(n, 30), rows, q)
    assert (lat > 0).all() and wall >= arrival[-1]
    st = srv.stats(reset=True)
    assert st["requests"] == n and st["queries"] == int(nq.sum())
    assert srv.stats()["requests"] == 0
    with pytest.raises(P.PannError):
        srv.submit_knn(q[:10], 11, 30)        # k above the server's bound
    with pytest.raises(P.PannError):
        srv.submit_knn(q[:200], 10, 30)       # more queries than a batch holds
    with pytest.raises(P.PannError):
        srv.submit_knn(q[:10], 10, 5)         # beam below k
    srv.close()
    idx.close()


def test_server_admission_by_scratch(lib_built):
    """A slot admits requests while the batch they form fits its scratch arena: with an arena that
    holds 256 queries at k = 20, beam 80, batches of small-k, short-beam requests hold more queries
    than batches of large ones; a request that alone needs more than the arena is refused; answers
    equal the same requests run alone."""
    base = random_points(np.float32, 20000, 16, 121)
    g = O.random_graph(20000, 32, 122)
    q = random_points(np.float32, 4000, 16, 123)
    idx = P.Index(base, 32)
    idx.set_graph(g)
    probe = P.Server(idx, max_batch_queries=256, inflight=1, max_k=20, max_beam=80)
    budget = probe.admission()["scratch_bytes"]
    probe.close()
    srv = P.Server(idx, max_batch_queries=4000, inflight=1, max_k=20, max_beam=80, scratch_bytes=budget)

    def run(k, beam, n_req, per):
        rows = np.arange(n_req) * per
        alone = [idx.search(q[r:r + per], k, beam) for r in rows]
        srv.admission(reset=True)
        tickets = [srv.submit_knn(q[r:r + per], k, beam) for r in rows]
        for t, a in zip(tickets, alone):
            ids, dists, _ = srv.wait(t)
            np.testing.assert_array_equal(ids, a.ids)
            np.testing.assert_array_equal(dists.view(np.uint32), a.dists.view(np.uint32))
        adm = srv.admission()
        assert adm["scratch_peak"] <= budget
        return adm["queries"] / adm["batches"]

    small = run(5, 10, 60, 50)
    large = run(20, 80, 60, 50)
    assert small > large, (small, large)
    with pytest.raises(P.PannError):
        srv.submit_knn(q[:3000], 20, 80)      # alone more than the arena holds
    srv.close()
    idx.close()
