"""ctypes bindings of the oracle libraries (TEST INFRASTRUCTURE ONLY).

  libpann_oracle.so   the C restatement of the reference's hot path (pann_oracle.c)
  _ref/libpann_ref.so the reference's own headers compiled in place (ref_driver.cpp)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker / the timed reference. The product never imports it.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import sys
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libpann_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpann_ref.so")
_DT = {np.dtype(np.uint8): 0, np.dtype(np.int8): 1, np.dtype(np.float32): 2}

_P = ctypes.c_void_p
_U32, _U64, _I, _D = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double


def build():
    """Compile the oracle (and the in-place reference where its checkout exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


_olib = None
_rlib = None


def olib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.oracle_search.restype = _I
        L.oracle_search.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, _U32, _P, _U32, _U32, _U64, _U32, _D, _U32, _P,
                                    _P, _P, _P, _P, _P, _P, _P, _P, _U32, _P, _P]
        L.oracle_robust_prune.restype = _I
        L.oracle_robust_prune.argtypes = [_I, _I, _U32, _P, _U32, _P, _U32, _U32, _P, _P, _D, _I, _P, _P, _P]
        L.oracle_build.restype = _I
        L.oracle_build.argtypes = [_I, _I, _U32, _U32, _P, _U32, _U32, _D, _I, _D, _P, _U64, _I, _P, _P]
        L.oracle_groundtruth.restype = _I
        L.oracle_groundtruth.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, _U32, _P, _P]
        L.oracle_permutation.restype = None
        L.oracle_permutation.argtypes = [_U32, _U64, _P]
        L.oracle_batch_schedule.restype = _U32
        L.oracle_batch_schedule.argtypes = [_U64, _U64, _D, _D, _P, _P, _U32]
        L.oracle_range_search.restype = _I
        L.oracle_range_search.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, _U32, _P, _U32, _U32, _I, _D, _D, _U32,
                                          _P, _P, _U64, _P, _P, _P]
        L.oracle_range_groundtruth.restype = _I
        L.oracle_range_groundtruth.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, ctypes.c_float, _P, _P, _U64]
        L.oracle_search_quantized.restype = _I
        L.oracle_search_quantized.argtypes = [_I, _U32, _U32, _P, _U32, _P, _U32, _P, _U32, _U32, _U64, _U32, _D,
                                              _D, _U32, _P, _P, _P, _P]
        L.oracle_quant_params_mips.restype = None
        L.oracle_quant_params_mips.argtypes = [_U32, _U32, _P, _P, _P]
        L.oracle_quant_params.restype = None
        L.oracle_quant_params.argtypes = [_U32, _U32, _P, _P, _P]
        L.oracle_distance.restype = ctypes.c_float
        L.oracle_distance.argtypes = [_I, _I, ctypes.c_uint, _P, _P]
        _olib = L
    return _olib


def have_ref() -> bool:
    return os.path.exists(REF_SO)


def rlib():
    global _rlib
    if _rlib is None:
        L = ctypes.CDLL(REF_SO)
        L.ref_search.restype = _I
        L.ref_search.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, _U32, _P, _U32, _U32, _U64, _U32, _D, _U32, _P, _P,
                                 _P, _P, _P, _P, _P, _P, _U32, _P, _P]
        L.ref_qsearch_time.restype = _D
        L.ref_qsearch_time.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, _U32, _P, _U32, _U32, _D, _P, _P, _P, _P]
        L.ref_check_recall.restype = _I
        L.ref_check_recall.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, _U32, _P, ctypes.c_char_p, _U32, _U32, _U64,
                                       _U32, _D, _P]
        L.ref_synth_mixture.restype = _I
        L.ref_synth_mixture.argtypes = [_I, _U64, _U32, _U32, _U64, _U32, _D, _D, _D, _I, _P]
        L.ref_robust_prune.restype = _I
        L.ref_robust_prune.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, _U32, _U32, _P, _P, _D, _I, _P, _P, _P]
        L.ref_build.restype = _I
        L.ref_build.argtypes = [_I, _I, _U32, _U32, _P, _U32, _U32, _D, _I, _D, _P, _P, _P, _P]
        L.ref_range_search.restype = _I
        L.ref_range_search.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, _U32, _P, _U32, _U32, _I, _D, _D, _U32, _P,
                                       _P, _U64, _P, _P]
        L.ref_range_groundtruth.restype = _I
        L.ref_range_groundtruth.argtypes = [_I, _I, _U32, _U32, _P, _U32, _P, ctypes.c_float, _P, _P, _U64]
        L.ref_search_quantized.restype = _I
        L.ref_search_quantized.argtypes = [_I, _U32, _U32, _P, _U32, _P, _U32, _P, _U32, _U32, _U64, _U32, _D, _D,
                                           _U32, _P, _P, _P, _P, _P, _P, _P]
        L.ref_num_workers.restype = _I
        L.ref_num_workers.argtypes = []
        _rlib = L
    return _rlib


def search(impl: str, base, queries, graph, k, L, limit=None, degree_limit=None, batch_factor=0.125, starts=(0,),
           metric=0, full=False, visited_cap=None):
    """Beam search per query through the oracle ('oracle') or the in-place reference ('ref').
    graph: n x (R+1) uint32 reference rows. Returns a dict of arrays."""
    base = np.ascontiguousarray(base)
    queries = np.ascontiguousarray(queries, dtype=base.dtype)
    graph = np.ascontiguousarray(graph, dtype=np.uint32)
    n, d = base.shape
    R = graph.shape[1] - 1
    nq = queries.shape[0]
    limit = n if limit is None else limit
    degree_limit = R if degree_limit is None else degree_limit
    st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint32))
    ids = np.zeros((nq, k), np.uint32)
    dists = np.zeros((nq, k), np.float32)
    vis = np.zeros(nq, np.uint32)
    cmps = np.zeros(nq, np.uint32)
    out = dict(ids=ids, dists=dists, visited=vis, cmps=cmps)
    fn = fi = fd = vi = vd = None
    vcap = 0
    if full:
        fn = np.zeros(nq, np.uint32)
        fi = np.zeros((nq, L), np.uint32)
        fd = np.zeros((nq, L), np.float32)
        vcap = visited_cap or 4 * L + 64
        vi = np.zeros((nq, vcap), np.uint32)
        vd = np.zeros((nq, vcap), np.float32)
        out.update(frontier_n=fn, frontier_ids=fi, frontier_d=fd, visited_ids=vi, visited_d=vd)
    dt = _DT[base.dtype]
    if impl == "oracle":
        grew = np.zeros(nq, np.int32)
        rc = olib().oracle_search(dt, metric, n, d, _p(base), nq, _p(queries), R, _p(graph), k, L, limit,
                                  degree_limit, batch_factor, len(st), _p(st), _p(ids), _p(dists), _p(vis), _p(cmps),
                                  _p(grew), _p(fn), _p(fi), _p(fd), vcap, _p(vi), _p(vd))
        out["hash_grew"] = grew
    else:
        rc = rlib().ref_search(dt, metric, n, d, _p(base), nq, _p(queries), R, _p(graph), k, L, limit, degree_limit,
                               batch_factor, len(st), _p(st), _p(ids), _p(dists), _p(vis), _p(cmps), _p(fn), _p(fi),
                               _p(fd), vcap, _p(vi), _p(vd))
    out["rc"] = rc
    return out


RANGE_GREEDY, RANGE_DOUBLING, RANGE_BEAM = 1, 2, 3  # rangeQueryType (types.h:153)


def range_search(impl, base, queries, graph, beam, radius, rtype=RANGE_GREEDY, start=0, esr=0.0, esc=0, metric=0,
                 cap=None):
    """Range search per query ('oracle': pann_oracle.c; 'ref': RangeSearch / DoubleBeamRangeSearch compiled in
    place). Returns dict(ids=[uint32 arrays], visited, cmps[, hash_grew])."""
    base = np.ascontiguousarray(base)
    queries = np.ascontiguousarray(queries, dtype=base.dtype)
    graph = np.ascontiguousarray(graph, dtype=np.uint32)
    n, d = base.shape
    R = graph.shape[1] - 1
    nq = queries.shape[0]
    cap = cap or n
    cnt = np.zeros(nq, np.uint64)
    ids = np.zeros((nq, cap), np.uint32)
    vis = np.zeros(nq, np.uint32)
    cmps = np.zeros(nq, np.uint64)
    dt = _DT[base.dtype]
    out = {}
    if impl == "oracle":
        grew = np.zeros(nq, np.int32)
        rc = olib().oracle_range_search(dt, metric, n, d, _p(base), nq, _p(queries), R, _p(graph), beam, start, rtype,
                                        radius, esr, esc, _p(cnt), _p(ids), cap, _p(vis), _p(cmps), _p(grew))
        out["hash_grew"] = grew
    else:
        rc = rlib().ref_range_search(dt, metric, n, d, _p(base), nq, _p(queries), R, _p(graph), beam, start, rtype,
                                     radius, esr, esc, _p(cnt), _p(ids), cap, _p(vis), _p(cmps))
    assert rc == 0, rc
    assert (cnt <= cap).all(), "raise cap"
    out.update(ids=[ids[i, : int(cnt[i])].copy() for i in range(nq)], visited=vis,
               cmps=(cmps & 0xFFFFFFFF).astype(np.uint32))
    return out


@contextlib.contextmanager
def _stdout_to_stderr():
    """The reference's tools print progress on stdout; keep it off a caller's stdout."""
    sys.stdout.flush()
    saved = os.dup(1)
    try:
        os.dup2(2, 1)
        yield
    finally:
        os.dup2(saved, 1)
        os.close(saved)


def range_groundtruth(impl, base, queries, radius, metric=0):
    """Every base id within `radius` of each query, in id order ('oracle': pann_oracle.c; 'ref':
    compute_range_groundtruth compiled in place, its progress line sent to stderr). Returns
    (offsets[nq + 1], ids)."""
    base = np.ascontiguousarray(base)
    queries = np.ascontiguousarray(queries, dtype=base.dtype)
    n, d = base.shape
    nq = queries.shape[0]
    fn = olib().oracle_range_groundtruth if impl == "oracle" else rlib().ref_range_groundtruth
    offs = np.zeros(nq + 1, np.uint64)
    cap = 0
    for _ in range(2):
        ids = np.zeros(max(cap, 1), np.uint32)
        with _stdout_to_stderr():
            rc = fn(_DT[base.dtype], metric, n, d, _p(base), nq, _p(queries), radius, _p(offs), _p(ids), cap)
        assert rc in (0, 1), rc
        if rc == 0:
            return offs, ids[: int(offs[nq])]
        cap = int(offs[nq])
    raise AssertionError("range groundtruth did not fit")


def search_quantized(impl, base, queries, graph, k, L, rerank_factor=100.0, limit=None, degree_limit=None,
                     batch_factor=0.125, start=0, metric=0):
    """beam_search_rerank over one-byte scalar-quantized float points with a float re-rank ('oracle':
    pann_oracle.c; 'ref': the reference compiled in place); metric 0 Euclidian_Point<uint8_t>, 1
    Quantized_Mips_Point<8, true>. Returns dict(ids, dists, visited, cmps, slope, offset[, seconds]); for
    mips slope is the scale and offset 0."""
    base = np.ascontiguousarray(base, dtype=np.float32)
    queries = np.ascontiguousarray(queries, dtype=np.float32)
    graph = np.ascontiguousarray(graph, dtype=np.uint32)
    n, d = base.shape
    R = graph.shape[1] - 1
    nq = queries.shape[0]
    limit = n if limit is None else limit
    degree_limit = R if degree_limit is None else degree_limit
    ids = np.zeros((nq, k), np.uint32)
    dists = np.zeros((nq, k), np.float32)
    vis = np.zeros(nq, np.uint32)
    cmps = np.zeros(nq, np.uint32)
    slope = np.zeros(1, np.float32)
    offset = np.zeros(1, np.int32)
    out = {}
    if impl == "oracle":
        rc = olib().oracle_search_quantized(metric, n, d, _p(base), nq, _p(queries), R, _p(graph), k, L, limit,
                                            degree_limit, rerank_factor, batch_factor, start, _p(ids), _p(dists),
                                            _p(vis), _p(cmps))
        if metric == 0:
            olib().oracle_quant_params(n, d, _p(base), _p(slope), _p(offset))
        else:
            bound = np.zeros(1, np.float32)
            olib().oracle_quant_params_mips(n, d, _p(base), _p(slope), _p(bound))
    else:
        secs = np.zeros(1, np.float64)
        with _stdout_to_stderr():
            rc = rlib().ref_search_quantized(metric, n, d, _p(base), nq, _p(queries), R, _p(graph), k, L, limit,
                                             degree_limit, rerank_factor, batch_factor, start, _p(ids), _p(dists),
                                             _p(vis), _p(cmps), _p(slope), _p(offset), _p(secs))
        out["seconds"] = float(secs[0])
    assert rc == 0, rc
    out.update(ids=ids, dists=dists, visited=vis, cmps=cmps, slope=float(slope[0]), offset=int(offset[0]))
    return out


def robust_prune(impl, base, graph, p, cand_ids, cand_d, alpha, add=True, metric=0):
    base = np.ascontiguousarray(base)
    graph = np.ascontiguousarray(graph, dtype=np.uint32)
    n, d = base.shape
    R = graph.shape[1] - 1
    ci = np.ascontiguousarray(cand_ids, dtype=np.uint32)
    cd = np.ascontiguousarray(cand_d, dtype=np.float32)
    out = np.zeros(R + 1, np.uint32)
    nout = np.zeros(1, np.uint32)
    cm = np.zeros(1, np.int64)
    dt = _DT[base.dtype]
    if impl == "oracle":
        olib().oracle_robust_prune(dt, metric, d, _p(base), R, _p(graph), p, len(ci), _p(ci), _p(cd), alpha, int(add),
                                   _p(out), _p(nout), _p(cm))
    else:
        rlib().ref_robust_prune(dt, metric, n, d, _p(base), R, _p(graph), p, len(ci), _p(ci), _p(cd), alpha, int(add),
                                _p(out), _p(nout), _p(cm))
    return out[: int(nout[0])].copy(), int(cm[0])


def build_graph(impl, base, R, L, alpha, passes, batch_factor=0.125, perm=None, perm_seed=0x5EED5EED5EED,
                sort_neighbors=True, metric=0):
    """Vamana build; returns (n x (R+1) reference rows, total distance comparisons)."""
    base = np.ascontiguousarray(base)
    n, d = base.shape
    g = np.zeros((n, R + 1), np.uint32)
    dt = _DT[base.dtype]
    tot = np.zeros(1, np.uint64)
    if impl == "oracle":
        pm = None if perm is None else np.ascontiguousarray(perm, dtype=np.uint32)
        rc = olib().oracle_build(dt, metric, n, d, _p(base), R, L, alpha, passes, batch_factor, _p(pm), perm_seed,
                                 int(sort_neighbors), _p(g), _p(tot))
    else:
        secs = np.zeros(1, np.float64)
        vis = np.zeros(n, np.uint32)
        rc = rlib().ref_build(dt, metric, n, d, _p(base), R, L, alpha, passes, batch_factor, _p(g), _p(secs), _p(tot),
                              _p(vis))
    assert rc == 0, rc
    return g, int(tot[0])


def groundtruth(base, queries, k, metric=0):
    base = np.ascontiguousarray(base)
    queries = np.ascontiguousarray(queries, dtype=base.dtype)
    n, d = base.shape
    ids = np.zeros((queries.shape[0], k), np.uint32)
    dd = np.zeros((queries.shape[0], k), np.float64)
    olib().oracle_groundtruth(_DT[base.dtype], metric, n, d, _p(base), queries.shape[0], _p(queries), k, _p(ids),
                              _p(dd))
    return ids, dd


def groundtruth_fast(base, queries, k, metric=0, cand=None, chunk=256, threads=None):
    """Exact top-k by FP64 distance (ties by id), for float32 points, on the host cores: a float32
    pass (torch CPU matmul of the |q|^2 + |b|^2 - 2 q.b expansion) keeps the `cand` best candidates
    per query; their FP64 distances give the answer. The float32 distance of every point is within
    `bound` of its FP64 distance (a forward error bound of the expansion), so when the cand-th
    float32 distance exceeds the k-th by more than 2 bound the candidates hold every true top-k
    point; a query where it does not is recomputed in FP64 over all points. metric 1 = mips
    (distance -q.b). Returns (ids uint32, dists float64)."""
    import torch

    base = np.ascontiguousarray(base, dtype=np.float32)
    queries = np.ascontiguousarray(queries, dtype=np.float32)
    n, d = base.shape
    nq = queries.shape[0]
    cand = min(n, cand or max(4 * k, 64))
    if threads:
        torch.set_num_threads(threads)
    B = torch.from_numpy(base)
    b64 = base.astype(np.float64)
    bn = (b64 * b64).sum(1)
    bn32 = torch.from_numpy(bn.astype(np.float32))
    bmax = float(np.sqrt(bn.max()))
    ids = np.zeros((nq, k), np.uint32)
    dd = np.zeros((nq, k), np.float64)
    u = 2.0 ** -23
    for s in range(0, nq, chunk):
        q = queries[s:s + chunk]
        Q = torch.from_numpy(q)
        if metric == 0:
            D = torch.addmm(bn32[None, :], Q, B.t(), beta=1.0, alpha=-2.0)
        else:
            D = -(Q @ B.t())
        top = torch.topk(D, cand, dim=1, largest=False, sorted=True)
        tv = top.values.numpy().astype(np.float64)
        ti = top.indices.numpy()
        q64 = q.astype(np.float64)
        qn = np.sqrt((q64 * q64).sum(1))
        # |error| of a float32 dot of length d is <= d u sum|q_t b_t| <= d u |q||b|; the norms add less
        bound = (d + 8) * u * (qn * bmax + (qn * qn + bmax * bmax if metric == 0 else 0.0)) * 2.0
        for j in range(q.shape[0]):
            if cand < n and not (tv[j, cand - 1] - tv[j, k - 1] > 2.0 * bound[j]):
                c = np.arange(n)
            else:
                c = ti[j]
            rows = b64[c]
            dj = ((rows - q64[j]) ** 2).sum(1) if metric == 0 else -(rows @ q64[j])
            o = np.lexsort((c, dj))[:k]
            ids[s + j] = c[o]
            dd[s + j] = dj[o]
    return ids, dd


def write_ibin(path, ids, dists):
    """groundTruth's .ibin file (types.h:48-73): int32 n, int32 k, int32 ids[n k], float dists[n k]."""
    with open(path, "wb") as fh:
        np.array(ids.shape, np.int32).tofile(fh)
        np.ascontiguousarray(ids, dtype=np.int32).tofile(fh)
        np.ascontiguousarray(dists, dtype=np.float32).tofile(fh)


def permutation(n, seed=0x5EED5EED5EED):
    out = np.zeros(n, np.uint32)
    olib().oracle_permutation(n, seed, _p(out))
    return out


def batch_schedule(n, m=None):
    m = n if m is None else m
    fl = np.zeros(8192, np.uint64)
    ce = np.zeros(8192, np.uint64)
    nb = olib().oracle_batch_schedule(n, m, 2.0, 0.02, _p(fl), _p(ce), 8192)
    return list(zip(fl[:nb].tolist(), ce[:nb].tolist()))


def qsearch_time(base, queries, graph, k, L, batch_factor=0.125, metric=0):
    """The reference's qsearchAll timed as checkRecall times it (check_nn_recall.h:46-59). Returns
    (seconds, ids, visited, comparisons, distances); the distances of the returned ids come from the
    reference's Point::distance, outside the timed region."""
    base = np.ascontiguousarray(base)
    queries = np.ascontiguousarray(queries, dtype=base.dtype)
    graph = np.ascontiguousarray(graph, dtype=np.uint32)
    n, d = base.shape
    R = graph.shape[1] - 1
    nq = queries.shape[0]
    ids = np.zeros((nq, k), np.uint32)
    dists = np.zeros((nq, k), np.float32)
    vis = np.zeros(nq, np.uint32)
    cmps = np.zeros(nq, np.uint32)
    secs = rlib().ref_qsearch_time(_DT[base.dtype], metric, n, d, _p(base), nq, _p(queries), R, _p(graph), k, L,
                                   batch_factor, _p(ids), _p(vis), _p(cmps), _p(dists))
    return secs, ids, vis, cmps, dists


def check_recall(base, queries, graph, gt_path, k, L, limit=None, degree_limit=None, batch_factor=0.125, metric=0):
    """The reference's checkRecall (check_nn_recall.h:17-128) over a groundtruth .ibin file: returns
    dict(recall, qps, avg_cmps, tail_cmps, avg_visited, tail_visited)."""
    base = np.ascontiguousarray(base)
    queries = np.ascontiguousarray(queries, dtype=base.dtype)
    graph = np.ascontiguousarray(graph, dtype=np.uint32)
    n, d = base.shape
    R = graph.shape[1] - 1
    out = np.zeros(6, np.float64)
    with _stdout_to_stderr():
        rc = rlib().ref_check_recall(_DT[base.dtype], metric, n, d, _p(base), queries.shape[0], _p(queries), R,
                                     _p(graph), os.fsencode(gt_path), k, L, n if limit is None else limit,
                                     R if degree_limit is None else degree_limit, batch_factor, _p(out))
    if rc != 0:
        raise RuntimeError(f"ref_check_recall failed ({rc})")
    return dict(zip(("recall", "qps", "avg_cmps", "tail_cmps", "avg_visited", "tail_visited"), out.tolist()))


def synth_mixture(dtype, n, d, components, seed, stream, lo=32.0, hi=224.0, sigma=20.0, normalize=False):
    """The seeded Gaussian-mixture rows, generated by the in-place reference library (the same values
    as the product's pann_synth_mixture; a reference run loads no other library)."""
    out = np.empty((n, d), dtype=np.uint8 if dtype == 0 else np.float32)
    if rlib().ref_synth_mixture(dtype, n, d, components, seed, stream, lo, hi, sigma, int(normalize), _p(out)) != 0:
        raise ValueError("ref_synth_mixture: bad arguments")
    return out


def random_graph(n, R, seed, min_deg=1):
    """Seeded random graph in the reference layout (degree slot + padded rows)."""
    rng = np.random.default_rng(seed)
    g = np.zeros((n, R + 1), np.uint32)
    for i in range(n):
        deg = int(rng.integers(min_deg, R + 1))
        nb = rng.choice(n, size=deg, replace=False)
        g[i, 0] = deg
        g[i, 1:1 + deg] = nb
    return g
