"""parlayann_b200: B200 (sm_100a) beam search and Vamana build behind
ParlayANN's interfaces.

The product is the C ABI in ``include/parlayann_b200.h``, implemented by
``parlayann_b200/libparlayann_b200.so`` (CUDA kernels + host orchestration).
This module is a thin ctypes binding of that ABI, shaped like the reference's
Python surface (``GraphIndex.batch_search``, ``build_vamana_index``;
python/graph_index.cpp:192-216, python/builder.cpp:36-99) and its C++ types
(``QueryParams`` / ``BuildParams``, algorithms/utils/types.h:155-268).

There is no CPU fallback: if the shared library is missing, importing the
binding raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# PANN_LIB_PATH loads another build of the same library (a debug or variant build)
LIB_PATH = os.environ.get("PANN_LIB_PATH") or os.path.join(_HERE, "libparlayann_b200.so")

PANN_OK, PANN_EINVAL, PANN_ENOMEM, PANN_ETIMEOUT, PANN_EDEVICE, PANN_EOVERFLOW, PANN_ESHORT = range(7)
U8, I8, F32 = 0, 1, 2
SCORER_CUDA, SCORER_TENSOR = 0, 1  # pann_search_options::scorer (tile search)
L2, MIPS = 0, 1
PREC_F32, PREC_BF16, PREC_FP8 = 0, 1, 2
PANN_NOALLOC_SCRATCH_BYTES = 32 << 20  # static scratch of pann_search_device_noalloc, per device
_DTYPES = {np.dtype(np.uint8): U8, np.dtype(np.int8): I8, np.dtype(np.float32): F32}
_NP_OF = {U8: np.uint8, I8: np.int8, F32: np.float32}


class PannError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"parlayann_b200 error {code}: {msg}")
        self.code = code


class QueryParams(ctypes.Structure):
    """QueryParams (types.h:233-252): k, beamSize, limit, degree_limit, batch_factor."""

    _fields_ = [
        ("k", ctypes.c_uint32),
        ("beam", ctypes.c_uint32),
        ("limit", ctypes.c_uint64),
        ("degree_limit", ctypes.c_uint32),
        ("batch_factor", ctypes.c_double),
    ]


class SearchOptions(ctypes.Structure):
    """pann_search_options: precision form and re-rank count."""

    _fields_ = [("precision", ctypes.c_int32), ("rerank", ctypes.c_uint32), ("parents", ctypes.c_uint32),
                ("scorer", ctypes.c_uint32)]


class BatchOptions(ctypes.Structure):
    """pann_batch_options: CUDA-graph replay, autotuning, fixed tier-0 shape."""

    _fields_ = [("use_graph", ctypes.c_int32), ("autotune", ctypes.c_int32), ("seen_slots", ctypes.c_uint32),
                ("warps_per_block", ctypes.c_uint32), ("cta_per_query", ctypes.c_int32)]


class RangeParams(ctypes.Structure):
    """pann_range_params: RangeSearch / DoubleBeamRangeSearch parameters (types.h:254-259)."""

    _fields_ = [("beam", ctypes.c_uint32), ("type", ctypes.c_int32), ("radius", ctypes.c_double),
                ("early_stopping_radius", ctypes.c_double), ("early_stopping_count", ctypes.c_uint32)]


RANGE_GREEDY, RANGE_DOUBLING, RANGE_BEAM = 1, 2, 3


class ServerOptions(ctypes.Structure):
    """pann_server_options: slots, admission unit and the bounds of k-NN requests."""

    _fields_ = [("max_batch_queries", ctypes.c_uint32), ("inflight", ctypes.c_uint32), ("max_k", ctypes.c_uint32),
                ("max_beam", ctypes.c_uint32), ("limit", ctypes.c_uint64), ("degree_limit", ctypes.c_uint32),
                ("batch_factor", ctypes.c_double), ("precision", ctypes.c_int32), ("parents", ctypes.c_uint32),
                ("scorer", ctypes.c_uint32), ("scratch_bytes", ctypes.c_uint64)]


class BuildParams(ctypes.Structure):
    """BuildParams fields of the Vamana build (types.h:155-230)."""

    _fields_ = [
        ("R", ctypes.c_uint32),
        ("L", ctypes.c_uint32),
        ("alpha", ctypes.c_double),
        ("num_passes", ctypes.c_int32),
        ("batch_factor", ctypes.c_double),
        ("perm_seed", ctypes.c_uint64),
        ("sort_neighbors", ctypes.c_int32),
    ]


class BuildStats(ctypes.Structure):
    _fields_ = [
        ("seconds", ctypes.c_double),
        ("search_seconds", ctypes.c_double),
        ("prune_seconds", ctypes.c_double),
        ("reverse_seconds", ctypes.c_double),
        ("dist_cmps", ctypes.c_uint64),
        ("visited_total", ctypes.c_uint64),
        ("batches", ctypes.c_uint32),
        ("flagged", ctypes.c_uint32),
        ("search_cmps", ctypes.c_uint64),
        ("prune_candidates", ctypes.c_uint64),
        ("edge_pairs", ctypes.c_uint64),
        ("reprunes", ctypes.c_uint64),
        ("inserted", ctypes.c_uint64),
    ]


# Every symbol include/parlayann_b200.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_U32, _U64, _I = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
SIGNATURES = {
    "pann_index_create": (_I, [ctypes.POINTER(_P), _I, _I, _U64, _U32, _U32]),
    "pann_index_destroy": (_I, [_P]),
    "pann_index_set_points": (_I, [_P, _P, _I]),
    "pann_graph_upload": (_I, [_P, _P, _I]),
    "pann_graph_download": (_I, [_P, _P]),
    "pann_graph_load": (_I, [_P, ctypes.c_char_p]),
    "pann_graph_save": (_I, [_P, ctypes.c_char_p]),
    "pann_search": (_I, [_P, _P, _U32, ctypes.POINTER(QueryParams), _P, _U32, _P, _P, _P, _P, _P]),
    "pann_search_device": (_I, [_P, _P, _U32, ctypes.POINTER(QueryParams), _P, _U32, _P, _P, _P, _P, _P, _P]),
    "pann_search_device_noalloc": (_I, [_P, _P, _U32, ctypes.POINTER(QueryParams), _P, _U32, _P, _P, _P, _P, _P, _P]),
    "pann_search_lists": (_I, [_P, _P, _U32, ctypes.POINTER(QueryParams), _P, _U32, _P, _P, _P, _U32, _P, _P, _P,
                               _P]),
    "pann_index_set_precision": (_I, [_P, _I]),
    "pann_search_ex": (_I, [_P, _P, _U32, ctypes.POINTER(QueryParams), ctypes.POINTER(SearchOptions), _P, _U32, _P,
                            _P, _P, _P, _P, _I, _P]),
    "pann_range_search": (_I, [_P, _P, _U32, ctypes.POINTER(RangeParams), _U32, _P, _P, _U64, _P, _P, _P]),
    "pann_range_fetch": (_I, [_P, _P, _U64]),
    "pann_index_set_quantized": (_I, [_P]),
    "pann_index_quant_params": (_I, [_P, _P, _P]),
    "pann_search_quantized": (_I, [_P, _P, _U32, ctypes.POINTER(QueryParams), ctypes.c_double, _P, _U32, _P, _P, _P,
                                   _P]),
    "pann_range_groundtruth": (_I, [_P, _P, _U32, ctypes.c_float, _P, _P, _U64]),
    "pann_server_create": (_I, [ctypes.POINTER(_P), _P, ctypes.POINTER(ServerOptions), _P, _U32]),
    "pann_server_submit_knn": (_I, [_P, _P, _U32, _U32, _U32, ctypes.POINTER(_U64)]),
    "pann_server_submit_range": (_I, [_P, _P, _U32, ctypes.POINTER(RangeParams), _U32, ctypes.POINTER(_U64)]),
    "pann_server_wait_knn": (_I, [_P, _U64, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "pann_server_wait_range": (_I, [_P, _U64, _P, _P, _U64, ctypes.POINTER(ctypes.c_double)]),
    "pann_server_stats": (_I, [_P, _I, ctypes.POINTER(_U64), ctypes.POINTER(_U64), ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "pann_server_admission": (_I, [_P, _I, ctypes.POINTER(_U64), ctypes.POINTER(_U64), ctypes.POINTER(_U64),
                                   ctypes.POINTER(_U64)]),
    "pann_server_replay": (_I, [_P, _U32, _P, _P, _P, _P, _P, _P, _P, ctypes.POINTER(RangeParams), _U32, _P,
                                ctypes.POINTER(ctypes.c_double)]),
    "pann_server_destroy": (_I, [_P]),
    "pann_batch_create": (_I, [ctypes.POINTER(_P), _P, _U32, ctypes.POINTER(QueryParams), _P, _U32,
                               ctypes.POINTER(SearchOptions), ctypes.POINTER(BatchOptions)]),
    "pann_batch_run": (_I, [_P, _P, _U32, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "pann_batch_mapping": (_I, [_P, ctypes.POINTER(_U32), ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "pann_batch_config": (_I, [_P, _P, _P, _P, _P]),
    "pann_batch_destroy": (_I, [_P]),
    "pann_build": (_I, [_P, ctypes.POINTER(BuildParams), _P, ctypes.POINTER(BuildStats)]),
    "pann_groundtruth": (_I, [_P, _P, _U32, _U32, _P, _P]),
    "pann_score": (_I, [_P, _P, _U32, _P, _U32, _I, _P]),
    "pann_last_error": (ctypes.c_char_p, []),
    "pann_synth_mixture": (_I, [_I, _U64, _U32, _U32, _U64, _U32, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, _I, _P]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libparlayann_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run python -c 'import __graft_entry__ as g; g.build()'")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int):
    if rc != PANN_OK:
        raise PannError(rc, lib().pann_last_error().decode())


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return a.ctypes.data_as(ctypes.c_void_p)


def synth_mixture(dtype: int, n: int, d: int, components: int, seed: int, stream: int,
                  lo: float = 32.0, hi: float = 224.0, sigma: float = 20.0, normalize: bool = False) -> np.ndarray:
    """Seeded Gaussian-mixture rows (see pann_synth_mixture)."""
    out = np.empty((n, d), dtype=_NP_OF[dtype])
    _check(lib().pann_synth_mixture(dtype, n, d, components, seed, stream, lo, hi, sigma, int(normalize), _ptr(out)))
    return out


def batch_schedule(n: int, m: int | None = None, base: float = 2.0, max_fraction: float = 0.02):
    """Prefix-doubling batch bounds of batch_insert (algorithms/vamana/index.h:206-240)."""
    m = n if m is None else m
    max_batch = min(int(max_fraction * float(np.float32(n))), 1000000)
    if max_batch == 0:
        max_batch = n
    out, count, inc = [], 0, 0
    while count < m:
        if base ** inc <= max_batch:
            f = int(base ** inc) - 1
            c = min(int(base ** (inc + 1)) - 1, m)
            count = c
        else:
            f = count
            c = min(count + max_batch, m)
            count += max_batch
        out.append((f, c))
        inc += 1
    return out


def permutation(n: int, seed: int = 0x5EED5EED5EED) -> np.ndarray:
    """Insertion order used when no permutation is given: indices ordered by splitmix64(seed + i)."""
    x = (np.arange(n, dtype=np.uint64) + np.uint64(seed)).astype(np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    return np.argsort(x, kind="stable").astype(np.uint32)


@dataclass
class SearchResult:
    ids: np.ndarray
    dists: np.ndarray
    visited: np.ndarray
    cmps: np.ndarray
    flags: np.ndarray


class Index:
    """Device-resident PointRange + Graph (point_range.h, graph.h) on one GPU."""

    def __init__(self, points: np.ndarray, R: int, metric: int = L2):
        points = np.ascontiguousarray(points)
        self.dtype = _DTYPES[points.dtype]
        self.n, self.d = points.shape
        self.R = R
        self.metric = metric
        h = ctypes.c_void_p()
        _check(lib().pann_index_create(ctypes.byref(h), self.dtype, metric, self.n, self.d, R))
        self._h = h
        _check(lib().pann_index_set_points(self._h, _ptr(points), 0))

    def close(self):
        if getattr(self, "_h", None):
            lib().pann_index_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # graph in the reference layout: n x (R+1), slot 0 = degree
    def set_graph(self, rows: np.ndarray):
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        assert rows.shape == (self.n, self.R + 1)
        _check(lib().pann_graph_upload(self._h, _ptr(rows), 0))

    def get_graph(self) -> np.ndarray:
        out = np.empty((self.n, self.R + 1), dtype=np.uint32)
        _check(lib().pann_graph_download(self._h, _ptr(out)))
        return out

    def save_graph(self, path: str):
        _check(lib().pann_graph_save(self._h, path.encode()))

    def load_graph(self, path: str):
        _check(lib().pann_graph_load(self._h, path.encode()))

    def build(self, L: int, alpha: float, num_passes: int = 1, batch_factor: float = 0.125,
              perm: np.ndarray | None = None, perm_seed: int = 0x5EED5EED5EED, sort_neighbors: bool = True) -> BuildStats:
        bp = BuildParams(self.R, L, alpha, num_passes, batch_factor, perm_seed, int(sort_neighbors))
        st = BuildStats()
        p = None if perm is None else np.ascontiguousarray(perm, dtype=np.uint32)
        _check(lib().pann_build(self._h, ctypes.byref(bp), _ptr(p), ctypes.byref(st)))
        return st

    def set_quantized(self):
        """One-byte scalar-quantized copy of float Euclidean points (pann_index_set_quantized)."""
        _check(lib().pann_index_set_quantized(self._h))

    def quant_params(self):
        slope = np.zeros(1, np.float32)
        offset = np.zeros(1, np.int32)
        _check(lib().pann_index_quant_params(self._h, _ptr(slope), _ptr(offset)))
        return float(slope[0]), int(offset[0])

    def search_quantized(self, queries: np.ndarray, k: int, L: int, rerank_factor: float = 100.0,
                         limit: int | None = None, degree_limit: int | None = None, batch_factor: float = 0.125,
                         starts=(0,)) -> SearchResult:
        """The reference's quantized search with a float re-rank (beam_search_rerank, pann_search_quantized)."""
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        nq = queries.shape[0]
        qp = QueryParams(k, L, self.n if limit is None else limit, self.R if degree_limit is None else degree_limit,
                         batch_factor)
        st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint32))
        ids = np.empty((nq, k), np.uint32)
        dists = np.empty((nq, k), np.float32)
        vis = np.empty(nq, np.uint32)
        cmps = np.empty(nq, np.uint32)
        _check(lib().pann_search_quantized(self._h, _ptr(queries), nq, ctypes.byref(qp), rerank_factor, _ptr(st),
                                           len(st), _ptr(ids), _ptr(dists), _ptr(vis), _ptr(cmps)))
        return SearchResult(ids, dists, vis, cmps, np.zeros(nq, np.uint32))

    def set_precision(self, precision: int):
        """Build the low-precision copy used by the precision form (float32 indexes)."""
        _check(lib().pann_index_set_precision(self._h, precision))

    def score(self, queries: np.ndarray, ids: np.ndarray, precision: int = PREC_F32) -> np.ndarray:
        """Distances of queries[i] to the points ids[i, j] (pann_score): Point::distance exactly, or the
        precision form's approximate score."""
        queries = np.ascontiguousarray(queries, dtype=_NP_OF[self.dtype])
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        out = np.empty(ids.shape, np.float32)
        _check(lib().pann_score(self._h, _ptr(queries), queries.shape[0], _ptr(ids), ids.shape[1], precision,
                                _ptr(out)))
        return out

    def search(self, queries: np.ndarray, k: int, L: int, limit: int | None = None, degree_limit: int | None = None,
               batch_factor: float = 0.125, starts=(0,), allow_short: bool = False, precision: int = PREC_F32,
               rerank: int = 0, parents: int = 0, scorer: int = 0) -> SearchResult:
        queries = np.ascontiguousarray(queries, dtype=_NP_OF[self.dtype])
        nq = queries.shape[0]
        qp = QueryParams(k, L, self.n if limit is None else limit, self.R if degree_limit is None else degree_limit,
                         batch_factor)
        st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint32))
        ids = np.empty((nq, k), np.uint32)
        dists = np.empty((nq, k), np.float32)
        vis = np.empty(nq, np.uint32)
        cmps = np.empty(nq, np.uint32)
        flags = np.empty(nq, np.uint32)
        if precision == PREC_F32 and rerank == 0 and parents == 0:
            rc = lib().pann_search(self._h, _ptr(queries), nq, ctypes.byref(qp), _ptr(st), len(st), _ptr(ids),
                                   _ptr(dists), _ptr(vis), _ptr(cmps), _ptr(flags))
        else:
            opt = SearchOptions(precision, rerank, parents, scorer)
            rc = lib().pann_search_ex(self._h, _ptr(queries), nq, ctypes.byref(qp), ctypes.byref(opt), _ptr(st),
                                      len(st), _ptr(ids), _ptr(dists), _ptr(vis), _ptr(cmps), _ptr(flags), 0, None)
        if not (allow_short and rc == PANN_ESHORT):
            _check(rc)
        return SearchResult(ids, dists, vis, cmps, flags)

    def batch(self, max_queries: int, max_k: int, max_beam: int, limit: int | None = None,
              degree_limit: int | None = None, batch_factor: float = 0.125, starts=(0,), precision: int = PREC_F32,
              rerank: int = 0, use_graph: bool = True, autotune: bool = False, seen_slots: int = 0,
              warps_per_block: int = 0, parents: int = 0, scorer: int = 0, cta_per_query: bool = False) -> "Batch":
        """A reusable batch for queries with per-query k and beam (pann_batch_create)."""
        return Batch(self, max_queries, max_k, max_beam, limit, degree_limit, batch_factor, starts, precision, rerank,
                     use_graph, autotune, seen_slots, warps_per_block, parents, scorer, cta_per_query)

    def range_search(self, queries: np.ndarray, beam: int, radius: float, rtype: int = RANGE_GREEDY, start: int = 0,
                     early_stopping_radius: float = 0.0, early_stopping_count: int = 0):
        """Range search (pann_range_search). Returns dict(ids=[uint32 array per query], offsets, visited, cmps,
        flags); ids are in the reference's answer order."""
        queries = np.ascontiguousarray(queries, dtype=_NP_OF[self.dtype])
        nq = queries.shape[0]
        rp = RangeParams(beam, rtype, radius, early_stopping_radius, early_stopping_count)
        offs = np.zeros(nq + 1, np.uint64)
        vis = np.zeros(nq, np.uint32)
        cmps = np.zeros(nq, np.uint32)
        flags = np.zeros(nq, np.uint32)
        cap = max(1, nq * beam * 4)
        ids = np.zeros(cap, np.uint32)
        rc = lib().pann_range_search(self._h, _ptr(queries), nq, ctypes.byref(rp), start, _ptr(offs), _ptr(ids),
                                     cap, _ptr(vis), _ptr(cmps), _ptr(flags))
        if rc == PANN_EOVERFLOW and int(offs[nq]) > cap:   # the answers are held on the device
            ids = np.zeros(int(offs[nq]), np.uint32)
            rc = lib().pann_range_fetch(self._h, _ptr(ids), len(ids))
        _check(rc)
        lists = [ids[int(offs[i]):int(offs[i + 1])].copy() for i in range(nq)]
        return dict(ids=lists, offsets=offs, visited=vis, cmps=cmps, flags=flags)

    def search_lists(self, queries: np.ndarray, L: int, limit: int | None = None, degree_limit: int | None = None,
                     batch_factor: float = 0.125, starts=(0,), visited_cap: int | None = None):
        """Full beam_search output: frontier (<= L) and sorted visited list per query."""
        queries = np.ascontiguousarray(queries, dtype=_NP_OF[self.dtype])
        nq = queries.shape[0]
        vc = visited_cap or 4 * L + 64
        qp = QueryParams(L, L, self.n if limit is None else limit, self.R if degree_limit is None else degree_limit,
                         batch_factor)
        st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint32))
        fi = np.zeros((nq, L), np.uint32)
        fd = np.zeros((nq, L), np.float32)
        fn = np.zeros(nq, np.uint32)
        vi = np.zeros((nq, vc), np.uint32)
        vd = np.zeros((nq, vc), np.float32)
        vn = np.zeros(nq, np.uint32)
        cm = np.zeros(nq, np.uint32)
        _check(lib().pann_search_lists(self._h, _ptr(queries), nq, ctypes.byref(qp), _ptr(st), len(st), _ptr(fi),
                                       _ptr(fd), _ptr(fn), vc, _ptr(vi), _ptr(vd), _ptr(vn), _ptr(cm)))
        return dict(frontier_ids=fi, frontier_d=fd, frontier_n=fn, visited_ids=vi, visited_d=vd, visited=vn, cmps=cm)

    def groundtruth(self, queries: np.ndarray, k: int):
        queries = np.ascontiguousarray(queries, dtype=_NP_OF[self.dtype])
        ids = np.empty((queries.shape[0], k), np.uint32)
        dd = np.empty((queries.shape[0], k), np.float64)
        _check(lib().pann_groundtruth(self._h, _ptr(queries), queries.shape[0], k, _ptr(ids), _ptr(dd)))
        return ids, dd

    def range_groundtruth(self, queries: np.ndarray, radius: float):
        """Every base id within `radius` of each query, in id order (pann_range_groundtruth). Returns
        (offsets[nq + 1], ids): answer i = ids[offsets[i]:offsets[i + 1]]."""
        queries = np.ascontiguousarray(queries, dtype=_NP_OF[self.dtype])
        nq = queries.shape[0]
        offs = np.zeros(nq + 1, np.uint64)
        rc = lib().pann_range_groundtruth(self._h, _ptr(queries), nq, radius, _ptr(offs), None, 0)
        if rc != PANN_EOVERFLOW:
            _check(rc)
            return offs, np.zeros(0, np.uint32)
        ids = np.zeros(int(offs[nq]), np.uint32)   # the answers are held on the device
        _check(lib().pann_range_fetch(self._h, _ptr(ids), len(ids)))
        return offs, ids


class Batch:
    """Batched form: runs of up to max_queries queries, each with its own k and
    beam, through one persistent launch sequence (optionally a replayed CUDA
    graph). Per query the results equal Index.search with that k and beam."""

    def __init__(self, index: "Index", max_queries, max_k, max_beam, limit, degree_limit, batch_factor, starts,
                 precision, rerank, use_graph, autotune, seen_slots, warps_per_block, parents=0, scorer=0,
                 cta_per_query=False):
        self.index = index
        self.max_k = max_k
        qp = QueryParams(max_k, max_beam, index.n if limit is None else limit,
                         index.R if degree_limit is None else degree_limit, batch_factor)
        st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint32))
        opt = SearchOptions(precision, rerank, parents, scorer)
        bo = BatchOptions(int(use_graph), int(autotune), seen_slots, warps_per_block, int(cta_per_query))
        h = ctypes.c_void_p()
        _check(lib().pann_batch_create(ctypes.byref(h), index.handle, max_queries, ctypes.byref(qp), _ptr(st), len(st),
                                       ctypes.byref(opt), ctypes.byref(bo)))
        self._h = h

    def run(self, queries: np.ndarray, k, beam, allow_short: bool = False) -> SearchResult:
        queries = np.ascontiguousarray(queries, dtype=_NP_OF[self.index.dtype])
        nq = queries.shape[0]
        k = np.ascontiguousarray(np.broadcast_to(np.asarray(k, np.uint32), (nq,)))
        beam = np.ascontiguousarray(np.broadcast_to(np.asarray(beam, np.uint32), (nq,)))
        ids = np.empty((nq, self.max_k), np.uint32)
        dists = np.empty((nq, self.max_k), np.float32)
        vis = np.empty(nq, np.uint32)
        cmps = np.empty(nq, np.uint32)
        flags = np.empty(nq, np.uint32)
        rc = lib().pann_batch_run(self._h, _ptr(queries), nq, _ptr(k), _ptr(beam), _ptr(ids), _ptr(dists), _ptr(vis),
                                  _ptr(cmps), _ptr(flags), 0, None)
        if not (allow_short and rc == PANN_ESHORT):
            _check(rc)
        return SearchResult(ids, dists, vis, cmps, flags)

    def config(self) -> dict:
        s, w, b, g = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_int32()
        _check(lib().pann_batch_config(self._h, ctypes.byref(s), ctypes.byref(w), ctypes.byref(b), ctypes.byref(g)))
        c, m, t = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().pann_batch_mapping(self._h, ctypes.byref(c), ctypes.byref(m), ctypes.byref(t)))
        return dict(seen_slots=s.value, warps_per_block=w.value, blocks=b.value, graph=bool(g.value),
                    cta_per_query=bool(c.value), register_blocks=m.value, tile_rows=t.value)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().pann_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving form (pann_server_*): continuous batching of k-NN requests over
    `inflight` batch slots, range requests on a second worker. While it runs it
    is the only user of its index."""

    def __init__(self, index: "Index", max_batch_queries: int = 1024, inflight: int = 3, max_k: int = 100,
                 max_beam: int = 400, limit: int | None = None, degree_limit: int | None = None,
                 batch_factor: float = 0.125, precision: int = PREC_F32, starts=(0,), parents: int = 0,
                 scorer: int = 0, scratch_bytes: int = 0):
        self.index = index
        o = ServerOptions(max_batch_queries, inflight, max_k, max_beam, index.n if limit is None else limit,
                          index.R if degree_limit is None else degree_limit, batch_factor, precision, parents,
                          scorer, scratch_bytes)
        st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint32))
        h = ctypes.c_void_p()
        _check(lib().pann_server_create(ctypes.byref(h), index.handle, ctypes.byref(o), _ptr(st), len(st)))
        self._h = h
        self._kinds = {}

    def _q(self, queries):
        return np.ascontiguousarray(queries, dtype=_NP_OF[self.index.dtype])

    def submit_knn(self, queries, k: int, beam: int) -> int:
        q = self._q(queries)
        t = ctypes.c_uint64()
        _check(lib().pann_server_submit_knn(self._h, _ptr(q), q.shape[0], k, beam, ctypes.byref(t)))
        self._kinds[t.value] = ("knn", q.shape[0], k)
        return t.value

    def submit_range(self, queries, beam: int, radius: float, rtype: int = RANGE_GREEDY, start: int = 0,
                     early_stopping_radius: float = 0.0, early_stopping_count: int = 0) -> int:
        q = self._q(queries)
        rp = RangeParams(beam, rtype, radius, early_stopping_radius, early_stopping_count)
        t = ctypes.c_uint64()
        _check(lib().pann_server_submit_range(self._h, _ptr(q), q.shape[0], ctypes.byref(rp), start, ctypes.byref(t)))
        self._kinds[t.value] = ("range", q.shape[0], 0)
        return t.value

    def wait(self, ticket: int):
        """k-NN: (ids, dists, latency_s); range: (list of id arrays, latency_s)."""
        kind, nq, k = self._kinds.pop(ticket)
        lat = ctypes.c_double()
        if kind == "knn":
            ids = np.empty((nq, k), np.uint32)
            dists = np.empty((nq, k), np.float32)
            _check(lib().pann_server_wait_knn(self._h, ticket, _ptr(ids), _ptr(dists), ctypes.byref(lat)))
            return ids, dists, lat.value
        offs = np.zeros(nq + 1, np.uint64)
        cap = 1 << 22
        ids = np.empty(cap, np.uint32)
        _check(lib().pann_server_wait_range(self._h, ticket, _ptr(offs), _ptr(ids), cap, ctypes.byref(lat)))
        return [ids[int(offs[i]):int(offs[i + 1])].copy() for i in range(nq)], lat.value

    def stats(self, reset: bool = False) -> dict:
        r, q = ctypes.c_uint64(), ctypes.c_uint64()
        sec, p50, p99 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(lib().pann_server_stats(self._h, int(reset), ctypes.byref(r), ctypes.byref(q), ctypes.byref(sec),
                                       ctypes.byref(p50), ctypes.byref(p99)))
        return dict(requests=r.value, queries=q.value, seconds=sec.value, p50_s=p50.value, p99_s=p99.value)

    def admission(self, reset: bool = False) -> dict:
        """Batches launched, queries they held, the largest scratch a batch used and each slot's scratch."""
        b, q, peak, cap = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().pann_server_admission(self._h, int(reset), ctypes.byref(b), ctypes.byref(q), ctypes.byref(peak),
                                           ctypes.byref(cap)))
        return dict(batches=b.value, queries=q.value, scratch_peak=peak.value, scratch_bytes=cap.value)

    def replay(self, arrival_s, kind, nq, k, beam, q_row, query_pool, range_params: RangeParams | None = None,
               range_start: int = 0):
        """Open-loop load generation in native code; returns (latencies_s, wall_s)."""
        a = np.ascontiguousarray(arrival_s, np.float64)
        n = len(a)
        kd = np.ascontiguousarray(kind, np.uint32)
        nqa = np.ascontiguousarray(nq, np.uint32)
        ka = np.ascontiguousarray(k, np.uint32)
        ba = np.ascontiguousarray(beam, np.uint32)
        rows = np.ascontiguousarray(q_row, np.uint64)
        pool = self._q(query_pool)
        lat = np.zeros(n, np.float64)
        wall = ctypes.c_double()
        rp = range_params if range_params is not None else RangeParams(10, RANGE_BEAM, 0.0, 0.0, 0)
        _check(lib().pann_server_replay(self._h, n, _ptr(a), _ptr(kd), _ptr(nqa), _ptr(ka), _ptr(ba), _ptr(rows),
                                        _ptr(pool), ctypes.byref(rp), range_start, _ptr(lat), ctypes.byref(wall)))
        return lat, wall.value

    def close(self):
        if self._h:
            lib().pann_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def recall_at_k(ids: np.ndarray, gt_ids: np.ndarray, k: int) -> float:
    """recall@k = |result[:k] ∩ gt[:k]| / k averaged over queries (check_nn_recall.h:86-112,
    without the tie extension; see recall_with_ties)."""
    hit = 0
    for a, b in zip(ids[:, :k], gt_ids[:, :k]):
        hit += len(set(a.tolist()) & set(b.tolist()))
    return hit / float(k * ids.shape[0])


def point_distances(queries: np.ndarray, base: np.ndarray, ids: np.ndarray, metric: int = L2) -> np.ndarray:
    """Point::distance of queries[i] to base[ids[i, j]] in the reference's arithmetic, for every
    (i, j): int32 sums returned as float for 8-bit points, and for float points one sequential sum of
    separately rounded float products (euclidian_point.h:54-90, mips_point.h:44-66). Returns float32
    of ids' shape."""
    ids = np.asarray(ids, dtype=np.int64)
    rows = base[ids.ravel()].reshape(ids.shape + (base.shape[1],))
    q = queries[:, None, :]
    if base.dtype != np.float32:
        a = q.astype(np.int64)
        b = rows.astype(np.int64)
        r = ((a - b) ** 2).sum(-1) if metric == L2 else -(a * b).sum(-1)
        return r.astype(np.float32)
    acc = np.zeros(ids.shape, np.float32)
    for t in range(base.shape[1]):
        if metric == L2:
            diff = rows[..., t] - q[..., t]
            acc = acc + diff * diff
        else:
            acc = acc + rows[..., t] * q[..., t]
    return acc if metric == L2 else -acc


def recall_with_ties(ids: np.ndarray, gt_ids: np.ndarray, k: int, queries: np.ndarray, base: np.ndarray,
                     metric: int = L2) -> float:
    """checkRecall's recall@k (check_nn_recall.h:86-112): the true set of a query is its first k
    groundtruth ids plus every later groundtruth id whose distance, recomputed with the reference's
    own float distance, equals that of the k-th; the hits are the true ids among the first k
    reported. Returns hits / (k * nq) rounded to float32, as the reference divides."""
    nq = ids.shape[0]
    m = gt_ids.shape[1]
    if m < k:
        raise ValueError(f"{k}@{k} too large for ground truth data of size {m}")
    truth = np.ascontiguousarray(gt_ids).astype(np.int64)
    keep = np.ones(truth.shape, bool)
    if m > k:
        d = point_distances(queries, base, truth[:, k - 1:], metric)
        keep[:, k:] = d[:, 1:] == d[:, :1]
    rep = np.asarray(ids)[:, :k].astype(np.int64)
    hits = 0
    for b in range(0, nq, 4096):
        t = truth[b:b + 4096]
        hit = (t[:, :, None] == rep[b:b + 4096, None, :]).any(-1) & keep[b:b + 4096]
        hits += int(hit.sum())
    return float(np.float32(hits) / np.float32(k * nq))
