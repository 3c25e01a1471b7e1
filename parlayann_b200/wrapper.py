"""The reference's Python surface (python/wrapper.py, python/_files.py,
python/graph_index.cpp, python/builder.cpp) over this library.

* Files: `vectors_to_file` / `vectors_from_file` / `vectors_metadata_from_file`
  (the .bin point format read by PointRange(char*), point_range.h:74-117:
  int32 n, int32 d, then n*d values), `groundtruth_to_file` /
  `groundtruth_from_file` (the .ibin groundtruth of groundTruth, types.h:38-107:
  int32 n, int32 k, int32 ids[n*k], float dists[n*k]) and
  `range_groundtruth_to_file` / `range_groundtruth_from_file` (the tool's
  write_rangeres, data_tools/compute_range_groundtruth.cpp:64-87: int32 n,
  int32 total, int32 sizes[n], int32 ids[total]).
* `build_vamana_index(metric, dtype, data_dir, index_dir, R, L, alpha,
  two_pass)` (python/wrapper.py:3-24, python/builder.cpp:36-99): reads the
  points, builds the Vamana graph on the GPU (pann_build), writes the graph
  file in the reference format. For mips it normalises the points and sets
  alpha to 1.0 below 100 dimensions and 0.98 up to 200, as the reference's
  builder does, with its batch_factor of 1.0. The reference's builder
  quantises float points to one byte before building; this one builds on the
  points themselves, as knn_index::build_index does.
* `load_index(metric, dtype, data_dir, index_dir)` (python/wrapper.py:96-116)
  and the classes `FloatEuclidianIndex`, `FloatMipsIndex`,
  `UInt8EuclidianIndex`, `UInt8MipsIndex`, `Int8EuclidianIndex`,
  `Int8MipsIndex` (GraphIndex, python/graph_index.cpp:49-120) with
  `batch_search`, `single_search`, `batch_search_from_string` and
  `check_recall` (graph_index.cpp:192-300). The reference binding builds its
  QueryParams with arguments in the wrong slots (a visit limit of 1); here
  `visit_limit <= 0` means no limit (G.size()), the degree limit is the
  graph's, and the start point is 0 as in search_dispatch. `quant=True` on a
  float Euclidian index runs the reference's own quantized search
  (pann_search_quantized: one-byte points, float re-rank of min(100 k, beam)
  entries, as search_dispatch does); on a float mips index it runs the same
  search over Quantized_Mips_Point<8, true> rows, with the query normalised
  first as search_dispatch does.
"""
from __future__ import annotations

from typing import NamedTuple

import numpy as np

from . import L2, MIPS, PREC_F32, Index, recall_with_ties

_DTYPE = {"float": np.float32, "uint8": np.uint8, "int8": np.int8}
_METRIC = {"Euclidian": L2, "mips": MIPS}


class Metadata(NamedTuple):
    num_vectors: int
    dimensions: int


class QueryResponseBatch(NamedTuple):
    identifiers: np.ndarray
    distances: np.ndarray


# ---------------------------------------------------------------- files
def vectors_metadata_from_file(vector_file: str) -> Metadata:
    n, d = np.fromfile(vector_file, dtype=np.int32, count=2)
    return Metadata(int(n), int(d))


def vectors_from_file(vector_file: str, dtype) -> np.ndarray:
    n, d = vectors_metadata_from_file(vector_file)
    return np.fromfile(vector_file, dtype=dtype, offset=8, count=n * d).reshape(n, d)


def vectors_to_file(vector_file: str, vectors: np.ndarray) -> None:
    vectors = np.ascontiguousarray(vectors)
    if vectors.ndim != 2 or vectors.dtype not in (np.float32, np.uint8, np.int8):
        raise ValueError("vectors must be a 2-d float32, uint8 or int8 array")
    with open(vector_file, "wb") as fh:
        fh.write(np.array(vectors.shape, dtype=np.int32).tobytes())
        fh.write(vectors.tobytes())


def groundtruth_to_file(path: str, ids: np.ndarray, dists: np.ndarray) -> None:
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    with open(path, "wb") as fh:
        fh.write(np.array(ids.shape, dtype=np.int32).tobytes())
        fh.write(ids.tobytes())
        fh.write(np.ascontiguousarray(dists, dtype=np.float32).tobytes())


def groundtruth_from_file(path: str):
    n, k = (int(x) for x in np.fromfile(path, dtype=np.int32, count=2))
    ids = np.fromfile(path, dtype=np.int32, offset=8, count=n * k).reshape(n, k)
    dists = np.fromfile(path, dtype=np.float32, offset=8 + 4 * n * k, count=n * k).reshape(n, k)
    return ids.astype(np.uint32), dists


def range_groundtruth_to_file(path: str, offsets: np.ndarray, ids: np.ndarray) -> None:
    offsets = np.asarray(offsets, dtype=np.int64)
    with open(path, "wb") as fh:
        fh.write(np.array([len(offsets) - 1, int(offsets[-1])], dtype=np.int32).tobytes())
        fh.write(np.diff(offsets).astype(np.int32).tobytes())
        fh.write(np.ascontiguousarray(ids, dtype=np.int32).tobytes())


def range_groundtruth_from_file(path: str):
    n, total = (int(x) for x in np.fromfile(path, dtype=np.int32, count=2))
    sizes = np.fromfile(path, dtype=np.int32, offset=8, count=n)
    ids = np.fromfile(path, dtype=np.int32, offset=8 + 4 * n, count=total).astype(np.uint32)
    offsets = np.zeros(n + 1, np.uint64)
    offsets[1:] = np.cumsum(sizes)
    return offsets, ids


def graph_metadata_from_file(graph_file: str):
    """(num_points, max_degree) of a graph file (graph.h:151-166)."""
    n, r = np.fromfile(graph_file, dtype=np.uint32, count=2)
    return int(n), int(r)


# ---------------------------------------------------------------- build
def _normalize(points: np.ndarray) -> np.ndarray:
    """Mips_Point::normalize (mips_point.h:120-129) row by row: float squares summed in double in
    order, one float inverse norm, float products."""
    norm = np.zeros(len(points), np.float64)
    for j in range(points.shape[1]):
        norm += (points[:, j] * points[:, j]).astype(np.float64)
    norm = np.sqrt(norm)
    norm[norm == 0] = 1.0
    inv = (1.0 / norm).astype(np.float32)
    return (points * inv[:, None]).astype(np.float32)


def _mips_prepare(points: np.ndarray, alpha: float):
    """Normalise float points and the reference builder's alpha rule (builder.cpp:46-58)."""
    if points.dtype == np.float32:
        points = _normalize(points)
    d = points.shape[1]
    if d <= 200:
        alpha = 1.0 if d < 100 else 0.98
    return points, alpha


def build_vamana_index(metric, dtype, data_dir, index_dir, R, L, alpha, two_pass):
    if metric not in _METRIC:
        raise Exception("Invalid metric " + str(metric))
    if dtype not in _DTYPE:
        raise Exception("Invalid data type " + str(dtype))
    points = vectors_from_file(data_dir, _DTYPE[dtype])
    if metric == "mips":
        points, alpha = _mips_prepare(points, alpha)
    idx = Index(points, int(R), _METRIC[metric])
    try:
        # BuildParams(R, L, alpha, passes) leaves batch_factor at 1.0 (types.h:176,209)
        idx.build(int(L), float(alpha), 2 if two_pass else 1, batch_factor=1.0)
        idx.save_graph(index_dir)
    finally:
        idx.close()


# ---------------------------------------------------------------- search
class GraphIndex:
    """A graph file and its points on the GPU (GraphIndex, python/graph_index.cpp:49-120). The *Index
    classes fix the point type and metric; GraphIndex itself takes them as keywords."""

    _metric = None
    _dtype = None

    def __init__(self, data_path: str, index_path: str, hnsw: bool = False, *, metric=None, dtype=None):
        if hnsw:
            raise NotImplementedError("HNSW indexes are not part of this library")
        self.metric = self._metric if metric is None else metric
        dt = self._dtype if dtype is None else dtype
        if self.metric is None or dt is None:
            raise ValueError("GraphIndex needs metric= and dtype= (or use one of the *Index classes)")
        points = vectors_from_file(data_path, dt)
        if self.metric == MIPS and points.dtype == np.float32:
            points, _ = _mips_prepare(points, 1.0)
        n, R = graph_metadata_from_file(index_path)
        if n != points.shape[0]:
            raise ValueError("graph size and point size do not match")
        self.points = points
        self.index = Index(points, R, self.metric)
        self.index.load_graph(index_path)
        self._lowprec = False
        self._quantized = False

    def close(self):
        self.index.close()

    def _search(self, queries, knn, beam_width, quant, visit_limit):
        queries = np.ascontiguousarray(queries, dtype=self.points.dtype)
        if quant and self.metric == MIPS and queries.dtype == np.float32:
            queries = _normalize(queries)   # search_dispatch normalises the query on its quantized path only
        limit = None if visit_limit is None or visit_limit <= 0 else int(visit_limit)
        if quant and self.points.dtype == np.float32:
            if not self._quantized:
                self.index.set_quantized()
                self._quantized = True
            r = self.index.search_quantized(queries, int(knn), int(beam_width), limit=limit)
        else:
            r = self.index.search(queries, int(knn), int(beam_width), limit=limit, precision=PREC_F32,
                                  allow_short=True)
        return r.ids, r.dists

    def batch_search(self, queries, knn, beam_width, quant=False, visit_limit=-1) -> QueryResponseBatch:
        ids, dists = self._search(queries, knn, beam_width, quant, visit_limit)
        return QueryResponseBatch(ids, dists)

    def single_search(self, q, knn, beam_width, quant=False, visit_limit=-1) -> np.ndarray:
        ids, _ = self._search(np.asarray(q).reshape(1, -1), knn, beam_width, quant, visit_limit)
        return ids[0]

    def batch_search_from_string(self, queries, knn, beam_width, quant=False, visit_limit=-1) -> QueryResponseBatch:
        return self.batch_search(vectors_from_file(queries, self.points.dtype), knn, beam_width, quant, visit_limit)

    def check_recall(self, queries_file, graph_file, neighbors, k) -> float:
        """Recall with ties at the k-th groundtruth distance, as graph_index.cpp:254-300 counts it;
        `graph_file` is the .ibin groundtruth. Prints and returns the recall."""
        gt_ids, _ = groundtruth_from_file(graph_file)
        queries = vectors_from_file(queries_file, self.points.dtype)
        neighbors = np.asarray(neighbors)
        if (neighbors[:, :k] >= self.points.shape[0]).any():
            raise ValueError("neighbor reported by query out of range")
        recall = recall_with_ties(neighbors, gt_ids, k, queries, self.points, self.metric)
        print(f"Recall: {recall:.6g}")
        return recall


def _distances(q: np.ndarray, rows: np.ndarray, metric: int) -> np.ndarray:
    """Point::distance of q against each row, in the reference's arithmetic: integer sums for 8-bit
    types, and for float a sequential sum of unfused float products (euclidian_point.h:83-90,
    mips_point.h:60-66)."""
    if q.dtype != np.float32:
        a = q.astype(np.int64)
        b = rows.astype(np.int64)
        r = ((a - b) ** 2).sum(1) if metric == L2 else -(a * b).sum(1)
        return r.astype(np.float32)
    r = np.zeros(len(rows), np.float32)
    for j in range(q.shape[0]):
        if metric == L2:
            t = np.float32(q[j]) - rows[:, j]
            r = r + t * t
        else:
            r = r + np.float32(q[j]) * rows[:, j]
    return r if metric == L2 else -r


def _index_class(name, dtype, metric):
    return type(name, (GraphIndex,), {"_dtype": dtype, "_metric": metric,
                                      "__doc__": f"GraphIndex over {np.dtype(dtype).name} points, "
                                                 f"{'Euclidian' if metric == L2 else 'mips'} distance."})


FloatEuclidianIndex = _index_class("FloatEuclidianIndex", np.float32, L2)
FloatMipsIndex = _index_class("FloatMipsIndex", np.float32, MIPS)
UInt8EuclidianIndex = _index_class("UInt8EuclidianIndex", np.uint8, L2)
UInt8MipsIndex = _index_class("UInt8MipsIndex", np.uint8, MIPS)
Int8EuclidianIndex = _index_class("Int8EuclidianIndex", np.int8, L2)
Int8MipsIndex = _index_class("Int8MipsIndex", np.int8, MIPS)


def load_index(metric, dtype, data_dir, index_dir, hnsw=False):
    if metric not in _METRIC:
        raise Exception("Invalid metric")
    if dtype not in _DTYPE:
        raise Exception("Invalid data type")
    cls = {("Euclidian", "float"): FloatEuclidianIndex, ("mips", "float"): FloatMipsIndex,
           ("Euclidian", "uint8"): UInt8EuclidianIndex, ("mips", "uint8"): UInt8MipsIndex,
           ("Euclidian", "int8"): Int8EuclidianIndex, ("mips", "int8"): Int8MipsIndex}[(metric, dtype)]
    return cls(data_dir, index_dir, hnsw)
