// parlayANN drop-in host API over the parlayann_b200 C ABI.
//
// Mirrors the reference's types and free functions for the beam-search /
// Vamana-build path, with the same names and argument meaning, so code
// written against ParlayANN's headers compiles against this one:
//
//   QueryParams, BuildParams          algorithms/utils/types.h:155-268
//   Euclidian_Point<T>, Mips_Point<T> algorithms/utils/euclidian_point.h:92-248,
//                                     algorithms/utils/mips_point.h:68-144
//   PointRange<Point>                 algorithms/utils/point_range.h:43-141
//   Graph<indexType>, edgeRange       algorithms/utils/graph.h:45-255
//   stats<indexType>                  algorithms/utils/stats.h:120-155
//   groundTruth<T>                    algorithms/utils/types.h:38-107
//   beam_search, searchAll, qsearchAll algorithms/utils/beamSearch.h:420-646
//   RangeSearch, DoubleBeamRangeSearch algorithms/utils/rangeSearch.h:183-276,
//                                     algorithms/utils/doublingSearch.h:50-157
//   knn_index<PR,QPR,indexType>::build_index   algorithms/vamana/index.h:42-186
//
// Points and graphs live on the host as in the reference; the first search or
// build on a (Graph, PointRange) pair uploads them to the GPU (a cached device
// index kept with the Graph, refreshed when the graph or the points change).
// Errors that make the reference abort() print a message and abort() here too.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../parlayann_b200.h"

namespace parlayANN {

inline void pann_check(int rc, const char* where) {
  if (rc != PANN_OK) {
    std::cout << "ERROR in " << where << ": " << pann_last_error() << std::endl;
    std::abort();
  }
}

// ---------------------------------------------------------------- params
enum rangeQueryType { None, Greedy, Doubling, Beam };  // types.h:153

struct QueryParams {
  long k;
  long beamSize;
  long limit;
  long degree_limit;
  double rerank_factor = 100;
  double batch_factor = .125;
  bool is_early_stop = false;
  double early_stopping_radius = 0;
  double early_stopping_count = 0;
  rangeQueryType range_query_type = None;
  double radius = 0;
  QueryParams(long k, long Q, long limit, long dg, double rerank_factor = 100, double batch_factor = .125)
      : k(k), beamSize(Q), limit(limit), degree_limit(dg), rerank_factor(rerank_factor), batch_factor(batch_factor) {}
  // range search (types.h:254-259)
  QueryParams(long k, long Q, long limit, long dg, long es, double esr, long esc, rangeQueryType range_query_type,
              double radius)
      : k(k), beamSize(Q), limit(limit), degree_limit(dg), is_early_stop(es), early_stopping_radius(esr),
        early_stopping_count((double)esc), range_query_type(range_query_type), radius(radius) {}
  QueryParams() : k(0), beamSize(0), limit(0), degree_limit(0) {}
  pann_query_params c() const {
    pann_query_params q;
    q.k = (uint32_t)k;
    q.beam = (uint32_t)beamSize;
    q.limit = (uint64_t)limit;
    q.degree_limit = (uint32_t)degree_limit;
    q.batch_factor = batch_factor;
    return q;
  }
};

struct BuildParams {
  long R = 0;
  long L = 0;
  double alpha = 1.0;
  int num_passes = 1;
  double rerank_factor = 100;
  double batch_factor = 1.0;  // the reference's default for this constructor (types.h:176)
  int single_batch = 0;
  bool verbose = false;
  BuildParams() {}
  BuildParams(long R, long L, double a, int num_passes, bool verbose = false)
      : R(R), L(L), alpha(a), num_passes(num_passes), verbose(verbose) {}
  long max_degree() { return R; }
};

// ---------------------------------------------------------------- points
// Host distance functions, restated from euclidian_point.h:54-90 and
// mips_point.h:44-66 (sequential sums), for callers that score points on the host.
template <typename T>
inline float pann_host_distance(const T* p, const T* q, unsigned d, int metric) {
  if constexpr (std::is_same<T, float>::value) {
    float r = 0.0f;
    if (metric == PANN_L2)
      for (unsigned i = 0; i < d; i++) { float t = q[i] - p[i]; float s = t * t; r = r + s; }
    else
      for (unsigned i = 0; i < d; i++) { float s = q[i] * p[i]; r = r + s; }
    return metric == PANN_L2 ? r : -r;
  } else {
    int32_t r = 0;
    for (unsigned i = 0; i < d; i++) {
      int32_t a = (int32_t)p[i], b = (int32_t)q[i];
      r += metric == PANN_L2 ? (a - b) * (a - b) : a * b;
    }
    return metric == PANN_L2 ? (float)r : -((float)r);
  }
}

template <typename T> struct pann_dtype_of;
template <> struct pann_dtype_of<uint8_t> { static constexpr int value = PANN_U8; };
template <> struct pann_dtype_of<int8_t> { static constexpr int value = PANN_I8; };
template <> struct pann_dtype_of<float> { static constexpr int value = PANN_F32; };

template <typename T_, int METRIC>
struct PannPoint {
  using T = T_;
  using distanceType = float;
  using byte = uint8_t;
  static constexpr int pann_metric = METRIC;
  static constexpr bool is_metric = METRIC == PANN_L2;
  // slope/offset: one-byte scalar quantization (euclidian_point.h:98-108)
  struct parameters {
    float slope;
    int32_t offset;
    int dims;
    parameters() : slope(0), offset(0), dims(0) {}
    parameters(int d) : slope(1.0f), offset(0), dims(d) {}
    parameters(float min_val, float max_val, int d)
        : slope(255.0f / (max_val - min_val)), offset((int32_t)std::round(min_val * slope)), dims(d) {}
    int num_bytes() const { return dims * (int)sizeof(T); }
  };
  // generate_parameters (euclidian_point.h:214-240) for one-byte points: the
  // minimum and maximum value with 0 included; all non-negative integers give
  // [0, 255]
  template <class PR>
  static parameters generate_parameters(const PR& pr) {
    static_assert(std::is_same<T, uint8_t>::value, "scalar quantization targets one-byte points");
    float min_val = 0.0f, max_val = 0.0f;
    bool all_ints = true;
    const auto* v = pr.data();
    for (size_t i = 0; i < pr.size() * (size_t)pr.dimension(); i++) {
      const float x = (float)v[i];
      all_ints = all_ints && (x >= 0) && (x - (float)(long)x) == 0;
      min_val = std::min(min_val, x);
      max_val = std::max(max_val, x);
    }
    if (all_ints) {
      if (max_val < 256) max_val = 255;
      min_val = 0;
    }
    return parameters(min_val, max_val, (int)pr.dimension());
  }
  // translate_point (euclidian_point.h:188-212): round(x * slope) - offset in [0, 255]
  template <class SrcPoint>
  static void translate_point(byte* out, const SrcPoint& p, const parameters& params) {
    static_assert(std::is_same<T, uint8_t>::value, "scalar quantization targets one-byte points");
    for (int j = 0; j < params.dims; j++) {
      if (params.slope == 1.0f && params.offset == 0) {
        out[j] = (T)p[j];
        continue;
      }
      int64_t r = (int64_t)std::round((float)p[j] * params.slope) - params.offset;
      out[j] = (T)(r < 0 ? 0 : (r > 255 ? 255 : r));
    }
  }
  PannPoint() : values(nullptr), id_(-1), params(0) {}
  PannPoint(byte* v, long id, parameters p) : values((T*)v), id_(id), params(p) {}
  T operator[](long i) const { return values[i]; }
  float distance(const PannPoint& x) const { return pann_host_distance(values, x.values, params.dims, METRIC); }
  bool same_as(const PannPoint& q) const { return values == q.values; }
  long id() const { return id_; }
  void prefetch() const {}
  static distanceType d_min() { return METRIC == PANN_L2 ? 0.0f : -std::numeric_limits<float>::max(); }
  T* values;
  long id_;
  parameters params;
};
template <typename T> using Euclidian_Point = PannPoint<T, PANN_L2>;
template <typename T> using Mips_Point = PannPoint<T, PANN_MIPS>;

template <class Point_>
struct PointRange {
  using Point = Point_;
  using T = typename Point::T;
  using parameters = typename Point::parameters;
  parameters params;

  PointRange() : n(0) {}
  // .bin file: uint32 n, uint32 d, then n*d values (point_range.h:74-117)
  PointRange(char* filename) : n(0) {
    if (filename == nullptr) return;
    std::ifstream reader(filename, std::ios::binary);
    if (!reader.is_open()) {
      std::cout << "Data file " << filename << " not found" << std::endl;
      std::abort();
    }
    uint32_t num_points = 0, d = 0;
    reader.read((char*)&num_points, 4);
    reader.read((char*)&d, 4);
    n = num_points;
    params = parameters((int)d);
    data_ = std::make_shared<std::vector<T>>((size_t)n * d);
    reader.read((char*)data_->data(), (std::streamsize)(sizeof(T) * (size_t)n * d));
    if (!reader) {
      std::cout << "Data file " << filename << " is truncated" << std::endl;
      std::abort();
    }
  }
  // from memory (copied)
  PointRange(const T* rows, size_t num, int dims) : params(dims), n(num) {
    data_ = std::make_shared<std::vector<T>>(rows, rows + num * (size_t)dims);
  }
  // a quantized copy of another range (point_range.h:55-71): with the given
  // parameters, or with parameters generated from that range
  template <class PR, typename std::enable_if<!std::is_same<typename PR::T, T>::value, int>::type = 0>
  PointRange(const PR& pr, const parameters& p) : params(p), n(pr.size()) {
    data_ = std::make_shared<std::vector<T>>(pr.size() * (size_t)p.dims);
    for (size_t i = 0; i < n; i++) Point::translate_point((uint8_t*)(data_->data() + i * (size_t)p.dims), pr[(long)i], p);
  }
  template <class PR, typename std::enable_if<!std::is_same<typename PR::T, T>::value, int>::type = 0>
  explicit PointRange(const PR& pr) : PointRange(pr, Point::generate_parameters(pr)) {}
  size_t size() const { return n; }
  long dimension() const { return params.dims; }
  unsigned int get_dims() const { return params.dims; }
  Point operator[](long i) const {
    if (i > (long)n) {
      std::cout << "ERROR: point index out of range: " << i << " from range " << n << ", " << std::endl;
      std::abort();
    }
    return Point((uint8_t*)(data_->data() + (size_t)i * params.dims), i, params);
  }
  const T* data() const { return data_ ? data_->data() : nullptr; }

 private:
  size_t n;
  std::shared_ptr<std::vector<T>> data_;
};

// ---------------------------------------------------------------- graph
struct PannDevice {
  pann_index* idx = nullptr;
  const void* points = nullptr;
  int dtype = -1, metric = -1;
  bool quantized = false;  // pann_index_set_quantized done on idx
  ~PannDevice() {
    if (idx) pann_index_destroy(idx);
  }
};

template <typename indexType>
struct edgeRange {
  edgeRange(indexType* row, long maxDeg, indexType id, bool* dirty) : e(row), maxDeg(maxDeg), id_(id), dirty(dirty) {}
  size_t size() const { return e[0]; }
  indexType id() const { return id_; }
  indexType operator[](indexType j) const {
    if (j > e[0]) {
      std::cout << "ERROR: index exceeds degree while accessing neighbors" << std::endl;
      std::abort();
    }
    return e[j + 1];
  }
  template <typename rangeType>
  void update_neighbors(const rangeType& r) {
    if ((long)r.size() > maxDeg) {
      std::cout << "ERROR in update_neighbors: cannot exceed max degree " << maxDeg << std::endl;
      std::abort();
    }
    e[0] = (indexType)r.size();
    for (size_t i = 0; i < r.size(); i++) e[i + 1] = r[i];
    *dirty = true;
  }
  void append_neighbor(indexType nbh) {
    if ((long)e[0] == maxDeg) {
      std::cout << "ERROR in append_neighbor: cannot exceed max degree " << maxDeg << std::endl;
      std::abort();
    }
    e[e[0] + 1] = nbh;
    e[0] += 1;
    *dirty = true;
  }
  void clear_neighbors() {
    e[0] = 0;
    *dirty = true;
  }
  template <typename F>
  void sort(F&& less) {
    std::sort(e + 1, e + 1 + e[0], less);
    *dirty = true;
  }
  indexType* begin() const { return e + 1; }
  indexType* end() const { return e + 1 + e[0]; }
  void prefetch() const {}

 private:
  indexType* e;
  long maxDeg;
  indexType id_;
  bool* dirty;
};

template <typename indexType_>
struct Graph {
  using indexType = indexType_;
  static_assert(sizeof(indexType) == 4, "the device graph stores 32-bit ids");
  Graph() : n(0), maxDeg(0) {}
  Graph(long maxDeg, size_t n) : n(n), maxDeg(maxDeg), rows(std::make_shared<std::vector<indexType>>(n * (maxDeg + 1), 0)) {}
  // the reference's graph file (graph.h:151-208)
  Graph(char* gFile) {
    std::ifstream reader(gFile, std::ios::binary);
    if (!reader.is_open()) {
      std::cout << "graph file " << gFile << " not found" << std::endl;
      std::abort();
    }
    uint32_t pre[2];
    reader.read((char*)pre, 8);
    n = pre[0];
    maxDeg = pre[1];
    rows = std::make_shared<std::vector<indexType>>(n * (maxDeg + 1), 0);
    std::vector<uint32_t> deg(n);
    reader.read((char*)deg.data(), 4 * (std::streamsize)n);
    for (size_t i = 0; i < n; i++) {
      indexType* r = rows->data() + i * (maxDeg + 1);
      r[0] = deg[i];
      reader.read((char*)(r + 1), 4 * (std::streamsize)deg[i]);
    }
    if (!reader) {
      std::cout << "graph file " << gFile << " is truncated" << std::endl;
      std::abort();
    }
  }
  long max_degree() const { return maxDeg; }
  size_t size() const { return n; }
  edgeRange<indexType> operator[](indexType i) const {
    if (i > n) {
      std::cout << "ERROR: graph index out of range: " << i << std::endl;
      std::abort();
    }
    return edgeRange<indexType>(rows->data() + (size_t)i * (maxDeg + 1), maxDeg, i, &dirty_->v);
  }
  // graph.h:210-237
  void save(char* oFile) {
    std::ofstream w(oFile, std::ios::binary);
    uint32_t pre[2] = {(uint32_t)n, (uint32_t)maxDeg};
    w.write((char*)pre, 8);
    for (size_t i = 0; i < n; i++) w.write((char*)(rows->data() + i * (maxDeg + 1)), 4);
    for (size_t i = 0; i < n; i++) {
      const indexType* r = rows->data() + i * (maxDeg + 1);
      w.write((char*)(r + 1), 4 * (std::streamsize)r[0]);
    }
  }
  const indexType* raw_rows() const { return rows->data(); }
  indexType* raw_rows() { return rows->data(); }

  // device mirror of (this graph, the given points)
  template <class PR>
  pann_index* device(const PR& Points) const {
    using P = typename PR::Point;
    const int dt = pann_dtype_of<typename P::T>::value, mt = P::pann_metric;
    PannDevice& d = *dev_;
    if (!d.idx || d.points != (const void*)Points.data() || d.dtype != dt || d.metric != mt) {
      if (d.idx) pann_index_destroy(d.idx);
      d.idx = nullptr;
      pann_check(pann_index_create(&d.idx, dt, mt, n, (uint32_t)Points.dimension(), (uint32_t)maxDeg),
                 "pann_index_create");
      pann_check(pann_index_set_points(d.idx, Points.data(), 0), "pann_index_set_points");
      d.points = Points.data();
      d.dtype = dt;
      d.metric = mt;
      d.quantized = false;
      dirty_->v = true;
    }
    if (dirty_->v) {
      pann_check(pann_graph_upload(d.idx, (const uint32_t*)rows->data(), 0), "pann_graph_upload");
      dirty_->v = false;
    }
    return d.idx;
  }
  // the device index with its one-byte quantized copy (pann_index_set_quantized)
  template <class PR>
  pann_index* device_quantized(const PR& Points) const {
    pann_index* idx = device(Points);
    if (!dev_->quantized) {
      pann_check(pann_index_set_quantized(idx), "pann_index_set_quantized");
      dev_->quantized = true;
    }
    return idx;
  }
  void pull_from_device() {
    pann_check(pann_graph_download(dev_->idx, (uint32_t*)rows->data()), "pann_graph_download");
    dirty_->v = false;
  }

 private:
  struct Flag { bool v = true; };
  size_t n;
  long maxDeg;
  std::shared_ptr<std::vector<indexType>> rows;
  std::shared_ptr<PannDevice> dev_ = std::make_shared<PannDevice>();
  std::shared_ptr<Flag> dirty_ = std::make_shared<Flag>();
};

// ---------------------------------------------------------------- stats, groundtruth
template <typename indexType>
struct stats {
  stats() {}
  stats(size_t n) : visited(n, 0), distances(n, 0) {}
  std::vector<indexType> visited;
  std::vector<indexType> distances;
  void increment_dist(indexType i, indexType j) { distances[i] += j; }
  void increment_visited(indexType i, indexType j) { visited[i] += j; }
  std::vector<indexType> visited_stats() { return statistics(visited); }
  std::vector<indexType> dist_stats() { return statistics(distances); }
  void clear() {
    std::fill(visited.begin(), visited.end(), 0);
    std::fill(distances.begin(), distances.end(), 0);
  }
  // mean and the 0.99 quantile (stats.h:147-153)
  static std::vector<indexType> statistics(std::vector<indexType> s) {
    long sum = 0;
    for (auto x : s) sum += (long)x;
    indexType avg = (indexType)(sum / (long)s.size());
    std::sort(s.begin(), s.end());
    indexType tail = s[(size_t)(.99 * ((float)s.size()))];
    return {avg, tail};
  }
};

// .ibin groundtruth: int32 n, int32 k, ids[n*k], float dists[n*k] (types.h:38-107)
template <typename T>
struct groundTruth {
  std::vector<T> coords;
  std::vector<float> dists;
  long dim = 0;
  size_t n = 0;
  groundTruth() {}
  groundTruth(char* gtFile) {
    if (!gtFile) return;
    std::ifstream r(gtFile, std::ios::binary);
    if (!r.is_open()) {
      std::cout << "groundtruth file " << gtFile << " not found" << std::endl;
      std::abort();
    }
    int32_t pre[2];
    r.read((char*)pre, 8);
    n = pre[0];
    dim = pre[1];
    coords.resize(n * dim);
    dists.resize(n * dim);
    r.read((char*)coords.data(), sizeof(T) * n * dim);
    r.read((char*)dists.data(), 4 * n * dim);
  }
  T coordinates(long i, long j) const { return coords[i * dim + j]; }
  float distances(long i, long j) const { return dists[i * dim + j]; }
  size_t size() const { return n; }
  long dimension() const { return dim; }
};

// ---------------------------------------------------------------- search
template <typename indexType>
using pann_pairs = std::vector<std::pair<indexType, float>>;

// beam_search (beamSearch.h:420-427): ((frontier, visited), full_dist_cmps)
template <typename Point, typename PointRange_, typename indexType>
std::pair<std::pair<pann_pairs<indexType>, pann_pairs<indexType>>, size_t>
beam_search(const Point p, const Graph<indexType>& G, const PointRange_& Points,
            const std::vector<indexType> starting_points, const QueryParams& QP) {
  pann_index* idx = G.device(Points);
  pann_query_params q = QP.c();
  const uint32_t L = (uint32_t)QP.beamSize;
  uint32_t vcap = 4 * L + 256;
  for (;;) {
    std::vector<uint32_t> fi(L), vi(vcap);
    std::vector<float> fd(L), vd(vcap);
    uint32_t fn = 0, vn = 0, cm = 0;
    std::vector<uint32_t> st(starting_points.begin(), starting_points.end());
    int rc = pann_search_lists(idx, p.values, 1, &q, st.data(), (uint32_t)st.size(), fi.data(), fd.data(), &fn, vcap,
                               vi.data(), vd.data(), &vn, &cm);
    if (rc == PANN_EOVERFLOW && vcap < (1u << 24)) {
      vcap *= 4;
      continue;
    }
    pann_check(rc, "beam_search");
    pann_pairs<indexType> fr, vis;
    for (uint32_t j = 0; j < fn; j++) fr.push_back({fi[j], fd[j]});
    for (uint32_t j = 0; j < vn; j++) vis.push_back({vi[j], vd[j]});
    return {{fr, vis}, (size_t)cm};
  }
}

template <typename Point, typename PointRange_, typename indexType>
std::pair<std::pair<pann_pairs<indexType>, pann_pairs<indexType>>, size_t>
beam_search(const Point p, const Graph<indexType>& G, const PointRange_& Points, const indexType starting_point,
            const QueryParams& QP) {
  return beam_search(p, G, Points, std::vector<indexType>{starting_point}, QP);
}

template <typename PointRange_, typename indexType>
std::vector<std::vector<indexType>> pann_batch(const PointRange_& Query_Points, const Graph<indexType>& G,
                                               const PointRange_& Base_Points, stats<indexType>& QueryStats,
                                               const std::vector<indexType>& starts, const QueryParams& QP,
                                               const char* who) {
  if (QP.k > QP.beamSize) {
    std::cout << "Error: beam search parameter Q = " << QP.beamSize << " same size or smaller than k = " << QP.k
              << std::endl;
    std::abort();
  }
  pann_index* idx = G.device(Base_Points);
  pann_query_params q = QP.c();
  const size_t nq = Query_Points.size(), k = (size_t)QP.k;
  std::vector<uint32_t> ids(nq * k), vis(nq), cmps(nq);
  std::vector<uint32_t> st(starts.begin(), starts.end());
  pann_check(pann_search(idx, Query_Points.data(), (uint32_t)nq, &q, st.data(), (uint32_t)st.size(), ids.data(),
                         nullptr, vis.data(), cmps.data(), nullptr),
             who);
  std::vector<std::vector<indexType>> out(nq);
  for (size_t i = 0; i < nq; i++) {
    out[i].assign(ids.begin() + i * k, ids.begin() + (i + 1) * k);
    if (QueryStats.visited.size() == nq) {
      QueryStats.increment_visited((indexType)i, vis[i]);
      QueryStats.increment_dist((indexType)i, cmps[i]);
    }
  }
  return out;
}

// searchAll (beamSearch.h:492-526)
template <typename PointRange_, typename indexType>
std::vector<std::vector<indexType>> searchAll(PointRange_& Query_Points, Graph<indexType>& G,
                                              PointRange_& Base_Points, stats<indexType>& QueryStats,
                                              std::vector<indexType> starting_points, QueryParams& QP) {
  return pann_batch(Query_Points, G, Base_Points, QueryStats, starting_points, QP, "searchAll");
}
template <typename PointRange_, typename indexType>
std::vector<std::vector<indexType>> searchAll(PointRange_& Query_Points, Graph<indexType>& G,
                                              PointRange_& Base_Points, stats<indexType>& QueryStats,
                                              indexType starting_point, QueryParams& QP) {
  return pann_batch(Query_Points, G, Base_Points, QueryStats, std::vector<indexType>{starting_point}, QP, "searchAll");
}

// qsearchAll (beamSearch.h:599-646). Unquantized (the three point ranges the
// same), or float Euclidian points with one-byte quantized ranges (QPR =
// PointRange<Euclidian_Point<uint8_t>>, QQ the same range: no second level),
// where each query runs beam_search_rerank (beamSearch.h:529-597) through
// pann_search_quantized. The quantized ranges must carry the parameters the
// device derives from the base points (PointRange<...>(Base_Points), and the
// queries translated with Q_Base_Points.params).
template <typename PR, typename QPR, typename QQPR, typename indexType>
std::vector<std::vector<indexType>> qsearchAll(const PR& Query_Points, const QPR& Q_Query_Points,
                                               const QQPR& QQ_Query_Points, const Graph<indexType>& G,
                                               const PR& Base_Points, const QPR& Q_Base_Points,
                                               const QQPR& QQ_Base_Points, stats<indexType>& QueryStats,
                                               const indexType starting_point, const QueryParams& QP,
                                               bool random = false) {
  if constexpr (std::is_same<typename PR::T, float>::value && std::is_same<typename QPR::T, uint8_t>::value &&
                PR::Point::pann_metric == PANN_L2 && QPR::Point::pann_metric == PANN_L2) {
    if ((const void*)&QQ_Base_Points != (const void*)&Q_Base_Points || random) {
      std::cout << "ERROR: qsearchAll supports one quantization level from a fixed start point" << std::endl;
      std::abort();
    }
    (void)Q_Query_Points;
    (void)QQ_Query_Points;
    pann_index* idx = G.device_quantized(Base_Points);
    float slope = 0.0f;
    int32_t offset = 0;
    pann_check(pann_index_quant_params(idx, &slope, &offset), "pann_index_quant_params");
    if (slope != Q_Base_Points.params.slope || offset != Q_Base_Points.params.offset) {
      std::cout << "ERROR: the quantized base points were not made from Base_Points" << std::endl;
      std::abort();
    }
    const size_t nq = Query_Points.size(), k = (size_t)QP.k;
    std::vector<uint32_t> ids(nq * k), vis(nq), cmps(nq);
    std::vector<float> dists(nq * k);
    const uint32_t start = (uint32_t)starting_point;
    pann_query_params qp = QP.c();
    pann_check(pann_search_quantized(idx, Query_Points.data(), (uint32_t)nq, &qp, QP.rerank_factor, &start, 1,
                                     ids.data(), dists.data(), vis.data(), cmps.data()),
               "qsearchAll (quantized)");
    std::vector<std::vector<indexType>> out(nq);
    for (size_t i = 0; i < nq; i++) {
      out[i].assign(ids.begin() + (long)(i * k), ids.begin() + (long)((i + 1) * k));
      if (QueryStats.visited.size() > i) {
        QueryStats.increment_visited((indexType)i, vis[i]);
        QueryStats.increment_dist((indexType)i, cmps[i]);
      }
    }
    return out;
  }
  if ((const void*)&Q_Base_Points != (const void*)&Base_Points ||
      (const void*)&QQ_Base_Points != (const void*)&Base_Points || random) {
    std::cout << "ERROR: qsearchAll supports the unquantized search from a fixed start point" << std::endl;
    std::abort();
  }
  (void)Q_Query_Points;
  (void)QQ_Query_Points;
  return pann_batch(Query_Points, G, Base_Points, QueryStats, std::vector<indexType>{starting_point}, QP,
                    "qsearchAll");
}

// ---------------------------------------------------------------- range search
// One pann_range_search over the given query rows; answers in the reference's
// order, QueryStats incremented as the reference does.
template <typename PointRange_, typename indexType>
std::vector<std::vector<indexType>> pann_range_batch(const PointRange_& Query_Points, const std::vector<long>& rows,
                                                     const Graph<indexType>& G, const PointRange_& Base_Points,
                                                     stats<indexType>& QueryStats, indexType start,
                                                     const QueryParams& QP, int type) {
  pann_index* idx = G.device(Base_Points);
  using T = typename PointRange_::T;
  const size_t nq = rows.size(), d = (size_t)Query_Points.dimension();
  std::vector<T> q(nq * d);
  for (size_t i = 0; i < nq; i++) std::memcpy(&q[i * d], Query_Points.data() + (size_t)rows[i] * d, sizeof(T) * d);
  pann_range_params rp;
  rp.beam = (uint32_t)QP.beamSize;
  rp.type = type;
  rp.radius = QP.radius;
  rp.early_stopping_radius = QP.early_stopping_radius;
  rp.early_stopping_count = (uint32_t)QP.early_stopping_count;
  std::vector<uint64_t> offs(nq + 1);
  std::vector<uint32_t> vis(nq), cmps(nq), ids(nq * (size_t)QP.beamSize + 16);
  int rc = pann_range_search(idx, q.data(), (uint32_t)nq, &rp, (uint32_t)start, offs.data(), ids.data(), ids.size(),
                             vis.data(), cmps.data(), nullptr);
  if (rc == PANN_EOVERFLOW && offs[nq] > ids.size()) {  // the answers are held on the device
    ids.resize(offs[nq]);
    rc = pann_range_fetch(idx, ids.data(), ids.size());
  }
  pann_check(rc, "range search");
  std::vector<std::vector<indexType>> out(nq);
  for (size_t i = 0; i < nq; i++) {
    out[i].assign(ids.begin() + (long)offs[i], ids.begin() + (long)offs[i + 1]);
    if (QueryStats.visited.size() > i) {
      QueryStats.increment_visited((indexType)i, vis[i]);
      QueryStats.increment_dist((indexType)i, cmps[i]);
    }
  }
  return out;
}

// RangeSearch (rangeSearch.h:183-276) on unquantized points; the second
// element is (seconds, 0), the reference's (beam, other) time split.
template <typename Point, typename PointRange_, typename QPointRange, typename indexType>
std::pair<std::vector<std::vector<indexType>>, std::pair<double, double>>
RangeSearch(Graph<indexType>& G, PointRange_& Query_Points, PointRange_& Base_Points, QPointRange& Q_Query_Points,
            QPointRange& Q_Base_Points, stats<indexType>& QueryStats, indexType starting_point, QueryParams& QP) {
  if ((const void*)&Q_Base_Points != (const void*)&Base_Points) {
    std::cout << "ERROR: RangeSearch supports unquantized points" << std::endl;
    std::abort();
  }
  (void)Q_Query_Points;
  std::vector<long> rows(Query_Points.size());
  for (size_t i = 0; i < rows.size(); i++) rows[i] = (long)i;
  const int type = QP.range_query_type == Beam ? PANN_RANGE_BEAM : PANN_RANGE_GREEDY;
  auto t0 = std::chrono::steady_clock::now();
  auto out = pann_range_batch(Query_Points, rows, G, Base_Points, QueryStats, starting_point, QP, type);
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return {out, {secs, 0.0}};
}

// DoubleBeamRangeSearch (doublingSearch.h:50-157) over active_indices.
template <typename PointRange_, typename QPointRange, typename indexType>
std::pair<std::vector<std::vector<indexType>>, std::pair<double, double>>
DoubleBeamRangeSearch(Graph<indexType>& G, PointRange_& Query_Points, PointRange_& Base_Points,
                      QPointRange& Q_Query_Points, QPointRange& Q_Base_Points, stats<indexType>& QueryStats,
                      std::vector<indexType> starting_points, QueryParams& QP,
                      std::vector<indexType> active_indices) {
  if ((const void*)&Q_Base_Points != (const void*)&Base_Points || starting_points.size() != 1) {
    std::cout << "ERROR: DoubleBeamRangeSearch supports unquantized points and one start point" << std::endl;
    std::abort();
  }
  (void)Q_Query_Points;
  std::vector<long> rows(active_indices.begin(), active_indices.end());
  auto t0 = std::chrono::steady_clock::now();
  auto out = pann_range_batch(Query_Points, rows, G, Base_Points, QueryStats, starting_points[0], QP,
                              PANN_RANGE_DOUBLING);
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return {out, {secs, 0.0}};
}

// ---------------------------------------------------------------- build
template <typename PointRange_, typename QPointRange, typename indexType>
struct knn_index {
  BuildParams BP;
  indexType start_point = 0;
  knn_index(BuildParams& BP) : BP(BP) {}
  indexType get_start() { return start_point; }
  void set_start() { start_point = 0; }
  // build_index (index.h:150-186): batch insertion with prefix doubling, on the GPU
  void build_index(Graph<indexType>& G, PointRange_& Points, QPointRange& QPoints, stats<indexType>& BuildStats,
                   bool sort_neighbors = true) {
    (void)QPoints;
    set_start();
    if (BP.single_batch != 0) {
      std::cout << "ERROR: single_batch builds are not offered" << std::endl;
      std::abort();
    }
    pann_index* idx = G.device(Points);
    pann_build_params bp;
    bp.R = (uint32_t)BP.R;
    bp.L = (uint32_t)BP.L;
    bp.alpha = BP.alpha;
    bp.num_passes = BP.num_passes;
    bp.batch_factor = BP.batch_factor;
    bp.perm_seed = 0x5EED5EED5EEDull;
    bp.sort_neighbors = sort_neighbors ? 1 : 0;
    pann_build_stats st;
    pann_check(pann_build(idx, &bp, nullptr, &st), "build_index");
    G.pull_from_device();
    if (BP.verbose)
      std::cout << "build: " << st.seconds << " s (search " << st.search_seconds << ", prune " << st.prune_seconds
                << ", reverse " << st.reverse_seconds << "), " << st.batches << " batches" << std::endl;
    (void)BuildStats;
  }
};

}  // namespace parlayANN
