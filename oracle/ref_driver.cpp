// Oracle driver around the REFERENCE's own code, compiled in place.
//
// TEST INFRASTRUCTURE ONLY. This file includes ParlayANN's headers from the
// reference checkout (algorithms/utils/*.h, algorithms/vamana/index.h) and
// wraps them in a C ABI so that tests and the CPU baseline can run the
// reference's beam search, robustPrune and Vamana build on in-memory data.
// It is built by oracle/Makefile into oracle/_ref/libpann_ref.so, against the
// project's own ParlayLib-API shim (oracle/parlay_shim), because ParlayLib is
// not vendored with the reference. Nothing in the product links or loads it.
//
// Entry points (dtype 0=uint8, 1=int8, 2=float32; metric 0=Euclidian, 1=mips):
//   ref_search       beam_search() per query          (beamSearch.h:420-427)
//   ref_qsearch_time qsearchAll() timed as checkRecall (check_nn_recall.h:46-59)
//   ref_robust_prune knn_index::robustPrune()          (index.h:63-120)
//   ref_build        knn_index::build_index()          (index.h:150-186)
//   ref_range_search RangeSearch() / DoubleBeamRangeSearch()
//                                        (rangeSearch.h:183-276, doublingSearch.h:50-157)
//   ref_range_groundtruth compute_range_groundtruth() (data_tools/compute_range_groundtruth.cpp:14-30;
//                    the tool's file is included with its main() renamed)
//   ref_search_quantized beam_search_rerank() over one-byte scalar-quantized
//                    points with a float re-rank, as GraphIndex::search_dispatch
//                    calls it for float indexes (beamSearch.h:529-597,
//                    python/graph_index.cpp:140-185): Euclidian_Point<uint8_t>
//                    (euclidian_point.h:186-240) for Euclidian, and
//                    Quantized_Mips_Point<8, true> (mips_point.h:293-499) for mips
//   ref_check_recall checkRecall() itself on a groundtruth .ibin file
//                    (check_nn_recall.h:17-128): recall with the groundtruth's
//                    ties at the k-th distance, QPS, mean visited / comparisons
//   ref_synth_mixture the seeded Gaussian-mixture generator of the data the
//                    benchmark and tests use (the same function of (seed,
//                    stream, row, dim) as the product's pann_synth_mixture), so
//                    a reference run needs no other library
//   ref_num_workers  threads used by parallel_for
#include <cmath>
#include <type_traits>
#include <cstdint>
#include <cstring>
#include <chrono>
#include <thread>
#include <vector>

#include "utils/euclidian_point.h"
#include "utils/mips_point.h"
#include "utils/point_range.h"
#include "utils/graph.h"
#include "utils/beamSearch.h"
#include "utils/stats.h"
#include "vamana/index.h"
#include "utils/rangeSearch.h"
#include "utils/doublingSearch.h"
#include "utils/check_nn_recall.h"

#define main pann_ref_range_groundtruth_tool_main
#include "../data_tools/compute_range_groundtruth.cpp"
#undef main

using namespace parlayANN;

namespace {

template <typename T>
struct MemRow {
  const T* p;
  T operator[](long j) const { return p[j]; }
};
template <typename T>
struct MemRows {
  const T* base; size_t n; size_t d;
  size_t size() const { return n; }
  long dimension() const { return (long)d; }
  MemRow<T> operator[](long i) const { return MemRow<T>{base + (size_t)i * d}; }
};

template <typename Point>
PointRange<Point> make_points(const void* data, size_t n, size_t d) {
  using T = typename Point::T;
  MemRows<T> rows{static_cast<const T*>(data), n, d};
  typename Point::parameters params((int)d);
  return PointRange<Point>(rows, params);
}

Graph<unsigned int> make_graph(const uint32_t* rows, size_t n, uint32_t R) {
  Graph<unsigned int> G((long)R, n);
  for (size_t i = 0; i < n; i++) {
    const uint32_t* r = rows + i * (size_t)(R + 1);
    uint32_t deg = r[0];
    if (deg > R) deg = R;
    auto s = parlay::make_slice(const_cast<uint32_t*>(r + 1), const_cast<uint32_t*>(r + 1 + deg));
    G[(unsigned)i].update_neighbors(s);
  }
  return G;
}

void export_graph(const Graph<unsigned int>& G, uint32_t* out, uint32_t R) {
  for (size_t i = 0; i < G.size(); i++) {
    uint32_t* r = out + i * (size_t)(R + 1);
    auto e = G[(unsigned)i];
    r[0] = (uint32_t)e.size();
    for (size_t j = 0; j < R; j++) r[1 + j] = j < e.size() ? e[(unsigned)j] : 0u;
  }
}

template <typename Point>
int search_t(uint32_t n, uint32_t d, const void* base, uint32_t nq, const void* queries,
             uint32_t R, const uint32_t* graph, uint32_t k, uint32_t L, uint64_t limit,
             uint32_t degree_limit, double batch_factor, uint32_t n_start, const uint32_t* starts,
             uint32_t* out_ids, float* out_dists, uint32_t* out_visited, uint32_t* out_cmps,
             uint32_t* out_frontier_n, uint32_t* out_frontier_ids, float* out_frontier_d,
             uint32_t visited_cap, uint32_t* out_visited_ids, float* out_visited_d) {
  auto B = make_points<Point>(base, n, d);
  auto Q = make_points<Point>(queries, nq, d);
  auto G = make_graph(graph, n, R);
  QueryParams QP((long)k, (long)L, (long)limit, (long)degree_limit, 100.0, batch_factor);
  parlay::sequence<unsigned int> sp(starts, starts + n_start);
  int bad = 0;
  parlay::parallel_for(0, (long)nq, [&](long i) {
    auto [pairElts, cmps] = beam_search(Q[i], G, B, sp, QP);
    auto& fr = pairElts.first;
    auto& vis = pairElts.second;
    if (fr.size() < k) { __atomic_store_n(&bad, 1, __ATOMIC_RELAXED); }
    for (uint32_t j = 0; j < k; j++) {
      out_ids[(size_t)i * k + j] = j < fr.size() ? fr[j].first : 0xFFFFFFFFu;
      out_dists[(size_t)i * k + j] = j < fr.size() ? fr[j].second : 0.0f;
    }
    out_visited[i] = (uint32_t)vis.size();
    out_cmps[i] = (uint32_t)cmps;
    if (out_frontier_n) {
      out_frontier_n[i] = (uint32_t)fr.size();
      for (size_t j = 0; j < fr.size() && j < L; j++) {
        out_frontier_ids[(size_t)i * L + j] = fr[j].first;
        out_frontier_d[(size_t)i * L + j] = fr[j].second;
      }
    }
    if (out_visited_ids) {
      for (size_t j = 0; j < vis.size() && j < visited_cap; j++) {
        out_visited_ids[(size_t)i * visited_cap + j] = vis[j].first;
        out_visited_d[(size_t)i * visited_cap + j] = vis[j].second;
      }
    }
  });
  return bad ? 1 : 0;
}

template <typename Point>
double qsearch_time_t(uint32_t n, uint32_t d, const void* base, uint32_t nq, const void* queries,
                      uint32_t R, const uint32_t* graph, uint32_t k, uint32_t L,
                      double batch_factor, uint32_t* out_ids, uint32_t* out_visited,
                      uint32_t* out_cmps, float* out_dists) {
  using PR = PointRange<Point>;
  auto B = make_points<Point>(base, n, d);
  auto Q = make_points<Point>(queries, nq, d);
  auto G = make_graph(graph, n, R);
  QueryParams QP((long)k, (long)L, (long)n, (long)R, 10.0, batch_factor);
  stats<unsigned int> QueryStats(nq);
  QueryStats.clear();
  // cache flush then a timer around qsearchAll only, as checkRecall does
  auto volatile xx = parlay::random_permutation<long>(5000000);
  (void)xx;
  auto t0 = std::chrono::steady_clock::now();
  auto all = qsearchAll<PR, PR, PR, unsigned int>(Q, Q, Q, G, B, B, B, QueryStats, 0u, QP);
  auto t1 = std::chrono::steady_clock::now();
  for (uint32_t i = 0; i < nq; i++) {
    for (uint32_t j = 0; j < k; j++) out_ids[(size_t)i * k + j] = all[i][j];
    out_visited[i] = QueryStats.visited[i];
    out_cmps[i] = QueryStats.distances[i];
  }
  // outside the timed region: the reference's distance of each returned id
  if (out_dists)
    parlay::parallel_for(0, (long)nq, [&](long i) {
      for (uint32_t j = 0; j < k; j++) out_dists[(size_t)i * k + j] = Q[i].distance(B[all[i][j]]);
    });
  return std::chrono::duration<double>(t1 - t0).count();
}

template <typename Point>
int check_recall_t(uint32_t n, uint32_t d, const void* base, uint32_t nq, const void* queries, uint32_t R,
                   const uint32_t* graph, const char* gt_path, uint32_t k, uint32_t L, uint64_t limit,
                   uint32_t degree_limit, double batch_factor, double* out) {
  using PR = PointRange<Point>;
  auto B = make_points<Point>(base, n, d);
  auto Q = make_points<Point>(queries, nq, d);
  auto G = make_graph(graph, n, R);
  groundTruth<unsigned int> GT(const_cast<char*>(gt_path));
  QueryParams QP((long)k, (long)L, (long)limit, (long)degree_limit, 100.0, batch_factor);
  nn_result r = checkRecall<PR, PR, PR, unsigned int>(G, B, Q, B, Q, B, Q, GT, false, 0, (long)k, QP, false);
  out[0] = r.recall;
  out[1] = r.QPS;
  out[2] = r.avg_cmps;
  out[3] = r.tail_cmps;
  out[4] = r.avg_visited;
  out[5] = r.tail_visited;
  return 0;
}

// Data generator (see ref_synth_mixture below).
inline uint64_t sm_mix(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
inline uint64_t sm_key(uint64_t seed, uint64_t stream, uint64_t a, uint64_t b) {
  return sm_mix(sm_mix(sm_mix(seed ^ (stream << 56)) + a) + b);
}
inline double sm_unif(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
inline double sm_normal(uint64_t h1, uint64_t h2) {
  const double r = std::sqrt(-2.0 * std::log(1.0 - sm_unif(h1)));
  return r * std::cos(6.283185307179586476925286766559 * sm_unif(h2));
}

template <typename Point>
int prune_t(uint32_t n, uint32_t d, const void* base, uint32_t R, const uint32_t* graph,
            uint32_t p, uint32_t n_cand, const uint32_t* cand_ids, const float* cand_d,
            double alpha, int add, uint32_t* out_nbrs, uint32_t* out_n, long* out_cmps) {
  using PR = PointRange<Point>;
  auto B = make_points<Point>(base, n, d);
  auto G = make_graph(graph, n, R);
  BuildParams BP((long)R, 64, alpha, 1);
  knn_index<PR, PR, unsigned int> I(BP);
  parlay::sequence<std::pair<unsigned int, float>> cand;
  for (uint32_t i = 0; i < n_cand; i++) cand.push_back(std::make_pair(cand_ids[i], cand_d[i]));
  auto [nb, dc] = I.robustPrune(p, cand, G, B, alpha, add != 0);
  *out_n = (uint32_t)nb.size();
  for (size_t i = 0; i < nb.size(); i++) out_nbrs[i] = nb[i];
  *out_cmps = dc;
  return 0;
}

template <typename Point>
int build_t(uint32_t n, uint32_t d, const void* base, uint32_t R, uint32_t L, double alpha,
            int passes, double batch_factor, uint32_t* out_graph, double* seconds,
            uint64_t* out_dist_total, uint32_t* out_visited) {
  using PR = PointRange<Point>;
  auto B = make_points<Point>(base, n, d);
  BuildParams BP((long)R, (long)L, alpha, passes, 0, 0, 0, 0.0, false, 0, false, 0, 0, 0.0,
                 10.0, batch_factor);
  Graph<unsigned int> G((long)R, n);
  knn_index<PR, PR, unsigned int> I(BP);
  stats<unsigned int> BuildStats(G.size());
  auto t0 = std::chrono::steady_clock::now();
  I.build_index(G, B, B, BuildStats);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  export_graph(G, out_graph, R);
  if (out_dist_total) {
    uint64_t s = 0;
    for (size_t i = 0; i < n; i++) s += BuildStats.distances[i];
    *out_dist_total = s;
  }
  if (out_visited) for (size_t i = 0; i < n; i++) out_visited[i] = BuildStats.visited[i];
  return 0;
}

template <typename Point>
int range_t(uint32_t n, uint32_t d, const void* base, uint32_t nq, const void* queries, uint32_t R,
            const uint32_t* graph, uint32_t beam, uint32_t start, int type, double radius, double esr,
            uint32_t esc, uint64_t* out_count, uint32_t* out_ids, uint64_t cap, uint32_t* out_visited,
            uint64_t* out_cmps) {
  using PR = PointRange<Point>;
  auto B = make_points<Point>(base, n, d);
  auto Q = make_points<Point>(queries, nq, d);
  auto G = make_graph(graph, n, R);
  // as range_search_wrapper builds it (check_range_recall.h:132-133)
  QueryParams QP((long)beam, (long)beam, (long)G.size(), (long)G.max_degree(), (long)(esc > 0), esr, (long)esc,
                 (rangeQueryType)type, radius);
  stats<unsigned int> QS(nq);
  QS.clear();
  auto emit = [&](size_t i, const auto& v) {
    out_count[i] = v.size();
    for (size_t j = 0; j < v.size() && j < cap; j++) out_ids[i * cap + j] = v[j];
  };
  if (type == Doubling) {
    parlay::sequence<unsigned int> sp = {start};
    auto active = parlay::tabulate(nq, [](size_t i) { return (unsigned int)i; });
    auto res = DoubleBeamRangeSearch(G, Q, B, Q, B, QS, sp, QP, active);
    for (size_t i = 0; i < nq; i++) emit(i, res.first[i]);
  } else {
    auto res = RangeSearch<Point, PR, PR, unsigned int>(G, Q, B, Q, B, QS, start, QP);
    for (size_t i = 0; i < nq; i++) emit(i, res.first[i]);
  }
  for (size_t i = 0; i < nq; i++) {
    if (out_visited) out_visited[i] = QS.visited[i];
    if (out_cmps) out_cmps[i] = QS.distances[i];
  }
  return 0;
}

template <typename Point>
int range_gt_t(uint32_t n, uint32_t d, const void* base, uint32_t nq, const void* queries, float radius,
               uint64_t* out_offsets, uint32_t* out_ids, uint64_t cap) {
  using PR = PointRange<Point>;
  auto B = make_points<Point>(base, n, d);
  auto Q = make_points<Point>(queries, nq, d);
  auto ans = compute_range_groundtruth<PR>(B, Q, radius);
  uint64_t total = 0;
  for (size_t i = 0; i < nq; i++) {
    out_offsets[i] = total;
    for (size_t j = 0; j < ans[i].size(); j++)
      if (total + j < cap) out_ids[total + j] = (uint32_t)ans[i][j];
    total += ans[i].size();
  }
  out_offsets[nq] = total;
  return total > cap ? 1 : 0;
}

// Euclidian: Euclidian_Point<uint8_t> (slope, offset); mips: Quantized_Mips_Point<8, true>, the
// quantizer GraphIndex uses for float mips indexes (python/graph_index.cpp:69), whose parameters are
// reported as (scale, 0).
template <typename Point, typename QPoint>
int quantized_t(uint32_t n, uint32_t d, const float* base, uint32_t nq, const float* queries, uint32_t R,
                const uint32_t* graph, uint32_t k, uint32_t L, uint64_t limit, uint32_t degree_limit,
                double rerank_factor, double batch_factor, uint32_t start, uint32_t* out_ids, float* out_dists,
                uint32_t* out_visited, uint32_t* out_cmps, float* out_slope, int32_t* out_offset, double* seconds) {
  auto B = make_points<Point>(base, n, d);
  auto Q = make_points<Point>(queries, nq, d);
  auto G = make_graph(graph, n, R);
  PointRange<QPoint> QB(B);  // generate_parameters + translate_point per row
  if constexpr (std::is_same_v<Point, Euclidian_Point<float>>) {
    *out_slope = QB.params.slope;
    *out_offset = QB.params.offset;
  } else {
    *out_slope = QB.params.scale;
    *out_offset = 0;
  }
  QueryParams QP((long)k, (long)L, (long)limit, (long)degree_limit, rerank_factor, batch_factor);
  stats<unsigned int> QS(nq);
  QS.clear();
  parlay::sequence<unsigned int> starts = {start};
  auto t0 = std::chrono::steady_clock::now();
  parlay::parallel_for(0, nq, [&](size_t i) {
    std::vector<uint8_t> buf(QB.params.num_bytes() + 16);
    QPoint::translate_point(buf.data(), Q[i], QB.params);
    QPoint qq(buf.data(), (long)i, QB.params);
    auto res = beam_search_rerank(Q[i], qq, qq, G, B, QB, QB, QS, starts, QP, true);
    for (size_t j = 0; j < k; j++) {
      out_ids[i * k + j] = res[j].first;
      out_dists[i * k + j] = res[j].second;
    }
  });
  *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (size_t i = 0; i < nq; i++) {
    out_visited[i] = QS.visited[i];
    out_cmps[i] = QS.distances[i];
  }
  return 0;
}

}  // namespace

#define DISPATCH(dtype, metric, FN, ...)                                                  \
  do {                                                                                    \
    if (metric == 0) {                                                                    \
      if (dtype == 0) return FN<Euclidian_Point<uint8_t>>(__VA_ARGS__);                   \
      if (dtype == 1) return FN<Euclidian_Point<int8_t>>(__VA_ARGS__);                    \
      if (dtype == 2) return FN<Euclidian_Point<float>>(__VA_ARGS__);                     \
    } else {                                                                              \
      if (dtype == 0) return FN<Mips_Point<uint8_t>>(__VA_ARGS__);                        \
      if (dtype == 1) return FN<Mips_Point<int8_t>>(__VA_ARGS__);                         \
      if (dtype == 2) return FN<Mips_Point<float>>(__VA_ARGS__);                          \
    }                                                                                     \
  } while (0)

extern "C" {

int ref_num_workers(void) { return (int)parlay::num_workers(); }

int ref_search(int dtype, int metric, uint32_t n, uint32_t d, const void* base, uint32_t nq,
               const void* queries, uint32_t R, const uint32_t* graph, uint32_t k, uint32_t L,
               uint64_t limit, uint32_t degree_limit, double batch_factor, uint32_t n_start,
               const uint32_t* starts, uint32_t* out_ids, float* out_dists, uint32_t* out_visited,
               uint32_t* out_cmps, uint32_t* out_frontier_n, uint32_t* out_frontier_ids,
               float* out_frontier_d, uint32_t visited_cap, uint32_t* out_visited_ids,
               float* out_visited_d) {
  DISPATCH(dtype, metric, search_t, n, d, base, nq, queries, R, graph, k, L, limit, degree_limit,
           batch_factor, n_start, starts, out_ids, out_dists, out_visited, out_cmps,
           out_frontier_n, out_frontier_ids, out_frontier_d, visited_cap, out_visited_ids,
           out_visited_d);
  return -1;
}

double ref_qsearch_time(int dtype, int metric, uint32_t n, uint32_t d, const void* base,
                        uint32_t nq, const void* queries, uint32_t R, const uint32_t* graph,
                        uint32_t k, uint32_t L, double batch_factor, uint32_t* out_ids,
                        uint32_t* out_visited, uint32_t* out_cmps, float* out_dists) {
  DISPATCH(dtype, metric, qsearch_time_t, n, d, base, nq, queries, R, graph, k, L, batch_factor,
           out_ids, out_visited, out_cmps, out_dists);
  return -1.0;
}

// out: recall, QPS, mean and p99 comparisons, mean and p99 visited (nn_result)
int ref_check_recall(int dtype, int metric, uint32_t n, uint32_t d, const void* base, uint32_t nq,
                     const void* queries, uint32_t R, const uint32_t* graph, const char* gt_path, uint32_t k,
                     uint32_t L, uint64_t limit, uint32_t degree_limit, double batch_factor, double* out) {
  DISPATCH(dtype, metric, check_recall_t, n, d, base, nq, queries, R, graph, gt_path, k, L, limit, degree_limit,
           batch_factor, out);
  return -1;
}

// Seeded Gaussian mixture, every value a function of (seed, stream, row, dim)
// through a splitmix64 chain: uint8 centres uniform in [lo, hi], float centres
// N(0,1); the row's component is a hash of (seed, 2 + 2 stream, row) modulo
// the component count; the noise is N(0,1) (Box-Muller on two hashes of
// (seed, 3 + 2 stream, row, 2t / 2t+1)) times sigma; uint8 values are
// rounded half away from zero and clipped to [0, 255]; float rows are
// optionally L2-normalised in double and rounded to float.
int ref_synth_mixture(int dtype, uint64_t n, uint32_t d, uint32_t comps, uint64_t seed, uint32_t stream, double lo,
                      double hi, double sigma, int normalize, void* out) {
  if (!out || d == 0 || comps == 0 || (dtype != 0 && dtype != 2)) return -1;
  std::vector<double> cen((size_t)comps * d);
  for (uint32_t c = 0; c < comps; c++)
    for (uint32_t t = 0; t < d; t++)
      cen[(size_t)c * d + t] = dtype == 0 ? lo + (hi - lo) * sm_unif(sm_key(seed, 1, c, t))
                                          : sm_normal(sm_key(seed, 1, c, 2ull * t), sm_key(seed, 1, c, 2ull * t + 1));
  const uint64_t s_comp = 2 + 2ull * stream, s_noise = 3 + 2ull * stream;
  unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  auto rows = [&](unsigned tid) {
    std::vector<double> v(d);
    for (uint64_t i = tid; i < n; i += nt) {
      const double* c = &cen[(size_t)(sm_key(seed, s_comp, i, 0) % comps) * d];
      for (uint32_t t = 0; t < d; t++)
        v[t] = c[t] + sigma * sm_normal(sm_key(seed, s_noise, i, 2ull * t), sm_key(seed, s_noise, i, 2ull * t + 1));
      if (dtype == 0) {
        uint8_t* o = static_cast<uint8_t*>(out) + i * d;
        for (uint32_t t = 0; t < d; t++) {
          const double r = std::round(v[t]);
          o[t] = (uint8_t)(r < 0.0 ? 0.0 : (r > 255.0 ? 255.0 : r));
        }
      } else {
        double norm = 1.0;
        if (normalize) {
          double ss = 0.0;
          for (uint32_t t = 0; t < d; t++) ss += v[t] * v[t];
          norm = std::sqrt(ss);
          if (norm == 0.0) norm = 1.0;
        }
        float* o = static_cast<float*>(out) + i * d;
        for (uint32_t t = 0; t < d; t++) o[t] = (float)(v[t] / norm);
      }
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; t++) th.emplace_back(rows, t);
  rows(0);
  for (auto& x : th) x.join();
  return 0;
}

int ref_robust_prune(int dtype, int metric, uint32_t n, uint32_t d, const void* base, uint32_t R,
                     const uint32_t* graph, uint32_t p, uint32_t n_cand, const uint32_t* cand_ids,
                     const float* cand_d, double alpha, int add, uint32_t* out_nbrs,
                     uint32_t* out_n, long* out_cmps) {
  DISPATCH(dtype, metric, prune_t, n, d, base, R, graph, p, n_cand, cand_ids, cand_d, alpha, add,
           out_nbrs, out_n, out_cmps);
  return -1;
}

int ref_build(int dtype, int metric, uint32_t n, uint32_t d, const void* base, uint32_t R,
              uint32_t L, double alpha, int passes, double batch_factor, uint32_t* out_graph,
              double* seconds, uint64_t* out_dist_total, uint32_t* out_visited) {
  DISPATCH(dtype, metric, build_t, n, d, base, R, L, alpha, passes, batch_factor, out_graph,
           seconds, out_dist_total, out_visited);
  return -1;
}

int ref_range_search(int dtype, int metric, uint32_t n, uint32_t d, const void* base, uint32_t nq,
                     const void* queries, uint32_t R, const uint32_t* graph, uint32_t beam, uint32_t start,
                     int type, double radius, double esr, uint32_t esc, uint64_t* out_count, uint32_t* out_ids,
                     uint64_t cap, uint32_t* out_visited, uint64_t* out_cmps) {
  DISPATCH(dtype, metric, range_t, n, d, base, nq, queries, R, graph, beam, start, type, radius, esr, esc,
           out_count, out_ids, cap, out_visited, out_cmps);
  return -1;
}

int ref_search_quantized(int metric, uint32_t n, uint32_t d, const float* base, uint32_t nq, const float* queries,
                         uint32_t R, const uint32_t* graph, uint32_t k, uint32_t L, uint64_t limit,
                         uint32_t degree_limit, double rerank_factor, double batch_factor, uint32_t start,
                         uint32_t* out_ids, float* out_dists, uint32_t* out_visited, uint32_t* out_cmps,
                         float* out_slope, int32_t* out_offset, double* seconds) {
  if (metric == 0)
    return quantized_t<Euclidian_Point<float>, Euclidian_Point<uint8_t>>(
        n, d, base, nq, queries, R, graph, k, L, limit, degree_limit, rerank_factor, batch_factor, start, out_ids,
        out_dists, out_visited, out_cmps, out_slope, out_offset, seconds);
  return quantized_t<Mips_Point<float>, Quantized_Mips_Point<8, true>>(
      n, d, base, nq, queries, R, graph, k, L, limit, degree_limit, rerank_factor, batch_factor, start, out_ids,
      out_dists, out_visited, out_cmps, out_slope, out_offset, seconds);
}

int ref_range_groundtruth(int dtype, int metric, uint32_t n, uint32_t d, const void* base, uint32_t nq,
                          const void* queries, float radius, uint64_t* out_offsets, uint32_t* out_ids,
                          uint64_t cap) {
  DISPATCH(dtype, metric, range_gt_t, n, d, base, nq, queries, radius, out_offsets, out_ids, cap);
  return -1;
}

}  // extern "C"
