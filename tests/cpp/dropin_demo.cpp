// A ParlayANN-style program (the shape of neighborsTime.C + ANN_Quantized:
// build a Vamana index, save/load the graph, search, check recall) written
// against include/parlayANN/parlayann.hpp. Exit status 0 when recall@10 of
// qsearchAll is >= 0.9 and beam_search agrees with qsearchAll.
#include <algorithm>
#include <cstdio>
#include <set>
#include <string>
#include <vector>

#include "parlayANN/parlayann.hpp"

using namespace parlayANN;

int main(int argc, char** argv) {
  std::string graph_path = argc > 1 ? argv[1] : "/tmp/pann_dropin.graph";
  const size_t n = 20000, nq = 200;
  const int d = 32;
  std::vector<uint8_t> base(n * d), q(nq * d);
  pann_check(pann_synth_mixture(PANN_U8, n, d, 16, 0, 0, 32.0, 224.0, 20.0, 0, base.data()), "synth");
  pann_check(pann_synth_mixture(PANN_U8, nq, d, 16, 0, 1, 32.0, 224.0, 20.0, 0, q.data()), "synth");
  using Point = Euclidian_Point<uint8_t>;
  using PR = PointRange<Point>;
  PR Points(base.data(), n, d), Query_Points(q.data(), nq, d);

  Graph<unsigned int> G(32, n);
  BuildParams BP(32, 64, 1.2, 2);
  BP.batch_factor = .125;
  knn_index<PR, PR, unsigned int> I(BP);
  stats<unsigned int> BuildStats(n);
  I.build_index(G, Points, Points, BuildStats);
  G.save((char*)graph_path.c_str());
  Graph<unsigned int> G2((char*)graph_path.c_str());

  QueryParams QP(10, 64, (long)n, 32, 10, .125);
  stats<unsigned int> QueryStats(nq);
  auto all = qsearchAll(Query_Points, Query_Points, Query_Points, G2, Points, Points, Points, QueryStats, 0u, QP);

  // recall@10 against an exact host scan
  long hit = 0;
  for (size_t i = 0; i < nq; i++) {
    std::vector<std::pair<float, unsigned>> ds;
    for (size_t j = 0; j < n; j++) ds.push_back({Query_Points[i].distance(Points[j]), (unsigned)j});
    std::partial_sort(ds.begin(), ds.begin() + 10, ds.end());
    std::set<unsigned> truth;
    for (int t = 0; t < 10; t++) truth.insert(ds[t].second);
    for (auto id : all[i]) hit += truth.count(id);
  }
  double recall = hit / (10.0 * nq);
  auto vs = QueryStats.visited_stats(), cs = QueryStats.dist_stats();

  // single-query beam_search agrees with the batch
  auto [lists, cmps] = beam_search(Query_Points[0], G2, Points, std::vector<unsigned int>{0u}, QP);
  bool same = lists.first.size() >= 10 && cmps == QueryStats.distances[0] && lists.second.size() == QueryStats.visited[0];
  for (int t = 0; t < 10 && same; t++) same = lists.first[t].first == all[0][t];
  std::printf("recall@10 %.4f  visited avg %u p99 %u  cmps avg %u p99 %u  beam_search agrees %d\n", recall, vs[0], vs[1],
              cs[0], cs[1], (int)same);

  // range search (RangeSearch, greedy; DoubleBeamRangeSearch), radius at the
  // 20th nearest distance of query 0: every answer is within the radius, and
  // most points within it are found
  std::vector<float> d0;
  for (size_t j = 0; j < n; j++) d0.push_back(Query_Points[0].distance(Points[j]));
  std::nth_element(d0.begin(), d0.begin() + 20, d0.end());
  const double radius = d0[20];
  QueryParams RQ(10, 10, (long)n, 32, 0, 0.0, 0, Greedy, radius);
  stats<unsigned int> RS(nq);
  auto [rr, rt] = RangeSearch<Point>(G2, Query_Points, Points, Query_Points, Points, RS, 0u, RQ);
  long found = 0, truth_n = 0;
  bool within = true;
  for (size_t i = 0; i < nq; i++) {
    for (auto id : rr[i]) within &= Query_Points[i].distance(Points[id]) <= radius;
    for (size_t j = 0; j < n; j++) truth_n += Query_Points[i].distance(Points[j]) <= radius;
    found += (long)std::set<unsigned>(rr[i].begin(), rr[i].end()).size();
  }
  std::vector<unsigned int> active(nq);
  for (size_t i = 0; i < nq; i++) active[i] = (unsigned)i;
  QueryParams DQ(10, 10, (long)n, 32, 0, 0.0, 0, Doubling, radius);
  stats<unsigned int> DS(nq);
  auto [dr, dt] = DoubleBeamRangeSearch(G2, Query_Points, Points, Query_Points, Points, DS,
                                        std::vector<unsigned int>{0u}, DQ, active);
  for (size_t i = 0; i < nq; i++)
    for (auto id : dr[i]) within &= Query_Points[i].distance(Points[id]) <= radius;
  double range_recall = truth_n ? (double)found / (double)truth_n : 1.0;
  std::printf("range: cumulative recall %.4f  all within radius %d\n", range_recall, (int)within);

  // the quantized search (ANN_Quantized's shape: float points, one-byte
  // quantized ranges, beam_search_rerank per query inside qsearchAll)
  const size_t nf = 8000;
  std::vector<float> fb(nf * 24), fq(nq * 24);
  pann_check(pann_synth_mixture(PANN_F32, nf, 24, 16, 3, 0, 0.0, 0.0, 0.3, 1, fb.data()), "synth");
  pann_check(pann_synth_mixture(PANN_F32, nq, 24, 16, 3, 1, 0.0, 0.0, 0.3, 1, fq.data()), "synth");
  using FPR = PointRange<Euclidian_Point<float>>;
  using QR = PointRange<Euclidian_Point<uint8_t>>;
  FPR FPoints(fb.data(), nf, 24), FQuery(fq.data(), nq, 24);
  QR QBase(FPoints);                    // generate_parameters + translate_point
  QR QQuery(FQuery, QBase.params);      // the queries with the base's parameters
  Graph<unsigned int> GF(24, nf);
  BuildParams FBP(24, 48, 1.2, 2);
  knn_index<FPR, FPR, unsigned int> FI(FBP);
  stats<unsigned int> FBS(nf);
  FI.build_index(GF, FPoints, FPoints, FBS);
  QueryParams FQP(10, 48, (long)nf, 24, 100, .125);
  stats<unsigned int> QS1(nq), QS2(nq);
  auto exact = qsearchAll(FQuery, FQuery, FQuery, GF, FPoints, FPoints, FPoints, QS1, 0u, FQP);
  auto quant = qsearchAll(FQuery, QQuery, QQuery, GF, FPoints, QBase, QBase, QS2, 0u, FQP);
  long qhit = 0, ehit = 0;
  for (size_t i = 0; i < nq; i++) {
    std::vector<std::pair<float, unsigned>> ds;
    for (size_t j = 0; j < nf; j++) ds.push_back({FQuery[i].distance(FPoints[j]), (unsigned)j});
    std::partial_sort(ds.begin(), ds.begin() + 10, ds.end());
    std::set<unsigned> truth;
    for (int t = 0; t < 10; t++) truth.insert(ds[t].second);
    for (auto id : quant[i]) qhit += truth.count(id);
    for (auto id : exact[i]) ehit += truth.count(id);
  }
  const double qrec = qhit / (10.0 * nq), erec = ehit / (10.0 * nq);
  std::printf("quantized: slope %.4f offset %d  recall@10 %.4f (float search %.4f)\n", QBase.params.slope,
              QBase.params.offset, qrec, erec);
  return (recall >= 0.9 && same && within && range_recall >= 0.8 && qrec >= erec - 0.05 && qrec >= 0.8) ? 0 : 1;
}
