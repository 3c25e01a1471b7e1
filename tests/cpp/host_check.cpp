// Host-side pieces of the drop-in header, with no device call: PointRange
// read from .bin files, Point::distance for both metrics and both element
// types, one-byte scalar quantization, the graph file read, edgeRange edits
// and the graph file write.
// Usage: host_check base_f32.bin base_u8.bin graph_in graph_out
#include <cstdio>
#include <vector>

#include "parlayANN/parlayann.hpp"

using namespace parlayANN;

int main(int argc, char** argv) {
  if (argc != 5) return 2;
  PointRange<Euclidian_Point<float>> F(argv[1]);
  PointRange<Mips_Point<float>> FM(argv[1]);
  PointRange<Euclidian_Point<uint8_t>> U(argv[2]);
  PointRange<Mips_Point<uint8_t>> UM(argv[2]);
  std::printf("sizes %zu %ld %zu %ld\n", F.size(), F.dimension(), U.size(), U.dimension());
  for (long i = 0; i < 6; i++)
    for (long j = 0; j < 6; j++)
      std::printf("d %ld %ld %a %a %a %a\n", i, j, F[i].distance(F[j]), FM[i].distance(FM[j]), U[i].distance(U[j]),
                  UM[i].distance(UM[j]));
  // one-byte scalar quantization of the float range (point_range.h:55-71)
  PointRange<Euclidian_Point<uint8_t>> Q(F);
  std::printf("quant %a %d\n", Q.params.slope, Q.params.offset);
  for (long i = 0; i < 3; i++) {
    std::printf("qrow %ld", i);
    for (long j = 0; j < Q.dimension(); j++) std::printf(" %d", (int)Q[i][j]);
    std::printf("\n");
  }
  Graph<uint32_t> G(argv[3]);
  std::printf("graph %zu %ld %zu\n", G.size(), G.max_degree(), G[4].size());
  G[0].clear_neighbors();
  G[0].append_neighbor(7);
  G[0].append_neighbor(3);
  G[0].append_neighbor(5);
  G[1].sort([](uint32_t a, uint32_t b) { return a > b; });
  std::vector<uint32_t> r2 = {1, 2};
  G[2].update_neighbors(r2);
  G.save(argv[4]);
  return 0;
}
