// Stub for parlaylib/examples/helper/graph_utils.h, included by
// algorithms/utils/stats.h; only print_graph_statistics (never instantiated by
// the oracle) uses it.
#pragma once
#include "parlay/internal/shim_core.h"
template <typename V>
struct graph_utils {
  template <typename G> static G transpose(const G& g) { return g; }
};
