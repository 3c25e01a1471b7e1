// Stub for parlaylib/examples/BFS.h, which algorithms/utils/stats.h includes.
// Only print_graph_statistics (never instantiated by the oracle) calls it.
#pragma once
#include "parlay/internal/shim_core.h"
template <typename V, typename G>
parlay::sequence<parlay::sequence<V>> BFS(V, const G&) { return {}; }
