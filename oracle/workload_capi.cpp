// workload_capi.cpp - TEST INFRASTRUCTURE. A C ABI over the seeded graph
// generators of the benchmark workloads (mosp-cuda_b200/csrc/host/
// graphGenerators.cpp, compiled into oracle/_gen/libworkload.so by
// oracle/Makefile), so that the benchmark's reference arm builds the same
// graphs as the library's arm without loading the library itself.
#include <algorithm>
#include <cstddef>
#include <cstdint>

#include "csrGraph.cuh"
#include "mospGenerators.h"

extern "C" {

/// A generated graph, owned by the caller until wl_free.
void *wl_grid_road(int width, int height, double keep, double shortcut, int K, int wmin, int wmax,
                   unsigned seed, int *n, long long *m) {
  CsrGraph *g = new CsrGraph();
  if (!generateGridRoad(width, height, keep, shortcut, K, wmin, wmax, seed, *g)) {
    delete g;
    return nullptr;
  }
  *n = g->numberOfNodes;
  *m = g->numberOfEdges();
  return g;
}

void *wl_rmat(int scale, int edge_factor, double a, double b, double c, int K, int wmin, int wmax,
              int log_uniform, unsigned seed, int *n, long long *m) {
  CsrGraph *g = new CsrGraph();
  if (!generateRmat(scale, edge_factor, a, b, c, K, wmin, wmax, log_uniform != 0, seed, *g)) {
    delete g;
    return nullptr;
  }
  *n = g->numberOfNodes;
  *m = g->numberOfEdges();
  return g;
}

/// Copy the CSR (n + 1 offsets, m heads, m * K edge-major weights) out.
void wl_copy(const void *graph, int *row, int *col, int *w) {
  const CsrGraph *g = static_cast<const CsrGraph *>(graph);
  std::copy(g->rowPtr.begin(), g->rowPtr.end(), row);
  std::copy(g->colInd.begin(), g->colInd.end(), col);
  std::copy(g->weights.begin(), g->weights.end(), w);
}

void wl_free(void *graph) { delete static_cast<CsrGraph *>(graph); }

}  // extern "C"
