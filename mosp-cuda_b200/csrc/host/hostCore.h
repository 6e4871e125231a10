// hostCore.h - internal host-side views and helpers shared by the C++ API
// and the C ABI of this library (not installed).
#pragma once

#include <functional>

#include <cuda_runtime.h>
#include <string>
#include <vector>

#include "csrGraph.cuh"

namespace mospb200 {

/// Writes `count` lines to path, formatting chunks of lines on all host
/// cores (line(i, out) appends line i to out); the bytes equal a sequential
/// writer's.
bool writeLinesParallel(const std::string &path, size_t count,
                        const std::function<void(size_t, std::string &)> &line);

/// Sets the calling thread's last-error message of the C ABI
/// (mosp_last_error) and returns `status` (defined with the C ABI).
int recordFailure(int status, const char *message);

/// Read-only view of a CSR graph (edge-major weights).
struct GraphView {
  int n = 0, K = 0;
  const int *row = nullptr, *col = nullptr, *w = nullptr;
  long long edges() const { return row == nullptr ? 0 : row[n]; }
  int weight(long long e, int k) const { return w[e * K + k]; }
};

/// Read-only view of a change batch (insertion-major weights).
struct BatchView {
  int K = 0, nIns = 0, nDel = 0;
  const int *insFrom = nullptr, *insTo = nullptr, *insW = nullptr;
  const int *delFrom = nullptr, *delTo = nullptr;
};

inline GraphView viewOf(const CsrGraph &g) {
  return GraphView{g.numberOfNodes, g.numberOfObjectives, g.rowPtr.data(), g.colInd.data(),
                   g.weights.data()};
}

inline BatchView viewOf(const ChangeBatch &b) {
  return BatchView{b.numberOfObjectives, b.numberOfInserts(), b.numberOfDeletes(),
                   b.insertFrom.data(), b.insertTo.data(), b.insertWeights.data(),
                   b.deleteFrom.data(), b.deleteTo.data()};
}

/// Batch application on views (the semantics of applyChangeBatch); mask
/// receives the weight-increase bits of every insertion.
bool applyBatchView(const GraphView &g, const BatchView &b, CsrGraph &updated,
                    std::vector<unsigned> &mask);

}  // namespace mospb200

struct MospOptions;
struct MospResult;

/// mospUpdate() that also computes the MOSP path costs (n * KG, original
/// weights of the updated graph, DISTANCE_INF when unreachable) on the GPU
/// when costs is non-null.
bool mospUpdateWithCosts(const CsrGraph &original, ChangeBatch &batch,
                         const std::vector<long long> &initialDistances,
                         const std::vector<int> &initialParents, const MospOptions &options,
                         CsrGraph &updated, MospResult &result, std::vector<long long> *costs);
