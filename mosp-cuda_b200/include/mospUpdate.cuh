#ifndef MOSP_B200_MOSP_UPDATE_CUH
#define MOSP_B200_MOSP_UPDATE_CUH

// In-memory MOSP update, declared as in the reference (SMShovan/MOSP-CUDA
// headers/mospUpdate.cuh:17-85). The K SOSP updates run as one fused
// persistent launch and Steps 2-3 as a second one, queued back to back
// (mosp_update_device).

#include "combinedGraphGpu.cuh"

#include <vector>

struct CsrGraph;
struct ChangeBatch;

/// Options of mospUpdate().
struct MospOptions {
  int source = 0;
  int numberOfObjectives = 0;   ///< 0: every objective of the graph
  std::vector<int> preferences; ///< Pref vector; empty = all 1s
  long long delta = 0;          ///< near-far bucket width; <= 0: default
  /// The initial trees follow the lowest-id tie rule (canonicalizeTree,
  /// or any tree this library returns): distance-only objectives then
  /// recover parents only where the batch reaches (same result for such
  /// trees); see mosp_workspace_set_canonical_trees.
  bool canonicalTrees = false;
};

/// Wall-clock times (milliseconds) of the stages of mospUpdate().
struct MospTimings {
  double applyBatch = 0;          ///< host: apply the batch to the CSR
  double upload = 0;              ///< graph, trees and batch to the GPU
  /// GPU: SOSP updates. The K updates share one launch; its time is split
  /// evenly over the K entries, so their sum is the launch time.
  std::vector<double> objectives;
  double combined = 0;            ///< GPU: combined graph + its SOSP tree
  double download = 0;            ///< results back to the host

  /// The timed region of the papers: the K SOSP updates and Steps 2-3.
  double gpuCompute() const;
};

/// Output of mospUpdate().
struct MospResult {
  int numberOfObjectives = 0;
  std::vector<long long> distances;         ///< K * n, objective-major
  std::vector<int> parents;                 ///< K * n, objective-major
  std::vector<long long> combinedDistances; ///< units of 1/L
  std::vector<int> combinedParent;          ///< the MOSP tree
  std::vector<SospStats> objectiveStats;
  CombineStats combineStats;
  MospTimings timings;
};

/// One MOSP update on an in-memory graph: apply the batch (host), upload
/// once, run the K SOSP updates and Steps 2-3 on the GPU, download. The
/// initial trees (K * n, objective-major) must be rooted at
/// options.source. batch.weightIncreaseMask is filled; `updated` receives
/// the updated graph.
bool mospUpdate(const CsrGraph &original, ChangeBatch &batch,
                const std::vector<long long> &initialDistances,
                const std::vector<int> &initialParents,
                const MospOptions &options, CsrGraph &updated,
                MospResult &result);

/// Force the lowest-id tie rule on a tree of graph: parent[v] becomes the
/// lowest u with dist[u] + w(u,v) == dist[v] (one pass over the edges).
void canonicalizeTree(const CsrGraph &graph, int objective, int source,
                      const std::vector<long long> &distances, int *parent);

#endif // MOSP_B200_MOSP_UPDATE_CUH
