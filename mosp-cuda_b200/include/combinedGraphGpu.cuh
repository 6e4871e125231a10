#ifndef MOSP_B200_COMBINED_GRAPH_GPU_CUH
#define MOSP_B200_COMBINED_GRAPH_GPU_CUH

// Steps 2-3 of the MOSP update on the GPU, declared as in the reference
// (SMShovan/MOSP-CUDA headers/combinedGraphGpu.cuh:17-69). The combined
// graph and its SSSP run in one persistent launch (mosp_combined_sosp).

#include "sospUpdateGpu.cuh"

#include <vector>

/// Counters of combinedGraphSospGpu().
struct CombineStats {
  int numberOfEdges = 0; ///< edges of the combined graph
  long long scale = 1;   ///< L: combined distances are in units of 1/L
  long long delta = 0;   ///< near-far bucket width of Step 3
  SospStats search;      ///< Step 3 counters
};

/// Sizes reserved for the combined step. The device buffers live in the
/// engine workspace (SospWorkspace); this records the reservation.
struct CombineWorkspace {
  CombineWorkspace() = default;
  ~CombineWorkspace();
  CombineWorkspace(const CombineWorkspace &) = delete;
  CombineWorkspace &operator=(const CombineWorkspace &) = delete;

  /// Record a reservation for numberOfNodes vertices and K trees.
  bool reserve(int numberOfNodes, int K);
  void release();

  int capacity = 0;
  int trees = 0;
};

/// Build the combined graph of the K trees d_parents[k * n + v] and run
/// its SSSP from source: edge (p, v) iff p = Parent_i[v] for some i, with
/// weight L * (K + 1) - sum_{i : Parent_i[v] == p} L / Pref_i (L =
/// lcm(Pref), so weights stay integral). preferences: K values >= 1, empty
/// = all 1s. delta <= 0 selects the default width of the combined graph.
bool combinedGraphSospGpu(const int *d_parents, int numberOfNodes, int K,
                          const std::vector<int> &preferences, int source,
                          long long delta, CombineWorkspace &workspace,
                          SospWorkspace &sospWorkspace, long long *d_distances,
                          int *d_parent, CombineStats *stats = nullptr);

#endif // MOSP_B200_COMBINED_GRAPH_GPU_CUH
