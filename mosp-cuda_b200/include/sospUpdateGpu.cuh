#ifndef MOSP_B200_SOSP_UPDATE_GPU_CUH
#define MOSP_B200_SOSP_UPDATE_GPU_CUH

// C++ entry points of the SOSP update engine, declared as in the reference
// (SMShovan/MOSP-CUDA headers/sospUpdateGpu.cuh:14-110). They forward to the
// C ABI of this library (include/mosp_b200.h: mosp_sosp_update,
// mosp_sosp_from_scratch), which runs the sm_100a persistent kernels.

struct mosp_workspace;

/// Device CSR view with one weight column.
struct DeviceCsr {
  int numberOfNodes = 0;
  int numberOfEdges = 0;
  const int *rowPtr = nullptr;
  const int *colInd = nullptr;
  const int *weights = nullptr;
};

/// The change batch as one objective sees it (device arrays).
struct DeviceChanges {
  /// Deleted or weight-increased edges (changedFrom[i], changedTo[i]).
  const int *changedFrom = nullptr;
  const int *changedTo = nullptr;
  int numberOfChanged = 0;
  /// Heads of all inserted edges.
  const int *insertHeads = nullptr;
  int numberOfInsertHeads = 0;
};

/// Counters of one update.
struct SospStats {
  int invalidated = 0;  ///< vertices in invalidated subtrees
  int jumpRounds = 0;   ///< pointer-jumping rounds
  int iterations = 0;   ///< near-far push iterations
  int epochs = 0;       ///< far-pile threshold increases
  long long pushes = 0; ///< vertex expansions
  /// false: (n - 1) * maxWeight did not fit next to the parent ids; the
  /// search kept distances only and recovered the parents afterwards
  bool packedParents = true;
};

/// Device scratch of the engine; reserve once, reuse for every objective
/// and for the combined graph. Owns a C-ABI workspace (mosp_workspace).
struct SospWorkspace {
  SospWorkspace() = default;
  ~SospWorkspace();
  SospWorkspace(const SospWorkspace &) = delete;
  SospWorkspace &operator=(const SospWorkspace &) = delete;

  /// Allocate for graphs with up to capacity vertices (no-op if large
  /// enough); also fixes the grid of the persistent kernels.
  bool reserve(int capacity);
  /// Kept for interface compatibility: the engine advances its stamp
  /// generations on the device; returns the host-side call count.
  int nextGeneration();
  void release();

  int capacity = 0;
  int generation = 0;
  int gridBlocks = 0;               ///< co-resident CTAs of the engine
  mosp_workspace *handle = nullptr; ///< the C-ABI workspace
};

/// Default near-far bucket width: max(1, 32 * average weight / average
/// out-degree).
long long defaultDelta(long long numberOfEdges, int numberOfNodes,
                       long long weightSum);

/// Incremental SOSP update in place: d_distances / d_parent hold the tree
/// of the old graph on entry and the tree of the graph (out, in) on return
/// (canonical input trees give the canonical tree). Unreachable vertices
/// get DISTANCE_INF and parent -1. delta > 0; maxWeight bounds distances.
bool sospUpdateGpu(const DeviceCsr &out, const DeviceCsr &in,
                   const DeviceChanges &changes, int source, long long delta,
                   long long maxWeight, SospWorkspace &workspace,
                   long long *d_distances, int *d_parent,
                   SospStats *stats = nullptr);

/// Canonical single-source shortest paths from scratch.
bool sospFromScratchGpu(const DeviceCsr &out, int source, long long delta,
                        long long maxWeight, SospWorkspace &workspace,
                        long long *d_distances, int *d_parent,
                        SospStats *stats = nullptr);

#endif // MOSP_B200_SOSP_UPDATE_GPU_CUH
