#ifndef MOSP_B200_VALIDATION_CUH
#define MOSP_B200_VALIDATION_CUH

// Tree checks used by `mosp --validate`, declared as in the reference
// (SMShovan/MOSP-CUDA headers/validation.cuh:10-59).

#include <string>
#include <vector>

struct CsrGraph;

/// Result of checking an SOSP tree against reference distances.
struct TreeCheck {
  long long distanceMismatches = 0;  ///< dist[v] != reference[v]
  long long inconsistentParents = 0; ///< no edge (p,v) with d[p]+w == d[v]
  long long nonCanonicalParents = 0; ///< consistent, but not the lowest id
  long long parentMismatches = 0;    ///< parent[v] != referenceParent[v]

  bool ok(bool requireCanonical) const {
    return distanceMismatches == 0 && inconsistentParents == 0 &&
           parentMismatches == 0 &&
           (!requireCanonical || nonCanonicalParents == 0);
  }
  std::string summary() const;
};

/// Check distances (equal to the reference, INF where unreachable), parent
/// consistency (source and unreachable: -1; otherwise an edge (p,v) with
/// d[p] + w == d[v]), canonical parents (the lowest such p) and, if
/// referenceParents is given, equality with it. reverse: in-edge CSR.
TreeCheck checkSospTree(const CsrGraph &reverse, int objective, int source,
                        const std::vector<long long> &distances,
                        const std::vector<int> &parents,
                        const std::vector<long long> &referenceDistances,
                        const std::vector<int> *referenceParents = nullptr);

/// Host construction of the combined graph of K trees (one objective).
CsrGraph combinedGraphReference(const std::vector<int> &parents, int n, int K,
                                int source,
                                const std::vector<int> &preferences);

#endif // MOSP_B200_VALIDATION_CUH
