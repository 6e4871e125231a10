#ifndef MOSP_B200_PARALLEL_COMBINED_GRAPH_CUH
#define MOSP_B200_PARALLEL_COMBINED_GRAPH_CUH

// File-based combined-graph step and the preference helpers, declared as in
// the reference (SMShovan/MOSP-CUDA headers/parallelCombinedGraph.cuh:46-89).

#include <string>
#include <vector>

/// Read K parent files, build the combined graph of the K trees on the GPU,
/// run its SSSP from source and write distances (units of 1/L) and parents.
/// originalCsrPrefix only supplies the vertex count; workDir is unused.
bool parallelCombinedGraph(
    const std::string &originalCsrPrefix,
    const std::vector<std::string> &treeInputPaths, int K, int source = 0,
    const std::string &workDir = "output/combinedGraph",
    const std::string &distancesOutputPath =
        "output/combinedGraph/distancesCsr.txt",
    const std::string &treeOutputPath = "output/combinedGraph/SSSPTreeCsr.txt",
    const std::vector<int> &preferences = std::vector<int>());

/// L = lcm(Pref_1..Pref_K); 0 if a value is < 1, the size is not K, or
/// L > 2^20. Empty preferences = all 1s (L = 1).
long long preferenceScale(const std::vector<int> &preferences, int K);

/// Scaled combined-graph weight of an edge in the trees of treeMask:
/// L * (K + 1) - sum_{i in treeMask} L / Pref_i.
long long combinedEdgeWeight(unsigned int treeMask,
                             const std::vector<int> &preferences, int K,
                             long long scale);

struct CsrGraph;

/// MOSP cost vectors: costs[v * K + k] is the objective-k length (original
/// weights of graph, edge (p,v) = first occurrence of v in row p) of the
/// tree path source -> v; DISTANCE_INF if v is unreachable. false if a tree
/// edge is not in graph.
bool mospPathCosts(const CsrGraph &graph, const std::vector<int> &parent,
                   int source, std::vector<long long> &costs);

#endif // MOSP_B200_PARALLEL_COMBINED_GRAPH_CUH
