#ifndef MOSP_B200_DIJKSTRA_CUH
#define MOSP_B200_DIJKSTRA_CUH

// Host Dijkstra for `mospPrep init|expected` and `mosp --validate`,
// declared as in the reference (SMShovan/MOSP-CUDA headers/dijkstra.cuh:
// 45-56). Ties go to the lowest parent id.

#include <string>
#include <vector>

struct CsrGraph;

/// Dijkstra of one objective on the text CSR at inputPrefix; writes the
/// distance and tree files.
bool runDijkstraCSR(const std::string &inputPrefix, int objectiveNumber, int source,
                    const std::string &distanceOutputPath = "output/distancesCsr.txt",
                    const std::string &treeOutputPath = "output/SSSPTreeCsr.txt");

void dijkstraCsrGraph(const CsrGraph &graph, int objective, int source,
                      std::vector<long long> &distances,
                      std::vector<int> &parent);

#endif // MOSP_B200_DIJKSTRA_CUH
