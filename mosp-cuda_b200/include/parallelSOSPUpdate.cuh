#ifndef MOSP_B200_PARALLEL_SOSP_UPDATE_CUH
#define MOSP_B200_PARALLEL_SOSP_UPDATE_CUH

// File-based SOSP update of one objective, declared as in the reference
// (SMShovan/MOSP-CUDA headers/parallelSOSPUpdate.cuh:32-40): read the
// graph, the tree and the batch, apply the batch, update on the GPU, write
// the updated distances and tree.

#include <string>

bool parallelSOSPUpdate(
    const std::string &originalCsrPrefix, const std::string &distancesInputPath,
    const std::string &treeInputPath, const std::string &insertPath,
    const std::string &deletePath, int objectiveIndex, int source = 0,
    const std::string &distancesOutputPath =
        "output/parallelSospUpdateDistancesTrees/distancesCsr.txt",
    const std::string &treeOutputPath =
        "output/parallelSospUpdateDistancesTrees/SSSPTreeCsr.txt");

#endif // MOSP_B200_PARALLEL_SOSP_UPDATE_CUH
