#ifndef MOSP_B200_CHANGE_GENERATOR_CUH
#define MOSP_B200_CHANGE_GENERATOR_CUH

// Seeded change-batch generator (`mospPrep changes`), declared as in the
// reference (SMShovan/MOSP-CUDA headers/changeGenerator.cuh:9-62). For the
// same graph, options and seed it draws the same batch as the reference.
//
// Modes: Uniform (random vertex pairs with random weights; deletions
// sampled with replacement from the existing edges), Targeted (inserted
// weights below each objective's average weight; deletions of distinct
// SOSP-tree edges), Reweight (new random weights on existing edges),
// Increase (raise every weight of distinct tree edges by [1, weightMax]).

#include <string>

struct CsrGraph;
struct ChangeBatch;

enum class ChangeMode { Uniform, Targeted, Reweight, Increase };

/// Parse "uniform", "targeted", "reweight" or "increase".
bool parseChangeMode(const std::string &name, ChangeMode &mode);

struct ChangeGeneratorOptions {
  int numberOfChanges = 0;
  double insertionPercentage = 50; ///< Uniform / Targeted
  ChangeMode mode = ChangeMode::Uniform;
  int weightMin = 1;
  int weightMax = 100;
  unsigned int seed = 1;
  /// > 0: every endpoint within this many undirected hops of a random
  /// centre vertex
  int localHops = 0;
  /// drop deletions that would disconnect a vertex reachable from source
  bool safeDeletions = false;
  int source = 0;
};

bool generateChangeBatch(const CsrGraph &graph,
                         const ChangeGeneratorOptions &options,
                         ChangeBatch &batch, std::string *report = nullptr);

/// Write a batch as insert.txt / delete.txt.
bool writeChangeBatch(const ChangeBatch &batch, const std::string &insertPath,
                      const std::string &deletePath);

#endif // MOSP_B200_CHANGE_GENERATOR_CUH
