// deletionFilter.h - the round structure of the `--safe` connectivity
// filter, shared by its host and GPU reachability back-ends
// (changeGenerator.cpp, safeFilterGpu.cpp).
#pragma once

#include <vector>

#include "csrGraph.cuh"

/// The connectivity filter of `--safe` batches, in rounds: apply the batch
/// (all insertions, the deletions kept so far), find the vertices that were
/// reachable from the source before and are not now, drop every deletion
/// with such an endpoint, and repeat until nothing is lost (or nothing was
/// dropped). The rounds, and so the kept deletions, are the reference's
/// (src/changeGenerator.cu:78-114); only how reachability is computed
/// differs between the host and the GPU path. `after(batch)` returns the
/// reachability of the updated graph, or an empty vector on failure.
template <typename ReachAfter>
int filterDeletionRounds(const std::vector<char> &before, ChangeBatch &batch, ReachAfter after) {
  int rounds = 0;
  while (batch.numberOfDeletes() > 0) {
    ++rounds;
    const std::vector<char> now = after(batch);
    if (now.empty()) return -1;
    auto lost = [&](int v) { return before[v] && !now[v]; };
    size_t kept = 0;
    const size_t count = batch.deleteFrom.size();
    for (size_t i = 0; i < count; ++i) {
      const int u = batch.deleteFrom[i], v = batch.deleteTo[i];
      if (lost(u) || lost(v)) continue;
      batch.deleteFrom[kept] = u;
      batch.deleteTo[kept] = v;
      ++kept;
    }
    if (kept == count) break;  // nothing lost, or no deletion touches it
    batch.deleteFrom.resize(kept);
    batch.deleteTo.resize(kept);
  }
  return rounds;
}
