// generators.cpp - seeded synthetic change batches (interface:
// include/mospGenerators.h); the graphs are in graphGenerators.cpp.
#include "mospGenerators.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <iostream>
#include <numeric>
#include <random>
#include <unordered_set>
#include <utility>
#include <vector>

#include "csrGraph.cuh"

bool generateNearBatch(const CsrGraph &graph, int gridWidth, int nIns, int nDel, int maxManhattan,
                       bool safe, unsigned seed, int source, int wmin, int wmax,
                       ChangeBatch &batch) {
  const int n = graph.numberOfNodes, K = graph.numberOfObjectives;
  batch = ChangeBatch();
  batch.numberOfObjectives = K;
  if (gridWidth < 1 || n % gridWidth != 0 || nIns < 0 || nDel < 0 || maxManhattan < 1 ||
      source < 0 || source >= n || wmin < 1 || wmin > wmax || K < 1) {
    std::cout << "Error: invalid near-batch parameters.\n";
    return false;
  }
  const int height = n / gridWidth;
  std::mt19937_64 rng(seed);
  auto key = [](int u, int v) { return (static_cast<uint64_t>(u) << 32) | static_cast<uint32_t>(v); };
  std::unordered_set<uint64_t> existing;
  for (int u = 0; u < n; ++u) {
    for (int e = graph.rowPtr[u]; e < graph.rowPtr[u + 1]; ++e) existing.insert(key(u, graph.colInd[e]));
  }
  std::vector<std::pair<int, int>> offsets;
  for (int dy = -maxManhattan; dy <= maxManhattan; ++dy) {
    for (int dx = -maxManhattan; dx <= maxManhattan; ++dx) {
      if ((dx != 0 || dy != 0) && std::abs(dx) + std::abs(dy) <= maxManhattan) offsets.push_back({dx, dy});
    }
  }
  std::uniform_int_distribution<int> vertex(0, n - 1);
  std::uniform_int_distribution<int> offset(0, static_cast<int>(offsets.size()) - 1);
  std::uniform_int_distribution<int> weight(wmin, wmax);
  std::unordered_set<uint64_t> chosen;
  long long attempts = 0;
  while (batch.numberOfInserts() < nIns && attempts < 100LL * (nIns + 1)) {
    ++attempts;
    const int u = vertex(rng);
    const auto d = offsets[offset(rng)];
    const int x = u % gridWidth + d.first, y = u / gridWidth + d.second;
    if (x < 0 || x >= gridWidth || y < 0 || y >= height) continue;
    const int v = y * gridWidth + x;
    if (existing.count(key(u, v)) || !chosen.insert(key(u, v)).second) continue;
    batch.insertFrom.push_back(u);
    batch.insertTo.push_back(v);
    for (int k = 0; k < K; ++k) batch.insertWeights.push_back(weight(rng));
  }
  std::vector<std::pair<int, int>> pool;
  pool.reserve(graph.colInd.size());
  for (int u = 0; u < n; ++u) {
    for (int e = graph.rowPtr[u]; e < graph.rowPtr[u + 1]; ++e) pool.push_back({u, graph.colInd[e]});
  }
  std::shuffle(pool.begin(), pool.end(), rng);
  for (int i = 0; i < nDel && i < static_cast<int>(pool.size()); ++i) {
    batch.deleteFrom.push_back(pool[i].first);
    batch.deleteTo.push_back(pool[i].second);
  }
  if (safe) filterUnsafeDeletions(graph, source, batch);
  return true;
}
