// checks.cpp - host shortest paths and tree checks used by `mospPrep
// init|expected` and `mosp --validate` (interfaces: include/dijkstra.cuh,
// include/validation.cuh; semantics of SMShovan/MOSP-CUDA
// src/Dijkstra.cu:239-272 and src/validation.cu:28-125).
#include <algorithm>
#include <queue>
#include <sstream>
#include <utility>
#include <vector>

#include "csrGraph.cuh"
#include "dijkstra.cuh"
#include "parallelCombinedGraph.cuh"
#include "validation.cuh"

void dijkstraCsrGraph(const CsrGraph &graph, int objective, int source,
                      std::vector<long long> &distances, std::vector<int> &parent) {
  const int n = graph.numberOfNodes;
  distances.assign(n, DISTANCE_INF);
  parent.assign(n, -1);
  if (source < 0 || source >= n) return;
  using Item = std::pair<long long, int>;
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
  distances[source] = 0;
  heap.push({0, source});
  while (!heap.empty()) {
    const auto [d, u] = heap.top();
    heap.pop();
    if (d != distances[u]) continue;  // stale entry
    for (int e = graph.rowPtr[u]; e < graph.rowPtr[u + 1]; ++e) {
      const int v = graph.colInd[e];
      const long long cand = d + graph.weight(e, objective);
      if (cand < distances[v]) {
        distances[v] = cand;
        parent[v] = u;
        heap.push({cand, v});
      } else if (cand == distances[v] && v != source && u < parent[v]) {
        parent[v] = u;  // equal distance: the lowest parent id wins
      }
    }
  }
}

bool runDijkstraCSR(const std::string &inputPrefix, int objectiveNumber, int source,
                    const std::string &distanceOutputPath, const std::string &treeOutputPath) {
  CsrGraph g;
  if (!readCsrGraph(inputPrefix, g)) return false;
  if (objectiveNumber < 0 || objectiveNumber >= g.numberOfObjectives || source < 0 ||
      source >= g.numberOfNodes) {
    return false;
  }
  std::vector<long long> d;
  std::vector<int> p;
  dijkstraCsrGraph(g, objectiveNumber, source, d, p);
  return writeDistances(distanceOutputPath, d) && writeParents(treeOutputPath, p);
}

std::string TreeCheck::summary() const {
  std::ostringstream out;
  out << "distance mismatches=" << distanceMismatches
      << " inconsistent parents=" << inconsistentParents
      << " non-canonical parents=" << nonCanonicalParents
      << " parent mismatches=" << parentMismatches;
  return out.str();
}

TreeCheck checkSospTree(const CsrGraph &reverse, int objective, int source,
                        const std::vector<long long> &distances, const std::vector<int> &parents,
                        const std::vector<long long> &referenceDistances,
                        const std::vector<int> *referenceParents) {
  TreeCheck check;
  const int n = reverse.numberOfNodes;
  auto finite = [](long long d) { return d < DISTANCE_INF / 2; };
  for (int v = 0; v < n; ++v) {
    const long long dv = distances[v];
    const bool reach = finite(dv);
    if (reach != finite(referenceDistances[v]) || (reach && dv != referenceDistances[v])) {
      ++check.distanceMismatches;
    }
    if (referenceParents != nullptr && parents[v] != (*referenceParents)[v]) {
      ++check.parentMismatches;
    }
    if (v == source) {
      if (parents[v] != -1 || dv != 0) ++check.inconsistentParents;
      continue;
    }
    if (!reach) {
      if (parents[v] != -1) ++check.inconsistentParents;
      continue;
    }
    const int p = parents[v];
    bool tight = false;
    int lowest = -1;
    for (int e = reverse.rowPtr[v]; e < reverse.rowPtr[v + 1]; ++e) {
      const int u = reverse.colInd[e];
      if (!finite(distances[u]) || distances[u] + reverse.weight(e, objective) != dv) continue;
      if (u == p) tight = true;
      if (lowest < 0 || u < lowest) lowest = u;
    }
    if (!tight) {
      ++check.inconsistentParents;
    } else if (p != lowest) {
      ++check.nonCanonicalParents;
    }
  }
  return check;
}

CsrGraph combinedGraphReference(const std::vector<int> &parents, int n, int K, int source,
                                const std::vector<int> &preferences) {
  const long long scale = preferenceScale(preferences, K);
  CsrGraph g;
  g.numberOfNodes = n;
  g.numberOfObjectives = 1;
  std::vector<std::vector<std::pair<int, int>>> rows(n);
  for (int v = 0; v < n; ++v) {
    if (v == source) continue;
    for (int k = 0; k < K; ++k) {
      const int p = parents[static_cast<size_t>(k) * n + v];
      bool seen = p < 0;
      for (int j = 0; j < k && !seen; ++j) seen = parents[static_cast<size_t>(j) * n + v] == p;
      if (seen) continue;
      unsigned mask = 0;
      for (int j = 0; j < K; ++j) {
        if (parents[static_cast<size_t>(j) * n + v] == p) mask |= 1u << j;
      }
      rows[p].push_back({v, static_cast<int>(combinedEdgeWeight(mask, preferences, K, scale))});
    }
  }
  g.rowPtr.assign(static_cast<size_t>(n) + 1, 0);
  for (int u = 0; u < n; ++u) {
    g.rowPtr[u + 1] = g.rowPtr[u] + static_cast<int>(rows[u].size());
    for (const auto &e : rows[u]) {
      g.colInd.push_back(e.first);
      g.weights.push_back(e.second);
    }
  }
  return g;
}
