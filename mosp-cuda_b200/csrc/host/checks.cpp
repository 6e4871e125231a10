// checks.cpp - host shortest paths and tree checks used by `mospPrep
// init|expected` and `mosp --validate` (interfaces: include/dijkstra.cuh,
// include/validation.cuh; semantics of SMShovan/MOSP-CUDA
// src/Dijkstra.cu:239-272 and src/validation.cu:28-125).
#include <algorithm>
#include <queue>
#include <sstream>
#include <thread>
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
  out << "distances off: " << distanceMismatches << ", parents not on a tight edge: "
      << inconsistentParents << ", tight but not the lowest id: " << nonCanonicalParents
      << ", parents unlike the reference: " << parentMismatches;
  return out.str();
}

namespace {

/// The four counts of TreeCheck for the vertices [lo, hi).
struct RangeVerdict {
  long long distance = 0, inconsistent = 0, nonCanonical = 0, mismatch = 0;
};

bool reachable(long long d) { return d < DISTANCE_INF / 2; }

/// Lowest in-neighbour u of v with d[u] + w(u, v) == d[v] (-1 if none), and
/// whether `p` is one of them.
std::pair<int, bool> tightParents(const CsrGraph &reverse, int objective,
                                  const std::vector<long long> &d, int v, int p) {
  int lowest = -1;
  bool pTight = false;
  for (int e = reverse.rowPtr[v]; e < reverse.rowPtr[v + 1]; ++e) {
    const int u = reverse.colInd[e];
    if (!reachable(d[u]) || d[u] + reverse.weight(e, objective) != d[v]) continue;
    lowest = lowest < 0 ? u : std::min(lowest, u);
    pTight = pTight || u == p;
  }
  return {lowest, pTight};
}

}  // namespace

TreeCheck checkSospTree(const CsrGraph &reverse, int objective, int source,
                        const std::vector<long long> &distances, const std::vector<int> &parents,
                        const std::vector<long long> &referenceDistances,
                        const std::vector<int> *referenceParents) {
  const int n = reverse.numberOfNodes;
  auto checkRange = [&](int lo, int hi) {
    RangeVerdict r;
    for (int v = lo; v < hi; ++v) {
      const long long dv = distances[v], rv = referenceDistances[v];
      if (reachable(dv) != reachable(rv) || (reachable(dv) && dv != rv)) ++r.distance;
      if (referenceParents != nullptr && parents[v] != (*referenceParents)[v]) ++r.mismatch;
      const int p = parents[v];
      if (v == source || !reachable(dv)) {
        // the source (distance 0) and unreachable vertices have no parent
        if (p != -1 || (v == source && dv != 0)) ++r.inconsistent;
        continue;
      }
      const auto [lowest, pTight] = tightParents(reverse, objective, distances, v, p);
      if (!pTight) {
        ++r.inconsistent;
      } else if (p != lowest) {
        ++r.nonCanonical;
      }
    }
    return r;
  };
  // vertex ranges checked side by side; every range's counts are summed
  const int workers = std::max(1, std::min<int>(std::thread::hardware_concurrency(), n / 65536 + 1));
  std::vector<RangeVerdict> part(workers);
  std::vector<std::thread> pool;
  for (int t = 1; t < workers; ++t) {
    pool.emplace_back([&, t] {
      part[t] = checkRange(static_cast<int>(static_cast<long long>(n) * t / workers),
                      static_cast<int>(static_cast<long long>(n) * (t + 1) / workers));
    });
  }
  part[0] = checkRange(0, static_cast<int>(static_cast<long long>(n) / workers));
  for (std::thread &th : pool) th.join();
  TreeCheck check;
  for (const RangeVerdict &r : part) {
    check.distanceMismatches += r.distance;
    check.inconsistentParents += r.inconsistent;
    check.nonCanonicalParents += r.nonCanonical;
    check.parentMismatches += r.mismatch;
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
