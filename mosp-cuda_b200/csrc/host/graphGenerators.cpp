// graphGenerators.cpp - seeded synthetic graphs of the benchmark workloads
// (interface: include/mospGenerators.h): the road-network grid and R-MAT.
// Self-contained (only the CsrGraph struct), so the benchmark's reference
// arm can build the same graphs without this library.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <iostream>
#include <numeric>
#include <random>
#include <utility>
#include <vector>

#include "csrGraph.cuh"
#include "mospGenerators.h"

namespace {

/// CSR from an undirected edge list over n vertices (both directions),
/// rows sorted by head, duplicates and self-loops removed.
void symmetricCsr(int n, std::vector<std::pair<int, int>> &edges, int K, CsrGraph &g) {
  std::vector<uint64_t> keys;
  keys.reserve(edges.size() * 2);
  for (const auto &e : edges) {
    if (e.first == e.second) continue;
    keys.push_back((static_cast<uint64_t>(e.first) << 32) | static_cast<uint32_t>(e.second));
    keys.push_back((static_cast<uint64_t>(e.second) << 32) | static_cast<uint32_t>(e.first));
  }
  std::vector<std::pair<int, int>>().swap(edges);
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  g = CsrGraph();
  g.numberOfNodes = n;
  g.numberOfObjectives = K;
  g.rowPtr.assign(static_cast<size_t>(n) + 1, 0);
  g.colInd.resize(keys.size());
  for (size_t i = 0; i < keys.size(); ++i) {
    ++g.rowPtr[(keys[i] >> 32) + 1];
    g.colInd[i] = static_cast<int>(keys[i] & 0xffffffffu);
  }
  for (int u = 0; u < n; ++u) g.rowPtr[u + 1] += g.rowPtr[u];
}

}  // namespace

bool generateGridRoad(int width, int height, double keep, double shortcutFraction, int K, int wmin,
                      int wmax, unsigned seed, CsrGraph &graph) {
  if (width < 1 || height < 1 || static_cast<long long>(width) * height > 0x7fffffffLL || K < 1 ||
      K > 32 || wmin < 1 || wmin > wmax) {
    std::cout << "Error: invalid grid-road parameters.\n";
    return false;
  }
  const int n = width * height;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> coin(0.0, 1.0);
  std::vector<std::pair<int, int>> edges;
  edges.reserve(static_cast<size_t>(2.0 * n * keep) + 16);
  for (int y = 0; y < height; ++y) {
    for (int x = 0; x < width; ++x) {
      const int u = y * width + x;
      if (x + 1 < width && coin(rng) < keep) edges.push_back({u, u + 1});
      if (y + 1 < height && coin(rng) < keep) edges.push_back({u, u + width});
    }
  }
  for (int u = 0; u < n && shortcutFraction > 0; ++u) {
    if (coin(rng) >= shortcutFraction) continue;
    const int x = u % width, y = u / width;
    const int dir = static_cast<int>(rng() & 3u);
    const int nx = x + ((dir & 1) ? 1 : -1), ny = y + ((dir & 2) ? 1 : -1);
    if (nx < 0 || nx >= width || ny < 0 || ny >= height) continue;
    edges.push_back({u, ny * width + nx});
  }
  // largest connected component (union-find), renumbered in row-major order
  std::vector<int> root(n);
  std::iota(root.begin(), root.end(), 0);
  auto find = [&](int v) {
    while (root[v] != v) {
      root[v] = root[root[v]];
      v = root[v];
    }
    return v;
  };
  for (const auto &e : edges) {
    const int a = find(e.first), b = find(e.second);
    if (a != b) root[std::max(a, b)] = std::min(a, b);
  }
  std::vector<int> size(n, 0);
  for (int v = 0; v < n; ++v) ++size[find(v)];
  const int big = static_cast<int>(std::max_element(size.begin(), size.end()) - size.begin());
  std::vector<int> id(n, -1);
  int kept = 0;
  for (int v = 0; v < n; ++v) {
    if (find(v) == big) id[v] = kept++;
  }
  std::vector<std::pair<int, int>> inside;
  inside.reserve(edges.size());
  for (const auto &e : edges) {
    if (id[e.first] >= 0 && id[e.second] >= 0) inside.push_back({id[e.first], id[e.second]});
  }
  std::vector<std::pair<int, int>>().swap(edges);
  symmetricCsr(kept, inside, K, graph);
  std::uniform_int_distribution<int> weight(wmin, wmax);
  graph.weights.resize(graph.colInd.size() * static_cast<size_t>(K));
  for (int &w : graph.weights) w = weight(rng);
  return true;
}

bool generateRmat(int scale, int edgeFactor, double a, double b, double c, int K, int wmin,
                  int wmax, bool logUniform, unsigned seed, CsrGraph &graph) {
  if (scale < 1 || scale > 30 || edgeFactor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1 ||
      K < 1 || K > 32 || wmin < 1 || wmin > wmax) {
    std::cout << "Error: invalid R-MAT parameters.\n";
    return false;
  }
  const int n = 1 << scale;
  const long long draws = static_cast<long long>(edgeFactor) * n / 2;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> coin(0.0, 1.0);
  std::vector<std::pair<int, int>> edges;
  edges.reserve(static_cast<size_t>(draws));
  for (long long i = 0; i < draws; ++i) {
    int u = 0, v = 0;
    for (int bit = scale - 1; bit >= 0; --bit) {
      const double r = coin(rng);
      if (r < a) {
      } else if (r < a + b) {
        v |= 1 << bit;
      } else if (r < a + b + c) {
        u |= 1 << bit;
      } else {
        u |= 1 << bit;
        v |= 1 << bit;
      }
    }
    edges.push_back({u, v});
  }
  symmetricCsr(n, edges, K, graph);
  graph.weights.resize(graph.colInd.size() * static_cast<size_t>(K));
  if (logUniform) {
    const double lo = std::log(static_cast<double>(wmin));
    const double hi = std::log(static_cast<double>(wmax) + 1.0);
    std::uniform_real_distribution<double> expo(lo, hi);
    for (int &w : graph.weights) {
      const double x = std::floor(std::exp(expo(rng)));
      w = static_cast<int>(std::min<double>(std::max<double>(x, wmin), wmax));
    }
  } else {
    std::uniform_int_distribution<int> weight(wmin, wmax);
    for (int &w : graph.weights) w = weight(rng);
  }
  return true;
}
