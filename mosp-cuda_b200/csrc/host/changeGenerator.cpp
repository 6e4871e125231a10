// changeGenerator.cpp - seeded change batches (`mospPrep changes`).
//
// Interface: include/changeGenerator.cuh. For a given graph, options and
// seed the batch must equal the reference's (SMShovan/MOSP-CUDA
// src/changeGenerator.cu:133-344), so the random draws happen in the same
// order from the same std::mt19937 stream: local-ball centre, insertion
// endpoints, deletion / re-weight picks, insertion weights, re-weight
// weights; deletions are then optionally filtered for connectivity.
#include "changeGenerator.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_set>
#include <utility>
#include <vector>

#include "csrGraph.cuh"
#include "deletionFilter.h"
#include "dijkstra.cuh"
#include "mospGenerators.h"

namespace {

using Edge = std::pair<int, int>;

uint64_t pairKey(int u, int v) {
  return (static_cast<uint64_t>(u) << 32) ^ static_cast<uint32_t>(v);
}

/// Vertices within `hops` undirected hops of centre, in BFS order (out-
/// edges before in-edges of each vertex).
std::vector<int> ball(const CsrGraph &g, const CsrGraph &rev, int centre, int hops) {
  std::vector<int> depth(g.numberOfNodes, -1), order{centre};
  depth[centre] = 0;
  for (size_t i = 0; i < order.size(); ++i) {
    const int u = order[i];
    if (depth[u] == hops) continue;
    for (const CsrGraph *h : {&g, &rev}) {
      for (int e = h->rowPtr[u]; e < h->rowPtr[u + 1]; ++e) {
        const int w = h->colInd[e];
        if (depth[w] < 0) {
          depth[w] = depth[u] + 1;
          order.push_back(w);
        }
      }
    }
  }
  return order;
}

/// Vertices reachable from source (host BFS over the out-edges).
std::vector<char> reachable(const CsrGraph &g, int source) {
  std::vector<char> seen(g.numberOfNodes, 0);
  std::vector<int> queue{source};
  seen[source] = 1;
  for (size_t i = 0; i < queue.size(); ++i) {
    const int u = queue[i];
    for (int e = g.rowPtr[u]; e < g.rowPtr[u + 1]; ++e) {
      const int w = g.colInd[e];
      if (!seen[w]) {
        seen[w] = 1;
        queue.push_back(w);
      }
    }
  }
  return seen;
}

std::atomic<bool> g_filterOnGpu{false};
double g_lastFilterMs = 0;

}  // namespace

int filterUnsafeDeletions(const CsrGraph &g, int source, ChangeBatch &batch) {
  const auto t0 = std::chrono::steady_clock::now();
  int rounds = -1;
  if (g_filterOnGpu.load()) rounds = filterUnsafeDeletionsGpu(g, source, batch);
  if (rounds < 0) {
    rounds = filterDeletionRounds(reachable(g, source), batch, [&](const ChangeBatch &b) {
      ChangeBatch applied = b;
      CsrGraph updated;
      applyChangeBatch(g, applied, updated);
      return reachable(updated, source);
    });
  }
  g_lastFilterMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return rounds;
}

void useGpuDeletionFilter(bool on) { g_filterOnGpu.store(on); }

double lastDeletionFilterMs() { return g_lastFilterMs; }

bool parseChangeMode(const std::string &name, ChangeMode &mode) {
  if (name == "uniform") {
    mode = ChangeMode::Uniform;
  } else if (name == "targeted") {
    mode = ChangeMode::Targeted;
  } else if (name == "reweight") {
    mode = ChangeMode::Reweight;
  } else if (name == "increase") {
    mode = ChangeMode::Increase;
  } else {
    return false;
  }
  return true;
}

bool generateChangeBatch(const CsrGraph &graph, const ChangeGeneratorOptions &opt,
                         ChangeBatch &batch, std::string *report) {
  const int n = graph.numberOfNodes, K = graph.numberOfObjectives;
  batch = ChangeBatch();
  batch.numberOfObjectives = K;
  if (n < 2 || K <= 0 || opt.numberOfChanges < 0 || opt.weightMin > opt.weightMax ||
      opt.weightMin < 1 || opt.source < 0 || opt.source >= n) {
    std::cout << "Error: invalid change generator options.\n";
    return false;
  }
  const ChangeMode mode = opt.mode;
  const bool insertDelete = mode == ChangeMode::Uniform || mode == ChangeMode::Targeted;
  const bool onTrees = mode == ChangeMode::Targeted || mode == ChangeMode::Increase;
  int nIns = 0, nDel = 0, nRe = 0;
  if (insertDelete) {
    nIns = static_cast<int>(std::llround(opt.numberOfChanges * opt.insertionPercentage / 100.0));
    nIns = std::max(0, std::min(nIns, opt.numberOfChanges));
    nDel = opt.numberOfChanges - nIns;
  } else {
    nRe = opt.numberOfChanges;
  }
  std::mt19937 rng(opt.seed);
  std::uniform_int_distribution<int> anyWeight(opt.weightMin, opt.weightMax);

  // region of a local batch
  std::vector<int> region;
  std::vector<char> inRegion;
  int centre = -1;
  if (opt.localHops > 0) {
    CsrGraph rev;
    transposeCsrGraph(graph, rev);
    centre = std::uniform_int_distribution<int>(0, n - 1)(rng);
    region = ball(graph, rev, centre, opt.localHops);
    inRegion.assign(n, 0);
    for (int v : region) inRegion[v] = 1;
    if (region.size() < 2) {
      std::cout << "Error: local region around vertex " << centre << " has fewer than 2 vertices.\n";
      return false;
    }
  }
  auto pickVertex = [&]() {
    if (region.empty()) return std::uniform_int_distribution<int>(0, n - 1)(rng);
    return region[std::uniform_int_distribution<size_t>(0, region.size() - 1)(rng)];
  };
  auto allowed = [&](int v) { return inRegion.empty() || inRegion[v]; };

  std::vector<std::vector<int>> trees;
  if (onTrees) {
    // the K trees are independent: one thread each
    trees.resize(K);
    std::vector<std::thread> threads;
    for (int k = 0; k < K; ++k) {
      threads.emplace_back([&graph, &trees, &opt, k] {
        std::vector<long long> dist;
        dijkstraCsrGraph(graph, k, opt.source, dist, trees[k]);
      });
    }
    for (auto &t : threads) t.join();
  }

  std::vector<Edge> inserts;
  inserts.reserve(nIns);
  while (static_cast<int>(inserts.size()) < nIns) {
    const int u = pickVertex();
    const int v = pickVertex();
    if (u != v) inserts.push_back({u, v});
  }

  // existing edges that may be deleted / re-weighted: tree edges (by head,
  // objective order) or all edges (row order), first occurrence of each
  // pair, no self-loops
  std::vector<Edge> deletes, reweights;
  if (nDel > 0 || nRe > 0) {
    // A pair (u,v) can repeat only inside row u (all edges) or among the K
    // parents of v (tree edges), so the first occurrences are found per row
    // / per vertex, in parallel over vertex ranges, and concatenated in
    // order: the pool equals a sequential scan with a global seen-set.
    std::vector<Edge> pool;
    const int parts = static_cast<int>(std::max<long long>(
        1, std::min<long long>(std::max(1u, std::thread::hardware_concurrency()),
                               (static_cast<long long>(graph.numberOfEdges()) + n) >> 18)));
    std::vector<std::vector<Edge>> pieces(parts);
    std::vector<std::thread> threads;
    for (int j = 0; j < parts; ++j) {
      threads.emplace_back([&, j] {
        const int lo = static_cast<int>(static_cast<long long>(n) * j / parts);
        const int hi = static_cast<int>(static_cast<long long>(n) * (j + 1) / parts);
        std::vector<Edge> &out = pieces[j];
        if (onTrees) {
          for (int v = lo; v < hi; ++v) {
            if (!allowed(v)) continue;
            for (int k = 0; k < K; ++k) {
              const int p = trees[k][v];
              bool first = p >= 0;
              for (int q = 0; q < k && first; ++q) first = trees[q][v] != p;
              if (first) out.push_back({p, v});
            }
          }
        } else {
          std::vector<int> stamp(n, -1);  // row that last listed v
          for (int u = lo; u < hi; ++u) {
            if (!allowed(u)) continue;
            for (int e = graph.rowPtr[u]; e < graph.rowPtr[u + 1]; ++e) {
              const int v = graph.colInd[e];
              if (u == v || !allowed(v) || stamp[v] == u) continue;
              stamp[v] = u;
              out.push_back({u, v});
            }
          }
        }
      });
    }
    for (auto &t : threads) t.join();
    for (auto &piece : pieces) pool.insert(pool.end(), piece.begin(), piece.end());
    if (pool.empty()) {
      std::cout << "Error: No existing edges available for the batch.\n";
      return false;
    }
    const int wanted = std::max(nDel, nRe);
    std::vector<Edge> &chosen = nDel > 0 ? deletes : reweights;
    if (mode == ChangeMode::Uniform || mode == ChangeMode::Reweight) {
      std::uniform_int_distribution<int> pick(0, static_cast<int>(pool.size()) - 1);
      for (int i = 0; i < wanted; ++i) chosen.push_back(pool[pick(rng)]);
    } else {
      std::shuffle(pool.begin(), pool.end(), rng);
      chosen.assign(pool.begin(), pool.begin() + std::min<size_t>(pool.size(), wanted));
    }
  }

  std::vector<int> lowWeight(K, opt.weightMax);
  if (mode == ChangeMode::Targeted && graph.numberOfEdges() > 0) {
    for (int k = 0; k < K; ++k) {
      double sum = 0;
      for (int e = 0; e < graph.numberOfEdges(); ++e) sum += graph.weight(e, k);
      const int average = static_cast<int>(sum / graph.numberOfEdges());
      lowWeight[k] = std::max(opt.weightMin, average - 1);
    }
  }
  for (const Edge &x : inserts) {
    batch.insertFrom.push_back(x.first);
    batch.insertTo.push_back(x.second);
    for (int k = 0; k < K; ++k) {
      const int w = mode == ChangeMode::Targeted
                        ? std::uniform_int_distribution<int>(opt.weightMin, lowWeight[k])(rng)
                        : anyWeight(rng);
      batch.insertWeights.push_back(w);
    }
  }
  for (const Edge &x : reweights) {
    const int u = x.first, v = x.second;
    int e = graph.rowPtr[u];
    while (graph.colInd[e] != v) ++e;
    batch.insertFrom.push_back(u);
    batch.insertTo.push_back(v);
    for (int k = 0; k < K; ++k) {
      const int w = mode == ChangeMode::Increase
                        ? graph.weight(e, k) + std::uniform_int_distribution<int>(1, opt.weightMax)(rng)
                        : anyWeight(rng);
      batch.insertWeights.push_back(w);
    }
  }
  for (const Edge &x : deletes) {
    batch.deleteFrom.push_back(x.first);
    batch.deleteTo.push_back(x.second);
  }
  int rounds = 0;
  const int requested = batch.numberOfDeletes();
  if (opt.safeDeletions) rounds = filterUnsafeDeletions(graph, opt.source, batch);
  if (report != nullptr) {
    std::ostringstream out;
    out << "inserts=" << batch.numberOfInserts() - static_cast<int>(reweights.size())
        << " reweights=" << reweights.size() << " deletes=" << batch.numberOfDeletes();
    if (opt.safeDeletions) {
      out << " (safe: kept " << batch.numberOfDeletes() << " of " << requested << " after "
          << rounds << " rounds)";
    }
    if (centre >= 0) {
      out << " local centre=" << centre << " hops=" << opt.localHops << " region=" << region.size()
          << " vertices";
    }
    *report = out.str();
  }
  return true;
}

bool writeChangeBatch(const ChangeBatch &batch, const std::string &insertPath,
                      const std::string &deletePath) {
  for (const std::string &p : {insertPath, deletePath}) {
    const std::filesystem::path parent = std::filesystem::path(p).parent_path();
    if (!parent.empty()) {
      std::error_code ec;
      std::filesystem::create_directories(parent, ec);
    }
  }
  std::ofstream ins(insertPath), del(deletePath);
  if (!ins.is_open() || !del.is_open()) {
    std::cout << "Error: Could not open change-edge output files for writing.\n";
    return false;
  }
  const int K = batch.numberOfObjectives;
  std::string line;
  for (int i = 0; i < batch.numberOfInserts(); ++i) {
    line = std::to_string(batch.insertFrom[i]) + " " + std::to_string(batch.insertTo[i]);
    for (int k = 0; k < K; ++k) {
      line += " " + std::to_string(batch.insertWeights[static_cast<size_t>(i) * K + k]);
    }
    line += "\n";
    ins << line;
  }
  for (int i = 0; i < batch.numberOfDeletes(); ++i) {
    del << batch.deleteFrom[i] << " " << batch.deleteTo[i] << "\n";
  }
  return ins.good() && del.good();
}
