// engineApi.cpp - the reference's C++ engine interface on top of the C ABI
// (include/mosp_b200.h). Failures print the C ABI's message to stderr and
// return false, as the reference's entry points do
// (SMShovan/MOSP-CUDA src/sospUpdateGpu.cu:95-103, 685-745,
// src/deviceGraph.cu:87-135, src/combinedGraphGpu.cu:129-317).
#include <algorithm>
#include <iostream>
#include <numeric>
#include <vector>

#include "combinedGraphGpu.cuh"
#include "csrGraph.cuh"
#include "deviceGraph.cuh"
#include "mosp_b200.h"
#include "parallelCombinedGraph.cuh"
#include "sospUpdateGpu.cuh"

namespace {

bool report(int status) {
  if (status == MOSP_OK) return true;
  std::cerr << mosp_last_error() << "\n";
  return false;
}

void copyStats(const mosp_sosp_stats &from, SospStats &to) {
  to.invalidated = from.invalidated;
  to.jumpRounds = from.jump_rounds;
  to.iterations = from.iterations;
  to.epochs = from.epochs;
  to.pushes = from.pushes;
  to.packedParents = from.packed_parents != 0;
}

bool ensureHandle(SospWorkspace &ws) {
  if (ws.handle != nullptr) return true;
  return report(mosp_workspace_create(&ws.handle));
}

}  // namespace

// ---------------------------------------------------------------------------
// SospWorkspace
// ---------------------------------------------------------------------------
SospWorkspace::~SospWorkspace() { release(); }

void SospWorkspace::release() {
  if (handle != nullptr) mosp_workspace_destroy(handle);
  handle = nullptr;
  capacity = 0;
  generation = 0;
  gridBlocks = 0;
}

bool SospWorkspace::reserve(int requested) {
  if (!ensureHandle(*this)) return false;
  if (requested <= capacity) return true;
  if (!report(mosp_workspace_reserve(handle, std::max(requested, 1), 1))) return false;
  capacity = requested;
  return report(mosp_workspace_grid(handle, &gridBlocks));
}

int SospWorkspace::nextGeneration() { return ++generation; }

long long defaultDelta(long long numberOfEdges, int numberOfNodes, long long weightSum) {
  return mosp_default_delta(numberOfEdges, numberOfNodes, weightSum);
}

bool sospUpdateGpu(const DeviceCsr &out, const DeviceCsr &in, const DeviceChanges &changes,
                   int source, long long delta, long long maxWeight, SospWorkspace &ws,
                   long long *d_distances, int *d_parent, SospStats *stats) {
  const int n = out.numberOfNodes;
  SospStats local;
  SospStats &s = stats != nullptr ? *stats : local;
  s = SospStats();
  if (n == 0) return true;
  if (!ws.reserve(n) || delta <= 0) return false;
  mosp_sosp_stats st{};
  const bool ok = report(mosp_sosp_update(
      ws.handle, n, out.numberOfEdges, out.rowPtr, out.colInd, out.weights, in.rowPtr, in.colInd,
      in.weights, changes.changedFrom, changes.changedTo, changes.numberOfChanged,
      changes.insertHeads, changes.numberOfInsertHeads, source, delta, maxWeight, d_distances,
      d_parent, &st, nullptr));
  if (!ok) return false;
  copyStats(st, s);
  ws.nextGeneration();
  return true;
}

bool sospFromScratchGpu(const DeviceCsr &out, int source, long long delta, long long maxWeight,
                        SospWorkspace &ws, long long *d_distances, int *d_parent,
                        SospStats *stats) {
  const int n = out.numberOfNodes;
  SospStats local;
  SospStats &s = stats != nullptr ? *stats : local;
  s = SospStats();
  if (n == 0) return true;
  if (!ws.reserve(n) || delta <= 0 || source < 0 || source >= n) return false;
  mosp_sosp_stats st{};
  const bool ok = report(mosp_sosp_from_scratch(ws.handle, n, out.numberOfEdges, out.rowPtr,
                                                out.colInd, out.weights, source, delta, maxWeight,
                                                d_distances, d_parent, &st, nullptr));
  if (!ok) return false;
  copyStats(st, s);
  ws.nextGeneration();
  return true;
}

// ---------------------------------------------------------------------------
// DeviceGraph
// ---------------------------------------------------------------------------
DeviceCsr DeviceGraph::out(int k) const {
  DeviceCsr v;
  v.numberOfNodes = numberOfNodes;
  v.numberOfEdges = numberOfEdges;
  v.rowPtr = outRowPtr.data();
  v.colInd = outColInd.data();
  v.weights = outWeights.data() + static_cast<size_t>(k) * numberOfEdges;
  return v;
}

DeviceCsr DeviceGraph::in(int k) const {
  DeviceCsr v;
  v.numberOfNodes = numberOfNodes;
  v.numberOfEdges = numberOfEdges;
  v.rowPtr = inRowPtr.data();
  v.colInd = inColInd.data();
  v.weights = inWeights.data() + static_cast<size_t>(k) * numberOfEdges;
  return v;
}

bool uploadDeviceGraph(const CsrGraph &graph, DeviceGraph &device) {
  const int n = graph.numberOfNodes, m = graph.numberOfEdges(), K = graph.numberOfObjectives;
  device.numberOfNodes = n;
  device.numberOfEdges = m;
  device.numberOfObjectives = K;
  DeviceArray<int> edgeMajor;
  if (!device.outRowPtr.upload(graph.rowPtr) || !device.outColInd.upload(graph.colInd) ||
      !edgeMajor.upload(graph.weights) ||
      !device.outWeights.allocate(static_cast<size_t>(m) * std::max(K, 1)) ||
      !device.inRowPtr.allocate(static_cast<size_t>(n) + 1) || !device.inColInd.allocate(m) ||
      !device.inWeights.allocate(static_cast<size_t>(m) * std::max(K, 1))) {
    std::cerr << "Error: could not allocate the graph on the GPU.\n";
    return false;
  }
  if (n == 0) return true;
  mosp_workspace *ws = nullptr;
  if (!report(mosp_workspace_create(&ws))) return false;
  const bool ok = report(mosp_build_device_graph(
      ws, n, m, std::max(K, 1), device.outRowPtr.data(), device.outColInd.data(), edgeMajor.data(),
      device.outWeights.data(), device.inRowPtr.data(), device.inColInd.data(),
      device.inWeights.data(), nullptr));
  mosp_workspace_destroy(ws);
  return ok;
}

// ---------------------------------------------------------------------------
// Combined graph
// ---------------------------------------------------------------------------
CombineWorkspace::~CombineWorkspace() { release(); }

void CombineWorkspace::release() {
  capacity = 0;
  trees = 0;
}

bool CombineWorkspace::reserve(int numberOfNodes, int K) {
  capacity = std::max(capacity, numberOfNodes);
  trees = std::max(trees, K);
  return true;
}

bool combinedGraphSospGpu(const int *d_parents, int n, int K, const std::vector<int> &preferences,
                          int source, long long delta, CombineWorkspace &workspace,
                          SospWorkspace &sospWorkspace, long long *d_distances, int *d_parent,
                          CombineStats *stats) {
  CombineStats local;
  CombineStats &s = stats != nullptr ? *stats : local;
  s = CombineStats();
  if (K <= 0 || K > 32 || n <= 0 || source < 0 || source >= n) {
    std::cerr << "Error: invalid combined-graph parameters.\n";
    return false;
  }
  if (preferenceScale(preferences, K) == 0) {
    std::cerr << "Error: invalid preference vector (need K values >= 1).\n";
    return false;
  }
  if (!workspace.reserve(n, K) || !sospWorkspace.reserve(n)) return false;
  mosp_combine_stats cs{};
  const bool ok = report(mosp_combined_sosp(sospWorkspace.handle, n, K, d_parents,
                                            preferences.empty() ? nullptr : preferences.data(),
                                            source, delta, d_distances, d_parent, &cs, nullptr));
  if (!ok) return false;
  s.numberOfEdges = cs.edges;
  s.scale = cs.scale;
  s.delta = cs.delta;
  copyStats(cs.search, s.search);
  return true;
}

long long preferenceScale(const std::vector<int> &preferences, int K) {
  if (preferences.empty()) return 1;
  if (static_cast<int>(preferences.size()) != K) return 0;
  return mosp_preference_scale(preferences.data(), K);
}

long long combinedEdgeWeight(unsigned int treeMask, const std::vector<int> &preferences, int K,
                             long long scale) {
  long long w = scale * (K + 1);
  for (int i = 0; i < K; ++i) {
    if (treeMask & (1u << i)) w -= preferences.empty() ? scale : scale / preferences[i];
  }
  return w;
}

bool mospPathCosts(const CsrGraph &graph, const std::vector<int> &parent, int source,
                   std::vector<long long> &costs) {
  // Host version for in-memory callers: children lists, then a walk down
  // the tree from the source.
  const int n = graph.numberOfNodes, K = graph.numberOfObjectives;
  costs.assign(static_cast<size_t>(n) * K, DISTANCE_INF);
  std::vector<int> first(static_cast<size_t>(n) + 1, 0), kids(n);
  for (int v = 0; v < n; ++v) {
    if (v != source && parent[v] >= 0) ++first[parent[v] + 1];
  }
  for (int v = 0; v < n; ++v) first[v + 1] += first[v];
  std::vector<int> fill(first.begin(), first.end() - 1);
  for (int v = 0; v < n; ++v) {
    if (v != source && parent[v] >= 0) kids[fill[parent[v]]++] = v;
  }
  for (int k = 0; k < K; ++k) costs[static_cast<size_t>(source) * K + k] = 0;
  std::vector<int> order{source};
  for (size_t i = 0; i < order.size(); ++i) {
    const int p = order[i];
    for (int c = first[p]; c < first[p + 1]; ++c) {
      const int v = kids[c];
      int edge = -1;
      for (int e = graph.rowPtr[p]; e < graph.rowPtr[p + 1]; ++e) {
        if (graph.colInd[e] == v) {
          edge = e;
          break;
        }
      }
      if (edge < 0) return false;
      for (int k = 0; k < K; ++k) {
        costs[static_cast<size_t>(v) * K + k] =
            costs[static_cast<size_t>(p) * K + k] + graph.weight(edge, k);
      }
      order.push_back(v);
    }
  }
  return true;
}
