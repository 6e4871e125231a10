// mospPipeline.cpp - one MOSP update from host memory (the reference's
// in-memory pipeline, SMShovan/MOSP-CUDA src/mospUpdate.cu:57-225) and the
// file-based wrappers (src/parallelSOSPUpdate.cu, src/parallelCombinedGraph
// .cu). Stages: upload the original out-CSR, the batch and the trees; apply
// the batch on the GPU (Step 1), build the reverse CSR and weight columns on
// the GPU, run the K SOSP updates as one fused launch and Steps 2-3 as a
// second one, optionally the MOSP path costs on the GPU, download.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "combinedGraphGpu.cuh"
#include "csrGraph.cuh"
#include "deviceGraph.cuh"
#include "hostCore.h"
#include "mospUpdate.cuh"
#include "mosp_b200.h"
#include "parallelCombinedGraph.cuh"
#include "parallelSOSPUpdate.cuh"
#include "sospUpdateGpu.cuh"
#include "stageTimer.cuh"

namespace mospb200 {
namespace {

double msSince(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

/// Device buffers of one pipeline run, taken from workspace slots so that
/// repeated runs reuse them.
enum Slot : int {
  kOutRow, kOutCol, kEdgeW, kOutW, kInRow, kInCol, kInW, kDist, kParent, kHeads,
  kChFrom, kChTo, kCombDist, kCombParent, kCosts, kOrigRow, kOrigCol, kOrigW, kInsFrom,
  kInsW, kDelFrom, kDelTo, kMask
};

template <typename T>
bool slot(mosp_workspace *ws, int s, size_t count, T *&ptr, std::string &err) {
  void *p = nullptr;
  if (mosp_workspace_buffer(ws, s, std::max<size_t>(count, 1) * sizeof(T), &p) != MOSP_OK) {
    err = mosp_last_error();
    return false;
  }
  ptr = static_cast<T *>(p);
  return true;
}

template <typename T>
bool toDevice(T *dst, const T *src, size_t count, std::string &err) {
  if (count == 0) return true;
  const cudaError_t e = cudaMemcpy(dst, src, count * sizeof(T), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    err = std::string("CUDA error: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

template <typename T>
bool toHost(T *dst, const T *src, size_t count, std::string &err) {
  if (count == 0) return true;
  const cudaError_t e = cudaMemcpy(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    err = std::string("CUDA error: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

template <typename T>
bool toDeviceAsync(T *dst, const T *src, size_t count, cudaStream_t s, std::string &err) {
  if (count == 0) return true;
  const cudaError_t e = cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) {
    err = std::string("CUDA error: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

template <typename T>
bool toHostAsync(T *dst, const T *src, size_t count, cudaStream_t s, std::string &err) {
  if (count == 0) return true;
  const cudaError_t e = cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) {
    err = std::string("CUDA error: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

bool syncStream(cudaStream_t s, std::string &err) {
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    err = std::string("CUDA error: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

/// The pipeline's two streams (per host thread): the main stream runs the
/// batch upload, Step 1 and the engine; the side stream moves the trees
/// (upload while Step 1 runs, the K trees' download while the combined step
/// runs, the combined tree's while the path costs run).
struct PipelineStreams {
  cudaStream_t main = nullptr, side = nullptr;
  cudaEvent_t treesIn = nullptr, updated = nullptr, combined = nullptr;
  int device = -1;
  ~PipelineStreams() { release(); }
  void release() {
    if (device < 0) return;
    int current = -1;
    cudaGetDevice(&current);
    cudaSetDevice(device);
    if (treesIn) cudaEventDestroy(treesIn);
    if (updated) cudaEventDestroy(updated);
    if (combined) cudaEventDestroy(combined);
    if (main) cudaStreamDestroy(main);
    if (side) cudaStreamDestroy(side);
    treesIn = updated = combined = nullptr;
    main = side = nullptr;
    device = -1;
    if (current >= 0) cudaSetDevice(current);
  }
  /// Streams of the current device (recreated when the thread's device
  /// changed since the last call).
  bool ready(std::string &err) {
    int dev = -1;
    cudaGetDevice(&dev);
    if (main != nullptr && dev == device) return true;
    release();
    if (cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&treesIn, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&updated, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&combined, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      err = "Error: stream creation failed.";
      return false;
    }
    device = dev;
    return true;
  }
};

}  // namespace

struct PipelineIn {
  GraphView g;
  BatchView b;
  const long long *initDist = nullptr;  // K * n
  const int *initParent = nullptr;      // K * n
  int K = 0;
  int source = 0;
  const int *pref = nullptr;            // K values or null
  long long delta = 0;
  bool costs = false;
  bool wantUpdated = false;  // download the updated graph into PipelineOut::updated
};

struct PipelineOut {
  CsrGraph updated;
  std::vector<unsigned> mask;
  long long *dist = nullptr;       // K * n (host)
  int *parent = nullptr;           // K * n (host)
  long long *combDist = nullptr;   // n
  int *combParent = nullptr;       // n
  long long *costs = nullptr;      // n * KG (when requested)
  std::vector<mosp_sosp_stats> stats;
  mosp_combine_stats cstats{};
  mosp_timings t{};
};

/// Returns a MOSP status; on failure `err` holds the message.
int runPipeline(mosp_workspace *ws, const PipelineIn &in, PipelineOut &out, std::string &err) {
  const int n = in.g.n, KG = in.g.K, K = in.K;
  if (n <= 0 || K <= 0 || K > KG || K > MOSP_MAX_OBJECTIVES || in.source < 0 || in.source >= n ||
      in.initDist == nullptr || in.initParent == nullptr) {
    err = "Error: invalid MOSP update input.";
    return MOSP_ERR_INVALID;
  }
  for (int k = 0; k < K; ++k) {
    const size_t at = static_cast<size_t>(k) * n + in.source;
    if (in.initDist[at] != 0 || in.initParent[at] != -1) {
      err = "Error: the initial tree of objective " + std::to_string(k) +
            " is not rooted at the source " + std::to_string(in.source) + " (its distance is " +
            (in.initDist[at] >= DISTANCE_INF / 2 ? std::string("INF")
                                                  : std::to_string(in.initDist[at])) +
            ", its parent " + std::to_string(in.initParent[at]) +
            "); compute the trees for this source.";
      return MOSP_ERR_INVALID;
    }
  }
  if (in.b.K != KG) {
    err = "Error: change batch has " + std::to_string(in.b.K) + " objectives, graph has " +
          std::to_string(KG) + ".";
    return MOSP_ERR_INVALID;
  }
  const long long m0 = in.g.edges();
  const int nIns = in.b.nIns, nDel = in.b.nDel;
  const size_t kn = static_cast<size_t>(K) * n;
  const size_t cap = static_cast<size_t>(m0) + nIns;

  // make the workspace's device current (the workspace checks it on every
  // call), then take this thread's streams of that device
  int ctas = 0;
  if (mosp_workspace_grid(ws, &ctas) != MOSP_OK) {
    err = mosp_last_error();
    return MOSP_ERR_CUDA;
  }
  thread_local PipelineStreams streams;
  if (!streams.ready(err)) return MOSP_ERR_CUDA;
  cudaStream_t sm = streams.main, ss = streams.side;
  // every return waits for both streams, so no copy into a caller's buffer
  // is still in flight when the call returns (error paths included)
  struct Drain {
    cudaStream_t a, b;
    ~Drain() {
      cudaStreamSynchronize(a);
      cudaStreamSynchronize(b);
    }
  } drain{sm, ss};

  // --- upload the original graph, the batch and the trees -----------------------
  auto t0 = std::chrono::steady_clock::now();
  int *dOrigRow, *dOrigCol, *dOrigW, *dInsFrom, *dInsTo, *dInsW, *dDelFrom, *dDelTo;
  unsigned *dMask;
  int *dOutRow, *dOutCol, *dEdgeW, *dOutW, *dInRow, *dInCol, *dInW, *dParent, *dChFrom, *dChTo,
      *dCombParent;
  long long *dDist, *dCombDist, *dCosts = nullptr;
  {
    ScopedStage stage("upload", true);
    if (!slot(ws, kOrigRow, static_cast<size_t>(n) + 1, dOrigRow, err) ||
        !slot(ws, kOrigCol, m0, dOrigCol, err) ||
        !slot(ws, kOrigW, static_cast<size_t>(m0) * KG, dOrigW, err) ||
        !slot(ws, kInsFrom, nIns, dInsFrom, err) || !slot(ws, kHeads, nIns, dInsTo, err) ||
        !slot(ws, kInsW, static_cast<size_t>(nIns) * KG, dInsW, err) ||
        !slot(ws, kDelFrom, nDel, dDelFrom, err) || !slot(ws, kDelTo, nDel, dDelTo, err) ||
        !slot(ws, kMask, nIns, dMask, err) || !slot(ws, kDist, kn, dDist, err) ||
        !slot(ws, kParent, kn, dParent, err)) {
      return MOSP_ERR_OOM;
    }
    // graph and batch on the main stream (Step 1 needs them); the trees on
    // the side stream, overlapping Step 1 and the graph build
    if (!toDeviceAsync(dOrigRow, in.g.row, static_cast<size_t>(n) + 1, sm, err) ||
        !toDeviceAsync(dOrigCol, in.g.col, m0, sm, err) ||
        !toDeviceAsync(dOrigW, in.g.w, static_cast<size_t>(m0) * KG, sm, err) ||
        !toDeviceAsync(dInsFrom, in.b.insFrom, nIns, sm, err) ||
        !toDeviceAsync(dInsTo, in.b.insTo, nIns, sm, err) ||
        !toDeviceAsync(dInsW, in.b.insW, static_cast<size_t>(nIns) * KG, sm, err) ||
        !toDeviceAsync(dDelFrom, in.b.delFrom, nDel, sm, err) ||
        !toDeviceAsync(dDelTo, in.b.delTo, nDel, sm, err) ||
        !toDeviceAsync(dDist, in.initDist, kn, ss, err) ||
        !toDeviceAsync(dParent, in.initParent, kn, ss, err) ||
        cudaEventRecord(streams.treesIn, ss) != cudaSuccess || !syncStream(sm, err)) {
      return MOSP_ERR_CUDA;
    }
  }
  out.t.upload = msSince(t0);

  // --- Step 1 on the GPU: apply the batch ------------------------------------------
  // per objective: largest weight (original edges and inserts), weight sum
  // of the original edges, and the changes that may invalidate a subtree
  t0 = std::chrono::steady_clock::now();
  std::vector<long long> maxWeight(KG, 1), weightSum(KG, 0), delta(K, in.delta);
  int m = 0;
  {
    ScopedStage stage("apply_batch_gpu", true);
    if (!slot(ws, kOutRow, static_cast<size_t>(n) + 1, dOutRow, err) ||
        !slot(ws, kOutCol, cap, dOutCol, err) || !slot(ws, kEdgeW, cap * KG, dEdgeW, err)) {
      return MOSP_ERR_OOM;
    }
    int st = mosp_apply_batch_device(ws, n, KG, static_cast<int>(m0), dOrigRow, dOrigCol, dOrigW,
                                     nIns, dInsFrom, dInsTo, dInsW, nDel, dDelFrom, dDelTo,
                                     dOutRow, dOutCol, dEdgeW, static_cast<long long>(cap), &m,
                                     dMask, maxWeight.data(), weightSum.data(), sm);
    if (st != MOSP_OK) {
      err = mosp_last_error();
      return st;
    }
    out.mask.assign(nIns, 0u);
    if (!toHostAsync(out.mask.data(), dMask, nIns, sm, err) || !syncStream(sm, err)) {
      return MOSP_ERR_CUDA;
    }
  }
  std::vector<int> chFrom, chTo, chOffset(K + 1, 0);
  for (int k = 0; k < K; ++k) {
    chFrom.insert(chFrom.end(), in.b.delFrom, in.b.delFrom + nDel);
    chTo.insert(chTo.end(), in.b.delTo, in.b.delTo + nDel);
    for (int i = 0; i < nIns; ++i) {
      if (out.mask[i] & (1u << k)) {
        chFrom.push_back(in.b.insFrom[i]);
        chTo.push_back(in.b.insTo[i]);
      }
    }
    chOffset[k + 1] = static_cast<int>(chFrom.size());
    if (in.delta <= 0) {
      delta[k] = mosp_default_delta(m0 > 0 ? m0 : std::max(m, 1), n, weightSum[k]);
    }
  }
  if (!slot(ws, kChFrom, chFrom.size(), dChFrom, err) ||
      !slot(ws, kChTo, chTo.size(), dChTo, err) ||
      !toDeviceAsync(dChFrom, chFrom.data(), chFrom.size(), sm, err) ||
      !toDeviceAsync(dChTo, chTo.data(), chTo.size(), sm, err)) {
    return MOSP_ERR_CUDA;
  }
  if (in.wantUpdated) {
    // the reference API returns the updated graph on the host
    CsrGraph &up = out.updated;
    up = CsrGraph();
    up.numberOfNodes = n;
    up.numberOfObjectives = KG;
    up.rowPtr.resize(static_cast<size_t>(n) + 1);
    up.colInd.resize(m);
    up.weights.resize(static_cast<size_t>(m) * KG);
    if (!toHostAsync(up.rowPtr.data(), dOutRow, up.rowPtr.size(), sm, err) ||
        !toHostAsync(up.colInd.data(), dOutCol, up.colInd.size(), sm, err) ||
        !toHostAsync(up.weights.data(), dEdgeW, up.weights.size(), sm, err) || !syncStream(sm, err)) {
      return MOSP_ERR_CUDA;
    }
  }
  out.t.apply_batch = msSince(t0);

  // --- device graph: weight columns and reverse CSR, built on the GPU --------------
  t0 = std::chrono::steady_clock::now();
  {
    ScopedStage stage("build_device_graph", true);
    if (!slot(ws, kOutW, static_cast<size_t>(m) * KG, dOutW, err) ||
        !slot(ws, kInRow, static_cast<size_t>(n) + 1, dInRow, err) ||
        !slot(ws, kInCol, m, dInCol, err) ||
        !slot(ws, kInW, static_cast<size_t>(m) * KG, dInW, err) ||
        !slot(ws, kCombDist, n, dCombDist, err) || !slot(ws, kCombParent, n, dCombParent, err) ||
        (in.costs && !slot(ws, kCosts, static_cast<size_t>(n) * KG, dCosts, err))) {
      return MOSP_ERR_OOM;
    }
    const int st = mosp_build_device_graph(ws, n, m, KG, dOutRow, dOutCol, dEdgeW, dOutW, dInRow,
                                           dInCol, dInW, sm);
    if (st != MOSP_OK) {
      err = mosp_last_error();
      return st;
    }
  }
  out.t.upload += msSince(t0);

  // --- K SOSP updates (one fused launch) ------------------------------------------
  t0 = std::chrono::steady_clock::now();
  out.stats.assign(K, mosp_sosp_stats{});
  {
    ScopedStage stage("sosp_update_gpu", true);
    const int *outW[MOSP_MAX_OBJECTIVES], *inW[MOSP_MAX_OBJECTIVES];
    const int *cf[MOSP_MAX_OBJECTIVES], *ct[MOSP_MAX_OBJECTIVES];
    int nc[MOSP_MAX_OBJECTIVES];
    long long *dd[MOSP_MAX_OBJECTIVES];
    int *dp[MOSP_MAX_OBJECTIVES];
    for (int k = 0; k < K; ++k) {
      outW[k] = dOutW + static_cast<size_t>(k) * m;
      inW[k] = dInW + static_cast<size_t>(k) * m;
      cf[k] = dChFrom + chOffset[k];
      ct[k] = dChTo + chOffset[k];
      nc[k] = chOffset[k + 1] - chOffset[k];
      dd[k] = dDist + static_cast<size_t>(k) * n;
      dp[k] = dParent + static_cast<size_t>(k) * n;
    }
    // the trees must have arrived
    if (cudaStreamWaitEvent(sm, streams.treesIn, 0) != cudaSuccess) {
      err = "Error: stream wait failed.";
      return MOSP_ERR_CUDA;
    }
    const int st = mosp_sosp_update_multi(ws, n, m, K, dOutRow, dOutCol, outW, dInRow, dInCol, inW,
                                          cf, ct, nc, dInsTo, in.b.nIns, in.source, delta.data(),
                                          maxWeight.data(), dd, dp, out.stats.data(), sm);
    if (st != MOSP_OK) {
      err = mosp_last_error();
      return st;
    }
  }
  out.t.objectives = msSince(t0);
  // the K trees go back on the side stream while Steps 2-3 run
  if (cudaEventRecord(streams.updated, sm) != cudaSuccess ||
      cudaStreamWaitEvent(ss, streams.updated, 0) != cudaSuccess ||
      !toHostAsync(out.dist, dDist, kn, ss, err) || !toHostAsync(out.parent, dParent, kn, ss, err)) {
    if (err.empty()) err = "Error: stream wait failed.";
    return MOSP_ERR_CUDA;
  }

  // --- Steps 2-3: combined graph and its SOSP tree ----------------------------
  t0 = std::chrono::steady_clock::now();
  {
    ScopedStage stage("combined_graph_gpu", true);
    const int st = mosp_combined_sosp(ws, n, K, dParent, in.pref, in.source, 0, dCombDist,
                                      dCombParent, &out.cstats, sm);
    if (st != MOSP_OK) {
      err = mosp_last_error();
      return st;
    }
  }
  out.t.combined = msSince(t0);
  // the combined tree goes back on the side stream while the costs run
  if (cudaEventRecord(streams.combined, sm) != cudaSuccess ||
      cudaStreamWaitEvent(ss, streams.combined, 0) != cudaSuccess ||
      !toHostAsync(out.combDist, dCombDist, static_cast<size_t>(n), ss, err) ||
      !toHostAsync(out.combParent, dCombParent, static_cast<size_t>(n), ss, err)) {
    if (err.empty()) err = "Error: stream wait failed.";
    return MOSP_ERR_CUDA;
  }

  if (in.costs) {
    t0 = std::chrono::steady_clock::now();
    ScopedStage stage("mosp_costs_gpu", true);
    const int st = mosp_path_costs(ws, n, m, KG, dOutRow, dOutCol, dOutW, dCombParent, in.source,
                                   dCosts, sm);
    if (st != MOSP_OK) {
      err = mosp_last_error();
      return st;
    }
    out.t.costs = msSince(t0);
  }

  // --- download -------------------------------------------------------------------
  t0 = std::chrono::steady_clock::now();
  {
    ScopedStage stage("download", true);
    if ((in.costs && !toHostAsync(out.costs, dCosts, static_cast<size_t>(n) * KG, sm, err)) ||
        !syncStream(sm, err) || !syncStream(ss, err)) {
      return MOSP_ERR_CUDA;
    }
  }
  out.t.download = msSince(t0);
  return MOSP_OK;
}

/// Per-thread default workspace of the C++ entry points.
mosp_workspace *defaultWorkspace() {
  struct Holder {
    mosp_workspace *ws = nullptr;
    ~Holder() {
      if (ws != nullptr) mosp_workspace_destroy(ws);
    }
  };
  thread_local Holder holder;
  if (holder.ws == nullptr && mosp_workspace_create(&holder.ws) != MOSP_OK) holder.ws = nullptr;
  return holder.ws;
}

}  // namespace mospb200

using namespace mospb200;

// ---------------------------------------------------------------------------
// C++ API
// ---------------------------------------------------------------------------
double MospTimings::gpuCompute() const {
  double total = combined;
  for (double t : objectives) total += t;
  return total;
}

void canonicalizeTree(const CsrGraph &graph, int objective, int source,
                      const std::vector<long long> &distances, int *parent) {
  for (int u = 0; u < graph.numberOfNodes; ++u) {
    const long long du = distances[u];
    if (du >= DISTANCE_INF / 2) continue;
    for (int e = graph.rowPtr[u]; e < graph.rowPtr[u + 1]; ++e) {
      const int v = graph.colInd[e];
      if (v != source && u < parent[v] && du + graph.weight(e, objective) == distances[v]) {
        parent[v] = u;
      }
    }
  }
}

bool mospUpdate(const CsrGraph &original, ChangeBatch &batch,
                const std::vector<long long> &initialDistances,
                const std::vector<int> &initialParents, const MospOptions &options,
                CsrGraph &updated, MospResult &result) {
  return mospUpdateWithCosts(original, batch, initialDistances, initialParents, options, updated,
                             result, nullptr);
}

bool mospUpdateWithCosts(const CsrGraph &original, ChangeBatch &batch,
                         const std::vector<long long> &initialDistances,
                         const std::vector<int> &initialParents, const MospOptions &options,
                         CsrGraph &updated, MospResult &result, std::vector<long long> *costs) {
  const int n = original.numberOfNodes;
  const int KG = original.numberOfObjectives;
  const int K = options.numberOfObjectives > 0 ? std::min(options.numberOfObjectives, KG) : KG;
  const size_t kn = static_cast<size_t>(K) * n;
  result = MospResult();
  result.numberOfObjectives = K;
  if (n <= 0 || K <= 0 || options.source < 0 || options.source >= n ||
      initialDistances.size() < kn || initialParents.size() < kn) {
    std::cerr << "Error: invalid MOSP update input.\n";
    return false;
  }
  if (!options.preferences.empty() && static_cast<int>(options.preferences.size()) != K) {
    std::cerr << "Error: invalid preference vector (need K values >= 1).\n";
    return false;
  }
  mosp_workspace *ws = defaultWorkspace();
  if (ws == nullptr) {
    std::cerr << mosp_last_error() << "\n";
    return false;
  }
  mosp_workspace_set_canonical_trees(ws, options.canonicalTrees ? 1 : 0);
  PipelineIn in;
  in.g = viewOf(original);
  in.b = viewOf(batch);
  in.initDist = initialDistances.data();
  in.initParent = initialParents.data();
  in.K = K;
  in.source = options.source;
  in.pref = options.preferences.empty() ? nullptr : options.preferences.data();
  in.delta = options.delta;
  in.costs = costs != nullptr;
  in.wantUpdated = true;
  if (costs != nullptr) costs->assign(static_cast<size_t>(n) * KG, DISTANCE_INF);
  result.distances.resize(kn);
  result.parents.resize(kn);
  result.combinedDistances.resize(n);
  result.combinedParent.resize(n);
  PipelineOut out;
  out.dist = result.distances.data();
  out.parent = result.parents.data();
  out.combDist = result.combinedDistances.data();
  out.combParent = result.combinedParent.data();
  out.costs = costs != nullptr ? costs->data() : nullptr;
  std::string err;
  const int st = runPipeline(ws, in, out, err);
  if (!out.mask.empty() || batch.numberOfInserts() == 0) batch.weightIncreaseMask = out.mask;
  updated = std::move(out.updated);
  if (st != MOSP_OK) {
    std::cerr << err << "\n";
    return false;
  }
  MospTimings &tm = result.timings;
  tm.applyBatch = out.t.apply_batch;
  tm.upload = out.t.upload;
  tm.objectives.assign(K, out.t.objectives / K);
  tm.combined = out.t.combined;
  tm.download = out.t.download;
  result.objectiveStats.resize(K);
  for (int k = 0; k < K; ++k) {
    SospStats &s = result.objectiveStats[k];
    const mosp_sosp_stats &x = out.stats[k];
    s.invalidated = x.invalidated;
    s.jumpRounds = x.jump_rounds;
    s.iterations = x.iterations;
    s.epochs = x.epochs;
    s.pushes = x.pushes;
    s.packedParents = x.packed_parents != 0;
  }
  CombineStats &c = result.combineStats;
  c.numberOfEdges = out.cstats.edges;
  c.scale = out.cstats.scale;
  c.delta = out.cstats.delta;
  c.search.iterations = out.cstats.search.iterations;
  c.search.epochs = out.cstats.search.epochs;
  c.search.pushes = out.cstats.search.pushes;
  c.search.packedParents = out.cstats.search.packed_parents != 0;
  return true;
}

// ---------------------------------------------------------------------------
// C ABI: the whole update from host buffers
// ---------------------------------------------------------------------------
extern "C" int mosp_update_host(mosp_workspace *ws, int n, int KG, int m, const int *h_row,
                                const int *h_col, const int *h_w, int n_ins,
                                const int *h_ins_from, const int *h_ins_to, const int *h_ins_w,
                                int n_del, const int *h_del_from, const int *h_del_to,
                                const long long *h_init_dist, const int *h_init_parent, int K,
                                int source, const int *h_pref, long long delta, long long *h_dist,
                                int *h_parent, long long *h_comb_dist, int *h_comb_parent,
                                long long *h_costs, mosp_timings *timings) {
  if (ws == nullptr || n <= 0 || KG <= 0 || m < 0 || h_row == nullptr ||
      (m > 0 && (h_col == nullptr || h_w == nullptr)) || n_ins < 0 || n_del < 0 ||
      (n_ins > 0 && (h_ins_from == nullptr || h_ins_to == nullptr || h_ins_w == nullptr)) ||
      (n_del > 0 && (h_del_from == nullptr || h_del_to == nullptr)) || h_dist == nullptr ||
      h_parent == nullptr || h_comb_dist == nullptr || h_comb_parent == nullptr ||
      h_row[n] != m) {
    std::fprintf(stderr, "Error: invalid MOSP update input.\n");
    return MOSP_ERR_INVALID;
  }
  for (int i = 0; i < n_ins; ++i) {
    if (h_ins_from[i] < 0 || h_ins_from[i] >= n || h_ins_to[i] < 0 || h_ins_to[i] >= n) {
      std::fprintf(stderr, "Error: inserted edge endpoint out of range.\n");
      return MOSP_ERR_INVALID;
    }
  }
  for (int i = 0; i < n_del; ++i) {
    if (h_del_from[i] < 0 || h_del_from[i] >= n || h_del_to[i] < 0 || h_del_to[i] >= n) {
      std::fprintf(stderr, "Error: deleted edge endpoint out of range.\n");
      return MOSP_ERR_INVALID;
    }
  }
  PipelineIn in;
  in.g = GraphView{n, KG, h_row, h_col, h_w};
  in.b = BatchView{KG, n_ins, n_del, h_ins_from, h_ins_to, h_ins_w, h_del_from, h_del_to};
  in.initDist = h_init_dist;
  in.initParent = h_init_parent;
  in.K = K > 0 ? std::min(K, KG) : KG;
  in.source = source;
  in.pref = h_pref;
  in.delta = delta;
  in.costs = h_costs != nullptr;
  PipelineOut out;
  out.dist = h_dist;
  out.parent = h_parent;
  out.combDist = h_comb_dist;
  out.combParent = h_comb_parent;
  out.costs = h_costs;
  std::string err;
  const int st = runPipeline(ws, in, out, err);
  if (st != MOSP_OK) {
    std::fprintf(stderr, "%s\n", err.c_str());
    return st;
  }
  if (timings != nullptr) *timings = out.t;
  return MOSP_OK;
}

// ---------------------------------------------------------------------------
// File-based wrappers
// ---------------------------------------------------------------------------
bool parallelSOSPUpdate(const std::string &originalCsrPrefix, const std::string &distancesInputPath,
                        const std::string &treeInputPath, const std::string &insertPath,
                        const std::string &deletePath, int objectiveIndex, int source,
                        const std::string &distancesOutputPath, const std::string &treeOutputPath) {
  CsrGraph graph, updated;
  if (!readCsrGraph(originalCsrPrefix, graph)) {
    std::cout << "Error: Could not read original CSR graph.\n";
    return false;
  }
  const int n = graph.numberOfNodes;
  if (objectiveIndex < 0 || objectiveIndex >= graph.numberOfObjectives) {
    std::cout << "Error: objectiveIndex out of range.\n";
    return false;
  }
  if (source < 0 || source >= n) {
    std::cout << "Error: source vertex out of range.\n";
    return false;
  }
  std::vector<long long> dist;
  std::vector<int> parent;
  ChangeBatch batch;
  if (!readDistances(distancesInputPath, n, dist) || !readParents(treeInputPath, n, parent) ||
      !readChangeBatch(insertPath, deletePath, graph.numberOfObjectives, n, batch) ||
      !applyChangeBatch(graph, batch, updated)) {
    return false;
  }
  const int k = objectiveIndex;
  std::vector<int> chFrom(batch.deleteFrom), chTo(batch.deleteTo);
  for (int i = 0; i < batch.numberOfInserts(); ++i) {
    if (batch.weightIncreaseMask[i] & (1u << k)) {
      chFrom.push_back(batch.insertFrom[i]);
      chTo.push_back(batch.insertTo[i]);
    }
  }
  // the bound on the distances covers the old tree (original weights) and
  // the new one (updated weights)
  long long weightSum = 0, maxWeight = 1;
  for (int e = 0; e < graph.numberOfEdges(); ++e) {
    maxWeight = std::max(maxWeight, static_cast<long long>(graph.weight(e, k)));
  }
  for (int e = 0; e < updated.numberOfEdges(); ++e) {
    weightSum += updated.weight(e, k);
    maxWeight = std::max(maxWeight, static_cast<long long>(updated.weight(e, k)));
  }
  const long long delta = defaultDelta(updated.numberOfEdges(), n, weightSum);
  DeviceGraph device;
  DeviceArray<int> dFrom, dTo, dHeads, dParent;
  DeviceArray<long long> dDist;
  SospWorkspace ws;
  if (!uploadDeviceGraph(updated, device) || !dFrom.upload(chFrom) || !dTo.upload(chTo) ||
      !dHeads.upload(batch.insertTo) || !dDist.upload(dist) || !dParent.upload(parent) ||
      !ws.reserve(n)) {
    std::cout << "Error: could not copy the graph to the GPU.\n";
    return false;
  }
  DeviceChanges changes;
  changes.changedFrom = dFrom.data();
  changes.changedTo = dTo.data();
  changes.numberOfChanged = static_cast<int>(chFrom.size());
  changes.insertHeads = dHeads.data();
  changes.numberOfInsertHeads = batch.numberOfInserts();
  SospStats stats;
  if (!sospUpdateGpu(device.out(k), device.in(k), changes, source, delta, maxWeight, ws,
                     dDist.data(), dParent.data(), &stats)) {
    std::cout << "Error: SOSP update failed on the GPU.\n";
    return false;
  }
  recordCounter("sosp/invalidated", stats.invalidated);
  recordCounter("sosp/iterations", stats.iterations);
  recordCounter("sosp/pushes", static_cast<double>(stats.pushes));
  if (!dDist.download(dist) || !dParent.download(parent)) {
    std::cout << "Error: could not copy the result from the GPU.\n";
    return false;
  }
  return writeDistances(distancesOutputPath, dist) && writeParents(treeOutputPath, parent);
}

namespace {

/// Vertex count of a text CSR: values in <prefix>RowPtr.txt minus one.
int csrNodeCount(const std::string &prefix) {
  FILE *f = std::fopen((prefix + "RowPtr.txt").c_str(), "rb");
  if (f == nullptr) return -1;
  static thread_local char buf[1 << 16];
  long long values = 0;
  bool inNumber = false;
  size_t got;
  while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) {
    for (size_t i = 0; i < got; ++i) {
      const bool digit = buf[i] >= '0' && buf[i] <= '9';
      if (digit && !inNumber) ++values;
      inNumber = digit;
    }
  }
  std::fclose(f);
  return static_cast<int>(values - 1);
}

}  // namespace

bool parallelCombinedGraph(const std::string &originalCsrPrefix,
                           const std::vector<std::string> &treeInputPaths, int K, int source,
                           const std::string & /*workDir*/, const std::string &distancesOutputPath,
                           const std::string &treeOutputPath, const std::vector<int> &preferences) {
  if (K <= 0 || static_cast<int>(treeInputPaths.size()) < K) {
    std::cout << "Error: K=" << K << " but only " << treeInputPaths.size()
              << " tree paths supplied.\n";
    return false;
  }
  if (K > 32) {
    std::cout << "Error: at most 32 objectives are supported.\n";
    return false;
  }
  if (preferenceScale(preferences, K) == 0) {
    std::cout << "Error: invalid preference vector (need K values >= 1).\n";
    return false;
  }
  const int n = csrNodeCount(originalCsrPrefix);
  if (n <= 0) {
    std::cout << "Error: Could not read the vertex count of " << originalCsrPrefix << "\n";
    return false;
  }
  if (source < 0 || source >= n) {
    std::cout << "Error: source vertex " << source << " out of range.\n";
    return false;
  }
  std::vector<int> parents(static_cast<size_t>(n) * K);
  for (int k = 0; k < K; ++k) {
    std::vector<int> p;
    if (!readParents(treeInputPaths[k], n, p)) return false;
    std::copy(p.begin(), p.end(), parents.begin() + static_cast<size_t>(k) * n);
  }
  DeviceArray<int> dParents, dParent(n);
  DeviceArray<long long> dDist(n);
  CombineWorkspace cws;
  SospWorkspace ws;
  if (!dParents.upload(parents) || !cws.reserve(n, K) || !ws.reserve(n)) {
    std::cout << "Error: could not allocate the combined graph on the GPU.\n";
    return false;
  }
  CombineStats stats;
  if (!combinedGraphSospGpu(dParents.data(), n, K, preferences, source, 0, cws, ws, dDist.data(),
                            dParent.data(), &stats)) {
    std::cout << "Error: combined graph failed on the GPU.\n";
    return false;
  }
  std::vector<long long> dist;
  std::vector<int> parent;
  if (!dDist.download(dist) || !dParent.download(parent) ||
      !writeDistances(distancesOutputPath, dist) || !writeParents(treeOutputPath, parent)) {
    std::cout << "Error: could not write the combined graph result.\n";
    return false;
  }
  std::cout << "parallelCombinedGraph: " << stats.numberOfEdges << " edges, " << n
            << " vertices; output written to:\n  Distances: " << distancesOutputPath
            << "\n  SSSP Tree: " << treeOutputPath << "\n";
  return true;
}
