// capi.cu - the C ABI of the engine (include/mosp_b200.h): workspace
// management, argument checks, packing choice, launches and the readback
// of the device control blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "engine.h"
#include "mosp_b200.h"

using namespace mospb200;

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
namespace {
thread_local std::string g_lastError;

int fail(int status, const std::string &message) {
  g_lastError = message;
  return status;
}

int cudaFail(cudaError_t err, const char *what) {
  return fail(MOSP_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(err) + " (" +
                                 what + ")");
}

#define MOSP_CUDA(call)                                   \
  do {                                                    \
    cudaError_t err_ = (call);                            \
    if (err_ != cudaSuccess) return cudaFail(err_, #call); \
  } while (0)

constexpr int kControlBlocks = 4;  // 0: update/scratch, 1: combined, 2: build, 3: costs

}  // namespace

int mospb200::recordFailure(int status, const char *message) { return fail(status, message); }

// ---------------------------------------------------------------------------
// Workspace
// ---------------------------------------------------------------------------
struct mosp_workspace {
  int device = -1;
  long long timeoutNs = 10000LL * 1000000LL;
  int ctasPerSm = 0;
  bool shapeValid = false;
  LaunchShape shape{};
  // engine lists: kCap objectives x nCap vertices
  long long nCap = 0;
  int kCap = 0;
  u64 *packed = nullptr;
  int *val = nullptr, *stamp = nullptr, *inFar = nullptr, *cand = nullptr;
  int *far0 = nullptr, *far1 = nullptr;
  // near lists (vertex, distance tag): kCap objectives x nearCap entries
  long long nearCap = 0;
  int nearK = 0;
  int *nearV0 = nullptr, *nearV1 = nullptr;
  u64 *nearD0 = nullptr, *nearD1 = nullptr;
  int *gen = nullptr;  // device stamp generation
  bool dirty = false;  // an aborted run may have left inFar/stamp set (or queue slots filled)
  // asynchronous near queue: aqCap slots (all ~0 between launches) in
  // kAsyncShards shards, two counter sets
  u64 *aqSlots = nullptr;
  long long aqCap = 0;
  AsyncShard *aqCtr = nullptr;
  // near-far loop: 1 asynchronous where the graph allows it, 0 bulk
  // (mosp_workspace_set_async); results do not depend on it
  int asyncMode = 1;
  long long asyncSlots = 0;  // queue size set by the caller (0: asyncSlotsFor)
  // the last launch of each kind (0: update / scratch, 1: combined) found
  // hub rows, so the next one goes straight to the bulk loop with its full
  // stage
  bool heavySeen[2] = {false, false};
  // grid of the persistent engine launches (0: one CTA per SM, all SMs) and
  // the hub-row threshold (0: the engine's default); autotuned, results do
  // not depend on them
  int gridCtas = 0;
  int heavyDeg = 0;
  int graphCtas = 0;  // grid of the captured CUDA graph
  // control blocks
  EngineControl *ctl = nullptr;
  EngineControl *hostCtl = nullptr;  // pinned
  long long *blockSums = nullptr;
  int blockSumsCap = 0;
  // combined graph
  long long combN = 0, combEdgesCap = 0;
  int *combDeg = nullptr, *combRow = nullptr, *combCol = nullptr, *combW = nullptr;
  // reverse-CSR build cursor
  long long cursorCap = 0;
  int *cursor = nullptr;
  // path costs
  long long costN = 0;
  int costKG = 0;
  int *edgeOf = nullptr, *anc0 = nullptr, *anc1 = nullptr;
  long long *acc0 = nullptr, *acc1 = nullptr;
  // per-launch timing (mosp_workspace_enable_timing)
  bool timing = false;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  float lastUpdateMs = 0, lastCombinedMs = 0;
  // caller buffers (mosp_workspace_buffer)
  void *user[32] = {nullptr};
  unsigned long long userBytes[32] = {0};
  // Step 1 scratch (mosp_apply_batch_device)
  void *applyScratch = nullptr;
  size_t applyBytes = 0;
  // roots of batched runs (mosp_workspace_set_sources): sorted, > 1 entries
  std::vector<int> hostSources;
  int *sources = nullptr;
  int nSources = 0;
  // near-far width of the combined step in mosp_update_device (0: default)
  long long combDelta = 0;
  // CTA-local expansion rounds per near-far iteration: update launches,
  // and from-scratch / combined-graph launches
  int roundsUpdate = 0;
  int roundsScratch = 2;
  // narrow iterations (few items) run on one CTA with many local rounds
  int narrowItems = 512;
  int narrowRounds = 64;
  // input trees declared canonical (mosp_workspace_set_canonical_trees):
  // distance-only objectives recover parents only where the batch reaches;
  // mark bytes (recMarkCap = K x n) and the list of long rows
  bool canonicalTrees = false;
  unsigned char *recMark = nullptr;
  int *recVerts = nullptr;  // changed lists, then scan lists (2 x recMarkCap)
  long long recMarkCap = 0;
  u64 *recChunks = nullptr;  // two chunk lists of recChunkCap entries
  long long recChunkCap = 0;
  // CUDA graph of mosp_update_device's launch sequence (mosp_workspace_use_graphs)
  bool useGraphs = false;
  cudaStream_t captureStream = nullptr;
  cudaGraphExec_t graphExec = nullptr;
  EngineParams graphPu{}, graphPc{};
  int graphReplays = 0;
};

namespace {

template <typename T>
int deviceAlloc(T **ptr, size_t count) {
  if (*ptr != nullptr) cudaFree(*ptr);
  *ptr = nullptr;
  cudaError_t err = cudaMalloc(reinterpret_cast<void **>(ptr), std::max<size_t>(count, 1) * sizeof(T));
  if (err != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    return fail(MOSP_ERR_OOM, std::string("device allocation of ") +
                                  std::to_string(count * sizeof(T)) + " bytes failed: " +
                                  cudaGetErrorString(err));
  }
  return MOSP_OK;
}

void releaseNear(mosp_workspace *ws) {
  for (void *p : {static_cast<void *>(ws->nearV0), static_cast<void *>(ws->nearV1),
                  static_cast<void *>(ws->nearD0), static_cast<void *>(ws->nearD1)}) {
    if (p) cudaFree(p);
  }
  ws->nearV0 = ws->nearV1 = nullptr;
  ws->nearD0 = ws->nearD1 = nullptr;
  ws->nearCap = 0;
  ws->nearK = 0;
}

void releaseAsync(mosp_workspace *ws) {
  if (ws->aqSlots) cudaFree(ws->aqSlots);
  if (ws->aqCtr) cudaFree(ws->aqCtr);
  ws->aqSlots = nullptr;
  ws->aqCtr = nullptr;
  ws->aqCap = 0;
}

void releaseLists(mosp_workspace *ws) {
  for (void *p : {static_cast<void *>(ws->packed), static_cast<void *>(ws->val),
                  static_cast<void *>(ws->stamp), static_cast<void *>(ws->inFar),
                  static_cast<void *>(ws->cand), static_cast<void *>(ws->far0),
                  static_cast<void *>(ws->far1)}) {
    if (p) cudaFree(p);
  }
  ws->packed = nullptr;
  ws->val = ws->stamp = ws->inFar = ws->cand = nullptr;
  ws->far0 = ws->far1 = nullptr;
  ws->nCap = 0;
  ws->kCap = 0;
  releaseNear(ws);
  releaseAsync(ws);
}

/// CTAs of a persistent launch whose occupancy-sized grid is `full`: that
/// grid, or fewer when the workspace asks for it (also what keeps several
/// workspaces' cooperative grids on disjoint SMs).
int limitCtas(const mosp_workspace *ws, int full) {
  return ws->gridCtas > 0 && ws->gridCtas < full ? ws->gridCtas : full;
}

int engineCtas(const mosp_workspace *ws) { return limitCtas(ws, ws->shape.engineCtas); }

int ensureShape(mosp_workspace *ws) {
  if (ws->shapeValid) return MOSP_OK;
  MOSP_CUDA(cudaSetDevice(ws->device));
  cudaError_t err = queryLaunchShape(ws->ctasPerSm, ws->shape);
  if (err == cudaErrorNotSupported) {
    return fail(MOSP_ERR_UNSUPPORTED, "the GPU does not support cooperative launches");
  }
  if (err != cudaSuccess) return cudaFail(err, "occupancy query");
  const int maxCtas = std::max({ws->shape.engineCtas, ws->shape.buildCtas, ws->shape.costCtas});
  if (maxCtas > ws->blockSumsCap) {
    int st = deviceAlloc(&ws->blockSums, maxCtas);
    if (st != MOSP_OK) return st;
    ws->blockSumsCap = maxCtas;
  }
  ws->shapeValid = true;
  return MOSP_OK;
}

/// Near lists of K objectives (bulk loop). One iteration appends at most one
/// entry per relaxation (<= m) and a split at most one per far-pile vertex
/// (<= n), but the lists hold min(n + m, max(2n, 2^20)) + 64 entries each:
/// appends past that go to the far pile (divertToFar), which the next split
/// brings back, so the cap bounds memory without changing results.
int reserveNear(mosp_workspace *ws, long long n, long long m, int K) {
  long long need = std::min(n + m, std::max(2 * n, 1LL << 20)) + 64;
  if (ws->asyncSlots > 0) {
    // the caller's bound on the near queue caps the bulk loop's lists too
    need = std::min(need, std::max(ws->asyncSlots, 1024LL));
    if (need == ws->nearCap && K <= ws->nearK && ws->nearV0 != nullptr) return MOSP_OK;
  } else if (need <= ws->nearCap && K <= ws->nearK && ws->nearV0 != nullptr) {
    return MOSP_OK;
  }
  const long long cap = std::max(need, ws->nearCap);
  const int kk = std::max(K, ws->nearK);
  releaseNear(ws);
  const size_t total = static_cast<size_t>(cap) * kk;
  int st = MOSP_OK;
  if ((st = deviceAlloc(&ws->nearV0, total)) != MOSP_OK) return st;
  if ((st = deviceAlloc(&ws->nearV1, total)) != MOSP_OK) return st;
  if ((st = deviceAlloc(&ws->nearD0, total)) != MOSP_OK) return st;
  if ((st = deviceAlloc(&ws->nearD1, total)) != MOSP_OK) return st;
  ws->nearCap = cap;
  ws->nearK = kk;
  return MOSP_OK;
}

/// Slots of the asynchronous near queue for K objectives of n vertices:
/// one entry per vertex and objective plus n, at least 2^20 (or the size
/// the caller set), in whole 32-slot claims per shard. A phase that pushes
/// more moves the excess to the far piles, so this bounds memory, not
/// correctness.
long long asyncSlotsFor(long long n, int K, long long fixed = 0) {
  const long long want = fixed > 0 ? fixed : std::max(n * K + n, 1LL << 20);
  const long long perShard = (want + kAsyncShards - 1) / kAsyncShards;
  return (perShard + 31) / 32 * 32 * kAsyncShards;
}

int reserveAsync(mosp_workspace *ws, long long n, int K) {
  if (ws->asyncMode == 0) return MOSP_OK;
  int st = MOSP_OK;
  if (ws->aqCtr == nullptr) {
    if ((st = deviceAlloc(&ws->aqCtr, 2 * kAsyncShards)) != MOSP_OK) return st;
  }
  const long long need = asyncSlotsFor(n, K, ws->asyncSlots);
  if (need == ws->aqCap && ws->aqSlots != nullptr) return MOSP_OK;
  if (ws->asyncSlots == 0 && need < ws->aqCap && ws->aqSlots != nullptr) return MOSP_OK;
  if ((st = deviceAlloc(&ws->aqSlots, need)) != MOSP_OK) {
    ws->aqCap = 0;
    return st;
  }
  MOSP_CUDA(cudaMemset(ws->aqSlots, 0xff, need * sizeof(u64)));
  ws->aqCap = need;
  return MOSP_OK;
}

int reserveLists(mosp_workspace *ws, long long n, int K) {
  if (n <= ws->nCap && K <= ws->kCap) return MOSP_OK;
  const long long newN = std::max(n, ws->nCap);
  const int newK = std::max(K, ws->kCap);
  releaseLists(ws);
  const size_t total = static_cast<size_t>(newN) * newK;
  int st = MOSP_OK;
  if ((st = deviceAlloc(&ws->packed, total)) != MOSP_OK) return st;
  for (int **p : {&ws->val, &ws->stamp, &ws->inFar, &ws->cand, &ws->far0, &ws->far1}) {
    if ((st = deviceAlloc(p, total)) != MOSP_OK) {
      releaseLists(ws);
      return st;
    }
  }
  MOSP_CUDA(cudaMemset(ws->stamp, 0, total * sizeof(int)));
  MOSP_CUDA(cudaMemset(ws->inFar, 0, total * sizeof(int)));
  MOSP_CUDA(cudaMemset(ws->gen, 0, sizeof(int)));
  ws->nCap = newN;
  ws->kCap = newK;
  ws->dirty = false;
  return MOSP_OK;
}

/// Clear the dedup state after an aborted run, or before the stamp
/// generation could overflow.
int cleanLists(mosp_workspace *ws, cudaStream_t s) {
  const size_t total = static_cast<size_t>(ws->nCap) * ws->kCap;
  if (ws->dirty) {
    MOSP_CUDA(cudaMemsetAsync(ws->inFar, 0, total * sizeof(int), s));
    MOSP_CUDA(cudaMemsetAsync(ws->stamp, 0, total * sizeof(int), s));
    MOSP_CUDA(cudaMemsetAsync(ws->gen, 0, sizeof(int), s));
    if (ws->aqSlots != nullptr) {
      MOSP_CUDA(cudaMemsetAsync(ws->aqSlots, 0xff, ws->aqCap * sizeof(u64), s));
    }
    ws->dirty = false;
  }
  return MOSP_OK;
}

/// After a synchronous run: restart the generations well before they wrap.
int maybeResetGenerations(mosp_workspace *ws, int finalGen, cudaStream_t s) {
  if (finalGen > INT_MAX / 2) {
    const size_t total = static_cast<size_t>(ws->nCap) * ws->kCap;
    MOSP_CUDA(cudaMemsetAsync(ws->stamp, 0, total * sizeof(int), s));
    MOSP_CUDA(cudaMemsetAsync(ws->gen, 0, sizeof(int), s));
    MOSP_CUDA(cudaStreamSynchronize(s));
  }
  return MOSP_OK;
}

int reserveCombined(mosp_workspace *ws, long long n, int K) {
  int st = MOSP_OK;
  if (n > ws->combN) {
    if ((st = deviceAlloc(&ws->combDeg, n + 1)) != MOSP_OK) return st;
    if ((st = deviceAlloc(&ws->combRow, n + 1)) != MOSP_OK) return st;
    ws->combN = n;
  }
  const long long edges = n * K;
  if (edges > ws->combEdgesCap) {
    if ((st = deviceAlloc(&ws->combCol, edges)) != MOSP_OK) return st;
    if ((st = deviceAlloc(&ws->combW, edges)) != MOSP_OK) return st;
    ws->combEdgesCap = edges;
  }
  return MOSP_OK;
}

cudaStream_t asStream(void *s) { return static_cast<cudaStream_t>(s); }

/// Bits of the parent field and the distance bound (reference
/// src/sospUpdateGpu.cu:133-143, 670-681).
int choosePacking(long long n, long long maxWeight, int &bits, u64 &maxDist) {
  const u64 outputMax = static_cast<u64>(MOSP_DISTANCE_INF / 2 - 1);
  const u64 weight = static_cast<u64>(std::max(maxWeight, 1LL));
  const u64 hops = static_cast<u64>(std::max(n - 1, 1LL));
  if (weight > outputMax / hops) {
    return fail(MOSP_ERR_OVERFLOW, "Error: distances up to " + std::to_string(weight) + " * " +
                                       std::to_string(hops) + " do not fit in 62 bits.");
  }
  maxDist = weight * hops;
  int b = 1;
  while ((1ULL << b) - 1 < static_cast<u64>(n)) ++b;
  const u64 storable = (kInfWord >> b) - 1;
  bits = maxDist <= storable ? b : 0;
  return MOSP_OK;
}

void setObjective(ObjectiveArgs &o, int bits, u64 maxDist, long long delta) {
  o.parentBits = bits;
  o.noParent = bits > 0 ? ((1ULL << bits) - 1) : 0;
  o.maxDist = maxDist;
  o.delta = static_cast<u64>(delta);
}

/// Tuning switches of the engine (EngineParams::flags) from the
/// environment variable MOSP_ENGINE_FLAGS (decimal); results do not depend
/// on them.
int engineFlags() {
  static const int flags = [] {
    const char *e = std::getenv("MOSP_ENGINE_FLAGS");
    return e != nullptr ? std::atoi(e) : 0;
  }();
  return flags;
}

/// A source argument must be one of the workspace's roots in batched mode.
int checkRoot(mosp_workspace *ws, int source) {
  if (ws->nSources > 1 &&
      !std::binary_search(ws->hostSources.begin(), ws->hostSources.end(), source)) {
    return fail(MOSP_ERR_INVALID, "Error: the source is not one of the workspace's roots "
                                  "(mosp_workspace_set_sources).");
  }
  return MOSP_OK;
}

void fillLists(EngineParams &p, mosp_workspace *ws, int block) {
  p.localRounds = p.mode == kModeUpdate ? ws->roundsUpdate : ws->roundsScratch;
  p.narrowItems = ws->narrowItems;
  p.narrowRounds = ws->narrowRounds;
  p.sources = ws->nSources > 1 ? ws->sources : nullptr;
  p.nSources = ws->nSources > 1 ? ws->nSources : 0;
  p.flags = engineFlags();
  if (p.mode == kModeUpdate && p.recMark != nullptr) p.flags |= kFlagCanonical;
  p.heavyDeg = ws->heavyDeg;
  // asynchronous loop unless it is off or the graph last seen here had hub
  // rows; its launches need a smaller stage (the pull pass stays staged up
  // to K tiles), which leaves more of the SM's memory to L1
  const bool async = ws->asyncMode != 0 && ws->aqSlots != nullptr &&
                     ws->aqCap >= asyncSlotsFor(p.n, p.K, ws->asyncSlots) &&
                     !ws->heavySeen[block == 1 ? 1 : 0];
  if (async) {
    p.flags |= kFlagAsync;
    p.aqSlots = ws->aqSlots;
    p.aqCtr = ws->aqCtr;
    p.aqShards = kAsyncShards;
    p.aqShardCap = static_cast<unsigned>(ws->aqCap / kAsyncShards);
    p.stageEntries = std::min(kStageEntriesMax, std::max(kStageEntriesAsync, p.K * kThreads));
  } else {
    p.stageEntries = kStageEntriesMax;
  }
  p.timeoutNs = ws->timeoutNs;
  p.genPtr = ws->gen;
  p.packed = ws->packed;
  p.val = ws->val;
  p.stamp = ws->stamp;
  p.inFar = ws->inFar;
  p.cand = ws->cand;
  p.nearV0 = ws->nearV0;
  p.nearV1 = ws->nearV1;
  p.nearD0 = ws->nearD0;
  p.nearD1 = ws->nearD1;
  p.strideNear = ws->nearCap;
  p.farL0 = ws->far0;
  p.farL1 = ws->far1;
  p.stride = ws->nCap;
  p.ctl = ws->ctl + block;
  p.blockSums = ws->blockSums;
}

int maxRoundsFor(long long n) {
  int rounds = 0;
  while ((1LL << rounds) < n) ++rounds;
  return rounds + 1;
}

int markEvent(mosp_workspace *ws, int i, cudaStream_t s) {
  if (!ws->timing) return MOSP_OK;
  if (ws->ev[i] == nullptr) MOSP_CUDA(cudaEventCreate(&ws->ev[i]));
  MOSP_CUDA(cudaEventRecord(ws->ev[i], s));
  return MOSP_OK;
}

/// Durations between the recorded events (after the stream was synced).
void readEvents(mosp_workspace *ws, float *first, float *second) {
  if (!ws->timing) return;
  if (first != nullptr) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ws->ev[0], ws->ev[1]) == cudaSuccess) *first = ms;
  }
  if (second != nullptr) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ws->ev[1], ws->ev[2]) == cudaSuccess) *second = ms;
  }
}

/// Queue one engine launch (control block `block` is cleared first).
int queueEngine(mosp_workspace *ws, const EngineParams &p, int block, cudaStream_t s) {
  MOSP_CUDA(cudaMemsetAsync(ws->ctl + block, 0, sizeof(EngineControl), s));
  if (needsHostRecovery(p)) {
    // distance-only objectives: the parent recovery follows as its own kernel
    EngineParams q = p;
    q.flags |= kFlagHostRecovery;
    MOSP_CUDA(launchEngine(q, engineCtas(ws), s));
    MOSP_CUDA(launchRecovery(q, s));
    return MOSP_OK;
  }
  MOSP_CUDA(launchEngine(p, engineCtas(ws), s));
  return MOSP_OK;
}

/// Copy control blocks [first, first + count) to the host and wait.
int readControl(mosp_workspace *ws, int first, int count, cudaStream_t s) {
  MOSP_CUDA(cudaMemcpyAsync(ws->hostCtl + first, ws->ctl + first, count * sizeof(EngineControl),
                            cudaMemcpyDeviceToHost, s));
  cudaError_t err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return cudaFail(err, "engine run");
  return MOSP_OK;
}

/// mosp_update_device's launch sequence (clear control block 0, update
/// launch, clear control block 1, combined launch, control blocks to the
/// pinned host copy) as one CUDA graph: captured on the workspace's own
/// stream the first time and again whenever the launch parameters change,
/// replayed on `s` otherwise. The caller waits on `s`.
int launchUpdateGraph(mosp_workspace *ws, const EngineParams &pu, const EngineParams &pc,
                      cudaStream_t s) {
  const bool same = ws->graphExec != nullptr && ws->graphCtas == engineCtas(ws) &&
                    std::memcmp(&ws->graphPu, &pu, sizeof(EngineParams)) == 0 &&
                    std::memcmp(&ws->graphPc, &pc, sizeof(EngineParams)) == 0;
  if (!same) {
    if (ws->graphExec) {
      cudaGraphExecDestroy(ws->graphExec);
      ws->graphExec = nullptr;
    }
    if (ws->captureStream == nullptr) {
      MOSP_CUDA(cudaStreamCreateWithFlags(&ws->captureStream, cudaStreamNonBlocking));
    }
    cudaStream_t c = ws->captureStream;
    MOSP_CUDA(cudaStreamBeginCapture(c, cudaStreamCaptureModeThreadLocal));
    cudaError_t err = cudaMemsetAsync(ws->ctl, 0, sizeof(EngineControl), c);
    if (needsHostRecovery(pu)) {
      EngineParams q = pu;
      q.flags |= kFlagHostRecovery;
      if (err == cudaSuccess) err = launchEngineEx(q, engineCtas(ws), c);
      if (err == cudaSuccess) err = launchRecovery(q, c);
    } else if (err == cudaSuccess) {
      err = launchEngineEx(pu, engineCtas(ws), c);
    }
    if (err == cudaSuccess) err = cudaMemsetAsync(ws->ctl + 1, 0, sizeof(EngineControl), c);
    if (err == cudaSuccess) err = launchEngineEx(pc, engineCtas(ws), c);
    if (err == cudaSuccess) {
      err = cudaMemcpyAsync(ws->hostCtl, ws->ctl, 2 * sizeof(EngineControl),
                            cudaMemcpyDeviceToHost, c);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t endErr = cudaStreamEndCapture(c, &graph);
    if (err == cudaSuccess) err = endErr;
    if (err == cudaSuccess) err = cudaGraphInstantiate(&ws->graphExec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (err != cudaSuccess) {
      cudaGetLastError();
      ws->graphExec = nullptr;
      return cudaFail(err, "capturing the update as a CUDA graph");
    }
    ws->graphPu = pu;
    ws->graphPc = pc;
    ws->graphCtas = engineCtas(ws);
  }
  MOSP_CUDA(cudaGraphLaunch(ws->graphExec, s));
  ++ws->graphReplays;
  return MOSP_OK;
}

/// Device-side status of a finished run.
int controlStatus(mosp_workspace *ws, const EngineControl &c) {
  if (c.status != 0) {
    ws->dirty = true;
    return fail(MOSP_ERR_TIMEOUT,
                "Error: a device-side wait of the persistent kernel exceeded its limit; the run "
                "was stopped.");
  }
  if (c.invalid) {
    ws->dirty = true;
    return fail(MOSP_ERR_INVALID,
                "Error: malformed input (a vertex id, parent or change endpoint out of range, a "
                "cycle in the parent array, or a tree edge missing from the graph).");
  }
  if (c.overflow) {
    return fail(MOSP_ERR_OVERFLOW,
                "Error: an input distance is negative or larger than (n - 1) * maxWeight; the "
                "initial tree does not belong to this graph.");
  }
  return MOSP_OK;
}

void fillStats(const EngineControl &c, int k, int bits, mosp_sosp_stats *s) {
  s->invalidated = c.invalidated[k];
  s->jump_rounds = c.rounds;
  s->iterations = c.iterations[k];
  s->epochs = c.epochs[k];
  s->pushes = c.pushes[k];
  s->packed_parents = bits > 0 ? 1 : 0;
  s->reserved = 0;
}

int checkWorkspace(mosp_workspace *ws) {
  if (ws == nullptr) return fail(MOSP_ERR_INVALID, "null workspace");
  int dev = -1;
  MOSP_CUDA(cudaGetDevice(&dev));
  if (dev != ws->device) MOSP_CUDA(cudaSetDevice(ws->device));
  return ensureShape(ws);
}

struct UpdateArgs {
  int n, m, K;
  const int *outRow, *outCol, *inRow, *inCol;
  const int *const *outW;
  const int *const *inW;
  const int *const *chFrom;
  const int *const *chTo;
  const int *nChanged;
  const int *heads;
  int nHeads, source;
  const long long *delta;
  const long long *maxWeight;
  long long *const *dist;
  int *const *parent;
};

/// Build the parameters of a fused K-objective update.
/// Buffers of the restricted parent recovery: per objective and vertex of
/// the engine lists one mark byte and two list slots (the changed and the
/// scan list), and two chunk lists with room for every chunk of every row
/// of more than kRecLightRow edges (at most m / kRecLightRow + 1 per
/// objective).
int reserveRecovery(mosp_workspace *ws, long long m, int K) {
  int st = MOSP_OK;
  const long long marks = ws->nCap * ws->kCap;
  if (marks > ws->recMarkCap) {
    ws->recMarkCap = 0;
    // whole 32-bit words: the marks are set with atomicOr on their word
    if ((st = deviceAlloc(&ws->recMark, (marks + 3) / 4 * 4)) != MOSP_OK) return st;
    if ((st = deviceAlloc(&ws->recVerts, 2 * marks)) != MOSP_OK) return st;
    ws->recMarkCap = marks;
  }
  const long long chunks = static_cast<long long>(K) * (m / kRecLightRow + 1) + 64;
  if (chunks > INT_MAX) return fail(MOSP_ERR_INVALID, "Error: graph too large for the parent recovery lists.");
  if (chunks > ws->recChunkCap) {
    ws->recChunkCap = 0;
    if ((st = deviceAlloc(&ws->recChunks, 2 * chunks)) != MOSP_OK) return st;
    ws->recChunkCap = chunks;
  }
  return MOSP_OK;
}

int prepareUpdate(mosp_workspace *ws, const UpdateArgs &a, EngineParams &p, int *bitsOut) {
  if (a.n <= 0 || a.m < 0 || a.K < 1 || a.K > kMaxK || a.source < 0 || a.source >= a.n ||
      a.nHeads < 0 || (a.nHeads > 0 && a.heads == nullptr) || a.outRow == nullptr ||
      a.inRow == nullptr || (a.m > 0 && (a.outCol == nullptr || a.inCol == nullptr))) {
    return fail(MOSP_ERR_INVALID, "Error: invalid SOSP update arguments.");
  }
  int st = checkRoot(ws, a.source);
  if (st != MOSP_OK) return st;
  st = reserveLists(ws, a.n, a.K);
  if (st != MOSP_OK) return st;
  if ((st = reserveNear(ws, a.n, a.m, a.K)) != MOSP_OK) return st;
  if ((st = reserveAsync(ws, a.n, a.K)) != MOSP_OK) return st;
  std::memset(&p, 0, sizeof(p));
  p.n = a.n;
  p.m = a.m;
  p.K = a.K;
  p.source = a.source;
  p.mode = kModeUpdate;
  p.maxRounds = maxRoundsFor(a.n);
  p.nHeads = a.nHeads;
  p.outRow = a.outRow;
  p.outCol = a.outCol;
  p.inRow = a.inRow;
  p.inCol = a.inCol;
  p.heads = a.heads;
  for (int k = 0; k < a.K; ++k) {
    if (a.delta[k] <= 0) return fail(MOSP_ERR_INVALID, "Error: delta must be positive.");
    if (a.nChanged[k] < 0 || (a.nChanged[k] > 0 && (a.chFrom[k] == nullptr || a.chTo[k] == nullptr)) ||
        a.dist[k] == nullptr || a.parent[k] == nullptr || (a.m > 0 && (a.outW[k] == nullptr || a.inW[k] == nullptr))) {
      return fail(MOSP_ERR_INVALID, "Error: invalid SOSP update arguments.");
    }
    int bits = 0;
    u64 maxDist = 0;
    if ((st = choosePacking(a.n, a.maxWeight[k], bits, maxDist)) != MOSP_OK) return st;
    ObjectiveArgs &o = p.obj[k];
    o.outW = a.outW[k];
    o.inW = a.inW[k];
    o.dist = a.dist[k];
    o.parent = a.parent[k];
    o.chFrom = a.chFrom[k];
    o.chTo = a.chTo[k];
    o.nChanged = a.nChanged[k];
    setObjective(o, bits, maxDist, a.delta[k]);
    bitsOut[k] = bits;
  }
  if (ws->canonicalTrees && std::any_of(bitsOut, bitsOut + a.K, [](int b) { return b == 0; })) {
    if ((st = reserveRecovery(ws, a.m, a.K)) != MOSP_OK) return st;
    p.recMark = ws->recMark;
    p.recChangedList = ws->recVerts;
    p.recScanList = ws->recVerts + ws->recMarkCap;
    p.recChunkList = ws->recChunks;
    p.recChunkCap = static_cast<int>(ws->recChunkCap);
  }
  return MOSP_OK;
}

/// Build the parameters of the combined-graph step.
int prepareCombined(mosp_workspace *ws, int n, int K, const int *d_parents, const int *h_pref,
                    int source, long long delta, long long *d_dist, int *d_parent,
                    EngineParams &p, long long &scale, int &bits) {
  if (K <= 0 || K > 32 || n <= 0 || source < 0 || source >= n || d_parents == nullptr ||
      d_dist == nullptr || d_parent == nullptr) {
    return fail(MOSP_ERR_INVALID, "Error: invalid combined-graph parameters.");
  }
  scale = mosp_preference_scale(h_pref, K);
  if (scale == 0) {
    return fail(MOSP_ERR_INVALID, "Error: invalid preference vector (need K values >= 1).");
  }
  int st = checkRoot(ws, source);
  if (st != MOSP_OK) return st;
  st = reserveLists(ws, n, 1);
  if (st != MOSP_OK) return st;
  if ((st = reserveCombined(ws, n, K)) != MOSP_OK) return st;
  if ((st = reserveNear(ws, n, static_cast<long long>(n) * K, 1)) != MOSP_OK) return st;
  if ((st = reserveAsync(ws, n, 1)) != MOSP_OK) return st;
  std::memset(&p, 0, sizeof(p));
  p.n = n;
  p.K = 1;
  p.source = source;
  p.mode = kModeCombined;
  p.combParents = d_parents;
  p.combDeg = ws->combDeg;
  p.combRow = ws->combRow;
  p.combCol = ws->combCol;
  p.combW = ws->combW;
  p.combK = K;
  p.combBase = static_cast<int>(scale * (K + 1));
  p.combDelta = delta;
  for (int k = 0; k < K; ++k) {
    p.prefTerms[k] = static_cast<int>(h_pref == nullptr ? scale : scale / h_pref[k]);
  }
  u64 maxDist = 0;
  if ((st = choosePacking(n, p.combBase, bits, maxDist)) != MOSP_OK) return st;
  ObjectiveArgs &o = p.obj[0];
  o.dist = d_dist;
  o.parent = d_parent;
  setObjective(o, bits, maxDist, delta > 0 ? delta : 1);
  return MOSP_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// extern "C"
// ---------------------------------------------------------------------------
extern "C" {

int mosp_abi_version(void) { return MOSP_ABI_VERSION; }

const char *mosp_last_error(void) { return g_lastError.c_str(); }

const char *mosp_status_name(int status) {
  switch (status) {
    case MOSP_OK: return "MOSP_OK";
    case MOSP_ERR_INVALID: return "MOSP_ERR_INVALID";
    case MOSP_ERR_OVERFLOW: return "MOSP_ERR_OVERFLOW";
    case MOSP_ERR_OOM: return "MOSP_ERR_OOM";
    case MOSP_ERR_CUDA: return "MOSP_ERR_CUDA";
    case MOSP_ERR_TIMEOUT: return "MOSP_ERR_TIMEOUT";
    case MOSP_ERR_UNSUPPORTED: return "MOSP_ERR_UNSUPPORTED";
    default: return "MOSP_ERR_UNKNOWN";
  }
}

long long mosp_default_delta(long long num_edges, int num_nodes, long long weight_sum) {
  if (num_edges <= 0 || num_nodes <= 0) return 1;
  // 32 * (average weight) / (average out-degree); only the speed depends on it
  const double averageWeight = static_cast<double>(weight_sum) / num_edges;
  const double averageDegree = static_cast<double>(num_edges) / num_nodes;
  return std::max(1LL, static_cast<long long>(32.0 * averageWeight / averageDegree));
}

int mosp_choose_packing(int n, long long max_weight, int *parent_bits,
                        unsigned long long *max_distance) {
  int bits = 0;
  u64 maxDist = 0;
  const int st = choosePacking(std::max(n, 1), max_weight, bits, maxDist);
  if (st != MOSP_OK) return st;
  if (parent_bits) *parent_bits = bits;
  if (max_distance) *max_distance = maxDist;
  return MOSP_OK;
}

long long mosp_preference_scale(const int *h_pref, int K) {
  // L = lcm(Pref) <= 2^20 (reference src/combinedGraphGpu.cu:129-147)
  if (h_pref == nullptr) return 1;
  if (K <= 0) return 0;
  long long scale = 1;
  for (int i = 0; i < K; ++i) {
    if (h_pref[i] < 1) return 0;
    scale = scale / std::gcd(scale, static_cast<long long>(h_pref[i])) * h_pref[i];
    if (scale > (1LL << 20)) return 0;
  }
  return scale;
}

int mosp_workspace_create(mosp_workspace **out) {
  if (out == nullptr) return fail(MOSP_ERR_INVALID, "null output pointer");
  *out = nullptr;
  mosp_workspace *ws = new mosp_workspace();
  MOSP_CUDA(cudaGetDevice(&ws->device));
  int st = deviceAlloc(&ws->ctl, kControlBlocks);
  if (st == MOSP_OK) st = deviceAlloc(&ws->gen, 1);
  if (st == MOSP_OK && cudaMemset(ws->gen, 0, sizeof(int)) != cudaSuccess) st = MOSP_ERR_CUDA;
  if (st == MOSP_OK &&
      cudaMallocHost(reinterpret_cast<void **>(&ws->hostCtl), kControlBlocks * sizeof(EngineControl)) !=
          cudaSuccess) {
    st = fail(MOSP_ERR_OOM, "pinned allocation failed");
  }
  if (st != MOSP_OK) {
    mosp_workspace_destroy(ws);
    return st;
  }
  *out = ws;
  return MOSP_OK;
}

void mosp_workspace_destroy(mosp_workspace *ws) {
  if (ws == nullptr) return;
  int dev = -1;
  cudaGetDevice(&dev);
  if (ws->device >= 0) cudaSetDevice(ws->device);
  releaseLists(ws);
  for (void *p : {static_cast<void *>(ws->ctl), static_cast<void *>(ws->gen),
                  static_cast<void *>(ws->blockSums), static_cast<void *>(ws->combDeg),
                  static_cast<void *>(ws->combRow), static_cast<void *>(ws->combCol),
                  static_cast<void *>(ws->combW), static_cast<void *>(ws->cursor),
                  static_cast<void *>(ws->edgeOf), static_cast<void *>(ws->anc0),
                  static_cast<void *>(ws->anc1), static_cast<void *>(ws->acc0),
                  static_cast<void *>(ws->acc1), static_cast<void *>(ws->recMark),
                  static_cast<void *>(ws->recVerts), static_cast<void *>(ws->recChunks)}) {
    if (p) cudaFree(p);
  }
  for (void *p : ws->user) {
    if (p) cudaFree(p);
  }
  if (ws->applyScratch) cudaFree(ws->applyScratch);
  if (ws->sources) cudaFree(ws->sources);
  if (ws->graphExec) cudaGraphExecDestroy(ws->graphExec);
  if (ws->captureStream) cudaStreamDestroy(ws->captureStream);
  for (cudaEvent_t e : ws->ev) {
    if (e) cudaEventDestroy(e);
  }
  if (ws->hostCtl) cudaFreeHost(ws->hostCtl);
  if (dev >= 0) cudaSetDevice(dev);
  delete ws;
}

int mosp_workspace_reserve(mosp_workspace *ws, int n, int K) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (n < 0 || K < 1 || K > kMaxK) return fail(MOSP_ERR_INVALID, "invalid reserve size");
  if ((st = reserveLists(ws, std::max(n, 1), K)) != MOSP_OK) return st;
  return reserveCombined(ws, std::max(n, 1), K);
}

int mosp_workspace_reserve_graph(mosp_workspace *ws, int n, long long m, int K) {
  int st = mosp_workspace_reserve(ws, n, K);
  if (st != MOSP_OK) return st;
  if (m < 0) return fail(MOSP_ERR_INVALID, "invalid reserve size");
  const long long nn = std::max(n, 1);
  // the update's near lists and queue, and those of the combined step
  if ((st = reserveNear(ws, nn, std::max(m, nn * K), K)) != MOSP_OK) return st;
  return reserveAsync(ws, nn, K);
}

int mosp_workspace_set_sources(mosp_workspace *ws, const int *h_sources, int count) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (count < 0 || (count > 0 && h_sources == nullptr)) {
    return fail(MOSP_ERR_INVALID, "Error: invalid root list.");
  }
  std::vector<int> roots(h_sources, h_sources + count);
  std::sort(roots.begin(), roots.end());
  if (std::adjacent_find(roots.begin(), roots.end()) != roots.end() ||
      (count > 0 && roots.front() < 0)) {
    return fail(MOSP_ERR_INVALID, "Error: the roots must be distinct vertex ids >= 0.");
  }
  if (ws->sources) cudaFree(ws->sources);
  ws->sources = nullptr;
  ws->nSources = 0;
  ws->hostSources.clear();
  if (count <= 1) return MOSP_OK;
  if ((st = deviceAlloc(&ws->sources, count)) != MOSP_OK) return st;
  MOSP_CUDA(cudaMemcpy(ws->sources, roots.data(), count * sizeof(int), cudaMemcpyHostToDevice));
  ws->hostSources = std::move(roots);
  ws->nSources = count;
  return MOSP_OK;
}

int mosp_workspace_set_combined_delta(mosp_workspace *ws, long long delta) {
  if (ws == nullptr || delta < 0) return fail(MOSP_ERR_INVALID, "invalid combined-graph delta");
  ws->combDelta = delta;
  return MOSP_OK;
}

int mosp_workspace_set_local_rounds(mosp_workspace *ws, int update_rounds, int scratch_rounds) {
  if (ws == nullptr || update_rounds < 0 || update_rounds > 16 || scratch_rounds < 0 ||
      scratch_rounds > 16) {
    return fail(MOSP_ERR_INVALID, "invalid local rounds");
  }
  ws->roundsUpdate = update_rounds;
  ws->roundsScratch = scratch_rounds;
  return MOSP_OK;
}

int mosp_workspace_set_narrow(mosp_workspace *ws, int max_items, int rounds) {
  if (ws == nullptr || max_items < 0 || rounds < 0 || rounds > 1024) {
    return fail(MOSP_ERR_INVALID, "invalid narrow-iteration settings");
  }
  ws->narrowItems = max_items;
  ws->narrowRounds = rounds;
  return MOSP_OK;
}

int mosp_workspace_set_async(mosp_workspace *ws, int on, long long queue_slots) {
  if (ws == nullptr || on < 0 || on > 1 || queue_slots < 0 || queue_slots > (1LL << 34)) {
    return fail(MOSP_ERR_INVALID, "invalid near-far loop mode");
  }
  ws->asyncMode = on;
  ws->asyncSlots = queue_slots;
  return MOSP_OK;
}

int mosp_workspace_set_canonical_trees(mosp_workspace *ws, int on) {
  if (ws == nullptr || on < 0 || on > 1) {
    return fail(MOSP_ERR_INVALID, "invalid canonical-trees setting");
  }
  ws->canonicalTrees = on != 0;
  return MOSP_OK;
}

int mosp_workspace_set_grid(mosp_workspace *ws, int ctas, int hub_edges) {
  if (ws == nullptr || ctas < 0 || hub_edges < 0 || (hub_edges > 0 && hub_edges < 64)) {
    return fail(MOSP_ERR_INVALID, "invalid grid settings");
  }
  ws->gridCtas = ctas;
  ws->heavyDeg = hub_edges;
  return MOSP_OK;
}

int mosp_workspace_tuning(mosp_workspace *ws, int *ctas, int *hub_edges, int *async_on) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (ctas) *ctas = engineCtas(ws);
  if (hub_edges) *hub_edges = ws->heavyDeg > 0 ? ws->heavyDeg : 2048;
  if (async_on) *async_on = ws->asyncMode;
  return MOSP_OK;
}

int mosp_workspace_use_graphs(mosp_workspace *ws, int on) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  ws->useGraphs = on != 0;
  if (!ws->useGraphs && ws->graphExec) {
    cudaGraphExecDestroy(ws->graphExec);
    ws->graphExec = nullptr;
  }
  return MOSP_OK;
}

int mosp_workspace_graph_launches(mosp_workspace *ws, int *count) {
  if (ws == nullptr || count == nullptr) return fail(MOSP_ERR_INVALID, "invalid arguments");
  *count = ws->graphReplays;
  return MOSP_OK;
}

int mosp_workspace_set_timeout_ms(mosp_workspace *ws, long long ms) {
  if (ws == nullptr || ms <= 0) return fail(MOSP_ERR_INVALID, "invalid timeout");
  ws->timeoutNs = ms * 1000000LL;
  return MOSP_OK;
}

int mosp_workspace_set_ctas_per_sm(mosp_workspace *ws, int ctas_per_sm) {
  if (ws == nullptr || ctas_per_sm < 0) return fail(MOSP_ERR_INVALID, "invalid launch shape");
  ws->ctasPerSm = ctas_per_sm;
  ws->shapeValid = false;
  return MOSP_OK;
}

int mosp_workspace_buffer(mosp_workspace *ws, int slot, unsigned long long bytes, void **d_ptr) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (slot < 0 || slot >= 32 || d_ptr == nullptr) return fail(MOSP_ERR_INVALID, "invalid buffer slot");
  if (bytes > ws->userBytes[slot] || ws->user[slot] == nullptr) {
    char *p = static_cast<char *>(ws->user[slot]);
    const unsigned long long grow = std::max(bytes, ws->userBytes[slot] + ws->userBytes[slot] / 8);
    if ((st = deviceAlloc(&p, grow)) != MOSP_OK) {
      ws->user[slot] = nullptr;
      ws->userBytes[slot] = 0;
      return st;
    }
    ws->user[slot] = p;
    ws->userBytes[slot] = grow;
  }
  *d_ptr = ws->user[slot];
  return MOSP_OK;
}

int mosp_workspace_enable_timing(mosp_workspace *ws, int on) {
  if (ws == nullptr) return fail(MOSP_ERR_INVALID, "null workspace");
  ws->timing = on != 0;
  return MOSP_OK;
}

int mosp_workspace_last_timing(mosp_workspace *ws, float *update_ms, float *combined_ms) {
  if (ws == nullptr) return fail(MOSP_ERR_INVALID, "null workspace");
  if (update_ms) *update_ms = ws->lastUpdateMs;
  if (combined_ms) *combined_ms = ws->lastCombinedMs;
  return MOSP_OK;
}

int mosp_workspace_last_phases(mosp_workspace *ws, int which, unsigned long long *ns) {
  if (ws == nullptr || ns == nullptr || which < 0 || which > 1) {
    return fail(MOSP_ERR_INVALID, "invalid phase query");
  }
  for (int i = 0; i < 8; ++i) ns[i] = ws->hostCtl[which].phaseNs[i];
  return MOSP_OK;
}

int mosp_workspace_loop_profile(mosp_workspace *ws, int which, unsigned long long *ns,
                                long long *iters, long long *items) {
  if (ws == nullptr || which < 0 || which > 1) return fail(MOSP_ERR_INVALID, "invalid query");
  const EngineControl &c = ws->hostCtl[which];
  if (ns) {
    for (int q = 0; q < 5; ++q) ns[2 + q] = c.iterSplitNs[q];
  }
  for (int q = 0; q < 2; ++q) {
    if (ns) ns[q] = c.loopNs[q];
    if (iters) iters[q] = c.loopIters[q];
    if (items) items[q] = c.loopItems[q];
  }
  return MOSP_OK;
}

int mosp_workspace_grid(mosp_workspace *ws, int *ctas) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (ctas) *ctas = engineCtas(ws);
  return MOSP_OK;
}

int mosp_build_device_graph(mosp_workspace *ws, int n, int m, int K, const int *d_out_row,
                            const int *d_out_col, const int *d_edge_major_w, int *d_out_w,
                            int *d_in_row, int *d_in_col, int *d_in_w, void *stream) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (n <= 0 || m < 0 || K < 1 || d_out_row == nullptr || d_in_row == nullptr ||
      (m > 0 && (d_out_col == nullptr || d_edge_major_w == nullptr || d_out_w == nullptr ||
                 d_in_col == nullptr || d_in_w == nullptr))) {
    return fail(MOSP_ERR_INVALID, "Error: invalid device graph arguments.");
  }
  if (n + 1 > ws->cursorCap) {
    if ((st = deviceAlloc(&ws->cursor, static_cast<size_t>(n) + 1)) != MOSP_OK) return st;
    ws->cursorCap = static_cast<long long>(n) + 1;
  }
  cudaStream_t s = asStream(stream);
  BuildParams b{};
  b.n = n;
  b.m = m;
  b.K = K;
  b.timeoutNs = ws->timeoutNs;
  b.outRow = d_out_row;
  b.outCol = d_out_col;
  b.edgeMajorW = d_edge_major_w;
  b.outW = d_out_w;
  b.inRow = d_in_row;
  b.inCol = d_in_col;
  b.inW = d_in_w;
  b.cursor = ws->cursor;
  b.blockSums = ws->blockSums;
  b.ctl = ws->ctl + 2;
  MOSP_CUDA(cudaMemsetAsync(ws->ctl + 2, 0, sizeof(EngineControl), s));
  MOSP_CUDA(launchBuild(b, limitCtas(ws, ws->shape.buildCtas), s));
  if ((st = readControl(ws, 2, 1, s)) != MOSP_OK) return st;
  const EngineControl &c = ws->hostCtl[2];
  if (c.status != 0) return fail(MOSP_ERR_TIMEOUT, "Error: device graph build timed out.");
  if (c.invalid) {
    return fail(MOSP_ERR_INVALID,
                "Error: malformed CSR (row offsets not monotone from 0 to m, or a column index "
                "outside [0, n)).");
  }
  return MOSP_OK;
}

int mosp_apply_batch_device(mosp_workspace *ws, int n, int K, int m, const int *d_row,
                            const int *d_col, const int *d_w, int n_ins, const int *d_ins_from,
                            const int *d_ins_to, const int *d_ins_w, int n_del,
                            const int *d_del_from, const int *d_del_to, int *d_new_row,
                            int *d_new_col, int *d_new_w, long long new_capacity, int *new_m,
                            unsigned *d_mask, long long *h_max_weight, long long *h_weight_sum,
                            void *stream) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (n <= 0 || K < 1 || K > kMaxK || m < 0 || n_ins < 0 || n_del < 0 || d_row == nullptr ||
      (m > 0 && (d_col == nullptr || d_w == nullptr)) ||
      (n_ins > 0 && (d_ins_from == nullptr || d_ins_to == nullptr || d_ins_w == nullptr ||
                     d_mask == nullptr)) ||
      (n_del > 0 && (d_del_from == nullptr || d_del_to == nullptr)) || d_new_row == nullptr ||
      d_new_col == nullptr || d_new_w == nullptr || new_m == nullptr ||
      new_capacity < static_cast<long long>(m) + n_ins ||
      static_cast<long long>(m) + n_ins > INT_MAX) {
    return fail(MOSP_ERR_INVALID, "Error: invalid change-batch arguments (the updated graph needs "
                                  "room for m + n_ins edges).");
  }
  const size_t need = applyScratchBytes(n, m, n_ins, n_del);
  if (need > ws->applyBytes) {
    // grow by half again: batches of varying size then rarely reallocate
    // (a reallocation's cudaFree waits for the whole device)
    const size_t want = std::max(need, ws->applyBytes + ws->applyBytes / 2);
    if (ws->applyScratch) cudaFree(ws->applyScratch);
    ws->applyScratch = nullptr;
    ws->applyBytes = 0;
    unsigned char *p = nullptr;
    if ((st = deviceAlloc(&p, want)) != MOSP_OK) return st;
    ws->applyScratch = p;
    ws->applyBytes = want;
  }
  int sms = 0;
  MOSP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws->device));
  ApplyParams P;
  std::memset(&P, 0, sizeof(P));
  P.n = n;
  P.m = m;
  P.K = K;
  P.row = d_row;
  P.col = d_col;
  P.w = d_w;
  P.nIns = n_ins;
  P.nDel = n_del;
  P.insFrom = d_ins_from;
  P.insTo = d_ins_to;
  P.insW = d_ins_w;
  P.delFrom = d_del_from;
  P.delTo = d_del_to;
  P.newRow = d_new_row;
  P.newCol = d_new_col;
  P.newW = d_new_w;
  P.mask = d_mask;
  int counters[kApplyCounters + 1] = {0};
  long long stats[2 * kMaxK] = {0};
  const bool wantStats = h_max_weight != nullptr || h_weight_sum != nullptr;
  MOSP_CUDA(applyBatchGpu(P, ws->applyScratch, sms, asStream(stream), counters,
                          wantStats ? stats : nullptr));
  if (counters[kApplyInvalid]) {
    return fail(MOSP_ERR_INVALID, "Error: a changed edge's endpoint is out of range.");
  }
  *new_m = counters[kApplyCounters];
  for (int k = 0; k < K && wantStats; ++k) {
    if (h_max_weight) h_max_weight[k] = stats[k];
    if (h_weight_sum) h_weight_sum[k] = stats[K + k];
  }
  return MOSP_OK;
}

int mosp_sosp_update_multi(mosp_workspace *ws, int n, int m, int K, const int *d_out_row,
                           const int *d_out_col, const int *const *h_out_w, const int *d_in_row,
                           const int *d_in_col, const int *const *h_in_w,
                           const int *const *h_changed_from, const int *const *h_changed_to,
                           const int *h_n_changed, const int *d_insert_heads, int n_heads,
                           int source, const long long *h_delta, const long long *h_max_weight,
                           long long *const *h_dist, int *const *h_parent,
                           mosp_sosp_stats *stats, void *stream) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (K < 1 || K > kMaxK || h_out_w == nullptr || h_in_w == nullptr || h_changed_from == nullptr ||
      h_changed_to == nullptr || h_n_changed == nullptr || h_delta == nullptr ||
      h_max_weight == nullptr || h_dist == nullptr || h_parent == nullptr) {
    return fail(MOSP_ERR_INVALID, "Error: invalid SOSP update arguments.");
  }
  UpdateArgs a{n,        m,           K,          d_out_row,      d_out_col,  d_in_row,
               d_in_col, h_out_w,     h_in_w,     h_changed_from, h_changed_to, h_n_changed,
               d_insert_heads, n_heads, source,   h_delta,        h_max_weight, h_dist,
               h_parent};
  EngineParams p;
  int bits[kMaxK] = {0};
  if ((st = prepareUpdate(ws, a, p, bits)) != MOSP_OK) return st;
  cudaStream_t s = asStream(stream);
  if ((st = cleanLists(ws, s)) != MOSP_OK) return st;
  fillLists(p, ws, 0);
  if ((st = markEvent(ws, 0, s)) != MOSP_OK) return st;
  if ((st = queueEngine(ws, p, 0, s)) != MOSP_OK) return st;
  if ((st = markEvent(ws, 1, s)) != MOSP_OK) return st;
  if ((st = readControl(ws, 0, 1, s)) != MOSP_OK) return st;
  readEvents(ws, &ws->lastUpdateMs, nullptr);
  const EngineControl &c = ws->hostCtl[0];
  ws->heavySeen[0] = c.heavy != 0;
  if ((st = controlStatus(ws, c)) != MOSP_OK) return st;
  if (stats) {
    for (int k = 0; k < K; ++k) fillStats(c, k, bits[k], stats + k);
  }
  return maybeResetGenerations(ws, c.finalGen, s);
}

int mosp_sosp_update(mosp_workspace *ws, int n, int m, const int *d_out_row, const int *d_out_col,
                     const int *d_out_w, const int *d_in_row, const int *d_in_col,
                     const int *d_in_w, const int *d_changed_from, const int *d_changed_to,
                     int n_changed, const int *d_insert_heads, int n_heads, int source,
                     long long delta, long long max_weight, long long *d_dist, int *d_parent,
                     mosp_sosp_stats *stats, void *stream) {
  return mosp_sosp_update_multi(ws, n, m, 1, d_out_row, d_out_col, &d_out_w, d_in_row, d_in_col,
                                &d_in_w, &d_changed_from, &d_changed_to, &n_changed,
                                d_insert_heads, n_heads, source, &delta, &max_weight, &d_dist,
                                &d_parent, stats, stream);
}

int mosp_sosp_from_scratch(mosp_workspace *ws, int n, int m, const int *d_out_row,
                           const int *d_out_col, const int *d_out_w, int source, long long delta,
                           long long max_weight, long long *d_dist, int *d_parent,
                           mosp_sosp_stats *stats, void *stream) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (n <= 0 || m < 0 || source < 0 || source >= n || delta <= 0 || d_out_row == nullptr ||
      (m > 0 && (d_out_col == nullptr || d_out_w == nullptr)) || d_dist == nullptr ||
      d_parent == nullptr) {
    return fail(MOSP_ERR_INVALID, "Error: invalid SSSP arguments.");
  }
  if ((st = checkRoot(ws, source)) != MOSP_OK) return st;
  if ((st = reserveLists(ws, n, 1)) != MOSP_OK) return st;
  if ((st = reserveNear(ws, n, m, 1)) != MOSP_OK) return st;
  if ((st = reserveAsync(ws, n, 1)) != MOSP_OK) return st;
  int bits = 0;
  u64 maxDist = 0;
  if ((st = choosePacking(n, max_weight, bits, maxDist)) != MOSP_OK) return st;
  EngineParams p;
  std::memset(&p, 0, sizeof(p));
  p.n = n;
  p.m = m;
  p.K = 1;
  p.source = source;
  p.mode = kModeScratch;
  p.outRow = d_out_row;
  p.outCol = d_out_col;
  p.obj[0].outW = d_out_w;
  p.obj[0].dist = d_dist;
  p.obj[0].parent = d_parent;
  setObjective(p.obj[0], bits, maxDist, delta);
  cudaStream_t s = asStream(stream);
  if ((st = cleanLists(ws, s)) != MOSP_OK) return st;
  fillLists(p, ws, 0);
  if ((st = queueEngine(ws, p, 0, s)) != MOSP_OK) return st;
  if ((st = readControl(ws, 0, 1, s)) != MOSP_OK) return st;
  const EngineControl &c = ws->hostCtl[0];
  ws->heavySeen[0] = c.heavy != 0;
  if ((st = controlStatus(ws, c)) != MOSP_OK) return st;
  if (stats) fillStats(c, 0, bits, stats);
  return maybeResetGenerations(ws, c.finalGen, s);
}

int mosp_combined_sosp(mosp_workspace *ws, int n, int K, const int *d_parents, const int *h_pref,
                       int source, long long delta, long long *d_dist, int *d_parent,
                       mosp_combine_stats *stats, void *stream) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  // delta <= 0: the workspace's width (mosp_workspace_set_combined_delta),
  // else the default heuristic
  if (delta <= 0) delta = ws->combDelta;
  EngineParams p;
  long long scale = 0;
  int bits = 0;
  if ((st = prepareCombined(ws, n, K, d_parents, h_pref, source, delta, d_dist, d_parent, p,
                            scale, bits)) != MOSP_OK) {
    return st;
  }
  cudaStream_t s = asStream(stream);
  if ((st = cleanLists(ws, s)) != MOSP_OK) return st;
  fillLists(p, ws, 1);
  if ((st = markEvent(ws, 1, s)) != MOSP_OK) return st;
  if ((st = queueEngine(ws, p, 1, s)) != MOSP_OK) return st;
  if ((st = markEvent(ws, 2, s)) != MOSP_OK) return st;
  if ((st = readControl(ws, 1, 1, s)) != MOSP_OK) return st;
  readEvents(ws, nullptr, &ws->lastCombinedMs);
  const EngineControl &c = ws->hostCtl[1];
  ws->heavySeen[1] = c.heavy != 0;
  if ((st = controlStatus(ws, c)) != MOSP_OK) return st;
  if (stats) {
    stats->edges = static_cast<int>(c.sums[0]);
    stats->reserved = 0;
    stats->scale = scale;
    stats->delta = delta > 0 ? delta
                             : mosp_default_delta(static_cast<long long>(c.sums[0]), n,
                                                  static_cast<long long>(c.sums[1]));
    fillStats(c, 0, bits, &stats->search);
  }
  return maybeResetGenerations(ws, c.finalGen, s);
}

int mosp_update_device(mosp_workspace *ws, int n, int m, int K, const int *d_out_row,
                       const int *d_out_col, const int *d_out_w, const int *d_in_row,
                       const int *d_in_col, const int *d_in_w, const int *d_changed_from,
                       const int *d_changed_to, const int *h_changed_offset,
                       const int *d_insert_heads, int n_heads, int source, const long long *h_delta,
                       const long long *h_max_weight, const int *h_pref, long long *d_dist,
                       int *d_parent, long long *d_comb_dist, int *d_comb_parent,
                       mosp_sosp_stats *stats, mosp_combine_stats *cstats, void *stream) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (K < 1 || K > kMaxK || h_changed_offset == nullptr || h_delta == nullptr ||
      h_max_weight == nullptr || d_dist == nullptr || d_parent == nullptr) {
    return fail(MOSP_ERR_INVALID, "Error: invalid MOSP update arguments.");
  }
  const int *outW[kMaxK], *inW[kMaxK], *chFrom[kMaxK], *chTo[kMaxK];
  int nChanged[kMaxK];
  long long *dist[kMaxK];
  int *parent[kMaxK];
  for (int k = 0; k < K; ++k) {
    outW[k] = d_out_w + static_cast<long long>(k) * m;
    inW[k] = d_in_w + static_cast<long long>(k) * m;
    chFrom[k] = d_changed_from + h_changed_offset[k];
    chTo[k] = d_changed_to + h_changed_offset[k];
    nChanged[k] = h_changed_offset[k + 1] - h_changed_offset[k];
    dist[k] = d_dist + static_cast<long long>(k) * n;
    parent[k] = d_parent + static_cast<long long>(k) * n;
  }
  UpdateArgs a{n,     m,     K,        d_out_row, d_out_col, d_in_row, d_in_col,
               outW,  inW,   chFrom,   chTo,      nChanged,  d_insert_heads, n_heads,
               source, h_delta, h_max_weight, dist, parent};
  EngineParams pu, pc;
  int bits[kMaxK] = {0};
  if ((st = prepareUpdate(ws, a, pu, bits)) != MOSP_OK) return st;
  long long scale = 0;
  int cbits = 0;
  if ((st = prepareCombined(ws, n, K, d_parent, h_pref, source, ws->combDelta, d_comb_dist,
                            d_comb_parent, pc, scale, cbits)) != MOSP_OK) {
    return st;
  }
  cudaStream_t s = asStream(stream);
  if ((st = cleanLists(ws, s)) != MOSP_OK) return st;
  fillLists(pu, ws, 0);
  fillLists(pc, ws, 1);
  if (ws->useGraphs) {
    if ((st = launchUpdateGraph(ws, pu, pc, s)) != MOSP_OK) return st;
    MOSP_CUDA(cudaStreamSynchronize(s));
  } else {
    if ((st = markEvent(ws, 0, s)) != MOSP_OK) return st;
    if ((st = queueEngine(ws, pu, 0, s)) != MOSP_OK) return st;
    if ((st = markEvent(ws, 1, s)) != MOSP_OK) return st;
    if ((st = queueEngine(ws, pc, 1, s)) != MOSP_OK) return st;
    if ((st = markEvent(ws, 2, s)) != MOSP_OK) return st;
    if ((st = readControl(ws, 0, 2, s)) != MOSP_OK) return st;
  }
  readEvents(ws, &ws->lastUpdateMs, &ws->lastCombinedMs);
  ws->heavySeen[0] = ws->hostCtl[0].heavy != 0;
  ws->heavySeen[1] = ws->hostCtl[1].heavy != 0;
  if ((st = controlStatus(ws, ws->hostCtl[0])) != MOSP_OK) return st;
  if ((st = controlStatus(ws, ws->hostCtl[1])) != MOSP_OK) return st;
  const EngineControl &cu = ws->hostCtl[0];
  const EngineControl &cc = ws->hostCtl[1];
  if (stats) {
    for (int k = 0; k < K; ++k) fillStats(cu, k, bits[k], stats + k);
  }
  if (cstats) {
    cstats->edges = static_cast<int>(cc.sums[0]);
    cstats->reserved = 0;
    cstats->scale = scale;
    cstats->delta = ws->combDelta > 0
                        ? ws->combDelta
                        : mosp_default_delta(static_cast<long long>(cc.sums[0]), n,
                                             static_cast<long long>(cc.sums[1]));
    fillStats(cc, 0, cbits, &cstats->search);
  }
  return maybeResetGenerations(ws, std::max(cu.finalGen, cc.finalGen), s);
}

int mosp_autotune_update(mosp_workspace *ws, int n, int m, int K, const int *d_out_row,
                         const int *d_out_col, const int *d_out_w, const int *d_in_row,
                         const int *d_in_col, const int *d_in_w, const int *d_changed_from,
                         const int *d_changed_to, const int *h_changed_offset,
                         const int *d_insert_heads, int n_heads, int source,
                         const long long *h_delta, const long long *h_max_weight,
                         const int *h_pref, long long *d_dist, int *d_parent,
                         long long *d_comb_dist, int *d_comb_parent, long long *h_best_delta,
                         long long *h_best_comb_delta, int *h_best_rounds, float *h_best_ms,
                         void *stream) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (K < 1 || K > kMaxK || h_delta == nullptr || h_best_delta == nullptr ||
      h_best_comb_delta == nullptr || d_dist == nullptr || d_parent == nullptr || n <= 0) {
    return fail(MOSP_ERR_INVALID, "Error: invalid autotuner arguments.");
  }
  cudaStream_t s = asStream(stream);
  const size_t kn = static_cast<size_t>(K) * n;
  // the trees are updated in place: keep a copy and restore it before every
  // trial and at the end
  long long *saveDist = nullptr;
  int *saveParent = nullptr;
  if ((st = deviceAlloc(&saveDist, kn)) != MOSP_OK) return st;
  if ((st = deviceAlloc(&saveParent, kn)) != MOSP_OK) {
    cudaFree(saveDist);
    return st;
  }
  struct Restore {
    mosp_workspace *ws;
    bool timing, graphs;
    long long combDelta;
    int roundsUpdate, roundsScratch;
    long long *d;
    int *p;
    ~Restore() {
      ws->timing = timing;
      ws->useGraphs = graphs;
      ws->combDelta = combDelta;
      ws->roundsUpdate = roundsUpdate;
      ws->roundsScratch = roundsScratch;
      cudaFree(d);
      cudaFree(p);
    }
  } restore{ws, ws->timing, ws->useGraphs, ws->combDelta, ws->roundsUpdate, ws->roundsScratch,
            saveDist, saveParent};
  MOSP_CUDA(cudaMemcpyAsync(saveDist, d_dist, kn * sizeof(long long), cudaMemcpyDeviceToDevice, s));
  MOSP_CUDA(cudaMemcpyAsync(saveParent, d_parent, kn * sizeof(int), cudaMemcpyDeviceToDevice, s));
  ws->timing = true;
  ws->useGraphs = false;
  // Trial t runs the update with (width factor, local rounds) uc[t] and the
  // combined step with cc[t]; the two launches are timed separately, so the
  // two lists are searched independently. Trial 0 gives the combined
  // default width the factors apply to.
  struct Choice {
    double factor;
    int rounds;
  };
  const Choice uc[] = {{1, 0}, {0.5, 0}, {2, 0}, {4, 0}, {1, 1}, {2, 1}, {0.25, 0}, {8, 0}, {2, 2}};
  const Choice cc[] = {{1, 2}, {4, 2}, {16, 2}, {2, 0}, {8, 0}, {32, 0}, {4, 4}, {16, 4}, {8, 3}};
  const int trials = 9;
  float bestU = 1e30f, bestC = 1e30f;
  Choice bestUc = uc[0];
  long long combDefault = 0, bestComb = 0;
  int bestCr = cc[0].rounds;
  std::vector<long long> deltas(K);
  for (int t = 0; t < trials; ++t) {
    for (int k = 0; k < K; ++k) {
      deltas[k] = std::max(1LL, static_cast<long long>(h_delta[k] * uc[t].factor));
    }
    ws->roundsUpdate = uc[t].rounds;
    ws->roundsScratch = cc[t].rounds;
    ws->combDelta = t == 0 ? 0 : std::max(1LL, static_cast<long long>(combDefault * cc[t].factor));
    // median of three runs: sub-millisecond launches vary from run to run
    float us[3], cs3[3];
    for (int rep = 0; rep < 3; ++rep) {
      MOSP_CUDA(cudaMemcpyAsync(d_dist, saveDist, kn * sizeof(long long), cudaMemcpyDeviceToDevice, s));
      MOSP_CUDA(cudaMemcpyAsync(d_parent, saveParent, kn * sizeof(int), cudaMemcpyDeviceToDevice, s));
      mosp_combine_stats cs{};
      st = mosp_update_device(ws, n, m, K, d_out_row, d_out_col, d_out_w, d_in_row, d_in_col,
                              d_in_w, d_changed_from, d_changed_to, h_changed_offset,
                              d_insert_heads, n_heads, source, deltas.data(), h_max_weight, h_pref,
                              d_dist, d_parent, d_comb_dist, d_comb_parent, nullptr, &cs, stream);
      if (st != MOSP_OK) return st;
      if (t == 0) combDefault = cs.delta;
      us[rep] = ws->lastUpdateMs;
      cs3[rep] = ws->lastCombinedMs;
    }
    std::sort(us, us + 3);
    std::sort(cs3, cs3 + 3);
    const float u = us[1], c = cs3[1];
    if (u < bestU) {
      bestU = u;
      bestUc = uc[t];
    }
    if (c < bestC) {
      bestC = c;
      bestComb = t == 0 ? combDefault : ws->combDelta;
      bestCr = cc[t].rounds;
    }
  }
  for (int k = 0; k < K; ++k) {
    h_best_delta[k] = std::max(1LL, static_cast<long long>(h_delta[k] * bestUc.factor));
  }
  *h_best_comb_delta = bestComb;

  // With those widths: the near-far loop (asynchronous or bulk), the grid
  // (all SMs, or fewer CTAs: cheaper grid barriers) and, for graphs with
  // hub rows, the hub threshold (a higher one lets the asynchronous loop
  // run). Timed on the whole update; the best stays set on the workspace.
  {
    for (int k = 0; k < K; ++k) deltas[k] = h_best_delta[k];
    ws->roundsUpdate = bestUc.rounds;
    ws->roundsScratch = bestCr;
    ws->combDelta = bestComb;
    auto timeIt = [&](float &total) -> int {
      float runs[3];
      for (int rep = 0; rep < 3; ++rep) {
        MOSP_CUDA(cudaMemcpyAsync(d_dist, saveDist, kn * sizeof(long long), cudaMemcpyDeviceToDevice, s));
        MOSP_CUDA(cudaMemcpyAsync(d_parent, saveParent, kn * sizeof(int), cudaMemcpyDeviceToDevice, s));
        const int rc = mosp_update_device(ws, n, m, K, d_out_row, d_out_col, d_out_w, d_in_row, d_in_col,
                                          d_in_w, d_changed_from, d_changed_to, h_changed_offset,
                                          d_insert_heads, n_heads, source, deltas.data(), h_max_weight,
                                          h_pref, d_dist, d_parent, d_comb_dist, d_comb_parent, nullptr,
                                          nullptr, stream);
        if (rc != MOSP_OK) return rc;
        runs[rep] = ws->lastUpdateMs + ws->lastCombinedMs;
      }
      std::sort(runs, runs + 3);
      total = runs[1];
      return MOSP_OK;
    };
    struct Shape {
      int async, grid, hub;
    };
    const int full = ws->shape.engineCtas;
    const bool hubs = ws->heavySeen[0] || ws->heavySeen[1];
    Shape best{ws->asyncMode, ws->gridCtas, ws->heavyDeg};
    float bestMs = 1e30f;
    auto trial = [&](Shape sh) -> int {
      ws->asyncMode = sh.async;
      ws->gridCtas = sh.grid;
      ws->heavyDeg = sh.hub;
      ws->heavySeen[0] = ws->heavySeen[1] = false;
      if (sh.async != 0) {
        int rc = reserveAsync(ws, n, K);
        if (rc != MOSP_OK) return rc;
      }
      float ms = 0;
      const int rc = timeIt(ms);
      if (rc != MOSP_OK) return rc;
      if (ms < bestMs) {
        bestMs = ms;
        best = sh;
      }
      return MOSP_OK;
    };
    const Shape start = best;
    if ((st = trial(start)) != MOSP_OK) return st;
    if ((st = trial(Shape{1 - start.async, start.grid, start.hub})) != MOSP_OK) return st;
    for (int grid : {full * 3 / 4, full / 2}) {
      if (grid >= 1 && (st = trial(Shape{best.async, grid, best.hub})) != MOSP_OK) return st;
    }
    if (hubs) {
      for (int hub : {16384, 1 << 20}) {
        if ((st = trial(Shape{1, best.grid, hub})) != MOSP_OK) return st;
      }
    }
    ws->asyncMode = best.async;
    ws->gridCtas = best.grid;
    ws->heavyDeg = best.hub;
    ws->heavySeen[0] = ws->heavySeen[1] = false;
    if (bestMs < bestU + bestC) {
      bestU = bestMs;
      bestC = 0;
    }
  }
  if (h_best_rounds) {
    h_best_rounds[0] = bestUc.rounds;
    h_best_rounds[1] = bestCr;
  }
  if (h_best_ms) *h_best_ms = bestU + bestC;
  MOSP_CUDA(cudaMemcpyAsync(d_dist, saveDist, kn * sizeof(long long), cudaMemcpyDeviceToDevice, s));
  MOSP_CUDA(cudaMemcpyAsync(d_parent, saveParent, kn * sizeof(int), cudaMemcpyDeviceToDevice, s));
  MOSP_CUDA(cudaStreamSynchronize(s));
  return MOSP_OK;
}

int mosp_path_costs(mosp_workspace *ws, int n, int m, int KG, const int *d_out_row,
                    const int *d_out_col, const int *d_out_w, const int *d_parent, int source,
                    long long *d_costs, void *stream) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (n <= 0 || m < 0 || KG < 1 || source < 0 || source >= n || d_out_row == nullptr ||
      d_parent == nullptr || d_costs == nullptr ||
      (m > 0 && (d_out_col == nullptr || d_out_w == nullptr))) {
    return fail(MOSP_ERR_INVALID, "Error: invalid path-cost arguments.");
  }
  if ((st = checkRoot(ws, source)) != MOSP_OK) return st;
  if (n > ws->costN || KG > ws->costKG) {
    const long long nn = std::max<long long>(n, ws->costN);
    const int kk = std::max(KG, ws->costKG);
    if ((st = deviceAlloc(&ws->edgeOf, nn)) != MOSP_OK) return st;
    if ((st = deviceAlloc(&ws->anc0, nn)) != MOSP_OK) return st;
    if ((st = deviceAlloc(&ws->anc1, nn)) != MOSP_OK) return st;
    if ((st = deviceAlloc(&ws->acc0, nn * kk)) != MOSP_OK) return st;
    if ((st = deviceAlloc(&ws->acc1, nn * kk)) != MOSP_OK) return st;
    ws->costN = nn;
    ws->costKG = kk;
  }
  cudaStream_t s = asStream(stream);
  CostParams c{};
  c.n = n;
  c.m = m;
  c.KG = KG;
  c.source = source;
  c.sources = ws->nSources > 1 ? ws->sources : nullptr;
  c.nSources = ws->nSources > 1 ? ws->nSources : 0;
  c.timeoutNs = ws->timeoutNs;
  c.outRow = d_out_row;
  c.outCol = d_out_col;
  c.outW = d_out_w;
  c.parent = d_parent;
  c.edgeOf = ws->edgeOf;
  c.anc0 = ws->anc0;
  c.anc1 = ws->anc1;
  c.acc0 = ws->acc0;
  c.acc1 = ws->acc1;
  c.costs = d_costs;
  c.ctl = ws->ctl + 3;
  MOSP_CUDA(cudaMemsetAsync(ws->ctl + 3, 0, sizeof(EngineControl), s));
  MOSP_CUDA(launchCosts(c, limitCtas(ws, ws->shape.costCtas), s));
  if ((st = readControl(ws, 3, 1, s)) != MOSP_OK) return st;
  const EngineControl &h = ws->hostCtl[3];
  if (h.status != 0) return fail(MOSP_ERR_TIMEOUT, "Error: path-cost kernel timed out.");
  if (h.invalid) {
    return fail(MOSP_ERR_INVALID,
                "Error: a tree edge (parent[v], v) of the MOSP tree is not in the graph.");
  }
  return MOSP_OK;
}

/// Failure-path check: runs a barrier that one CTA never reaches, with the
/// given bound; returns the status the kernel reported (MOSP_ERR_TIMEOUT
/// when the bounded wait works). The workspace stays usable.
int mosp_debug_barrier_timeout(mosp_workspace *ws, long long timeout_ms, int *device_status) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (timeout_ms <= 0 || timeout_ms > 10000) return fail(MOSP_ERR_INVALID, "invalid timeout");
  cudaStream_t s = nullptr;
  MOSP_CUDA(cudaMemsetAsync(ws->ctl + 3, 0, sizeof(EngineControl), s));
  MOSP_CUDA(launchBarrierProbe(ws->ctl + 3, timeout_ms * 1000000LL,
                               std::min(ws->shape.engineCtas, 8), s));
  if ((st = readControl(ws, 3, 1, s)) != MOSP_OK) return st;
  if (device_status) *device_status = ws->hostCtl[3].status;
  return MOSP_OK;
}

/// Device time of `rounds` grid barriers of the engine's launch shape
/// (with `reads`, plus the per-iteration control reads); for tuning.
int mosp_debug_barrier_cost(mosp_workspace *ws, int rounds, int reads, double *ns_per_round) {
  int st = checkWorkspace(ws);
  if (st != MOSP_OK) return st;
  if (rounds <= 0 || rounds > 1000000) return fail(MOSP_ERR_INVALID, "invalid round count");
  cudaStream_t s = nullptr;
  MOSP_CUDA(cudaMemsetAsync(ws->ctl + 3, 0, sizeof(EngineControl), s));
  MOSP_CUDA(launchBarrierCost(ws->ctl + 3, rounds, reads, ws->timeoutNs, ws->shape.engineCtas, s));
  if ((st = readControl(ws, 3, 1, s)) != MOSP_OK) return st;
  if (ws->hostCtl[3].status != 0) return fail(MOSP_ERR_TIMEOUT, "barrier cost run timed out");
  if (ns_per_round) *ns_per_round = static_cast<double>(ws->hostCtl[3].phaseNs[0]) / rounds;
  return MOSP_OK;
}

}  // extern "C"
