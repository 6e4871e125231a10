// noalloc.cu - SSSP from scratch that allocates nothing
// (mosp_sosp_from_scratch_static, include/mosp_b200.h).
//
// Some callers cannot allocate device memory at the moment they need a
// shortest-path tree: a host process whose device memory belongs to another
// allocator (a caching allocator or a fixed arena sized at start-up) and
// that must not grow its footprint behind that allocator's back; a
// latency-critical request handler, where cudaMalloc/cudaFree may
// synchronize the device and take unbounded time; and plugin hosts whose
// contract forbids allocation inside a call. For them the scratch of the
// engine (packed words, far piles, near lists, the control block) lives in
// one file-scope __device__ array that the module reserves when it is
// loaded, so a call needs only the caller's graph and output buffers.
//
// Limits: n <= MOSP_STATIC_MAX_VERTICES and m <= MOSP_STATIC_MAX_EDGES, one
// objective. Calls on the same device share the array: calls that overlap
// in time (two host threads, or two streams without an ordering between
// them) race on it and produce garbage; callers serialize them.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "engine.h"
#include "mosp_b200.h"

using namespace mospb200;

namespace {

constexpr long long kMaxVertices = MOSP_STATIC_MAX_VERTICES;
constexpr long long kMaxEdges = MOSP_STATIC_MAX_EDGES;
// near lists: one split appends at most one entry per far-pile vertex and
// one iteration at most one per relaxation, so n + m + 64 entries suffice
// (the same bound as the workspace's lists)
constexpr long long kNearCap = kMaxVertices + kMaxEdges + 64;
constexpr long long kMaxCtas = 4096;  // blockSums entries (148 SMs x 1-2 CTAs in practice)
constexpr int kMaxDevices = 64;
constexpr long long kTimeoutNs = 10000LL * 1000000LL;

constexpr long long roundUp(long long x) { return (x + 255) / 256 * 256; }

// Byte offsets of the regions inside the array, each 256-byte aligned.
constexpr long long kOffCtl = 0;
constexpr long long kOffGen = kOffCtl + roundUp(sizeof(EngineControl));
constexpr long long kOffBlockSums = kOffGen + 256;
constexpr long long kOffPacked = kOffBlockSums + roundUp(kMaxCtas * 8);
constexpr long long kOffNearD0 = kOffPacked + roundUp(kMaxVertices * 8);
constexpr long long kOffNearD1 = kOffNearD0 + roundUp(kNearCap * 8);
constexpr long long kOffNearV0 = kOffNearD1 + roundUp(kNearCap * 8);
constexpr long long kOffNearV1 = kOffNearV0 + roundUp(kNearCap * 4);
constexpr long long kOffInts = kOffNearV1 + roundUp(kNearCap * 4);
constexpr int kIntLists = 6;  // val, stamp, inFar, cand, far0, far1
constexpr long long kScratchBytes = kOffInts + kIntLists * roundUp(kMaxVertices * 4);

// The scratch. Static storage starts zeroed when the module is loaded; the
// regions that the engine reads before writing (control block, generation
// counter, stamps, in-far flags) are cleared again by every call.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Launch shape per device ordinal (an occupancy query, made once). The
// array's device address is looked up on every call instead: it is only
// valid while the module stays loaded in the device's current context, and
// a context that was torn down and created again (cudaDeviceReset) loads
// the module anew at another address.
struct DeviceSlot {
  bool ready = false;
  LaunchShape shape{};
};
DeviceSlot g_slots[kMaxDevices];
std::mutex g_setupMutex;

int failCuda(cudaError_t err, const char *what) {
  return recordFailure(MOSP_ERR_CUDA, (std::string("CUDA error: ") + cudaGetErrorString(err) +
                                       " (" + what + ")").c_str());
}

/// Device address of the current device's copy of the array (a host-side
/// name of a __device__ variable is not an address a kernel may use) and
/// the launch shape. The first call on a device makes the occupancy query;
/// every call looks the address up, with the device current.
int setup(int &device, DeviceSlot *&slot, unsigned char *&base) {
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) return failCuda(err, "cudaGetDevice");
  if (device < 0 || device >= kMaxDevices) {
    return recordFailure(MOSP_ERR_UNSUPPORTED,
                         "Error: mosp_sosp_from_scratch_static supports device ordinals below 64.");
  }
  void *ptr = nullptr;
  err = cudaGetSymbolAddress(&ptr, g_scratch);
  if (err != cudaSuccess) return failCuda(err, "cudaGetSymbolAddress of the static scratch");
  base = static_cast<unsigned char *>(ptr);
  std::lock_guard<std::mutex> lock(g_setupMutex);
  DeviceSlot &s = g_slots[device];
  if (!s.ready) {
    LaunchShape shape{};
    err = queryLaunchShape(0, shape);
    if (err == cudaErrorNotSupported) {
      return recordFailure(MOSP_ERR_UNSUPPORTED, "the GPU does not support cooperative launches");
    }
    if (err != cudaSuccess) return failCuda(err, "occupancy query");
    if (shape.engineCtas > kMaxCtas) {
      return recordFailure(MOSP_ERR_UNSUPPORTED,
                           "Error: the launch shape exceeds the static scratch's CTA limit.");
    }
    s.shape = shape;
    s.ready = true;
  }
  slot = &s;
  return MOSP_OK;
}

}  // namespace

extern "C" int mosp_sosp_from_scratch_static(int n, int m, const int *d_out_row,
                                             const int *d_out_col, const int *d_out_w, int source,
                                             long long delta, long long max_weight,
                                             long long *d_dist, int *d_parent,
                                             mosp_sosp_stats *stats, void *stream) {
  if (n <= 0 || m < 0 || source < 0 || source >= n || delta <= 0 || d_out_row == nullptr ||
      (m > 0 && (d_out_col == nullptr || d_out_w == nullptr)) || d_dist == nullptr ||
      d_parent == nullptr) {
    return recordFailure(MOSP_ERR_INVALID, "Error: invalid SSSP arguments.");
  }
  if (n > kMaxVertices || m > kMaxEdges) {
    return recordFailure(
        MOSP_ERR_INVALID,
        ("Error: mosp_sosp_from_scratch_static handles at most " + std::to_string(kMaxVertices) +
         " vertices and " + std::to_string(kMaxEdges) + " edges (its scratch is a fixed " +
         "device array); got n = " + std::to_string(n) + ", m = " + std::to_string(m) +
         ". Use mosp_sosp_from_scratch with a workspace for larger graphs.")
            .c_str());
  }
  int bits = 0;
  u64 maxDist = 0;
  int st = mosp_choose_packing(n, max_weight, &bits, &maxDist);
  if (st != MOSP_OK) return st;

  int device = -1;
  DeviceSlot *slot = nullptr;
  unsigned char *b = nullptr;
  st = setup(device, slot, b);
  if (st != MOSP_OK) return st;
  EngineControl *ctl = reinterpret_cast<EngineControl *>(b + kOffCtl);
  int *gen = reinterpret_cast<int *>(b + kOffGen);
  int *ints = reinterpret_cast<int *>(b + kOffInts);
  const long long intStride = roundUp(kMaxVertices * 4) / 4;

  EngineParams p;
  std::memset(&p, 0, sizeof(p));
  p.n = n;
  p.m = m;
  p.K = 1;
  p.source = source;
  p.mode = kModeScratch;
  p.timeoutNs = kTimeoutNs;
  p.genPtr = gen;
  p.outRow = d_out_row;
  p.outCol = d_out_col;
  p.packed = reinterpret_cast<u64 *>(b + kOffPacked);
  p.val = ints + 0 * intStride;
  p.stamp = ints + 1 * intStride;
  p.inFar = ints + 2 * intStride;
  p.cand = ints + 3 * intStride;
  p.farL0 = ints + 4 * intStride;
  p.farL1 = ints + 5 * intStride;
  p.stride = kMaxVertices;
  p.nearV0 = reinterpret_cast<int *>(b + kOffNearV0);
  p.nearV1 = reinterpret_cast<int *>(b + kOffNearV1);
  p.nearD0 = reinterpret_cast<u64 *>(b + kOffNearD0);
  p.nearD1 = reinterpret_cast<u64 *>(b + kOffNearD1);
  p.strideNear = kNearCap;
  p.stageEntries = kStageEntriesMax;
  p.ctl = ctl;
  p.blockSums = reinterpret_cast<long long *>(b + kOffBlockSums);
  ObjectiveArgs &o = p.obj[0];
  o.outW = d_out_w;
  o.dist = d_dist;
  o.parent = d_parent;
  o.parentBits = bits;
  o.noParent = bits > 0 ? ((1ULL << bits) - 1) : 0;
  o.maxDist = maxDist;
  o.delta = static_cast<u64>(delta);

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t err = cudaMemsetAsync(ctl, 0, sizeof(EngineControl), s);
  if (err == cudaSuccess) err = cudaMemsetAsync(gen, 0, sizeof(int), s);
  if (err == cudaSuccess) err = cudaMemsetAsync(p.stamp, 0, static_cast<size_t>(n) * 4, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(p.inFar, 0, static_cast<size_t>(n) * 4, s);
  if (err != cudaSuccess) return failCuda(err, "clearing the static scratch");
  err = launchEngine(p, slot->shape.engineCtas, s);
  if (err != cudaSuccess) return failCuda(err, "engine launch");
  // the control block comes back into host stack memory (pageable), so no
  // pinned buffer is needed
  EngineControl c;
  err = cudaMemcpyAsync(&c, ctl, sizeof(EngineControl), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return failCuda(err, "engine run");
  if (c.status != 0) {
    return recordFailure(MOSP_ERR_TIMEOUT,
                         "Error: a device-side wait of the persistent kernel exceeded its limit; "
                         "the run was stopped.");
  }
  if (c.invalid) {
    return recordFailure(MOSP_ERR_INVALID,
                         "Error: malformed CSR (row offsets not monotone from 0 to m, or a column "
                         "index outside [0, n)).");
  }
  if (stats != nullptr) {
    stats->invalidated = c.invalidated[0];
    stats->jump_rounds = c.rounds;
    stats->iterations = c.iterations[0];
    stats->epochs = c.epochs[0];
    stats->pushes = c.pushes[0];
    stats->packed_parents = bits > 0 ? 1 : 0;
    stats->reserved = 0;
  }
  return MOSP_OK;
}
