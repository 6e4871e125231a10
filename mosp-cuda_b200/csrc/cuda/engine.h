// engine.h - shared host/device definitions of the sm_100a MOSP engine.
//
// The engine is a set of persistent kernels (one CTA group resident per SM,
// launched cooperatively so that every CTA is co-resident) whose phases are
// separated by a software grid barrier with a bounded wait. All state a
// phase hands to the next one lives in the workspace (device memory) or in
// the control block; per-launch arguments travel as one __grid_constant__
// parameter block, so a launch needs no host-to-device copy and can be
// queued back to back with the next one.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "mosp_b200.h"

namespace mospb200 {

using u64 = unsigned long long;

constexpr int kThreads = 1024;                // threads per CTA
constexpr int kMaxK = MOSP_MAX_OBJECTIVES;    // objectives per launch
constexpr u64 kInfWord = ~0ULL;               // packed INF (all ones)
constexpr long long kDistInf = MOSP_DISTANCE_INF;
constexpr int kLaneRowMax = 32;               // rows above: warp-cooperative
#ifndef MOSP_STAGE_ENTRIES
#define MOSP_STAGE_ENTRIES 8192
#endif
// entries of the per-CTA append stage of a bulk near-far launch (16 bytes
// each, dynamic shared memory); asynchronous launches take fewer
constexpr int kStageEntriesMax = MOSP_STAGE_ENTRIES;
constexpr int kStageEntriesAsync = 1536;     // far buffers + local buffers of 32 warps

enum EngineMode : int { kModeUpdate = 0, kModeScratch = 1, kModeCombined = 2 };

/// Per-objective arguments of one engine launch.
struct ObjectiveArgs {
  const int *outW;       // out-edge weights of this objective [m]
  const int *inW;        // in-edge weights of this objective [m]
  long long *dist;       // tree in/out [n]
  int *parent;           // tree in/out [n]
  const int *chFrom;     // deleted / weight-increased edges
  const int *chTo;
  int nChanged;
  int parentBits;        // 0: distance-only words
  u64 noParent;          // all-ones parent field
  u64 maxDist;           // (n - 1) * maxWeight: no candidate above it
  u64 delta;             // near-far bucket width (> 0)
};

/// Control block of one launch: barrier, status and the per-objective list
/// counters. Counters that change from one iteration to the next live in
/// rings of three slots (read slot i, write slot i+1, clear slot i+2), so
/// one grid barrier per iteration suffices.
struct alignas(128) EngineControl {
  unsigned arrive;       // barrier arrivals (monotone)
  unsigned pad0[31];
  unsigned release;      // barrier epoch released by the last arrival
  unsigned pad1[31];
  unsigned asyncPhase;   // asynchronous near-far: phases completed (monotone)
  unsigned pad3[31];
  unsigned asyncSplit;   // asynchronous near-far: CTAs past their phase's split (monotone)
  unsigned pad4[31];
  int status;            // 0 or MOSP_ERR_TIMEOUT (run aborted)
  int overflow;          // an input distance does not fit the packing
  int invalid;           // malformed input (ids out of range, cycles)
  int rounds;            // pointer-jumping rounds
  int jumpActive[4];
  int finalGen;          // last stamp generation used
  int heavy;             // the graph has rows of more than kHeavyDeg edges
  int pad2[2];
  unsigned long long sums[2];  // combined graph: edges, weight sum
  int candCount[kMaxK];
  int invalidated[kMaxK];
  int nearCount[kMaxK][4];
  int farCount[kMaxK][4];
  u64 farMinC[kMaxK][4];       // complement of the far-pile minimum
  int iterations[kMaxK];
  int epochs[kMaxK];
  long long pushes[kMaxK];
  // %globaltimer at the phase boundaries, written by CTA 0 (see kPhase*)
  unsigned long long phaseNs[8];
  // near-far loop profile. Bulk loop (written by CTA 0): time and items of
  // iterations that split a far pile ([0]) and of pure push iterations
  // ([1]). Asynchronous loop: loopNs[0] its time, loopIters[0] its phases,
  // loopIters[1] warp rounds, loopNs[1] of which local rounds, loopItems
  // entries taken from the queue ([0]) and from local buffers ([1])
  unsigned long long loopNs[2];
  long long loopIters[2];
  long long loopItems[2];
  // bulk loop: time (ns) of CTA 0 summed over the push iterations: decision
  // step, thread 0's own items, waiting for the CTA's other warps, list
  // flush, grid barrier. Asynchronous loop: durations of phases 0-3 and of
  // the rest
  unsigned long long iterSplitNs[5];
  // restricted parent recovery (kFlagCanonical): vertices in the changed
  // and scan lists of each objective, and chunks in the two chunk lists
  int recChanged[kMaxK];
  int recScan[kMaxK];
  int recChunks[2];
};

// EngineParams::flags (tuning switches; results do not depend on them)
enum : int {
  kFlagPrecheck = 1,     // read the word before the atomicMin of a relaxation
  kFlagHostRecovery = 2, // leave the lowest-id parent recovery of distance-only
                         // objectives to recoverParents, launched right after
  kFlagAsync = 4,        // asynchronous near-far loop (one grid barrier per far-pile
                         // split instead of one per iteration) when the graph has
                         // no hub rows
  kFlagPullOnly = 8,     // always pull into the candidates (never push from the
                         // valid vertices)
  kFlagLocal = 16,       // asynchronous loop with warp-local continuation (a warp
                         // expands up to 32 of its own pushes next); measured
                         // slower on the road workload (more re-expansions)
  kFlagCanonical = 32    // the input trees follow the lowest-id tie rule: with
                         // kFlagHostRecovery, distance-only objectives recover
                         // parents only where the batch can change them
                         // (recover.cu); the same result as the full recovery
                         // for such inputs
};

// Mark bytes of the restricted parent recovery (EngineParams::recMark, one
// per objective and vertex): the update launch writes kRecChanged where a
// distance-only objective's distance changed; kRecScan marks the vertices
// whose in-row is scanned again.
enum : unsigned char { kRecChanged = 1, kRecScan = 2 };

/// Counters of one shard of the asynchronous near queue, each on its own
/// 128-byte line: `head` is advanced by the warps that claim slots, `tail`
/// by the warps that reserve slots for new entries, `done` counts the
/// reserved entries that are settled (expanded, skipped as stale, or moved to
/// the far pile because the shard was full). A phase is over when every
/// shard has done == tail.
struct alignas(128) AsyncShard {
  unsigned head;
  unsigned pad0[31];
  unsigned tail;
  unsigned pad1[31];
  unsigned done;
  unsigned pad2[31];
};
constexpr int kAsyncShards = 32;  // shards of the near queue (one counter set)

// Phase boundaries recorded in EngineControl::phaseNs.
enum : int {
  kPhaseStart = 0,     // kernel start
  kPhasePacked = 1,    // old trees packed (update) / graph built (combined)
  kPhaseRoots = 2,     // roots marked
  kPhaseJumped = 3,    // subtrees flagged by pointer jumping
  kPhaseCandidates = 4,
  kPhasePulled = 5,    // pull pass done; near-far loop starts
  kPhaseLoop = 6,      // near-far loop done
  kPhaseEnd = 7        // results written
};

/// Parameters of one engine launch (passed by value, < 4 KB).
struct EngineParams {
  int n, m, K, source;
  // A batched run (independent instances stored as one disjoint union)
  // has one root per instance: `sources` holds them sorted, `source` is the
  // first. nSources <= 1 means the single root `source`.
  const int *sources;
  int nSources;
  int mode, maxRounds, nHeads, flags;
  int localRounds;  // CTA-local expansion rounds per near-far iteration (0: none)
  int narrowItems;  // iterations with at most this many items run on CTA 0 alone
  int narrowRounds; // CTA-local rounds of such an iteration
  long long timeoutNs;
  int *genPtr;                 // stamp generation, advanced by every launch
  const int *outRow, *outCol, *inRow, *inCol;
  const int *heads;
  // workspace lists: objective k uses [k * stride, (k + 1) * stride) of the
  // per-vertex arrays and [k * strideNear, ...) of the near lists
  u64 *packed;
  int *val, *stamp, *inFar, *cand;
  int *farL0, *farL1;
  int *nearV0, *nearV1;        // near lists: vertices
  u64 *nearD0, *nearD1;        // near lists: distance when appended
  long long stride, strideNear;
  // asynchronous near queue (kFlagAsync): aqShards shards of aqShardCap
  // slots, every slot ~0 (empty) between launches; two counter sets of
  // aqShards shards (phase parity)
  u64 *aqSlots;
  AsyncShard *aqCtr;
  unsigned aqShardCap;
  int aqShards;
  int stageEntries;            // entries of the per-CTA append stage (dynamic shared memory)
  int heavyDeg;                // rows above this many edges: whole-CTA handling (0: 2,048)
  EngineControl *ctl;
  // combined graph (Steps 2-3)
  const int *combParents;      // K trees, objective-major
  int *combDeg, *combRow, *combCol, *combW;
  long long *blockSums;
  int combK, combBase;
  long long combDelta;         // > 0: fixed width; else default
  int prefTerms[kMaxK];        // L / Pref_i
  // restricted parent recovery (kFlagCanonical): mark bytes [k * stride +
  // v]; per objective the list of vertices whose distance changed
  // (recChanged + k * stride) and of the other vertices whose in-row is
  // scanned (recScanList + k * stride); chunks of rows of more than
  // kRecLightRow edges: out-rows of changed vertices in [0, recChunkCap) of
  // recChunkList, in-rows to scan in [recChunkCap, 2 recChunkCap)
  unsigned char *recMark;
  int *recChangedList;
  int *recScanList;
  u64 *recChunkList;
  int recChunkCap;
  ObjectiveArgs obj[kMaxK];
};
static_assert(sizeof(EngineParams) <= 4096, "kernel parameter block limit");

// rows of the restricted recovery up to this many edges are handled by the
// warp of their vertex; longer rows go to a chunk list in chunks of
// 2 kRecLightRow edges, one warp per chunk (so each chunk list needs at
// most K (m / kRecLightRow + 1) entries, and no warp walks more than
// 32 kRecLightRow edges of its own vertices)
constexpr int kRecLightRow = 64;

/// Parameters of the device-graph build.
struct BuildParams {
  int n, m, K;
  long long timeoutNs;
  const int *outRow, *outCol, *edgeMajorW;
  int *outW, *inRow, *inCol, *inW;
  int *cursor;
  long long *blockSums;
  EngineControl *ctl;
};

/// Parameters of the MOSP path-cost kernel.
struct CostParams {
  int n, m, KG, source;
  const int *sources;  // sorted roots of a batched run (nSources > 1), else unused
  int nSources;
  long long timeoutNs;
  const int *outRow, *outCol, *outW;  // outW: KG objective-major columns
  const int *parent;
  int *edgeOf;
  int *anc0, *anc1;
  long long *acc0, *acc1;
  long long *costs;
  EngineControl *ctl;
};

// Host-side launchers (engine.cu). Each returns a cudaError_t of the
// launch; device-side errors are reported through the control block.
struct LaunchShape {
  int engineCtas, buildCtas, costCtas;
};
cudaError_t queryLaunchShape(int ctasPerSm, LaunchShape &shape);
cudaError_t launchEngine(const EngineParams &p, int ctas, cudaStream_t s);
/// The same cooperative launch through cudaLaunchKernelEx with the
/// cooperative attribute, the form a CUDA graph can capture.
cudaError_t launchEngineEx(const EngineParams &p, int ctas, cudaStream_t s);

/// An update launch with a distance-only objective: its parent recovery
/// runs as a kernel of its own (all of L1 for the graph reads, where the
/// update launch gives most of the SM's on-chip memory to its stage).
bool needsHostRecovery(const EngineParams &p);

/// The lowest-id tight parent recovery of the distance-only objectives of
/// update launch `p` (which ran with kFlagHostRecovery), on stream s: over
/// all edges, or (kFlagCanonical) only where the batch can change a parent.
cudaError_t launchRecovery(const EngineParams &p, cudaStream_t s);
/// The restricted recovery (recover.cu): four launches on stream s.
cudaError_t launchRestrictedRecovery(const EngineParams &p, int sms, cudaStream_t s);
cudaError_t launchBuild(const BuildParams &p, int ctas, cudaStream_t s);
cudaError_t launchCosts(const CostParams &p, int ctas, cudaStream_t s);
cudaError_t launchBarrierProbe(EngineControl *ctl, long long timeoutNs,
                               int ctas, cudaStream_t s);
cudaError_t launchBarrierCost(EngineControl *ctl, int rounds, int reads,
                              long long timeoutNs, int ctas, cudaStream_t s);

// ---------------------------------------------------------------------------
// Step 1 on the GPU (apply.cu): a change batch applied to a device CSR
// ---------------------------------------------------------------------------
struct ApplyParams {
  long long n, m;
  int K;
  const int *row, *col, *w;  // original out-CSR, edge-major weights w[e*K+k]
  int nIns, nDel;
  const int *insFrom, *insTo, *insW, *delFrom, *delTo;
  int *newRow, *newCol, *newW;  // updated out-CSR (capacity m + nIns edges)
  unsigned *mask;               // nIns weight-increase masks
  // set by applyBatchGpu
  int vbits, ibits;
  const int *sortedVals;
};

/// Per (u,v) group of the sorted batch.
struct ApplyGroups {
  int *start;  // first entry of each group (+ end sentinel)
  int *u, *v, *cD, *cI, *firstIns, *lastIns, *occ, *first;
};

/// Rows with at least one change.
struct ApplyRows {
  int *row, *gs, *deg, *off;
};

enum ApplyCounter : int {
  kApplyInvalid = 0,
  kApplyEntries,
  kApplyGroups,
  kApplyRows,
  kApplyAppended,
  kApplyCounters
};

/// Scratch bytes of applyBatchGpu for these sizes.
size_t applyScratchBytes(long long n, long long m, long long nIns, long long nDel);
/// Runs Step 1 on stream `s` and waits for it. hostCounters receives the
/// kApplyCounters device counters followed by the new edge count; when
/// hostStats is non-null it receives per objective the largest weight of
/// the original edges and insertions (at least 1), then the weight sums of
/// the original edges (2K values).
cudaError_t applyBatchGpu(ApplyParams P, void *scratch, int sms, cudaStream_t s, int *hostCounters,
                          long long *hostStats);

/// Whether v is a root: the source, or one of the sorted batched roots.
__device__ __forceinline__ bool isRoot(int source, const int *sources, int nSources, int v) {
  if (v == source) return true;
  if (nSources <= 1) return false;
  int lo = 0, hi = nSources;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const int s = sources[mid];
    if (s == v) return true;
    if (s < v) lo = mid + 1; else hi = mid;
  }
  return false;
}

/// Sets the calling thread's last-error message of the C ABI
/// (mosp_last_error) and returns `status`.
int recordFailure(int status, const char *message);

}  // namespace mospb200
