// engine.cu - persistent sm_100a kernels of the DynaMOSP update path.
//
// sosp_engine<Mode> runs a whole SOSP update (or an SSSP from scratch, or
// Steps 2-3 of the MOSP update) in one cooperative launch. The phases
// follow the reference algorithm (SMShovan/MOSP-CUDA src/sospUpdateGpu.cu:
// 211-519 and src/combinedGraphGpu.cu:55-121), re-planned for B200:
//
//   * all K objectives of a MOSP update share one launch and run their
//     phases and near-far iterations side by side, so the grid barriers
//     (the latency floor of a high-diameter graph) are paid once for all
//     objectives instead of K times;
//   * one grid barrier per near-far iteration: list counters rotate
//     through three slots and the far-pile minimum is folded into the
//     appends, so the threshold step needs no separate reduction pass;
//   * the barrier is a release/arrive pair on separate L2 lines with a
//     wall-clock bound (%globaltimer): a run that stalls returns
//     MOSP_ERR_TIMEOUT instead of hanging the GPU;
//   * subtree invalidation packs "ancestor or flag" into one int per
//     vertex, so a pointer-jumping step is two dependent loads;
//   * list appends are staged per CTA in shared memory and written out
//     with one reservation per list and iteration; a warp spreads the
//     edges of its items over its lanes, and rows of more than 2,048 edges
//     (power-law hubs) go to the whole CTA, in launches whose graph has
//     them;
//   * the pull pass scans in-rows four edges per round with their loads
//     in flight together;
//   * the lowest-id parent recovery of distance-only objectives is
//     edge-balanced (equal edge slices per warp, a shuffle search for the
//     rows) and, after an update launch, runs as its own kernel
//     (recoverParents) so that L1 is not shared with the append stage;
//     with input trees declared canonical it is restricted to the vertices
//     the batch reaches (recover.cu: the unpack lists the vertices whose
//     distance changed).
//
// Result semantics (identical to the reference): words pack
// (distance << b | parent) and only strictly better words are kept
// (64-bit atomicMin), so among equal distances the lowest parent id wins;
// a vertex is expanded whenever its distance strictly decreases. The fixed
// point does not depend on the schedule, the grid size or the bucket width.
#include "engine.h"

#include <climits>

namespace mospb200 {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// Small device helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned laneId() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned long long globalNs() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ldAcquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void stRelease(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ldVolatile(const int *p) {
  return *reinterpret_cast<const volatile int *>(p);
}

__device__ __forceinline__ unsigned ldVolatileU(const unsigned *p) {
  return *reinterpret_cast<const volatile unsigned *>(p);
}

__device__ __forceinline__ unsigned long long ldAcquire64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void stRelease64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void stRelaxed64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void redRelease(unsigned *p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

/// Word helpers for one objective.
struct Pk {
  int bits;
  u64 noParent;
  __device__ __forceinline__ u64 pack(u64 d, int p) const {
    return bits == 0 ? d : ((d << bits) | (p < 0 ? noParent : static_cast<u64>(p)));
  }
  __device__ __forceinline__ u64 dist(u64 w) const { return w >> bits; }
  __device__ __forceinline__ int parent(u64 w) const {
    const u64 f = w & noParent;
    return f == noParent ? -1 : static_cast<int>(f);
  }
};

__device__ __forceinline__ Pk pkOf(const ObjectiveArgs &o) {
  return Pk{o.parentBits, o.noParent};
}

/// Barrier bookkeeping of one CTA: the barrier epoch and the wall-clock
/// deadline (%globaltimer) of the whole launch.
struct Sync {
  unsigned epoch;
  unsigned long long deadline;
};

__device__ __forceinline__ Sync startSync(long long timeoutNs) {
  return Sync{0u, globalNs() + static_cast<unsigned long long>(timeoutNs)};
}

/// Software grid barrier. Thread 0 of every CTA arrives on `arrive`; the
/// last arrival publishes the epoch on `release`, which the others poll
/// (acquire). The launch has one wall-clock deadline: a CTA that reaches a
/// barrier after it marks the run MOSP_ERR_TIMEOUT and returns false
/// without arriving, so the others cannot pass this barrier; a CTA that
/// waits past it, or sees the status set while it waits (checked every 32
/// polls, off the path of a release that arrives in time), does the same.
/// A CTA that passed a barrier before the status was set returns false at
/// the next one (the deadline has passed by then), and the kernel must
/// return. So a run ends by the deadline whether it stalls or keeps
/// iterating.
__device__ bool gridSync(EngineControl *c, Sync &sync) {
  __shared__ int sOk;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned epoch = ++sync.epoch;
    int ok = 1;
    if (globalNs() > sync.deadline) {
      atomicCAS(&c->status, 0, MOSP_ERR_TIMEOUT);
      ok = 0;
    } else {
      __threadfence();
      const unsigned prev = atomicAdd(&c->arrive, 1u);
      if (prev + 1u == epoch * gridDim.x) {
        stRelease(&c->release, epoch);
      } else {
        unsigned spin = 0;
        while (static_cast<int>(ldAcquire(&c->release) - epoch) < 0) {
          if ((++spin & 31u) == 0) {
            if (ldVolatile(&c->status) != 0) {
              ok = 0;
              break;
            }
            if (globalNs() > sync.deadline) {
              atomicCAS(&c->status, 0, MOSP_ERR_TIMEOUT);
              ok = 0;
              break;
            }
          }
        }
      }
      __threadfence();
    }
    sOk = ok;
  }
  __syncthreads();
  return sOk != 0;
}

/// CTA 0 records the time of a phase boundary.
__device__ __forceinline__ void markPhase(EngineControl *c, int phase) {
  if (blockIdx.x == 0 && threadIdx.x == 0) c->phaseNs[phase] = globalNs();
}

/// Reserve one slot of a list: one atomicAdd per group of lanes of the warp
/// that append to the same counter at the same time.
__device__ __forceinline__ int warpAppend(int *counter) {
  const unsigned mask = __activemask();
  const unsigned peers =
      __match_any_sync(mask, static_cast<unsigned long long>(reinterpret_cast<uintptr_t>(counter)));
  const int leader = __ffs(peers) - 1;
  const unsigned lane = laneId();
  int base = 0;
  if (static_cast<int>(lane) == leader) base = atomicAdd(counter, __popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}

/// Fold d into the minimum kept (as a complement, so 0 means "none") at
/// *minC: one atomicMax per group of lanes with the same target.
__device__ __forceinline__ void warpMinInto(u64 *minC, u64 d) {
  const unsigned mask = __activemask();
  const unsigned peers =
      __match_any_sync(mask, static_cast<unsigned long long>(reinterpret_cast<uintptr_t>(minC)));
  const unsigned hi = static_cast<unsigned>(d >> 32);
  const unsigned lo = static_cast<unsigned>(d);
  const unsigned mhi = __reduce_min_sync(peers, hi);
  const unsigned mlo = __reduce_min_sync(peers, hi == mhi ? lo : 0xffffffffu);
  if (static_cast<int>(laneId()) == __ffs(peers) - 1) {
    atomicMax(minC, ~((static_cast<u64>(mhi) << 32) | mlo));
  }
}

__device__ __forceinline__ u64 warpMinU64(u64 v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const u64 o = __shfl_xor_sync(kFull, v, off);
    v = o < v ? o : v;
  }
  return v;
}

/// Graph loads: the update and scratch modes read a graph that is
/// read-only for the whole launch (read-only path); the combined mode
/// reads a graph built earlier in the same launch (L2).
template <int Mode>
__device__ __forceinline__ int ldGraph(const int *p) {
  if constexpr (Mode == kModeCombined) {
    return __ldcg(p);
  } else {
    return __ldg(p);
  }
}

// Shared per-CTA view of the loop state (identical in every CTA).
struct LoopShared {
  long long off[kMaxK + 1];
  u64 thr[kMaxK];
  int mode[kMaxK];
  int fp[kMaxK];
  int fs[kMaxK];
  long long total;
};

enum : int { kDone = 0, kPush = 1, kSplit = 2 };

// ---------------------------------------------------------------------------
// Per-CTA staging of list appends
//
// Every append of an iteration (next near list, far piles) goes to a
// shared-memory buffer first: a shared atomic per warp group gives the slot
// and the rank within the destination list. At the end of the iteration the
// CTA reserves one range per list with a single global atomic and copies
// its entries out, so the same-address global counters see one atomic per
// CTA and list instead of one per warp group on the relaxation's critical
// path. Entries that do not fit the buffer take the direct global path.
// ---------------------------------------------------------------------------
constexpr int kStage = kStageEntriesMax;
// Rows with more edges than this are expanded (push) or reduced (pull) by a
// whole CTA instead of one warp: a power-law hub row (10^5 edges) would
// otherwise keep one warp busy for the whole iteration. A launch turns
// this on only when its graph has such rows (EngineControl::heavy, set in
// the first phase), so graphs without them take no extra CTA barriers.
constexpr int kHeavyDegDefault = 2048;  // EngineParams::heavyDeg when 0
constexpr int kHeavyCap = 64;

/// Rows above this many edges go to a whole CTA (and keep a launch in the
/// bulk loop); a launch parameter, so the autotuner can move it.
__device__ __forceinline__ int heavyDegOf(const EngineParams &P) {
  return P.heavyDeg > 0 ? P.heavyDeg : kHeavyDegDefault;
}

struct StageHeader {
  int cap;                     // entries per list partition (kStage / (2K))
  int pad;
  int count[2 * kMaxK];        // appends per list this iteration (may exceed cap)
  int start[2 * kMaxK];        // entries before this were expanded by the CTA itself
  int roundEnd[kMaxK];         // end of the near entries of the current local round
  int roundTotal;              // entries of the current local round (0: no round)
  int base[2 * kMaxK];         // global start of this CTA's range
  u64 farMin[kMaxK];           // minimum distance appended to far (plain)
  long long expanded[kMaxK];   // non-stale expansions (statistics)
  // heavy rows met by the CTA's warps, handled by the whole CTA afterwards
  // (rows beyond kHeavyCap stay with their warp)
  int heavyCount;
  int heavyK[kHeavyCap];
  int heavyU[kHeavyCap];
  int heavyBeg[kHeavyCap];
  int heavyDeg[kHeavyCap];
  u64 heavyD[kHeavyCap];       // push: the row's distance; pull: the word before the pass
  u64 heavyBest[kHeavyCap];    // pull: best word over the row, reduced by the CTA
  int asyncFar[kThreads / 32]; // async loop: entries in each warp's far buffer
  int asyncLocal[kThreads / 32]; // async loop: entries in each warp's local buffer (may overshoot)
};

struct StageEntry {
  int v;
  int meta;                    // list << 16 | rank
  u64 d;
};

constexpr size_t kStageHeaderBytes = (sizeof(StageHeader) + 15) / 16 * 16;
constexpr size_t kStageBytes = kStageHeaderBytes + kStage * sizeof(StageEntry);

/// Dynamic shared memory of a launch with `entries` stage entries.
constexpr size_t stageBytesFor(int entries) {
  return kStageHeaderBytes + static_cast<size_t>(entries) * sizeof(StageEntry);
}

__device__ __forceinline__ StageHeader &stageHeader() {
  extern __shared__ __align__(16) unsigned char dynSmem[];
  return *reinterpret_cast<StageHeader *>(dynSmem);
}

__device__ __forceinline__ StageEntry *stageEntries() {
  extern __shared__ __align__(16) unsigned char dynSmem[];
  return reinterpret_cast<StageEntry *>(dynSmem + kStageHeaderBytes);
}

/// Destination of list l in this iteration: near list of objective l (l <
/// K) or the far pile objective l - K appends to (the current pile while it
/// pushes, the other pile while its pile is split).
struct Target {
  int *counter;
  int *v;
  u64 *d;
  u64 *minC;
};

__device__ __forceinline__ Target listTarget(const EngineParams &P, const LoopShared &L, int l,
                                             int wrSlot, int *nearWV, u64 *nearWD) {
  const int K = P.K;
  if (l < K) {
    const long long kn = static_cast<long long>(l) * P.strideNear;
    return Target{&P.ctl->nearCount[l][wrSlot], nearWV + kn, nearWD + kn, nullptr};
  }
  const int k = l - K;
  const long long ko = static_cast<long long>(k) * P.stride;
  if (L.mode[k] == kSplit) {
    const int s = (L.fs[k] + 1) % 3;
    return Target{&P.ctl->farCount[k][s], (L.fp[k] == 0 ? P.farL1 : P.farL0) + ko, nullptr,
                  &P.ctl->farMinC[k][s]};
  }
  const int s = L.fs[k];
  return Target{&P.ctl->farCount[k][s], (L.fp[k] == 0 ? P.farL0 : P.farL1) + ko, nullptr,
                &P.ctl->farMinC[k][s]};
}

/// A near entry (v, d) of objective k that found its near list full goes to
/// the far pile instead (once, by the in-far flag); the split after the
/// near list has run dry brings it back below the threshold. So the near
/// lists can be smaller than the worst case of one iteration.
__device__ __forceinline__ void divertToFar(const EngineParams &P, const LoopShared &L, int k, int v,
                                            u64 d) {
  if (atomicExch(P.inFar + static_cast<long long>(k) * P.stride + v, 1) != 0) return;
  const Target t = listTarget(P, L, P.K + k, 0, nullptr, nullptr);
  const int idx = warpAppend(t.counter);
  t.v[idx] = v;
  warpMinInto(t.minC, d);
}

/// Append (v, d) to list l (far lists: d only feeds the pile minimum). The
/// staging buffer is split into one partition per list; the rank within the
/// list is the slot, so a warp group needs one shared atomic.
__device__ __forceinline__ void stageAppend(const EngineParams &P, const LoopShared &L, int l,
                                            int v, u64 d, int wrSlot, int *nearWV, u64 *nearWD) {
  StageHeader &H = stageHeader();
  StageEntry *E = stageEntries();
  const unsigned lane = laneId();
  const unsigned lt = (1u << lane) - 1u;
  const unsigned mask = __activemask();
  const unsigned peers = __match_any_sync(mask, l);
  const int leader = __ffs(peers) - 1;
  int rankBase = 0;
  if (static_cast<int>(lane) == leader) rankBase = atomicAdd(&H.count[l], __popc(peers));
  rankBase = __shfl_sync(peers, rankBase, leader);
  const int rank = rankBase + __popc(peers & lt);
  if (l >= P.K) {
    // far pile minimum of this CTA (shared), reduced over the group first
    const unsigned hi = static_cast<unsigned>(d >> 32), lo = static_cast<unsigned>(d);
    const unsigned mhi = __reduce_min_sync(peers, hi);
    const unsigned mlo = __reduce_min_sync(peers, hi == mhi ? lo : 0xffffffffu);
    if (static_cast<int>(lane) == leader) {
      atomicMin(&H.farMin[l - P.K], (static_cast<u64>(mhi) << 32) | mlo);
    }
  }
  if (rank < H.cap) {
    E[l * H.cap + rank] = StageEntry{v, 0, d};
  } else {
    // partition full: this entry takes the direct global path
    const Target t = listTarget(P, L, l, wrSlot, nearWV, nearWD);
    const int idx = warpAppend(t.counter);
    if (l < P.K && idx >= P.strideNear) {
      divertToFar(P, L, l, v, d);
      return;
    }
    t.v[idx] = v;
    if (t.d != nullptr) t.d[idx] = d;
  }
}

/// End of an iteration: reserve every list's range once per CTA, copy the
/// staged entries out, fold the far minima. (The expansion counts are
/// summed per CTA and folded into the statistics after the loop.)
__device__ void flushStage(const EngineParams &P, const LoopShared &L, int wrSlot, int *nearWV,
                           u64 *nearWD) {
  StageHeader &H = stageHeader();
  StageEntry *E = stageEntries();
  const int K = P.K;
  __syncthreads();
  const int t = threadIdx.x;
  if (t < 2 * K) {
    const int staged = (H.count[t] < H.cap ? H.count[t] : H.cap) - H.start[t];
    if (staged > 0) H.base[t] = atomicAdd(listTarget(P, L, t, wrSlot, nearWV, nearWD).counter, staged);
  }
  if (t < K && H.farMin[t] != kInfWord) {
    atomicMax(listTarget(P, L, K + t, wrSlot, nearWV, nearWD).minC, ~H.farMin[t]);
  }
  __syncthreads();
  for (int l = 0; l < 2 * K; ++l) {
    const int first = H.start[l];
    const int staged = (H.count[l] < H.cap ? H.count[l] : H.cap) - first;
    if (staged <= 0) continue;
    const Target tg = listTarget(P, L, l, wrSlot, nearWV, nearWD);
    const int b = H.base[l];
    for (int i = t; i < staged; i += blockDim.x) {
      const StageEntry e = E[l * H.cap + first + i];
      if (l < K && b + i >= P.strideNear) {
        divertToFar(P, L, l, e.v, e.d);  // the near list is full
        continue;
      }
      tg.v[b + i] = e.v;
      if (tg.d != nullptr) tg.d[b + i] = e.d;
    }
  }
}

/// Edge slots a lane relaxes at once (loads and atomics overlapped).
#ifndef MOSP_EDGE_SLOTS
#define MOSP_EDGE_SLOTS 2
#endif
constexpr int kSlots = MOSP_EDGE_SLOTS;
// asynchronous rounds: three slots per lane cover the ~90 edges of 32 road
// vertices in one pass (one chain of edge loads, atomicMin and reservation
// instead of two)
#ifndef MOSP_EDGE_SLOTS_ASYNC
#define MOSP_EDGE_SLOTS_ASYNC 3
#endif
constexpr int kSlotsAsync = MOSP_EDGE_SLOTS_ASYNC;

// ---------------------------------------------------------------------------
// Asynchronous near queue
//
// In the asynchronous loop the near entries of all objectives go to one
// queue of aqShards shards. An entry is one 64-bit word: the vertex and its
// objective (v << 5 | k) in the low half and the distance it was pushed with
// (saturated at kTagSat) in the high half; an empty slot holds all ones, so a
// consumer that claimed a slot before its entry was written sees it arrive.
// A warp reserves slots for the entries of one round with one atomic on the
// target shard's tail (shards rotate per round, which spreads the work), and
// claims 32 slots of its home shard with one atomic on the head; it settles
// what it consumed with one release add on the shard's `done` after its own
// reservations, so done == tail on every shard (read twice, identical) means
// that no entry is left and none can be produced. A reservation past the
// shard's capacity moves its vertex to the far pile instead (re-split in the
// next phase), so the queue never needs more than its fixed size.
// ---------------------------------------------------------------------------
constexpr unsigned long long kEmptySlot = ~0ULL;
constexpr unsigned kTagSat = 0xFFFFFFFEu;  // distances >= this are not carried in the entry
constexpr int kFarBuf = 128;               // per-warp far buffer entries (async loop)
constexpr int kLocalBuf = 32;              // per-warp local near entries (async loop)
constexpr int kWarps = kThreads / 32;

struct AsyncState {
  AsyncShard *ctr;   // this phase's counter set
  int target;        // shard that receives this warp round's near entries
  unsigned spilled;  // this lane's reservations past the shard's capacity
  bool local;        // near entries may stay in the warp's local buffer
};

/// Per-warp buffers of near entries the warp expands itself next (async
/// loop), after the far buffers in the stage region.
__device__ __forceinline__ u64 *asyncLocalBuffer(int warp) {
  return reinterpret_cast<u64 *>(reinterpret_cast<int *>(stageEntries()) + kWarps * kFarBuf) +
         warp * kLocalBuf;
}

/// Per-warp buffers of far-pile appends in the async loop (v << 5 | k), in
/// the stage region of the dynamic shared memory.
__device__ __forceinline__ int *asyncFarBuffer(int warp) {
  return reinterpret_cast<int *>(stageEntries()) + warp * kFarBuf;
}

/// Far-pile append in the async loop: into the warp's buffer (flushed by
/// flushAsyncFar before it can overflow), the CTA's far minimum in shared
/// memory. An append that finds the buffer full goes to the pile directly.
__device__ __forceinline__ void asyncFar(const EngineParams &P, const LoopShared &L, int k, int w,
                                         u64 d) {
  StageHeader &H = stageHeader();
  const int warp = threadIdx.x >> 5;
  atomicMin(&H.farMin[k], d);
  const int slot = atomicAdd(&H.asyncFar[warp], 1);
  if (slot < kFarBuf) {
    asyncFarBuffer(warp)[slot] = (w << 5) | k;
  } else {
    const Target t = listTarget(P, L, P.K + k, 0, nullptr, nullptr);
    const int idx = warpAppend(t.counter);
    t.v[idx] = w;
  }
}

/// The warp's buffered far appends to their piles (one reservation per
/// objective group of lanes). All 32 lanes call it.
__device__ void flushAsyncFar(const EngineParams &P, const LoopShared &L) {
  StageHeader &H = stageHeader();
  const int warp = threadIdx.x >> 5;
  const unsigned lane = laneId();
  __syncwarp();
  int cnt = H.asyncFar[warp];
  cnt = cnt < kFarBuf ? cnt : kFarBuf;
  const int *buf = asyncFarBuffer(warp);
  for (int i0 = 0; i0 < cnt; i0 += 32) {
    const int i = i0 + static_cast<int>(lane);
    if (i < cnt) {
      const int e = buf[i];
      const int k = e & 31;
      const int v = static_cast<int>(static_cast<unsigned>(e) >> 5);
      const Target t = listTarget(P, L, P.K + k, 0, nullptr, nullptr);
      const int idx = warpAppend(t.counter);
      t.v[idx] = v;
    }
  }
  __syncwarp();
  if (lane == 0) H.asyncFar[warp] = 0;
  __syncwarp();
}

/// Whether the warp's far buffer has fewer than `margin` free entries; the
/// same answer in every lane (all 32 lanes call it).
__device__ __forceinline__ bool farBufferFull(int margin) {
  __syncwarp();
  const int cnt = __shfl_sync(kFull, stageHeader().asyncFar[threadIdx.x >> 5], 0);
  return cnt > kFarBuf - margin;
}

/// Near-queue push of (w, d) for objective k into the round's target shard.
/// The active lanes share one reservation.
__device__ __forceinline__ void asyncNear(const EngineParams &P, const LoopShared &L, AsyncState &A,
                                          int k, int w, u64 d) {
  const unsigned lane = laneId();
  const unsigned tag = d < kTagSat ? static_cast<unsigned>(d) : kTagSat;
  if (A.local) {
    // the warp keeps up to kLocalBuf of its own pushes and expands them
    // next, without the queue's round trips
    const int warp = threadIdx.x >> 5;
    const int slot = atomicAdd(&stageHeader().asyncLocal[warp], 1);
    if (slot < kLocalBuf) {
      asyncLocalBuffer(warp)[slot] =
          (static_cast<u64>(tag) << 32) | ((static_cast<unsigned>(w) << 5) | static_cast<unsigned>(k));
      return;
    }
  }
  const unsigned mask = __activemask();
  const int leader = __ffs(mask) - 1;
  unsigned base = 0;
  if (static_cast<int>(lane) == leader) base = atomicAdd(&A.ctr[A.target].tail, __popc(mask));
  base = __shfl_sync(mask, base, leader);
  const unsigned idx = base + __popc(mask & ((1u << lane) - 1u));
  if (idx < P.aqShardCap) {
    const u64 e = (static_cast<u64>(tag) << 32) | ((static_cast<unsigned>(w) << 5) | static_cast<unsigned>(k));
    u64 *slot = P.aqSlots + static_cast<long long>(A.target) * P.aqShardCap + idx;
    // A consumer expands with min(tag, its read of the word), so only an
    // entry without a usable tag needs the word ordered before it.
    if (tag < kTagSat) stRelaxed64(slot, e); else stRelease64(slot, e);
  } else {
    ++A.spilled;
    if (atomicExch(P.inFar + static_cast<long long>(k) * P.stride + w, 1) == 0) asyncFar(P, L, k, w, d);
  }
}

/// A strict improvement of w's distance to d (objective k): to the next near
/// list (d below the threshold) or, once, to the far pile.
template <bool Async>
__device__ __forceinline__ void pushImproved(const EngineParams &P, const LoopShared &L, AsyncState *A,
                                             int k, int w, u64 d, int wrSlot, int *nearWV,
                                             u64 *nearWD) {
  if (d < L.thr[k]) {
    if constexpr (Async) {
      asyncNear(P, L, *A, k, w, d);
    } else {
      stageAppend(P, L, k, w, d, wrSlot, nearWV, nearWD);
    }
  } else if (atomicExch(P.inFar + static_cast<long long>(k) * P.stride + w, 1) == 0) {
    if constexpr (Async) {
      asyncFar(P, L, k, w, d);
    } else {
      stageAppend(P, L, P.K + k, w, d, wrSlot, nearWV, nearWD);
    }
  }
}

/// Lane of the warp whose edge range holds edge slot s: the number of
/// lanes whose inclusive edge count is <= s (binary search by shuffles).
__device__ __forceinline__ int slotOwner(int incl, int s) {
  int lo = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const int probe = __shfl_sync(kFull, incl, lo + step - 1);
    if (probe <= s) lo += step;
  }
  return lo;
}

/// Relaxation of edge e out of u (objective k, distance du): atomicMin of
/// the word of its head, and the stage append of a strict improvement.
template <int Mode>
__device__ __forceinline__ void relaxEdge(const EngineParams &P, const LoopShared &L,
                                          const int *outCol, const int *const *outWk, int k,
                                          int u, u64 du, int e, int wrSlot, int *nearWV,
                                          u64 *nearWD) {
  const ObjectiveArgs &O = P.obj[k];
  const Pk pk = pkOf(O);
  const long long ko = static_cast<long long>(k) * P.stride;
  const int w = ldGraph<Mode>(outCol + e);
  const u64 nd = du + static_cast<u64>(ldGraph<Mode>(outWk[k] + e));
  if (w == P.source || nd > O.maxDist) return;
  const u64 old = atomicMin(P.packed + ko + w, pk.pack(nd, u));
  if (nd >= pk.dist(old)) return;
  pushImproved<false>(P, L, nullptr, k, w, nd, wrSlot, nearWV, nearWD);
}

/// The CTA's queued heavy rows, each expanded by all threads of the CTA.
/// Every thread of the CTA calls it; it starts with a barrier (so it also
/// serves as the barrier after the expansion that queued the rows) and,
/// when rows were queued, ends with one.
template <int Mode>
__device__ void expandHeavy(const EngineParams &P, const LoopShared &L, const int *outCol,
                            const int *const *outWk, int wrSlot, int *nearWV, u64 *nearWD) {
  StageHeader &H = stageHeader();
  __syncthreads();
  const int queued = H.heavyCount;
  if (queued == 0) return;  // the same for every thread of the CTA
  // every thread has read the count before it is reset; no warp queues a
  // row again before the last barrier below
  __syncthreads();
  if (threadIdx.x == 0) H.heavyCount = 0;
  const int count = queued < kHeavyCap ? queued : kHeavyCap;
  for (int h = 0; h < count; ++h) {
    const int k = H.heavyK[h], u = H.heavyU[h], beg = H.heavyBeg[h], end = beg + H.heavyDeg[h];
    const u64 du = H.heavyD[h];
    for (int e = beg + static_cast<int>(threadIdx.x); e < end; e += blockDim.x) {
      relaxEdge<Mode>(P, L, outCol, outWk, k, u, du, e, wrSlot, nearWV, nearWD);
    }
  }
  __syncthreads();
}

/// One warp expands up to 32 near entries, one per lane (u < 0: none):
/// the edges of all lanes are spread over the warp, two slots per lane,
/// with their loads and 64-bit atomicMin overlapped; every strict
/// improvement is staged for the next near list or the far pile. All 32
/// lanes call it.
template <int Mode, bool Async = false>
__device__ __forceinline__ void expandWarp(const EngineParams &P, const LoopShared &L,
                                           const int *outRow, const int *outCol,
                                           const int *const *outWk, int k, int u, u64 du, int beg,
                                           int deg, int wrSlot, int *nearWV, u64 *nearWD,
                                           bool heavyOn, AsyncState *A = nullptr) {
  StageHeader &H = stageHeader();
  const unsigned lane = laneId();
  {
    // statistics: one shared add per objective present in the warp
    const unsigned live = __ballot_sync(kFull, u >= 0);
    if (live != 0) {
      const unsigned peers = __match_any_sync(kFull, u >= 0 ? k : -1);
      if (u >= 0 && static_cast<int>(lane) == __ffs(peers) - 1) {
        atomicAdd(reinterpret_cast<unsigned long long *>(&H.expanded[k]),
                  static_cast<unsigned long long>(__popc(peers)));
      }
    }
  }
  if (__ballot_sync(kFull, deg > 0) == 0) return;
  // heavy rows go to the CTA's queue (expanded by the whole CTA after this
  // round of items) when the launch has any
  if (heavyOn && deg > heavyDegOf(P)) {
    const int slot = atomicAdd(&H.heavyCount, 1);
    if (slot < kHeavyCap) {
      H.heavyK[slot] = k;
      H.heavyU[slot] = u;
      H.heavyBeg[slot] = beg;
      H.heavyDeg[slot] = deg;
      H.heavyD[slot] = du;
      deg = 0;
    }
  }
  // rows above 2^20 edges: whole-warp striding, one row at a time
  unsigned huge = __ballot_sync(kFull, deg > (1 << 20));
  while (huge != 0) {
    const int src = __ffs(huge) - 1;
    huge &= huge - 1;
    const int kb = __shfl_sync(kFull, k, src);
    const int ub = __shfl_sync(kFull, u, src);
    const u64 db = __shfl_sync(kFull, du, src);
    const int bb = __shfl_sync(kFull, beg, src);
    const int eb = bb + __shfl_sync(kFull, deg, src);
    const ObjectiveArgs &O = P.obj[kb];
    const Pk pk = pkOf(O);
    const long long kob = static_cast<long long>(kb) * P.stride;
    for (int e = bb + static_cast<int>(lane); e < eb; e += 32) {
      const int w = ldGraph<Mode>(outCol + e);
      const u64 nd = db + static_cast<u64>(ldGraph<Mode>(outWk[kb] + e));
      if (w == P.source || nd > O.maxDist) continue;
      const u64 old = atomicMin(P.packed + kob + w, pk.pack(nd, ub));
      if (nd >= pk.dist(old)) continue;
      pushImproved<Async>(P, L, A, kb, w, nd, wrSlot, nearWV, nearWD);
    }
  }
  if (deg > (1 << 20)) deg = 0;
  int incl = deg;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int o = __shfl_up_sync(kFull, incl, off);
    if (static_cast<int>(lane) >= off) incl += o;
  }
  const int edges = __shfl_sync(kFull, incl, 31);
  const int excl = incl - deg;
  constexpr int SL = Async ? kSlotsAsync : kSlots;
  for (int s0 = 0; s0 < edges; s0 += 32 * SL) {
    if constexpr (Async) {
      // room for this round's far appends in the warp's buffer
      if (farBufferFull(32 * SL)) flushAsyncFar(P, L);
    }
    // SL edge slots per lane, their loads and atomics overlapped
    int sl[SL], kk[SL], uu[SL], ee[SL], ww[SL], wt[SL];
    u64 dd[SL], nd[SL], old[SL];
    bool act[SL];
#pragma unroll
    for (int h = 0; h < SL; ++h) {
      sl[h] = s0 + 32 * h + static_cast<int>(lane);
      const int o = slotOwner(incl, sl[h]);
      kk[h] = __shfl_sync(kFull, k, o);
      uu[h] = __shfl_sync(kFull, u, o);
      dd[h] = __shfl_sync(kFull, du, o);
      ee[h] = __shfl_sync(kFull, beg, o) + sl[h] - __shfl_sync(kFull, excl, o);
      act[h] = sl[h] < edges;
    }
#pragma unroll
    for (int h = 0; h < SL; ++h) {
      ww[h] = act[h] ? ldGraph<Mode>(outCol + ee[h]) : 0;
      wt[h] = act[h] ? ldGraph<Mode>(outWk[kk[h]] + ee[h]) : 0;
    }
    u64 cw[SL];
#pragma unroll
    for (int h = 0; h < SL; ++h) {
      nd[h] = dd[h] + static_cast<u64>(wt[h]);
      act[h] = act[h] && ww[h] != P.source && nd[h] <= P.obj[kk[h]].maxDist;
      cw[h] = pkOf(P.obj[kk[h]]).pack(nd[h], uu[h]);
    }
    if (P.flags & kFlagPrecheck) {
      u64 cur[SL];
#pragma unroll
      for (int h = 0; h < SL; ++h) {
        cur[h] = act[h] ? __ldcg(P.packed + static_cast<long long>(kk[h]) * P.stride + ww[h]) : 0;
      }
#pragma unroll
      for (int h = 0; h < SL; ++h) act[h] = act[h] && cw[h] < cur[h];
    }
#pragma unroll
    for (int h = 0; h < SL; ++h) {
      old[h] = act[h] ? atomicMin(P.packed + static_cast<long long>(kk[h]) * P.stride + ww[h], cw[h])
                      : 0;
    }
#pragma unroll
    for (int h = 0; h < SL; ++h) {
      if (!act[h] || nd[h] >= pkOf(P.obj[kk[h]]).dist(old[h])) continue;
      pushImproved<Async>(P, L, A, kk[h], ww[h], nd[h], wrSlot, nearWV, nearWD);
    }
  }
}

// ---------------------------------------------------------------------------
// Near-far loop shared by every mode
//
// Near lists carry (vertex, distance) pairs: an entry is stale when the
// vertex's word has a smaller distance by the time it is read, and is then
// skipped (a newer entry exists). Every strict improvement appends exactly
// one entry, so no claim atomic is needed and a list never holds more
// entries than the relaxations of one iteration (<= m) plus the far pile
// (<= n). Far piles keep one entry per vertex (inFar flag).
// ---------------------------------------------------------------------------
template <int Mode>
__device__ bool nearFarLoop(const EngineParams &P, const int *outRow,
                            const int *outCol, const int *const *outWk,
                            Sync &epoch, u64 *deltaOverride, int genBase) {
  __shared__ LoopShared L;
  StageHeader &H = stageHeader();
  EngineControl *c = P.ctl;
  const int K = P.K;
  const unsigned lane = laneId();
  const int warp = threadIdx.x >> 5;
  const long long gwarp = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + warp;
  const long long nwarps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);

  // Per-objective loop state, held by lane k of warp 0 (same in every CTA).
  u64 thr = 0;
  int fp = 0, fs = 0;
  int iters = 0, epochs = 0;
  u64 delta = 1;
  if (warp == 0 && static_cast<int>(lane) < K) {
    delta = P.obj[lane].delta;
    if (deltaOverride != nullptr && lane == 0) delta = *deltaOverride;
  }

  if (threadIdx.x < kMaxK) H.expanded[threadIdx.x] = 0;
  // set before the grid barrier that precedes the loop, the same for all
  const bool heavyOn = __ldcg(&c->heavy) != 0;
  int it = 0;
  unsigned long long profNs[2] = {0, 0};
  long long profIters[2] = {0, 0}, profItems[2] = {0, 0};
  unsigned long long part[5] = {0, 0, 0, 0, 0};
  unsigned long long tDecided = 0, tWorked = 0;
  for (;; ++it) {
    const int rdSlot = it % 3, wrSlot = (it + 1) % 3, clrSlot = (it + 2) % 3;
    const unsigned long long itStart = globalNs();
    if (threadIdx.x < 2 * kMaxK) {
      H.count[threadIdx.x] = 0;
      H.start[threadIdx.x] = 0;
    }
    if (threadIdx.x < kMaxK) H.farMin[threadIdx.x] = kInfWord;
    if (threadIdx.x == 0) {
      H.cap = P.stageEntries / (2 * K);
      H.heavyCount = 0;
    }
    if (warp == 0) {
      const int k = static_cast<int>(lane);
      const bool act = k < K;
      int mode = kDone;
      long long items = 0;
      if (act) {
        // (a count past the list's capacity counts entries diverted to far)
        const int nc = static_cast<int>(
            min(static_cast<long long>(__ldcg(&c->nearCount[k][rdSlot])), P.strideNear));
        if (nc > 0) {
          mode = kPush;
          items = nc;
        } else {
          const int fc = __ldcg(&c->farCount[k][fs]);
          if (fc > 0) {
            mode = kSplit;
            items = fc;
            const u64 mnC = __ldcg(&c->farMinC[k][fs]);
            u64 lo = thr;
            if (mnC != 0) {
              const u64 mn = ~mnC;
              lo = mn > thr ? mn : thr;
            }
            thr = (lo > kInfWord - delta) ? kInfWord - 1 : lo + delta;
          }
        }
      }
      long long incl = items;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const long long o = __shfl_up_sync(kFull, incl, off);
        if (static_cast<int>(lane) >= off) incl += o;
      }
      if (act) {
        L.off[k] = incl - items;
        L.thr[k] = thr;
        L.mode[k] = mode;
        L.fp[k] = fp;
        L.fs[k] = fs;
      }
      const long long total = __shfl_sync(kFull, incl, 31);
      if (lane == 0) L.total = total;
      if (act) {
        if (blockIdx.x == 0) {
          c->nearCount[k][clrSlot] = 0;
          if (mode == kSplit) {
            c->farCount[k][(fs + 2) % 3] = 0;
            c->farMinC[k][(fs + 2) % 3] = 0;
          }
        }
        if (mode == kPush) {
          ++iters;
        } else if (mode == kSplit) {
          ++epochs;
          fp ^= 1;           // takes effect after this iteration
          fs = (fs + 1) % 3;
        }
      }
    }
    __syncthreads();
    const long long total = L.total;
    if (total == 0) break;
    if (blockIdx.x == 0 && threadIdx.x == 0) tDecided = globalNs();

    const int *nearRV = (it & 1) ? P.nearV1 : P.nearV0;
    const u64 *nearRD = (it & 1) ? P.nearD1 : P.nearD0;
    int *nearWV = (it & 1) ? P.nearV0 : P.nearV1;
    u64 *nearWD = (it & 1) ? P.nearD0 : P.nearD1;

    // items per warp: ceil(total / warps), between 8 and 32, so that an
    // iteration is spread over every warp of the grid rather than over
    // total / 32 of them (the edges of a warp's items still spread over
    // all 32 lanes)
    //
    // A narrow iteration (at most P.narrowItems items, e.g. a deep graph's
    // thin wavefront or the tail of an epoch) goes to CTA 0 alone, which
    // then keeps expanding the entries it produces (up to P.narrowRounds
    // CTA-local rounds, each a __syncthreads instead of a grid barrier)
    // while the other CTAs go straight to the barrier.
    const bool narrow = total <= P.narrowItems;
    const long long myWarp = narrow ? warp : gwarp;
    const long long allWarps = narrow ? static_cast<long long>(blockDim.x >> 5) : nwarps;
    long long chunk = (total + allWarps - 1) / allWarps;
    chunk = chunk < 8 ? 8 : (chunk > 32 ? 32 : chunk);
    const long long myEnd = (narrow && blockIdx.x != 0) ? 0 : total;
    for (long long base = myWarp * chunk; base < myEnd; base += allWarps * chunk) {
      const long long j = base + lane;
      const bool valid = static_cast<long long>(lane) < chunk && j < total;
      int k = 0;
      if (valid) {
        while (k + 1 < K && L.off[k + 1] <= j) ++k;
      }
      const int mode = valid ? L.mode[k] : kDone;
      const long long i = valid ? j - L.off[k] : 0;
      const long long ko = static_cast<long long>(k) * P.stride;

      if (mode == kSplit) {
        // far pile entry: to the near list below the new threshold
        const int v = __ldcg((L.fp[k] == 0 ? P.farL0 : P.farL1) + ko + i);
        const u64 word = __ldcg(P.packed + ko + v);
        const u64 d = word == kInfWord ? kInfWord : pkOf(P.obj[k]).dist(word);
        if (d < L.thr[k]) {
          P.inFar[ko + v] = 0;
          stageAppend(P, L, k, v, d, wrSlot, nearWV, nearWD);
        } else {
          stageAppend(P, L, K + k, v, d, wrSlot, nearWV, nearWD);
        }
      }

      // push: one non-stale near entry per lane, edges spread over the warp
      int u = -1, beg = 0, deg = 0;
      u64 du = 0;
      if (mode == kPush) {
        const long long kn = static_cast<long long>(k) * P.strideNear;
        // A stale entry (the word has dropped below its tag since) is
        // expanded with its tag: its offers are strictly larger than the
        // ones of the newer entry, so they never win a word. Skipping the
        // check saves a dependent load on every expansion.
        u = __ldcg(nearRV + kn + i);
        du = __ldcg(nearRD + kn + i);
        beg = ldGraph<Mode>(outRow + u);
        deg = ldGraph<Mode>(outRow + u + 1) - beg;
      }
      expandWarp<Mode>(P, L, outRow, outCol, outWk, k, u, du, beg, deg, wrSlot, nearWV, nearWD,
                       heavyOn);
    }
    if (heavyOn) expandHeavy<Mode>(P, L, outCol, outWk, wrSlot, nearWV, nearWD);
    // Local rounds: the CTA expands the near entries it has just staged
    // itself, up to P.localRounds times while its partitions are at most
    // half full, so a frontier advances several hops per grid barrier. An
    // entry expanded here is not flushed; the last round's appends are.
    // (Relaxations are monotone atomicMin, so expanding an entry earlier
    // than the next iteration would cannot change the fixed point.)
    const int rounds = narrow ? (blockIdx.x == 0 ? P.narrowRounds : 0) : P.localRounds;
    for (int r = 0; r < rounds; ++r) {
      __syncthreads();
      if (threadIdx.x == 0) {
        int tot = 0;
        bool room = true;
        for (int q = 0; q < K; ++q) {
          const int end = H.count[q] < H.cap ? H.count[q] : H.cap;
          H.roundEnd[q] = end;
          tot += end - H.start[q];
          room = room && H.count[q] <= H.cap / 2;
        }
        H.roundTotal = room ? tot : 0;
      }
      __syncthreads();
      const int tot = H.roundTotal;
      if (tot == 0) break;
      for (int b0 = warp * 32; b0 < tot; b0 += (blockDim.x >> 5) * 32) {
        const int j = b0 + static_cast<int>(lane);
        int kq = 0, uq = -1, begq = 0, degq = 0;
        u64 dq = 0;
        if (j < tot) {
          int rem = j;
          while (rem >= H.roundEnd[kq] - H.start[kq]) {
            rem -= H.roundEnd[kq] - H.start[kq];
            ++kq;
          }
          const StageEntry e = stageEntries()[kq * H.cap + H.start[kq] + rem];
          uq = e.v;
          dq = e.d;
          begq = ldGraph<Mode>(outRow + uq);
          degq = ldGraph<Mode>(outRow + uq + 1) - begq;
        }
        expandWarp<Mode>(P, L, outRow, outCol, outWk, kq, uq, dq, begq, degq, wrSlot, nearWV, nearWD,
                         heavyOn);
      }
      if (heavyOn) {
        expandHeavy<Mode>(P, L, outCol, outWk, wrSlot, nearWV, nearWD);
      } else {
        __syncthreads();
      }
      if (threadIdx.x < K) H.start[threadIdx.x] = H.roundEnd[threadIdx.x];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) tWorked = globalNs();
    __syncthreads();
    unsigned long long tAll = 0, tFlushed = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) tAll = globalNs();
    flushStage(P, L, wrSlot, nearWV, nearWD);
    if (blockIdx.x == 0 && threadIdx.x == 0) tFlushed = globalNs();
    if (!gridSync(c, epoch)) return false;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      bool split = false;
      for (int k = 0; k < K; ++k) split |= L.mode[k] == kSplit;
      const unsigned long long tEnd = globalNs();
      profNs[split ? 0 : 1] += tEnd - itStart;
      profIters[split ? 0 : 1] += 1;
      profItems[split ? 0 : 1] += total;
      if (!split) {
        part[0] += tDecided - itStart;
        part[1] += tWorked - tDecided;
        part[2] += tAll - tWorked;
        part[3] += tFlushed - tAll;
        part[4] += tEnd - tFlushed;
      }
    }
  }

  if (threadIdx.x < K && H.expanded[threadIdx.x] != 0) {
    atomicAdd(reinterpret_cast<unsigned long long *>(&c->pushes[threadIdx.x]),
              static_cast<unsigned long long>(H.expanded[threadIdx.x]));
  }
  if (blockIdx.x == 0 && warp == 0 && static_cast<int>(lane) < K) {
    c->iterations[lane] = iters;
    c->epochs[lane] = epochs;
    if (lane == 0) {
      c->finalGen = genBase + 1 + it;
      *P.genPtr = genBase + 1 + it;
      for (int q = 0; q < 2; ++q) {
        c->loopNs[q] = profNs[q];
        c->loopIters[q] = profIters[q];
        c->loopItems[q] = profItems[q];
      }
      for (int q = 0; q < 5; ++q) c->iterSplitNs[q] = part[q];
    }
  }
  return true;
}

// ---------------------------------------------------------------------------
// Asynchronous near-far loop
//
// The bulk loop above pays a grid barrier per iteration and, worse, waits in
// every iteration for the slowest warp of the grid. Here a phase runs one
// far-pile split and then expands the near entries asynchronously: every
// warp claims slots of the near queue, expands what has arrived and pushes
// what improves, with no barrier until the whole phase has run dry. Only the
// split of the far piles (a new threshold per objective) needs the grid to
// agree, so there is one grid barrier per phase (a few per launch) instead
// of one per iteration (80-150). Relaxations are the same monotone 64-bit
// atomicMin, so the fixed point, i.e. every word, is the one the bulk loop
// reaches.
// ---------------------------------------------------------------------------

/// Phase end detection (warp 0 of CTA 0 while it is idle): every CTA has
/// finished its split and, in two successive reads of all shards' counters,
/// done == tail everywhere with nothing changed in between (the counters
/// only grow, so the second read shows the state of one moment).
__device__ void detectPhaseEnd(const EngineParams &P, const AsyncShard *ctr, unsigned phase) {
  EngineControl *c = P.ctl;
  const unsigned lane = laneId();
  const int S = P.aqShards;
  unsigned split = 0;
  if (lane == 0) split = ldAcquire(&c->asyncSplit);
  split = __shfl_sync(kFull, split, 0);
  if (split < (phase + 1) * gridDim.x) return;
  unsigned d1 = 0, t1 = 0, d2 = 0, t2 = 0;
  if (static_cast<int>(lane) < S) {
    d1 = ldAcquire(&ctr[lane].done);
    t1 = ldAcquire(&ctr[lane].tail);
  }
  if (!__all_sync(kFull, d1 == t1)) return;
  if (static_cast<int>(lane) < S) {
    d2 = ldAcquire(&ctr[lane].done);
    t2 = ldAcquire(&ctr[lane].tail);
  }
  if (!__all_sync(kFull, d2 == d1 && t2 == t1)) return;
  if (lane == 0) stRelease(&c->asyncPhase, phase + 1);
}

/// Settle one warp round: `consumed` entries of shard `from` and the lanes'
/// reservations past the capacity of shard `to`, after the round's own
/// reservations (release).
__device__ __forceinline__ void settleRound(AsyncShard *ctr, int from, unsigned consumed, int to,
                                            unsigned spilled) {
  if (__any_sync(kFull, spilled != 0)) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) spilled += __shfl_xor_sync(kFull, spilled, off);
  }
  if (consumed == 0 && spilled == 0) return;  // the same in every lane
  // the warp barrier orders the lanes' reservations before lane 0's
  // release adds, which order them (cumulatively) before the new counts
  __syncwarp();
  if (laneId() == 0) {
    if (consumed != 0) redRelease(&ctr[from].done, consumed);
    if (spilled != 0) redRelease(&ctr[to].done, spilled);
  }
}

/// Decode a near entry: objective k, vertex u (-1 if the entry is stale:
/// a later, smaller distance has its own entry), the distance du to expand
/// with and u's row. A word read older than the entry is covered by
/// expanding with the entry's tag.
template <int Mode>
__device__ __forceinline__ void asyncEntry(const EngineParams &P, const int *outRow, u64 e, int &k,
                                           int &u, u64 &du, int &beg, int &deg) {
  const unsigned vk = static_cast<unsigned>(e);
  const unsigned tag = static_cast<unsigned>(e >> 32);
  k = static_cast<int>(vk & 31u);
  const int v = static_cast<int>(vk >> 5);
  const u64 word = __ldcg(P.packed + static_cast<long long>(k) * P.stride + v);
  const int b0 = ldGraph<Mode>(outRow + v);
  const int b1 = ldGraph<Mode>(outRow + v + 1);
  const u64 d = word == kInfWord ? kInfWord : pkOf(P.obj[k]).dist(word);
  u = -1;
  if (tag < kTagSat) {
    if (d >= tag) {
      u = v;
      du = tag;
    }
  } else if (d != kInfWord) {
    u = v;
    du = d;
  }
  if (u >= 0) {
    beg = b0;
    deg = b1 - b0;
  }
}

/// The consumer side of one phase for one warp: expand its own local
/// entries first, else claim slots and expand the entries that arrive,
/// until the phase is over (true) or the launch is stopped (false).
/// Per-warp counters of the asynchronous loop (lane 0): rounds and entries
/// taken from the queue and from the warp's local buffer.
struct AsyncCounts {
  long long queueRounds, localRounds, queueItems, localItems;
};

template <int Mode>
__device__ bool asyncConsume(const EngineParams &P, const LoopShared &L, const int *outRow,
                             const int *outCol, const int *const *outWk, AsyncShard *ctr,
                             unsigned phase, long long gwarp, const Sync &sync, AsyncCounts &cnt) {
  EngineControl *c = P.ctl;
  const unsigned lane = laneId();
  const int S = P.aqShards;
  const unsigned cap = P.aqShardCap;
  int cs = static_cast<int>(gwarp % S);  // shard this warp claims from
  int hops = 0;                          // shards found exhausted
  int target = static_cast<int>((gwarp * 7 + 3) % S);
  unsigned pend = 0, cb = 0, spins = 0, knownTail = 0;
  // entries of shard cs consumed but not yet settled: a warp settles them
  // only with its local buffer empty, so while it holds local work the
  // shard's done stays below its tail and the phase cannot end
  unsigned unsettled = 0;
  StageHeader &H = stageHeader();
  const int warp = threadIdx.x >> 5;
  u64 *localBuf = asyncLocalBuffer(warp);
  while (true) {
    __syncwarp();
    int nLocal = __shfl_sync(kFull, H.asyncLocal[warp], 0);
    if (nLocal > 0) {
      nLocal = nLocal < kLocalBuf ? nLocal : kLocalBuf;
      const u64 le = static_cast<int>(lane) < nLocal ? localBuf[lane] : kEmptySlot;
      __syncwarp();
      if (lane == 0) {
        H.asyncLocal[warp] = 0;
        ++cnt.localRounds;
        cnt.localItems += nLocal;
      }
      __syncwarp();
      int k = 0, u = -1, beg = 0, deg = 0;
      u64 du = 0;
      if (le != kEmptySlot) asyncEntry<Mode>(P, outRow, le, k, u, du, beg, deg);
      AsyncState A{ctr, target, 0u, (P.flags & kFlagLocal) != 0};
      expandWarp<Mode, true>(P, L, outRow, outCol, outWk, k, u, du, beg, deg, 0, nullptr, nullptr,
                             false, &A);
      settleRound(ctr, cs, 0u, target, A.spilled);
      target = target + 1 == S ? 0 : target + 1;
      continue;
    }
    if (unsettled != 0) {
      settleRound(ctr, cs, unsettled, 0, 0u);
      unsettled = 0;
    }
    if (pend == 0 && hops < S) {
      unsigned b = 0;
      if (lane == 0) b = atomicAdd(&ctr[cs].head, 32u);
      b = __shfl_sync(kFull, b, 0);
      if (b >= cap) {
        cs = (cs + 1) % S;
        ++hops;
        knownTail = 0;
        continue;
      }
      cb = b;
      const unsigned room = cap - b;
      pend = room >= 32u ? kFull : ((1u << room) - 1u);
    }
    u64 *slot = P.aqSlots + static_cast<long long>(cs) * cap + cb + lane;
    u64 e = kEmptySlot;
    // only slots below the shard's tail are reserved; the tail only grows,
    // so the last value read is reloaded only when a pending slot lies past
    // it (one load per warp, and none while the shard is ahead of the warp)
    const bool mine = (pend >> lane) & 1u;
    if (__any_sync(kFull, mine && cb + lane >= knownTail)) {
      unsigned t = 0;
      if (lane == 0) t = ldVolatileU(&ctr[cs].tail);
      knownTail = __shfl_sync(kFull, t, 0);
    }
    if (mine && cb + lane < knownTail) e = ldAcquire64(slot);
    const unsigned ready = __ballot_sync(kFull, e != kEmptySlot);
    if (ready == 0) {
      unsigned ph = 0;
      if (lane == 0) ph = ldAcquire(&c->asyncPhase);
      ph = __shfl_sync(kFull, ph, 0);
      if (ph > phase) return true;
      if (gwarp == 0) detectPhaseEnd(P, ctr, phase);
      if ((++spins & 63u) == 0) {
        int stop = 0;
        if (lane == 0) {
          stop = ldVolatile(&c->status) != 0;
          if (!stop && globalNs() > sync.deadline) {
            atomicCAS(&c->status, 0, MOSP_ERR_TIMEOUT);
            stop = 1;
          }
        }
        if (__shfl_sync(kFull, stop, 0)) return false;
      }
      __nanosleep(spins < 32 ? 32 : 256);
      continue;
    }
    spins = 0;
    pend &= ~ready;
    if (lane == 0) {
      ++cnt.queueRounds;
      cnt.queueItems += __popc(ready);
    }
    int k = 0, u = -1, beg = 0, deg = 0;
    u64 du = 0;
    if (e != kEmptySlot) {
      stRelaxed64(slot, kEmptySlot);
      asyncEntry<Mode>(P, outRow, e, k, u, du, beg, deg);
    }
    AsyncState A{ctr, target, 0u, (P.flags & kFlagLocal) != 0};
    expandWarp<Mode, true>(P, L, outRow, outCol, outWk, k, u, du, beg, deg, 0, nullptr, nullptr,
                           false, &A);
    unsettled += __popc(ready);
    settleRound(ctr, cs, 0u, target, A.spilled);
    target = target + 1 == S ? 0 : target + 1;
  }
}

template <int Mode>
__device__ bool asyncNearFar(const EngineParams &P, const int *outRow, const int *outCol,
                             const int *const *outWk, Sync &epoch, u64 *deltaOverride, int genBase) {
  __shared__ LoopShared L;
  StageHeader &H = stageHeader();
  EngineControl *c = P.ctl;
  const int K = P.K;
  const int S = P.aqShards;
  const unsigned lane = laneId();
  const int warp = threadIdx.x >> 5;
  const long long gwarp = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + warp;
  const long long nwarps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);

  // per-objective state, held by lane k of warp 0 (the same in every CTA)
  u64 thr = 0;
  int fp = 0, fs = 0, phasesK = 0;
  u64 delta = 1;
  if (warp == 0 && static_cast<int>(lane) < K) {
    delta = P.obj[lane].delta;
    if (deltaOverride != nullptr && lane == 0) delta = *deltaOverride;
  }
  if (threadIdx.x < kMaxK) H.expanded[threadIdx.x] = 0;
  if (threadIdx.x < kWarps) {
    H.asyncFar[threadIdx.x] = 0;
    H.asyncLocal[threadIdx.x] = 0;
  }
  const unsigned long long t0 = globalNs();
  unsigned long long tPhase = t0;
  AsyncCounts cnt{0, 0, 0, 0};
  unsigned phase = 0;
  for (;; ++phase) {
    if (threadIdx.x < kMaxK) H.farMin[threadIdx.x] = kInfWord;
    if (warp == 0) {
      const int k = static_cast<int>(lane);
      const bool act = k < K;
      int mode = kDone;
      long long items = 0;
      if (act) {
        const int fc = __ldcg(&c->farCount[k][fs]);
        if (fc > 0) {
          mode = kSplit;
          items = fc;
          const u64 mnC = __ldcg(&c->farMinC[k][fs]);
          u64 lo = thr;
          if (mnC != 0) {
            const u64 mn = ~mnC;
            lo = mn > thr ? mn : thr;
          }
          thr = (lo > kInfWord - delta) ? kInfWord - 1 : lo + delta;
        }
      }
      long long incl = items;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const long long o = __shfl_up_sync(kFull, incl, off);
        if (static_cast<int>(lane) >= off) incl += o;
      }
      if (act) {
        L.off[k] = incl - items;
        L.thr[k] = thr;
        L.mode[k] = mode;
        L.fp[k] = fp;
        L.fs[k] = fs;
      }
      const long long total = __shfl_sync(kFull, incl, 31);
      if (lane == 0) L.total = total;
      if (act && mode == kSplit) {
        if (blockIdx.x == 0) {
          c->farCount[k][(fs + 2) % 3] = 0;
          c->farMinC[k][(fs + 2) % 3] = 0;
        }
        ++phasesK;
        fp ^= 1;
        fs = (fs + 1) % 3;
      }
    }
    // the counter set of the next phase (last used two phases ago)
    if (blockIdx.x == 0 && static_cast<int>(threadIdx.x) < S) {
      AsyncShard &nx = P.aqCtr[((phase + 1) & 1u) * S + threadIdx.x];
      nx.head = 0;
      nx.tail = 0;
      nx.done = 0;
    }
    __syncthreads();
    const long long total = L.total;
    if (total == 0) break;
    AsyncShard *ctr = P.aqCtr + (phase & 1u) * S;

    // ---- split: this warp's share of the far piles, below the new
    // threshold to the near queue, the rest to the other pile
    {
      // (split pushes all go to the queue: a warp settles nothing in the
      // split, so it must not hold local work past it)
      AsyncState A{ctr, static_cast<int>(gwarp % S), 0u, false};
      for (long long base = gwarp * 32; base < total; base += nwarps * 32) {
        if (farBufferFull(32)) flushAsyncFar(P, L);
        const long long j = base + lane;
        if (j < total) {
          int k = 0;
          while (k + 1 < K && L.off[k + 1] <= j) ++k;
          const long long ko = static_cast<long long>(k) * P.stride;
          const int v = __ldcg((L.fp[k] == 0 ? P.farL0 : P.farL1) + ko + (j - L.off[k]));
          const u64 word = __ldcg(P.packed + ko + v);
          const u64 d = word == kInfWord ? kInfWord : pkOf(P.obj[k]).dist(word);
          if (d < L.thr[k]) {
            P.inFar[ko + v] = 0;
            asyncNear(P, L, A, k, v, d);
          } else {
            asyncFar(P, L, k, v, d);
          }
        }
        settleRound(ctr, 0, 0u, A.target, A.spilled);
        A.spilled = 0;
        A.target = A.target + 1 == S ? 0 : A.target + 1;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      redRelease(&c->asyncSplit, 1u);
    }

    // ---- expand until the phase runs dry
    if (!asyncConsume<Mode>(P, L, outRow, outCol, outWk, ctr, phase, gwarp, epoch, cnt)) return false;
    flushAsyncFar(P, L);
    __syncthreads();
    if (threadIdx.x < K && H.farMin[threadIdx.x] != kInfWord) {
      atomicMax(listTarget(P, L, K + threadIdx.x, 0, nullptr, nullptr).minC, ~H.farMin[threadIdx.x]);
    }
    if (!gridSync(c, epoch)) return false;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      // phase durations (the first four, then the rest summed)
      const unsigned long long now = globalNs();
      c->iterSplitNs[phase < 4 ? phase : 4] += now - tPhase;
      tPhase = now;
    }
  }
  if (lane == 0 && (cnt.queueRounds | cnt.localRounds) != 0) {
    atomicAdd(reinterpret_cast<unsigned long long *>(&c->loopIters[1]),
              static_cast<unsigned long long>(cnt.queueRounds + cnt.localRounds));
    atomicAdd(reinterpret_cast<unsigned long long *>(&c->loopItems[0]),
              static_cast<unsigned long long>(cnt.queueItems));
    atomicAdd(reinterpret_cast<unsigned long long *>(&c->loopItems[1]),
              static_cast<unsigned long long>(cnt.localItems));
    atomicAdd(reinterpret_cast<unsigned long long *>(&c->loopNs[1]),
              static_cast<unsigned long long>(cnt.localRounds));
  }

  if (threadIdx.x < K && H.expanded[threadIdx.x] != 0) {
    atomicAdd(reinterpret_cast<unsigned long long *>(&c->pushes[threadIdx.x]),
              static_cast<unsigned long long>(H.expanded[threadIdx.x]));
  }
  if (blockIdx.x == 0 && warp == 0 && static_cast<int>(lane) < K) {
    c->iterations[lane] = phasesK;
    c->epochs[lane] = phasesK;
    if (lane == 0) {
      c->finalGen = genBase + 1;
      *P.genPtr = genBase + 1;
      c->loopNs[0] = globalNs() - t0;
      c->loopIters[0] = phase;
    }
  }
  return true;
}

/// Lowest-id tight parent of every vertex of the distance-only objectives
/// (parent INT_MAX after the unpack, -1 for roots and unreached vertices);
/// thread tid of T.
template <int Mode>
__device__ void recoverTightParents(const EngineParams &P, const int *outRow, const int *outCol,
                                    const int *const *outWk, long long tid, long long T) {
  const int n = P.n, K = P.K;
  // Lowest-id tight parent of every vertex of a distance-only objective:
  // every edge (u, x) with d(u) + w = d(x) offers u to x by atomicMin, so
  // the result does not depend on which thread checks which edge.
  // Edge-balanced: warp w takes the w-th equal slice of the edge array and
  // its lanes read two windows of 32 consecutive edges at a time
  // (coalesced), so hub rows and hub-dense id ranges of power-law graphs
  // cost no more than any other slice. The warp finds the source rows of
  // its edges from the ends of the next 32 rows (one coalesced load) by a
  // 5-step shuffle search, moving on 32 rows at a time through runs of
  // empty rows. The row search and the head loads are shared by all
  // distance-only objectives, whose loads then go out together.
  const unsigned lane = laneId();
  const long long gwarp = tid >> 5;
  const long long nwarps = T >> 5;
  const long long m = ldGraph<Mode>(outRow + n);
  const long long wb = m * gwarp / nwarps, we = m * (gwarp + 1) / nwarps;
  if (wb >= we) return;  // warp-uniform
  // the row of the slice's first edge: the last r with rowPtr[r] <= wb
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = lo + ((hi - lo) >> 1);
    if (ldGraph<Mode>(outRow + mid) <= wb) lo = mid; else hi = mid;
  }
  int r0 = lo;  // no edge of the rest of the slice lies in a row before r0
  for (long long e0 = wb; e0 < we; e0 += 64) {
    const int ea = static_cast<int>(e0 + lane);
    const int eb = static_cast<int>(e0 + 32 + lane);
    const bool la = e0 + lane < we, lb = e0 + 32 + lane < we;
    const int xa = la ? ldGraph<Mode>(outCol + ea) : 0;
    const int xb = lb ? ldGraph<Mode>(outCol + eb) : 0;
    int rowA = la ? -1 : 0, rowB = lb ? -1 : 0;
    // at most ceil((n - r0) / 32) windows: the window holding row n - 1
    // ends every search, since rows past n count as ending at INT_MAX
    for (int base = r0; base < n; base += 32) {
      const int rr = base + static_cast<int>(lane);
      const int end = rr < n ? ldGraph<Mode>(outRow + rr + 1) : INT_MAX;
      // pos = how many of the window's rows end at or before the edge
      int posA = 0, posB = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const int probeA = __shfl_sync(kFull, end, posA + step - 1);
        const int probeB = __shfl_sync(kFull, end, posB + step - 1);
        if (probeA <= ea) posA += step;
        if (probeB <= eb) posB += step;
      }
      const int lastEnd = __shfl_sync(kFull, end, 31);
      if (rowA < 0 && ea < lastEnd) rowA = base + posA;
      if (rowB < 0 && eb < lastEnd) rowB = base + posB;
      if (__all_sync(kFull, rowA >= 0 && rowB >= 0)) break;
    }
    // lane 31 of the second window holds the largest row; when it is past
    // the slice the loop ends here anyway
    r0 = __shfl_sync(kFull, rowB, 31);
    const bool ca = la && rowA >= 0 && !isRoot(P.source, P.sources, P.nSources, xa);
    const bool cb = lb && rowB >= 0 && !isRoot(P.source, P.sources, P.nSources, xb);
    for (int k = 0; k < K; ++k) {
      const ObjectiveArgs &O = P.obj[k];
      if (O.parentBits > 0) continue;  // the same for every thread
      const long long ko = static_cast<long long>(k) * P.stride;
      const int *w = outWk[k];
      u64 da = kInfWord, db = kInfWord, pa = 0, pb = 0;
      int wa = 0, wbt = 0;
      if (ca) {
        da = __ldcg(P.packed + ko + rowA);
        pa = __ldcg(P.packed + ko + xa);
        wa = ldGraph<Mode>(w + ea);
      }
      if (cb) {
        db = __ldcg(P.packed + ko + rowB);
        pb = __ldcg(P.packed + ko + xb);
        wbt = ldGraph<Mode>(w + eb);
      }
      if (da != kInfWord && da + static_cast<u64>(wa) == pa) atomicMin(O.parent + xa, rowA);
      if (db != kInfWord && db + static_cast<u64>(wbt) == pb) atomicMin(O.parent + xb, rowB);
    }
  }
}

// ---------------------------------------------------------------------------
// Unpack words into (distance, parent); distance-only objectives recover
// the lowest-id tight parent (reference src/sospUpdateGpu.cu:478-512).
// ---------------------------------------------------------------------------
template <int Mode>
__device__ bool unpackResults(const EngineParams &P, const int *outRow,
                              const int *outCol, const int *const *outWk,
                              Sync &epoch) {
  const int n = P.n, K = P.K;
  const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long T = static_cast<long long>(gridDim.x) * blockDim.x;
  const bool restricted = Mode == kModeUpdate && P.recMark != nullptr && P.recChangedList != nullptr &&
                          (P.flags & (kFlagCanonical | kFlagHostRecovery)) ==
                              (kFlagCanonical | kFlagHostRecovery);
  bool anyFallback = false;
  for (int k = 0; k < K; ++k) {
    const ObjectiveArgs &O = P.obj[k];
    const Pk pk = pkOf(O);
    const long long ko = static_cast<long long>(k) * P.stride;
    if (O.parentBits > 0) {
      // four words per thread (v, v + T, v + 2T, v + 3T), loaded together
      for (long long v0 = tid; v0 < n; v0 += 4 * T) {
        u64 word[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const long long v = v0 + q * T;
          word[q] = v < n ? __ldcg(P.packed + ko + v) : kInfWord;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const long long v = v0 + q * T;
          if (v >= n) break;
          if (word[q] == kInfWord) {
            O.dist[v] = kDistInf;
            O.parent[v] = -1;
          } else {
            O.dist[v] = static_cast<long long>(pk.dist(word[q]));
            O.parent[v] = pk.parent(word[q]);
          }
        }
      }
    } else if (restricted) {
      // restricted recovery (recover.cu): the input parents stay; the mark
      // byte says whether the distance changed, and the changed vertices
      // are listed (one reservation per warp)
      anyFallback = true;
      unsigned char *mark = P.recMark + ko;
      int *changed = P.recChangedList + ko;
      const int lane = static_cast<int>(laneId());
      for (long long v0 = tid - lane; v0 < n; v0 += T) {  // the same v0 in the whole warp
        const long long v = v0 + lane;
        bool chg = false;
        if (v < n) {
          const u64 word = __ldcg(P.packed + ko + v);
          const long long d = word == kInfWord ? kDistInf : static_cast<long long>(word);
          chg = O.dist[v] != d;
          mark[v] = chg ? kRecChanged : 0;
          O.dist[v] = d;
          if (word == kInfWord || isRoot(P.source, P.sources, P.nSources, static_cast<int>(v))) {
            O.parent[v] = -1;
          }
        }
        const unsigned bal = __ballot_sync(kFull, chg);
        if (bal != 0) {
          int at = 0;
          if (lane == __ffs(bal) - 1) at = atomicAdd(&P.ctl->recChanged[k], __popc(bal));
          at = __shfl_sync(kFull, at, __ffs(bal) - 1);
          if (chg) changed[at + __popc(bal & ((1u << lane) - 1))] = static_cast<int>(v);
        }
      }
    } else {
      anyFallback = true;
      for (long long v = tid; v < n; v += T) {
        const u64 word = __ldcg(P.packed + ko + v);
        O.dist[v] = word == kInfWord ? kDistInf : static_cast<long long>(word);
        O.parent[v] = (word == kInfWord || isRoot(P.source, P.sources, P.nSources, static_cast<int>(v)))
                          ? -1
                          : INT_MAX;
      }
    }
  }
  if (!anyFallback || (P.flags & kFlagHostRecovery) != 0) return true;
  if (!gridSync(P.ctl, epoch)) return false;
  recoverTightParents<Mode>(P, outRow, outCol, outWk, tid, T);
  return true;
}

// ---------------------------------------------------------------------------
// Block-level scan helpers (combined-graph and reverse-CSR builds)
// ---------------------------------------------------------------------------

/// Inclusive scan of one value per thread over the CTA; *total = CTA sum.
__device__ long long blockInclusiveScan(long long x, long long *total) {
  __shared__ long long warpSums[kThreads / 32];
  const unsigned lane = laneId();
  const int warp = threadIdx.x >> 5;
  long long v = x;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const long long o = __shfl_up_sync(kFull, v, off);
    if (static_cast<int>(lane) >= off) v += o;
  }
  if (lane == 31) warpSums[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    long long s = static_cast<int>(lane) < nw ? warpSums[lane] : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const long long o = __shfl_up_sync(kFull, s, off);
      if (static_cast<int>(lane) >= off) s += o;
    }
    if (static_cast<int>(lane) < nw) warpSums[lane] = s;
  }
  __syncthreads();
  const long long prefix = warp > 0 ? warpSums[warp - 1] : 0;
  *total = warpSums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return prefix + v;
}

/// Sum of one value per thread over the CTA (every thread gets it).
__device__ long long blockSum(long long x) {
  long long total;
  blockInclusiveScan(x, &total);
  return total;
}

/// Exclusive scan in[0, len) -> out[0, len) (and copy -> cursor) across the
/// grid; two phases separated by one grid barrier. Returns the total.
__device__ bool gridExclusiveScan(const int *in, int *out, int *cursor, long long len,
                                  long long *blockSums, EngineControl *c,
                                  Sync &epoch, long long *grandTotal) {
  const long long chunk = (len + gridDim.x - 1) / gridDim.x;
  const long long lo = static_cast<long long>(blockIdx.x) * chunk;
  const long long hi = lo + chunk < len ? lo + chunk : len;
  long long local = 0;
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) local += __ldcg(in + i);
  const long long sum = blockSum(local);
  if (threadIdx.x == 0) blockSums[blockIdx.x] = sum;
  if (!gridSync(c, epoch)) return false;
  long long before = 0, all = 0;
  for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x) {
    const long long s = __ldcg(blockSums + b);
    all += s;
    if (b < static_cast<int>(blockIdx.x)) before += s;
  }
  before = blockSum(before);
  all = blockSum(all);
  long long carry = before;
  for (long long t = lo; t < hi; t += blockDim.x) {
    const long long i = t + threadIdx.x;
    const long long x = i < hi ? __ldcg(in + i) : 0;
    long long tileTotal;
    const long long incl = blockInclusiveScan(x, &tileTotal);
    if (i < hi) {
      out[i] = static_cast<int>(carry + incl - x);
      if (cursor != nullptr) cursor[i] = static_cast<int>(carry + incl - x);
    }
    carry += tileTotal;
  }
  *grandTotal = all;
  return true;
}

// ---------------------------------------------------------------------------
// Combined graph edge of parent k of v (reference
// src/combinedGraphGpu.cu:55-75): edge (p, v) is attributed to the first
// tree whose parent of v is p; its weight is base - sum of the preference
// terms of every tree with that parent.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool combinedEdge(const EngineParams &P, int v, int k,
                                             int &p, int &weight) {
  const long long n = P.n;
  p = __ldg(P.combParents + k * n + v);
  if (p < 0) return false;
  for (int j = 0; j < k; ++j) {
    if (__ldg(P.combParents + j * n + v) == p) return false;
  }
  weight = P.combBase - P.prefTerms[k];
  for (int j = k + 1; j < P.combK; ++j) {
    if (__ldg(P.combParents + j * n + v) == p) weight -= P.prefTerms[j];
  }
  return true;
}

template <int Mode>
__device__ void scratchOrCombined(const EngineParams &P, Sync &epoch, int genBase,
                                  const int **sOutWk);

/// The near-far loop of a launch: asynchronous when the launch asks for it
/// and the graph has no hub rows (which the bulk loop hands to whole CTAs);
/// the same decision in every CTA (the hub flag is set before a barrier).
template <int Mode>
__device__ bool runNearFar(const EngineParams &P, const int *outRow, const int *outCol,
                           const int *const *outWk, Sync &epoch, u64 *deltaOverride, int genBase) {
  const bool async = (P.flags & kFlagAsync) != 0 && P.aqSlots != nullptr && P.aqShards > 0 &&
                     P.aqShards <= kAsyncShards && P.n <= (1 << 27) &&
                     P.stageEntries * sizeof(StageEntry) >=
                         kWarps * (kFarBuf * sizeof(int) + kLocalBuf * sizeof(u64)) &&
                     __ldcg(&P.ctl->heavy) == 0;
  if (async) return asyncNearFar<Mode>(P, outRow, outCol, outWk, epoch, deltaOverride, genBase);
  return nearFarLoop<Mode>(P, outRow, outCol, outWk, epoch, deltaOverride, genBase);
}

// ---------------------------------------------------------------------------
// The engine kernel
// ---------------------------------------------------------------------------
/// Pull pass: the best word that the in-edges e = first, first + step, ...
/// (< end) offer to their head (objective with args O at offset ko), folded
/// into `best`. Four edges per round with their loads in flight together
/// (the column and weight loads, then the four tail words), so a long
/// in-row is not one chain of dependent loads per edge.
__device__ __forceinline__ u64 pullBest(const EngineParams &P, const ObjectiveArgs &O,
                                        const Pk &pk, long long ko, int first, int end,
                                        int step, u64 best) {
  for (long long e0 = first; e0 < end; e0 += 4LL * step) {
    int u[4], w[4];
    u64 wd[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long e = e0 + static_cast<long long>(q) * step;
      u[q] = e < end ? __ldg(P.inCol + e) : -1;
      w[q] = e < end ? __ldg(O.inW + e) : 0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) wd[q] = u[q] >= 0 ? __ldcg(P.packed + ko + u[q]) : kInfWord;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (wd[q] == kInfWord) continue;
      const u64 nd = pk.dist(wd[q]) + static_cast<u64>(w[q]);
      if (nd <= O.maxDist) {
        const u64 cw = pk.pack(nd, u[q]);
        best = cw < best ? cw : best;
      }
    }
  }
  return best;
}

/// The push direction of the pass before the near-far loop, for objective
/// k: every valid (finite, not invalidated) vertex offers its distance plus
/// the edge weight along each out-edge; strict improvements go to far pile
/// 0 once (in-far flag). Warp gwarp of nwarps; a lane per short row, the
/// whole warp per row of more than kLaneRowMax edges.
__device__ void pushFromValid(const EngineParams &P, int k, const int *w, long long gwarp,
                              long long nwarps) {
  EngineControl *c = P.ctl;
  const ObjectiveArgs &O = P.obj[k];
  const Pk pk = pkOf(O);
  const long long ko = static_cast<long long>(k) * P.stride;
  const unsigned lane = laneId();
  auto relax = [&](int u, u64 du, int e) {
    const int x = __ldg(P.outCol + e);
    const u64 nd = du + static_cast<u64>(__ldg(w + e));
    if (x == P.source || nd > O.maxDist) return;
    const u64 old = atomicMin(P.packed + ko + x, pk.pack(nd, u));
    if (nd >= pk.dist(old)) return;
    if (atomicExch(P.inFar + ko + x, 1) == 0) {
      const int idx = warpAppend(&c->farCount[k][0]);
      P.farL0[ko + idx] = x;
      warpMinInto(&c->farMinC[k][0], nd);
    }
  };
  for (long long base = gwarp * 32; base < P.n; base += nwarps * 32) {
    const long long v = base + lane;
    u64 word = kInfWord;
    int beg = 0, end = 0;
    if (v < P.n) {
      word = __ldcg(P.packed + ko + v);
      if (word != kInfWord) {
        beg = __ldg(P.outRow + v);
        end = __ldg(P.outRow + v + 1);
      }
    }
    const u64 dv = word == kInfWord ? 0 : pk.dist(word);
    const int deg = end - beg;
    if (deg <= kLaneRowMax) {
      for (int e = beg; e < end; ++e) relax(static_cast<int>(v), dv, e);
    }
    unsigned big = __ballot_sync(kFull, deg > kLaneRowMax);
    while (big != 0) {
      const int src = __ffs(big) - 1;
      big &= big - 1;
      const int ub = static_cast<int>(__shfl_sync(kFull, v, src));
      const u64 db = __shfl_sync(kFull, dv, src);
      const int bb = __shfl_sync(kFull, beg, src);
      const int eb = __shfl_sync(kFull, end, src);
      for (int e = bb + static_cast<int>(lane); e < eb; e += 32) relax(ub, db, e);
    }
  }
}

template <int Mode>
__global__ void __launch_bounds__(kThreads, 1) sospEngine(const __grid_constant__ EngineParams P) {
  EngineControl *c = P.ctl;
  const int n = P.n, K = P.K;
  const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long T = static_cast<long long>(gridDim.x) * blockDim.x;
  const unsigned lane = laneId();
  const int warp = threadIdx.x >> 5;
  Sync epoch = startSync(P.timeoutNs);
  // Stamp generations of this launch start after the previous launch's.
  const int genBase = __ldcg(P.genPtr) + 1;

  __shared__ const int *sOutWk[kMaxK];
  if (threadIdx.x < kMaxK) {
    sOutWk[threadIdx.x] =
        static_cast<int>(threadIdx.x) < K ? P.obj[threadIdx.x].outW : nullptr;
  }
  const int *outRow = P.outRow;
  const int *outCol = P.outCol;

  markPhase(c, kPhaseStart);
  // both counter sets of the asynchronous near queue start at zero (every
  // mode passes a grid barrier before its near-far loop)
  if ((P.flags & kFlagAsync) != 0 && P.aqCtr != nullptr) {
    for (long long i = tid; i < 2LL * P.aqShards; i += T) {
      P.aqCtr[i].head = 0;
      P.aqCtr[i].tail = 0;
      P.aqCtr[i].done = 0;
    }
  }
  if constexpr (Mode == kModeUpdate) {
    // ---- Heavy rows: does the graph have rows for whole-CTA handling? -----
    const int heavyDeg = heavyDegOf(P);
    bool heavyRow = false;  // one store at the end, so the loads run ahead
    for (long long v = tid; v < n; v += T) {
      heavyRow |= __ldg(outRow + v + 1) - __ldg(outRow + v) > heavyDeg ||
                  __ldg(P.inRow + v + 1) - __ldg(P.inRow + v) > heavyDeg;
    }
    if (heavyRow) c->heavy = 1;
    // ---- Pack the old trees; ancestors (reference :234-252) ---------------
    // four vertices per thread (v, v + T, v + 2T, v + 3T): their loads are
    // issued before any of their stores
    bool badParent = false, badDist = false;
    for (int k = 0; k < K; ++k) {
      const ObjectiveArgs &O = P.obj[k];
      const Pk pk = pkOf(O);
      const long long ko = static_cast<long long>(k) * P.stride;
      for (long long v0 = tid; v0 < n; v0 += 4 * T) {
        long long d[4];
        int p[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const long long v = v0 + q * T;
          d[q] = v < n ? O.dist[v] : kDistInf;
          p[q] = v < n ? O.parent[v] : -1;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const long long v = v0 + q * T;
          if (v >= n) break;
          if (p[q] < -1 || p[q] >= n) {
            badParent = true;
            p[q] = -1;
          }
          u64 word;
          if (d[q] >= kDistInf / 2) {
            word = kInfWord;
          } else if (d[q] < 0 || static_cast<u64>(d[q]) > O.maxDist) {
            badDist = true;
            word = kInfWord;
          } else {
            word = pk.pack(static_cast<u64>(d[q]), p[q]);
          }
          P.packed[ko + v] = word;
          P.val[ko + v] = p[q];  // >= 0: ancestor; -1: none; -2: invalidated
        }
      }
    }
    if (badParent) c->invalid = 1;
    if (badDist) c->overflow = 1;
    if (!gridSync(c, epoch)) return;
    markPhase(c, kPhasePacked);

    // ---- Roots: heads of changed tree edges -------------------------------
    long long changes = 0;
    for (int k = 0; k < K; ++k) {
      const ObjectiveArgs &O = P.obj[k];
      const long long ko = static_cast<long long>(k) * P.stride;
      changes += O.nChanged;
      for (long long i = tid; i < O.nChanged; i += T) {
        const int v = O.chTo[i], u = O.chFrom[i];
        if (v < 0 || v >= n || u < 0 || u >= n) {
          c->invalid = 1;
          continue;
        }
        if (O.parent[v] == u) P.val[ko + v] = -2;
      }
    }
    if (!gridSync(c, epoch)) return;
    markPhase(c, kPhaseRoots);

    // ---- Subtree invalidation by pointer jumping (reference :254-291) -----
    // val[v] >= 0: no root on the tree path from v up to (excluding)
    // val[v]; -1: no root above v at all; -2: a root is v or an ancestor.
    // Every value another thread can observe keeps this invariant, so the
    // updates are made in place.
    if (changes > 0) {
      for (int round = 0; round < P.maxRounds; ++round) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
          c->jumpActive[(round + 1) % 3] = 0;
          c->rounds = round + 1;
        }
        int jumping = 0;
        for (int k = 0; k < K; ++k) {
          if (P.obj[k].nChanged == 0) continue;
          int *val = P.val + static_cast<long long>(k) * P.stride;
          // up to four jumps per round, each along the pointers the other
          // vertices have already lengthened, so a round covers more than
          // twice the distance and fewer rounds (and full scans) are needed
          // four vertices per thread (v, v + T, v + 2T, v + 3T) with their
          // chains of dependent loads in flight together
          for (long long v0 = tid; v0 < n; v0 += 4 * T) {
            int a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const long long v = v0 + q * T;
              a[q] = v < n ? __ldcg(val + v) : -1;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = a[q] >= 0 ? __ldcg(val + a[q]) : -1;
#pragma unroll
            for (int hop = 1; hop < 4; ++hop) {
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                if (a[q] >= 0 && b[q] >= 0) {
                  a[q] = b[q];
                  b[q] = __ldcg(val + a[q]);
                }
              }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              if (a[q] < 0) continue;  // no ancestor pointer (or past n)
              val[v0 + q * T] = b[q];
              jumping |= b[q] >= 0;
            }
          }
        }
        if (__syncthreads_or(jumping) && threadIdx.x == 0) {
          atomicOr(&c->jumpActive[round % 3], 1);
        }
        if (!gridSync(c, epoch)) return;
        if (__ldcg(&c->jumpActive[round % 3]) == 0) break;
        if (round + 1 == P.maxRounds && blockIdx.x == 0 && threadIdx.x == 0) {
          c->invalid = 1;  // the parent arrays are not a forest
        }
      }
    }

    markPhase(c, kPhaseJumped);
    // ---- Invalidate; candidates = invalidated + insert heads (:293-313) ---
    // Each CTA compacts its contiguous vertex range with block scans and
    // reserves its part of the candidate list with one atomic per objective.
    {
      __shared__ int sBase;
      const long long chunk = (static_cast<long long>(n) + gridDim.x - 1) / gridDim.x;
      const long long lo = static_cast<long long>(blockIdx.x) * chunk < n
                               ? static_cast<long long>(blockIdx.x) * chunk : n;
      const long long hi = lo + chunk < n ? lo + chunk : n;
      for (int k = 0; k < K; ++k) {
        const long long ko = static_cast<long long>(k) * P.stride;
        long long cnt = 0;
        for (long long v = lo + threadIdx.x; v < hi; v += blockDim.x) {
          cnt += __ldcg(P.val + ko + v) == -2 ? 1 : 0;
        }
        const long long found = blockSum(cnt);
        if (threadIdx.x == 0) {
          sBase = found > 0 ? atomicAdd(&c->candCount[k], static_cast<int>(found)) : 0;
          if (found > 0) atomicAdd(&c->invalidated[k], static_cast<int>(found));
        }
        __syncthreads();
        long long carry = sBase;
        for (long long t0 = lo; t0 < hi; t0 += blockDim.x) {
          const long long v = t0 + threadIdx.x;
          const bool inv = v < hi && __ldcg(P.val + ko + v) == -2;
          long long tileTotal;
          const long long incl = blockInclusiveScan(inv ? 1 : 0, &tileTotal);
          if (inv) {
            P.packed[ko + v] = kInfWord;
            P.cand[ko + carry + incl - 1] = static_cast<int>(v);
          }
          carry += tileTotal;
        }
      }
    }
    for (int k = 0; k < K; ++k) {
      const long long ko = static_cast<long long>(k) * P.stride;
      for (long long i = tid; i < P.nHeads; i += T) {
        const int v = P.heads[i];
        if (v < 0 || v >= n) {
          c->invalid = 1;
          continue;
        }
        if (isRoot(P.source, P.sources, P.nSources, v) || __ldcg(P.val + ko + v) == -2) continue;
        if (atomicExch(P.stamp + ko + v, genBase) != genBase) {
          const int idx = warpAppend(&c->candCount[k]);
          P.cand[ko + idx] = v;
        }
      }
    }
    if (!gridSync(c, epoch)) return;
    markPhase(c, kPhaseCandidates);

    // ---- Pull pass over in-edges (reference :315-344) ----------------------
    // The improved candidates form far pile 0; the first iteration of the
    // loop sets the threshold to their minimum + delta and splits them.
    //
    // Direction per objective: when more than half of the vertices were
    // invalidated, the few valid vertices push along all their out-edges
    // instead (pushFromValid below). That makes the same offers to the
    // invalidated vertices (their valid in-neighbours) and to the insert
    // heads (every inserted edge leaves a valid or an invalidated vertex, and
    // the latter is re-expanded in the loop anyway), for the out-edges of the
    // valid part instead of the in-edges of the invalidated part.
    __shared__ int sPush[kMaxK];
    if (threadIdx.x < kMaxK) {
      sPush[threadIdx.x] = static_cast<int>(threadIdx.x) < K && (P.flags & kFlagPullOnly) == 0 &&
                           2LL * __ldcg(&c->invalidated[threadIdx.x]) > n;
    }
    __syncthreads();
    {
      __shared__ long long sOff[kMaxK + 1];
      if (warp == 0) {
        const long long cnt =
            static_cast<int>(lane) < K && !sPush[lane] ? __ldcg(&c->candCount[lane]) : 0;
        long long incl = cnt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const long long o = __shfl_up_sync(kFull, incl, off);
          if (static_cast<int>(lane) >= off) incl += o;
        }
        sOff[lane] = incl - cnt;
        if (lane == 31) sOff[kMaxK] = incl;
      }
      StageHeader &H = stageHeader();
      StageEntry *E = stageEntries();
      if (threadIdx.x < kMaxK) {
        H.count[threadIdx.x] = 0;
        H.farMin[threadIdx.x] = kInfWord;
      }
      if (threadIdx.x == 0) {
        H.cap = P.stageEntries / K;
        H.heavyCount = 0;
      }
      __syncthreads();
      const long long total = sOff[kMaxK];
      // set in the first phase, the same for every thread of the grid
      const bool heavyOn = __ldcg(&c->heavy) != 0;
      // Improved candidates go to far pile 0. With a partition of at least
      // one tile per objective (K * blockDim <= stage entries) the appends are
      // staged per CTA and written out with one reservation per objective
      // when a partition could fill up and at the end; otherwise each warp
      // appends to the global pile directly.
      const bool staged = K * static_cast<int>(blockDim.x) <= P.stageEntries;
      auto flushPull = [&]() {
        __syncthreads();
        if (threadIdx.x < K && H.count[threadIdx.x] > 0) {
          H.base[threadIdx.x] = atomicAdd(&c->farCount[threadIdx.x][0], H.count[threadIdx.x]);
          atomicMax(&c->farMinC[threadIdx.x][0], ~H.farMin[threadIdx.x]);
        }
        __syncthreads();
        for (int k = 0; k < K; ++k) {
          const int cnt = H.count[k];
          const long long ko = static_cast<long long>(k) * P.stride;
          for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
            P.farL0[ko + H.base[k] + q] = E[k * H.cap + q].v;
          }
        }
        __syncthreads();
        if (threadIdx.x < kMaxK) {
          H.count[threadIdx.x] = 0;
          H.farMin[threadIdx.x] = kInfWord;
        }
        __syncthreads();
      };
      const long long tileStride = static_cast<long long>(gridDim.x) * blockDim.x;
      for (long long tile = static_cast<long long>(blockIdx.x) * blockDim.x; tile < total;
           tile += tileStride) {
        const long long j = tile + threadIdx.x;
        const bool valid = j < total;
        int k = 0;
        if (valid) {
          while (k + 1 < K && sOff[k + 1] <= j) ++k;
        }
        const long long ko = static_cast<long long>(k) * P.stride;
        const ObjectiveArgs &O = P.obj[k];
        const Pk pk = pkOf(O);
        int v = -1, beg = 0, end = 0;
        u64 cur = kInfWord;
        if (valid) {
          v = __ldcg(P.cand + ko + (j - sOff[k]));
          cur = __ldcg(P.packed + ko + v);
          beg = __ldg(P.inRow + v);
          end = __ldg(P.inRow + v + 1);
        }
        // heavy in-rows are reduced by the whole CTA after the tile
        if (heavyOn && end - beg > heavyDegOf(P)) {
          const int slot = atomicAdd(&H.heavyCount, 1);
          if (slot < kHeavyCap) {
            H.heavyK[slot] = k;
            H.heavyU[slot] = v;
            H.heavyBeg[slot] = beg;
            H.heavyDeg[slot] = end - beg;
            H.heavyD[slot] = cur;
            end = beg;
          }
        }
        u64 best = cur;
        const int deg = end - beg;
        unsigned big = __ballot_sync(kFull, deg > kLaneRowMax);
        if (deg <= kLaneRowMax) best = pullBest(P, O, pk, ko, beg, end, 1, best);
        while (big != 0) {
          const int src = __ffs(big) - 1;
          big &= big - 1;
          const int kb = __shfl_sync(kFull, k, src);
          const int bb = __shfl_sync(kFull, beg, src);
          const int eb = __shfl_sync(kFull, end, src);
          const ObjectiveArgs &Ob = P.obj[kb];
          const Pk pb = pkOf(Ob);
          const long long kob = static_cast<long long>(kb) * P.stride;
          u64 part = pullBest(P, Ob, pb, kob, bb + static_cast<int>(lane), eb, 32, kInfWord);
          part = warpMinU64(part);
          if (static_cast<int>(lane) == src) best = part < best ? part : best;
        }
        if (valid && best < cur) {
          // only this thread writes the word of v during the pull pass
          P.packed[ko + v] = best;
          if (pk.dist(best) < (cur == kInfWord ? kInfWord : pk.dist(cur))) {
            P.inFar[ko + v] = 1;
            if (!staged) {
              const int idx = warpAppend(&c->farCount[k][0]);
              P.farL0[ko + idx] = v;
              warpMinInto(&c->farMinC[k][0], pk.dist(best));
            } else {
              const unsigned peers = __match_any_sync(__activemask(), k);
              const int leader = __ffs(peers) - 1;
              int rb = 0;
              if (static_cast<int>(lane) == leader) rb = atomicAdd(&H.count[k], __popc(peers));
              rb = __shfl_sync(peers, rb, leader);
              E[k * H.cap + rb + __popc(peers & ((1u << lane) - 1u))].v = v;
              const u64 d = pk.dist(best);
              const unsigned hi = static_cast<unsigned>(d >> 32), lo = static_cast<unsigned>(d);
              const unsigned mhi = __reduce_min_sync(peers, hi);
              const unsigned mlo = __reduce_min_sync(peers, hi == mhi ? lo : 0xffffffffu);
              if (static_cast<int>(lane) == leader) {
                atomicMin(&H.farMin[k], (static_cast<u64>(mhi) << 32) | mlo);
              }
            }
          }
        }
        if (heavyOn) {
          // the tile's heavy in-rows: every thread of the CTA takes a share
          // of each row, the partial minima meet in shared memory, and one
          // thread per row writes the word and appends an improved vertex
          // to the global far pile (as the unstaged path does)
          __syncthreads();
          const int queued = H.heavyCount;
          if (queued > 0) {  // the same for every thread of the CTA
            const int count = queued < kHeavyCap ? queued : kHeavyCap;
            if (static_cast<int>(threadIdx.x) < count) H.heavyBest[threadIdx.x] = kInfWord;
            __syncthreads();
            if (threadIdx.x == 0) H.heavyCount = 0;
            for (int h = 0; h < count; ++h) {
              const int kh = H.heavyK[h], eh = H.heavyBeg[h] + H.heavyDeg[h];
              const ObjectiveArgs &Oh = P.obj[kh];
              const Pk ph = pkOf(Oh);
              const long long koh = static_cast<long long>(kh) * P.stride;
              u64 part = pullBest(P, Oh, ph, koh, H.heavyBeg[h] + static_cast<int>(threadIdx.x), eh,
                                  static_cast<int>(blockDim.x), kInfWord);
              part = warpMinU64(part);
              if (lane == 0 && part != kInfWord) atomicMin(&H.heavyBest[h], part);
            }
            __syncthreads();
            if (static_cast<int>(threadIdx.x) < count) {
              const int h = threadIdx.x;
              const int kh = H.heavyK[h], vh = H.heavyU[h];
              const Pk ph = pkOf(P.obj[kh]);
              const long long koh = static_cast<long long>(kh) * P.stride;
              const u64 curh = H.heavyD[h], besth = H.heavyBest[h];
              if (besth < curh) {
                // only this thread writes the word of vh during the pull pass
                P.packed[koh + vh] = besth;
                if (ph.dist(besth) < (curh == kInfWord ? kInfWord : ph.dist(curh))) {
                  P.inFar[koh + vh] = 1;
                  const int idx = atomicAdd(&c->farCount[kh][0], 1);
                  P.farL0[koh + idx] = vh;
                  atomicMax(&c->farMinC[kh][0], ~ph.dist(besth));
                }
              }
            }
          }
          // every thread has read the queue (and the rows are done) before
          // the next tile queues rows again
          __syncthreads();
        }
        if (!staged) continue;
        // a tile appends at most blockDim entries: flush before a partition
        // could overflow
        __syncthreads();
        if (__syncthreads_or(threadIdx.x < static_cast<unsigned>(K) &&
                             H.count[threadIdx.x] > H.cap - static_cast<int>(blockDim.x))) {
          flushPull();
        }
      }
      if (staged) flushPull();
    }
    for (int k = 0; k < K; ++k) {
      if (sPush[k]) pushFromValid(P, k, sOutWk[k], tid >> 5, T >> 5);
    }
    if (!gridSync(c, epoch)) return;
    markPhase(c, kPhasePulled);
    if (!runNearFar<Mode>(P, outRow, outCol, sOutWk, epoch, nullptr, genBase)) return;
    markPhase(c, kPhaseLoop);
    unpackResults<Mode>(P, outRow, outCol, sOutWk, epoch);
    if (!gridSync(c, epoch)) return;
    markPhase(c, kPhaseEnd);
  } else {
    scratchOrCombined<Mode>(P, epoch, genBase, sOutWk);
  }
}

/// Steps 2-3 (combined mode) and the SSSP from scratch (both modes).
/// The combined edges into v of every tree at once, for combK <= 8: the K
/// parents are loaded once (combinedEdge reloads them per tree); has[k],
/// p[k] and w[k] are what combinedEdge(P, v, k, ...) gives.
__device__ __forceinline__ void combinedEdges8(const EngineParams &P, int v, int (&p)[8],
                                               int (&w)[8], bool (&has)[8]) {
  const long long n = P.n;
#pragma unroll
  for (int k = 0; k < 8; ++k) p[k] = k < P.combK ? __ldg(P.combParents + k * n + v) : -1;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    bool first = p[k] >= 0;
#pragma unroll
    for (int j = 0; j < k; ++j) first = first && p[j] != p[k];
    int weight = P.combBase - P.prefTerms[k];
#pragma unroll
    for (int j = k + 1; j < 8; ++j) {
      if (p[j] == p[k]) weight -= P.prefTerms[j];  // trees past combK hold -1
    }
    has[k] = first;
    w[k] = weight;
  }
}

template <int Mode>
__device__ void scratchOrCombined(const EngineParams &P, Sync &epoch, int genBase,
                                  const int **sOutWk) {
  EngineControl *c = P.ctl;
  const int n = P.n, K = P.K;
  const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long T = static_cast<long long>(gridDim.x) * blockDim.x;
  const unsigned lane = laneId();
  __shared__ u64 sCombDelta;
  const int *outRow = P.outRow;
  const int *outCol = P.outCol;

  if constexpr (Mode == kModeCombined) {
    // ---- Step 2: combined graph, count / scan / fill (reference
    // src/combinedGraphGpu.cu:80-121, 281-300), then Step 3 below --------
    for (long long v = tid; v <= n; v += T) P.combDeg[v] = 0;
    if (!gridSync(c, epoch)) return;
    // four vertices per thread (v, v + T, v + 2T, v + 3T) in the count and
    // fill passes, so their parent loads and atomics are in flight together
    unsigned long long edges = 0, wsum = 0;
    bool badParent = false;
    const bool regs = P.combK <= 8;  // the same for every thread
    for (long long v = tid; regs && v < n; v += T) {
      if (isRoot(P.source, P.sources, P.nSources, static_cast<int>(v))) continue;
      int p[8], w[8];
      bool has[8];
      combinedEdges8(P, static_cast<int>(v), p, w, has);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (!has[k]) continue;
        if (p[k] >= n) {
          badParent = true;
          continue;
        }
        atomicAdd(P.combDeg + p[k], 1);
        ++edges;
        wsum += static_cast<unsigned long long>(w[k]);
      }
    }
    for (long long v0 = tid; !regs && v0 < n; v0 += 4 * T) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const long long v = v0 + q * T;
        if (v >= n || isRoot(P.source, P.sources, P.nSources, static_cast<int>(v))) continue;
        for (int k = 0; k < P.combK; ++k) {
          int p, w;
          if (combinedEdge(P, static_cast<int>(v), k, p, w)) {
            if (p >= n) {
              badParent = true;
              continue;
            }
            atomicAdd(P.combDeg + p, 1);
            ++edges;
            wsum += static_cast<unsigned long long>(w);
          }
        }
      }
    }
    if (badParent) c->invalid = 1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      edges += __shfl_down_sync(kFull, edges, off);
      wsum += __shfl_down_sync(kFull, wsum, off);
    }
    if (lane == 0 && edges > 0) {
      atomicAdd(&c->sums[0], edges);
      atomicAdd(&c->sums[1], wsum);
    }
    if (!gridSync(c, epoch)) return;
    long long totalEdges = 0;
    if (__ldcg(&c->invalid) != 0) return;
    // row starts; the degree array becomes the fill cursor (each CTA reads
    // and rewrites only its own chunk)
    if (!gridExclusiveScan(P.combDeg, P.combRow, P.combDeg, static_cast<long long>(n) + 1,
                           P.blockSums, c, epoch, &totalEdges)) {
      return;
    }
    if (!gridSync(c, epoch)) return;
    for (long long v = tid; regs && v < n; v += T) {
      if (isRoot(P.source, P.sources, P.nSources, static_cast<int>(v))) continue;
      int p[8], w[8];
      bool has[8];
      combinedEdges8(P, static_cast<int>(v), p, w, has);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (!has[k]) continue;
        const int pos = atomicAdd(P.combDeg + p[k], 1);
        P.combCol[pos] = static_cast<int>(v);
        P.combW[pos] = w[k];
      }
    }
    for (long long v0 = tid; !regs && v0 < n; v0 += 4 * T) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const long long v = v0 + q * T;
        if (v >= n || isRoot(P.source, P.sources, P.nSources, static_cast<int>(v))) continue;
        for (int k = 0; k < P.combK; ++k) {
          int p, w;
          if (combinedEdge(P, static_cast<int>(v), k, p, w)) {
            const int pos = atomicAdd(P.combDeg + p, 1);
            P.combCol[pos] = static_cast<int>(v);
            P.combW[pos] = w;
          }
        }
      }
    }
    if (threadIdx.x == 0) {
      // Default bucket width of the combined graph (reference
      // src/combinedGraphGpu.cu:310-312 and :607-616 of sospUpdateGpu.cu).
      u64 d = static_cast<u64>(P.combDelta);
      if (P.combDelta <= 0) {
        const double e = static_cast<double>(__ldcg(&c->sums[0]));
        const double ws = static_cast<double>(__ldcg(&c->sums[1]));
        long long dd = 1;
        if (e > 0 && n > 0) {
          dd = static_cast<long long>(32.0 * (ws / e) / (e / static_cast<double>(n)));
          if (dd < 1) dd = 1;
        }
        d = static_cast<u64>(dd);
      }
      sCombDelta = d;
    }
    outRow = P.combRow;
    outCol = P.combCol;
    if (threadIdx.x == 0) sOutWk[0] = P.combW;
    markPhase(c, kPhasePacked);
    // fall through to the SSSP from scratch
  }

  if constexpr (Mode == kModeScratch) {
    // The caller's CSR is checked before any access that it indexes: row
    // offsets monotone from 0 to m, every column in [0, n). A malformed graph
    // ends the launch with `invalid` set, before the relaxations.
    if (tid == 0 && (__ldg(outRow) != 0 || __ldg(outRow + n) != P.m)) c->invalid = 1;
    for (long long v = tid; v < n; v += T) {
      if (__ldg(outRow + v + 1) < __ldg(outRow + v)) c->invalid = 1;
    }
    for (long long e = tid; e < P.m; e += T) {
      const int x = __ldg(outCol + e);
      if (x < 0 || x >= n) c->invalid = 1;
    }
    if (!gridSync(c, epoch)) return;
    if (__ldcg(&c->invalid) != 0) return;
  }

  // ---- SSSP from scratch: only the source (the roots) is finite ------------
  bool heavyRow = false;  // one store at the end, so the loads run ahead
  for (long long v = tid; v < n; v += T) {
    heavyRow |= ldGraph<Mode>(outRow + v + 1) - ldGraph<Mode>(outRow + v) > heavyDegOf(P);
  }
  if (heavyRow) c->heavy = 1;
  for (int k = 0; k < K; ++k) {
    const Pk pk = pkOf(P.obj[k]);
    const long long ko = static_cast<long long>(k) * P.stride;
    for (long long v = tid; v < n; v += T) {
      P.packed[ko + v] =
          isRoot(P.source, P.sources, P.nSources, static_cast<int>(v)) ? pk.pack(0, -1) : kInfWord;
    }
    const int roots = P.nSources > 1 ? P.nSources : 1;
    for (long long i = tid; i < roots; i += T) {
      const int r = P.nSources > 1 ? P.sources[i] : P.source;
      P.inFar[ko + r] = 1;
      P.farL0[ko + i] = r;
    }
    if (tid == 0) {
      c->farCount[k][0] = roots;
      c->farMinC[k][0] = ~0ULL;  // minimum 0
    }
  }
  if (!gridSync(c, epoch)) return;
  markPhase(c, kPhasePulled);
  u64 *deltaOverride = nullptr;
  if constexpr (Mode == kModeCombined) deltaOverride = &sCombDelta;
  if (!runNearFar<Mode>(P, outRow, outCol, sOutWk, epoch, deltaOverride, genBase)) return;
  markPhase(c, kPhaseLoop);
  unpackResults<Mode>(P, outRow, outCol, sOutWk, epoch);
  if (!gridSync(c, epoch)) return;
  markPhase(c, kPhaseEnd);
}

// ---------------------------------------------------------------------------
// Device graph: objective-major weights and the reverse CSR (reference
// src/deviceGraph.cu:28-63, 87-135), one cooperative launch.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1) buildGraph(const __grid_constant__ BuildParams B) {
  EngineControl *c = B.ctl;
  const int n = B.n, m = B.m, K = B.K;
  const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long T = static_cast<long long>(gridDim.x) * blockDim.x;
  const unsigned lane = laneId();
  const long long gwarp = tid >> 5, nwarps = T >> 5;
  Sync epoch = startSync(B.timeoutNs);

  // validate the CSR; split the weights; clear the degree counts
  if (tid == 0 && (__ldg(B.outRow) != 0 || __ldg(B.outRow + n) != m)) c->invalid = 1;
  for (long long v = tid; v < n; v += T) {
    if (__ldg(B.outRow + v + 1) < __ldg(B.outRow + v)) c->invalid = 1;
  }
  for (long long e = tid; e < m; e += T) {
    const int x = __ldg(B.outCol + e);
    if (x < 0 || x >= n) c->invalid = 1;
  }
  for (long long i = tid; i < static_cast<long long>(m) * K; i += T) {
    const long long e = i / K;
    const int k = static_cast<int>(i - e * K);
    B.outW[static_cast<long long>(k) * m + e] = __ldg(B.edgeMajorW + i);
  }
  for (long long v = tid; v <= n; v += T) B.cursor[v] = 0;
  if (!gridSync(c, epoch)) return;
  if (__ldcg(&c->invalid) != 0) return;

  for (long long e = tid; e < m; e += T) atomicAdd(B.cursor + __ldg(B.outCol + e), 1);
  if (!gridSync(c, epoch)) return;
  long long total = 0;
  if (!gridExclusiveScan(B.cursor, B.inRow, B.cursor, static_cast<long long>(n) + 1,
                         B.blockSums, c, epoch, &total)) {
    return;
  }
  if (!gridSync(c, epoch)) return;

  // fill: one lane per short row, one warp per long row
  for (long long base = gwarp * 32; base < n; base += nwarps * 32) {
    const long long u = base + lane;
    int beg = 0, end = 0;
    if (u < n) {
      beg = __ldg(B.outRow + u);
      end = __ldg(B.outRow + u + 1);
    }
    const int deg = end - beg;
    unsigned big = __ballot_sync(kFull, deg > kLaneRowMax);
    auto place = [&](int uu, int e) {
      const int pos = atomicAdd(B.cursor + __ldg(B.outCol + e), 1);
      B.inCol[pos] = uu;
      for (int k = 0; k < K; ++k) {
        B.inW[static_cast<long long>(k) * m + pos] =
            __ldg(B.edgeMajorW + static_cast<long long>(e) * K + k);
      }
    };
    if (deg <= kLaneRowMax) {
      for (int e = beg; e < end; ++e) place(static_cast<int>(u), e);
    }
    while (big != 0) {
      const int src = __ffs(big) - 1;
      big &= big - 1;
      const int ub = static_cast<int>(__shfl_sync(kFull, u, src));
      const int bb = __shfl_sync(kFull, beg, src);
      const int eb = __shfl_sync(kFull, end, src);
      for (int e = bb + static_cast<int>(lane); e < eb; e += 32) place(ub, e);
    }
  }
}

// ---------------------------------------------------------------------------
// MOSP path costs: sums of the original weights along the MOSP tree by
// pointer jumping with double buffering (replaces the host BFS of
// reference src/combinedGraphGpu.cu:161-208; same edge rule: the first
// occurrence of v in row p).
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long satAdd(long long a, long long b) {
  if (a >= kDistInf / 2 || b >= kDistInf / 2) return kDistInf;
  const long long s = a + b;
  return s >= kDistInf / 2 ? kDistInf : s;
}

__global__ void __launch_bounds__(kThreads, 1) pathCosts(const __grid_constant__ CostParams C) {
  EngineControl *c = C.ctl;
  const int n = C.n, KG = C.KG;
  const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long T = static_cast<long long>(gridDim.x) * blockDim.x;
  const unsigned lane = laneId();
  const long long gwarp = tid >> 5, nwarps = T >> 5;
  Sync epoch = startSync(C.timeoutNs);

  for (long long v = tid; v < n; v += T) C.edgeOf[v] = INT_MAX;
  if (!gridSync(c, epoch)) return;
  // first occurrence of the tree edge (parent[v], v): lowest e in row p.
  // Edge-balanced: warp w takes the w-th equal slice of the edge array and
  // finds the row of each of its 32 edges from the ends of the next 32 rows
  // (one coalesced load, a 5-step shuffle search), so hub rows are shared
  // by many warps instead of walked by one.
  {
    const long long m = __ldg(C.outRow + n);
    const long long wb = m * gwarp / nwarps, we = m * (gwarp + 1) / nwarps;
    if (wb < we) {  // the same for the whole warp
      int lo = 0, hi = n;  // the row of the slice's first edge: last r with row[r] <= wb
      while (hi - lo > 1) {
        const int mid = lo + ((hi - lo) >> 1);
        if (__ldg(C.outRow + mid) <= wb) lo = mid; else hi = mid;
      }
      int r0 = lo;
      for (long long e0 = wb; e0 < we; e0 += 32) {
        const bool valid = e0 + lane < we;
        const int e = static_cast<int>(e0 + lane);
        const int x = valid ? __ldg(C.outCol + e) : 0;
        int row = valid ? -1 : 0;
        for (int base = r0; base < n; base += 32) {
          const int rr = base + static_cast<int>(lane);
          const int end = rr < n ? __ldg(C.outRow + rr + 1) : INT_MAX;
          int pos = 0;  // rows of the window that end at or before e
#pragma unroll
          for (int step = 16; step >= 1; step >>= 1) {
            if (__shfl_sync(kFull, end, pos + step - 1) <= e) pos += step;
          }
          // every lane takes part in the shuffle, found or not
          const int lastEnd = __shfl_sync(kFull, end, 31);
          if (row < 0 && e < lastEnd) row = base + pos;
          if (__all_sync(kFull, row >= 0)) break;
        }
        r0 = __shfl_sync(kFull, row, 31);  // the largest row; past the slice the loop ends
        if (valid && row >= 0 && row < n && static_cast<unsigned>(x) < static_cast<unsigned>(n) &&
            !isRoot(C.source, C.sources, C.nSources, x) && __ldg(C.parent + x) == row) {
          atomicMin(C.edgeOf + x, e);
        }
      }
    }
  }
  if (!gridSync(c, epoch)) return;
  for (long long v = tid; v < n; v += T) {
    const int p = __ldg(C.parent + v);
    long long *acc = C.acc0 + v * KG;
    if (isRoot(C.source, C.sources, C.nSources, static_cast<int>(v))) {
      C.anc0[v] = -1;
      for (int k = 0; k < KG; ++k) acc[k] = 0;
    } else if (p < 0 || p >= n) {
      if (p >= n) c->invalid = 1;
      C.anc0[v] = -1;
      for (int k = 0; k < KG; ++k) acc[k] = kDistInf;
    } else {
      const int e = __ldcg(C.edgeOf + v);
      if (e == INT_MAX) {
        c->invalid = 1;  // the tree edge is not in the graph
        C.anc0[v] = -1;
        for (int k = 0; k < KG; ++k) acc[k] = kDistInf;
      } else {
        C.anc0[v] = p;
        for (int k = 0; k < KG; ++k) {
          acc[k] = __ldg(C.outW + static_cast<long long>(k) * C.m + e);
        }
      }
    }
  }
  if (!gridSync(c, epoch)) return;
  int round = 0;
  for (;; ++round) {
    const int *ancR = (round & 1) ? C.anc1 : C.anc0;
    int *ancW = (round & 1) ? C.anc0 : C.anc1;
    const long long *accR = (round & 1) ? C.acc1 : C.acc0;
    long long *accW = (round & 1) ? C.acc0 : C.acc1;
    if (blockIdx.x == 0 && threadIdx.x == 0) c->jumpActive[(round + 1) % 3] = 0;
    int active = 0;
    for (long long v = tid; v < n; v += T) {
      const int a = __ldcg(ancR + v);
      if (a >= 0) {
        const int b = __ldcg(ancR + a);
        for (int k = 0; k < KG; ++k) {
          accW[v * KG + k] = satAdd(__ldcg(accR + v * KG + k), __ldcg(accR + static_cast<long long>(a) * KG + k));
        }
        ancW[v] = b;
        active |= b >= 0;
      } else {
        for (int k = 0; k < KG; ++k) accW[v * KG + k] = __ldcg(accR + v * KG + k);
        ancW[v] = a;
      }
    }
    if (__syncthreads_or(active) && threadIdx.x == 0) atomicOr(&c->jumpActive[round % 3], 1);
    if (!gridSync(c, epoch)) return;
    if (__ldcg(&c->jumpActive[round % 3]) == 0 || round > 64) break;
  }
  const long long *accF = (round & 1) ? C.acc0 : C.acc1;
  for (long long i = tid; i < static_cast<long long>(n) * KG; i += T) {
    const long long x = __ldcg(accF + i);
    C.costs[i] = x >= kDistInf / 2 ? kDistInf : x;
  }
}

// ---------------------------------------------------------------------------
// Failure-path probe: every CTA but the first waits at a barrier that the
// first never reaches; the bounded wait must end with MOSP_ERR_TIMEOUT.
// ---------------------------------------------------------------------------
__global__ void barrierProbe(EngineControl *c, long long timeoutNs) {
  Sync epoch = startSync(timeoutNs);
  if (blockIdx.x == 0) return;
  gridSync(c, epoch);
}

/// Cost of the grid barrier alone: `rounds` barriers back to back; with
/// `reads`, every CTA also reads two control words after each barrier (the
/// loop's decision step). CTA 0 records the elapsed device time.
__global__ void barrierCost(EngineControl *c, int rounds, int reads, long long timeoutNs) {
  Sync epoch = startSync(timeoutNs);
  const unsigned long long t0 = globalNs();
  for (int r = 0; r < rounds; ++r) {
    if (reads && threadIdx.x < 32) {
      const int a = __ldcg(&c->nearCount[threadIdx.x & 7][r % 3]);
      const int b = __ldcg(&c->farCount[threadIdx.x & 7][r % 3]);
      if (a == 12345 && b == 678) c->invalid = 0;
    }
    if (!gridSync(c, epoch)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) c->phaseNs[0] = globalNs() - t0;
}

/// The parent recovery of an update launch that ran with kFlagHostRecovery,
/// as a kernel of its own: no shared-memory stage, so L1 keeps its full
/// size for the graph reads.
__global__ void __launch_bounds__(256) recoverParents(const __grid_constant__ EngineParams P) {
  __shared__ const int *sOutWk[kMaxK];
  if (threadIdx.x < kMaxK) {
    sOutWk[threadIdx.x] =
        static_cast<int>(threadIdx.x) < P.K ? P.obj[threadIdx.x].outW : nullptr;
  }
  __syncthreads();
  const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long T = static_cast<long long>(gridDim.x) * blockDim.x;
  recoverTightParents<kModeUpdate>(P, P.outRow, P.outCol, sOutWk, tid, T);
}

template <typename Kernel>
cudaError_t ctasFor(Kernel kernel, int sms, int ctasPerSm, int &ctas, size_t smem = 0) {
  int perSm = 0;
  if (smem > 0) {
    cudaError_t a = cudaFuncSetAttribute(reinterpret_cast<const void *>(kernel),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (a != cudaSuccess) return a;
  }
  cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kThreads, smem);
  if (err != cudaSuccess) return err;
  if (perSm < 1) return cudaErrorInvalidConfiguration;
  if (ctasPerSm > 0 && ctasPerSm < perSm) perSm = ctasPerSm;
  ctas = perSm * sms;
  return cudaSuccess;
}

}  // namespace

cudaError_t queryLaunchShape(int ctasPerSm, LaunchShape &shape) {
  int device = 0, sms = 0, coop = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  if (err != cudaSuccess) return err;
  if (!coop) return cudaErrorNotSupported;
  int a = 0, b = 0, d = 0, e = 0;
  if ((err = ctasFor(sospEngine<kModeUpdate>, sms, ctasPerSm, a, kStageBytes)) != cudaSuccess) return err;
  if ((err = ctasFor(sospEngine<kModeScratch>, sms, ctasPerSm, b, kStageBytes)) != cudaSuccess) return err;
  if ((err = ctasFor(sospEngine<kModeCombined>, sms, ctasPerSm, d, kStageBytes)) != cudaSuccess) return err;
  shape.engineCtas = a < b ? (a < d ? a : d) : (b < d ? b : d);
  if ((err = ctasFor(buildGraph, sms, ctasPerSm, e)) != cudaSuccess) return err;
  shape.buildCtas = e;
  if ((err = ctasFor(pathCosts, sms, ctasPerSm, e)) != cudaSuccess) return err;
  shape.costCtas = e;
  return cudaSuccess;
}

cudaError_t launchEngine(const EngineParams &p, int ctas, cudaStream_t s) {
  void *args[] = {const_cast<EngineParams *>(&p)};
  const void *fn = nullptr;
  switch (p.mode) {
    case kModeUpdate: fn = reinterpret_cast<const void *>(sospEngine<kModeUpdate>); break;
    case kModeScratch: fn = reinterpret_cast<const void *>(sospEngine<kModeScratch>); break;
    default: fn = reinterpret_cast<const void *>(sospEngine<kModeCombined>); break;
  }
  return cudaLaunchCooperativeKernel(fn, dim3(ctas), dim3(kThreads), args,
                                     stageBytesFor(p.stageEntries), s);
}

bool needsHostRecovery(const EngineParams &p) {
  if (p.mode != kModeUpdate) return false;
  for (int k = 0; k < p.K; ++k) {
    if (p.obj[k].parentBits == 0) return true;
  }
  return false;
}

cudaError_t launchRecovery(const EngineParams &p, cudaStream_t s) {
  int device = 0, sms = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (err != cudaSuccess) return err;
  if ((p.flags & kFlagCanonical) != 0 && p.recMark != nullptr) {
    return launchRestrictedRecovery(p, sms, s);
  }
  recoverParents<<<sms * 8, 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launchEngineEx(const EngineParams &p, int ctas, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = stageBytesFor(p.stageEntries);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  switch (p.mode) {
    case kModeUpdate: return cudaLaunchKernelEx(&cfg, sospEngine<kModeUpdate>, p);
    case kModeScratch: return cudaLaunchKernelEx(&cfg, sospEngine<kModeScratch>, p);
    default: return cudaLaunchKernelEx(&cfg, sospEngine<kModeCombined>, p);
  }
}

cudaError_t launchBuild(const BuildParams &p, int ctas, cudaStream_t s) {
  void *args[] = {const_cast<BuildParams *>(&p)};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(buildGraph), dim3(ctas),
                                     dim3(kThreads), args, 0, s);
}

cudaError_t launchCosts(const CostParams &p, int ctas, cudaStream_t s) {
  void *args[] = {const_cast<CostParams *>(&p)};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(pathCosts), dim3(ctas),
                                     dim3(kThreads), args, 0, s);
}

cudaError_t launchBarrierCost(EngineControl *ctl, int rounds, int reads, long long timeoutNs,
                              int ctas, cudaStream_t s) {
  void *args[] = {&ctl, &rounds, &reads, &timeoutNs};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(barrierCost), dim3(ctas),
                                     dim3(kThreads), args, 0, s);
}

cudaError_t launchBarrierProbe(EngineControl *ctl, long long timeoutNs, int ctas,
                               cudaStream_t s) {
  void *args[] = {&ctl, &timeoutNs};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(barrierProbe), dim3(ctas),
                                     dim3(kThreads), args, 0, s);
}

}  // namespace mospb200
