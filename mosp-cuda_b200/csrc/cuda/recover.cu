// recover.cu - lowest-id parent recovery of the distance-only objectives of
// an update launch, restricted to the vertices whose parent the batch can
// change (EngineParams::flags & kFlagCanonical).
//
// An objective whose packed word would need more than 64 bits runs on
// distances alone, and its parents are recovered afterwards: every
// reachable vertex other than a root takes the lowest-id tail of a tight
// in-edge, d(u) + w(u, v) == d(v) (reference src/sospUpdateGpu.cu:491-512,
// which scans every edge of the graph; recoverParents in engine.cu does the
// same). When the input trees already follow that rule (every tree this
// library returns does, and so do trees made by the lowest-id Dijkstra),
// the rule returns the input parent at every vertex v for which none of
// these holds:
//   (a) the distance of v changed;
//   (b) the distance of v's input parent changed;
//   (c) an edge into v was inserted or lowered (v is a head of the batch);
//   (d) the edge from v's input parent was deleted or raised.
// At such a v the input parent is still tight, and the only tails that can
// have become tight are in-neighbours whose distance changed. So the
// (a)-(d) vertices scan their in-rows again, and every reachable vertex
// whose distance changed pushes itself along its out-edges into the other
// vertices with atomicMin. Everything after the update launch runs over
// lists, so the work follows the rows of the vertices the batch reached
// instead of all m edges or all n vertices of every distance-only objective.
//
// The update launch wrote the new distances, kept the input parents (-1 at
// roots and unreachable vertices), set kRecChanged on the (a) vertices and
// listed them (the changed list). Then, on the same stream:
//   markReach    kRecScan on (c) and (d), and on (b) found from the
//                out-rows of the changed vertices (their tree children);
//                each vertex it marks first, unless changed, goes to the
//                scan list; out-rows longer than kRecLightRow edges go to
//                the first chunk list;
//   markChunks   the same (b) marks over the listed out-row chunks;
//   scanNeed     every reachable vertex of the changed and scan lists takes
//                the lowest tight tail of its in-row (in-rows longer than
//                kRecLightRow edges go to the second chunk list); then the
//                changed vertices push along their out-rows (the listed
//                chunks one per warp) into the vertices on neither list;
//   scanChunks   the listed in-row chunks, one per warp.
// A warp takes 32 list entries at a time and walks their rows as one flat
// range of edges. Every index read from memory is range-checked, and
// nothing runs when the update launch reported an error.
#include "engine.h"

#include <climits>

namespace mospb200 {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kRecThreads = 256;
// a listed row is split into chunks of kChunk edges, one list entry each;
// with kChunk = 2 kRecLightRow a row of d > kRecLightRow edges has at most
// d / kRecLightRow chunks, which bounds a chunk list by m / kRecLightRow + 1
// entries per objective
constexpr int kChunk = 2 * kRecLightRow;

__device__ __forceinline__ bool launchFailed(const EngineParams &P) {
  return __ldcg(&P.ctl->status) != 0 || __ldcg(&P.ctl->invalid) != 0 ||
         __ldcg(&P.ctl->overflow) != 0;
}

__device__ __forceinline__ bool inRange(int x, int n) {
  return static_cast<unsigned>(x) < static_cast<unsigned>(n);
}

__device__ __forceinline__ unsigned char *markOf(const EngineParams &P, int k) {
  return P.recMark + static_cast<long long>(k) * P.stride;
}

/// Set kRecScan on vertex x of objective k; the first mark of a vertex
/// that is not changed puts it on the scan list, when it is reachable and
/// not a root (the others keep parent -1).
__device__ void markScan(const EngineParams &P, int k, int x) {
  unsigned char *byte = markOf(P, k) + x;
  const uintptr_t at = reinterpret_cast<uintptr_t>(byte);
  const unsigned shift = static_cast<unsigned>(at & 3u) * 8u;
  const unsigned old = atomicOr(reinterpret_cast<unsigned *>(at & ~static_cast<uintptr_t>(3)),
                                static_cast<unsigned>(kRecScan) << shift);
  if (((old >> shift) & (kRecChanged | kRecScan)) != 0) return;
  if (__ldg(P.obj[k].dist + x) == kDistInf || isRoot(P.source, P.sources, P.nSources, x)) return;
  // each vertex is listed at most once (its first mark), so at most n
  const int slot = atomicAdd(&P.ctl->recScan[k], 1);
  if (slot < P.n) P.recScanList[static_cast<long long>(k) * P.stride + slot] = x;
}

/// Append the chunks of row [a, e) of vertex v (objective k) to chunk list
/// `which`: vertex << 32 | chunk << 8 | objective.
__device__ void listChunks(const EngineParams &P, int which, int v, int a, int e, int k) {
  const int chunks = (e - a + kChunk - 1) / kChunk;
  const int i0 = atomicAdd(&P.ctl->recChunks[which], chunks);
  if (static_cast<long long>(i0) + chunks > P.recChunkCap) {
    // a chunk list holds every chunk of every row above kRecLightRow edges,
    // so only row pointers that disagree with m get here
    atomicExch(&P.ctl->invalid, 1);
    return;
  }
  u64 *list = P.recChunkList + static_cast<long long>(which) * P.recChunkCap;
  for (int c = 0; c < chunks; ++c) {
    list[i0 + c] = (static_cast<u64>(v) << 32) | (static_cast<u64>(c) << 8) | static_cast<u64>(k);
  }
}

/// The rows of the warp's lanes (this lane's: edges [a, e) of vertex v at
/// distance d in objective k; a == e for none) taken as one flat range of
/// edges, 32 at a time, so that every lane has an edge while any remain:
/// edge(v, d, k, j) for each edge j, with the v, d and k of its row.
template <typename Edge>
__device__ __forceinline__ void flatRows(int v, long long d, int k, int a, int e, int lane, Edge edge) {
  const int len = e - a;
  int incl = len;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int t = __shfl_up_sync(kFull, incl, off);
    if (lane >= off) incl += t;
  }
  const int total = __shfl_sync(kFull, incl, 31);
  const int first = a - (incl - len);  // a minus the edges of the lanes before
  for (int base = 0; base < total; base += 32) {
    const int s = base + lane;
    // the owner: the number of lanes whose rows end at or before s
    int lo = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
      const int probe = __shfl_sync(kFull, incl, lo + step - 1);
      if (probe <= s) lo += step;
    }
    lo = min(lo, 31);
    const int ov = __shfl_sync(kFull, v, lo);
    const long long od = __shfl_sync(kFull, d, lo);
    const int ok = __shfl_sync(kFull, k, lo);
    const int of = __shfl_sync(kFull, first, lo);
    if (s < total) edge(ov, od, ok, of + s);
  }
}

/// The lists of all distance-only objectives as one flat index: objective
/// k's entries are [off[k], off[k + 1]) (shared memory, set by thread 0).
/// withScan: each objective's changed list followed by its scan list, else
/// the changed list alone.
__device__ void flatOffsets(const EngineParams &P, bool withScan, long long *off) {
  if (threadIdx.x == 0) {
    long long acc = 0;
    for (int k = 0; k < P.K; ++k) {
      off[k] = acc;
      if (P.obj[k].parentBits == 0) {
        acc += min(__ldcg(&P.ctl->recChanged[k]), P.n);
        if (withScan) acc += min(__ldcg(&P.ctl->recScan[k]), P.n);
      }
    }
    off[P.K] = acc;
  }
  __syncthreads();
}

/// Objective and list position of flat index g (g < off[K]): the vertex,
/// from the changed list and then (withScan) the scan list.
__device__ __forceinline__ int flatEntry(const EngineParams &P, const long long *off, long long g,
                                         int &k) {
  k = 0;
  while (k + 1 < P.K && off[k + 1] <= g) ++k;
  const long long i = g - off[k];
  const int nc = min(__ldcg(&P.ctl->recChanged[k]), P.n);
  const long long ko = static_cast<long long>(k) * P.stride;
  return i < nc ? P.recChangedList[ko + i] : P.recScanList[ko + (i - nc)];
}

/// Out-edge j of changed vertex u: a head whose input parent is u is a
/// tree child of a vertex whose distance changed, case (b).
__device__ __forceinline__ void childEdge(const EngineParams &P, int k, int u, int j) {
  const int x = __ldg(P.outCol + j);
  if (inRange(x, P.n) && P.obj[k].parent[x] == u) markScan(P, k, x);
}

/// In-edge j of vertex v (distance d): a tight tail lowers v's parent.
__device__ __forceinline__ void scanEdge(const EngineParams &P, const ObjectiveArgs &O, int v,
                                         long long d, int j) {
  const int u = __ldg(P.inCol + j);
  if (!inRange(u, P.n)) return;
  const long long du = __ldg(O.dist + u);
  if (du != kDistInf && du + __ldg(O.inW + j) == d) atomicMin(O.parent + v, u);
}

/// Out-edge j of u (distance du): a push into a vertex on neither list.
__device__ __forceinline__ void pushEdge(const EngineParams &P, const ObjectiveArgs &O,
                                         const unsigned char *mark, int u, long long du, int j) {
  const int x = __ldg(P.outCol + j);
  if (!inRange(x, P.n) || (mark[x] & (kRecChanged | kRecScan)) != 0) return;
  if (isRoot(P.source, P.sources, P.nSources, x)) return;
  const long long dx = __ldg(O.dist + x);
  if (dx != kDistInf && du + __ldg(O.outW + j) == dx) atomicMin(O.parent + x, u);
}

/// Row [a, e) of list entry `entry` of chunk list `which`, or false.
__device__ __forceinline__ bool chunkOf(const EngineParams &P, int which, u64 entry, int &v, int &k,
                                        int &a, int &e) {
  v = static_cast<int>(entry >> 32);
  k = static_cast<int>(entry & 31u);
  const int c = static_cast<int>((entry >> 8) & 0xffffffu);
  if (!inRange(v, P.n) || k >= P.K) return false;
  const int *row = which == 0 ? P.outRow : P.inRow;
  a = __ldg(row + v) + c * kChunk;
  e = min(__ldg(row + v + 1), a + kChunk);
  return true;
}

__global__ void __launch_bounds__(kRecThreads) markReach(const __grid_constant__ EngineParams P) {
  __shared__ long long off[kMaxK + 1];
  if (launchFailed(P)) return;
  flatOffsets(P, false, off);
  const int n = P.n;
  const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long T = static_cast<long long>(gridDim.x) * blockDim.x;
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const long long gwarp = tid >> 5, nwarps = T >> 5;
  for (int k = 0; k < P.K; ++k) {
    const ObjectiveArgs &O = P.obj[k];
    if (O.parentBits > 0) continue;  // the same for every thread
    for (long long i = tid; i < P.nHeads; i += T) {  // (c)
      const int x = P.heads[i];
      if (inRange(x, n)) markScan(P, k, x);
    }
    for (long long i = tid; i < O.nChanged; i += T) {  // (d)
      const int t = O.chTo[i];
      if (inRange(t, n) && O.parent[t] == O.chFrom[i]) markScan(P, k, t);
    }
  }
  // (b): the out-rows of the changed vertices of every objective
  const long long total = off[P.K];
  for (long long base = gwarp * 32; base < total; base += nwarps * 32) {
    int u = 0, k = 0, a = 0, e = 0;
    if (base + lane < total) {
      u = flatEntry(P, off, base + lane, k);
      if (inRange(u, n)) {
        a = __ldg(P.outRow + u);
        e = __ldg(P.outRow + u + 1);
        if (e - a > kRecLightRow) {
          listChunks(P, 0, u, a, e, k);
          a = e = 0;
        }
      }
    }
    flatRows(u, 0, k, a, e, lane, [&](int ou, long long, int ok, int j) { childEdge(P, ok, ou, j); });
  }
}

__global__ void __launch_bounds__(kRecThreads) markChunks(const __grid_constant__ EngineParams P) {
  if (launchFailed(P)) return;
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const long long gwarp = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  const int count = min(__ldcg(&P.ctl->recChunks[0]), P.recChunkCap);
  for (long long i = gwarp; i < count; i += nwarps) {  // one chunk per warp
    int u, k, a, e;
    if (!chunkOf(P, 0, __ldcg(P.recChunkList + i), u, k, a, e)) continue;
    for (int j = a + lane; j < e; j += 32) childEdge(P, k, u, j);
  }
}

__global__ void __launch_bounds__(kRecThreads, 6) scanNeed(const __grid_constant__ EngineParams P) {
  __shared__ long long off[kMaxK + 1];
  if (launchFailed(P)) return;
  const int n = P.n;
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const long long gwarp = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  // the in-rows of the changed and scan lists
  flatOffsets(P, true, off);
  long long total = off[P.K];
  for (long long base = gwarp * 32; base < total; base += nwarps * 32) {
    int v = 0, k = 0, a = 0, e = 0;
    long long dv = kDistInf;
    if (base + lane < total) {
      v = flatEntry(P, off, base + lane, k);
      if (inRange(v, n)) {
        const ObjectiveArgs &O = P.obj[k];
        dv = __ldg(O.dist + v);
        if (dv != kDistInf && !isRoot(P.source, P.sources, P.nSources, v)) {
          O.parent[v] = INT_MAX;  // the scan takes the minimum
          a = __ldg(P.inRow + v);
          e = __ldg(P.inRow + v + 1);
          if (e - a > kRecLightRow) {
            listChunks(P, 1, v, a, e, k);
            a = e = 0;
          }
        }
      }
    }
    __syncwarp();  // the INT_MAX stores before the lanes' atomicMin
    flatRows(v, dv, k, a, e, lane,
             [&](int ov, long long od, int ok, int j) { scanEdge(P, P.obj[ok], ov, od, j); });
  }
  // the pushes of the changed vertices: into vertices on neither list, so
  // they do not meet the scans above (the marks are final since markChunks)
  __syncthreads();
  flatOffsets(P, false, off);
  total = off[P.K];
  for (long long base = gwarp * 32; base < total; base += nwarps * 32) {
    int u = 0, k = 0, a = 0, e = 0;
    long long du = kDistInf;
    if (base + lane < total) {
      u = flatEntry(P, off, base + lane, k);
      if (inRange(u, n)) {
        du = __ldg(P.obj[k].dist + u);
        a = __ldg(P.outRow + u);
        e = __ldg(P.outRow + u + 1);
        // unreachable vertices push nothing; long rows are in chunk list 0
        if (du == kDistInf || e - a > kRecLightRow) a = e = 0;
      }
    }
    flatRows(u, du, k, a, e, lane, [&](int ou, long long od, int ok, int j) {
      pushEdge(P, P.obj[ok], markOf(P, ok), ou, od, j);
    });
  }
  // the listed out-row chunks, one per warp
  const int pushes = min(__ldcg(&P.ctl->recChunks[0]), P.recChunkCap);
  for (long long i = gwarp; i < pushes; i += nwarps) {
    int u, k, a, e;
    if (!chunkOf(P, 0, __ldcg(P.recChunkList + i), u, k, a, e)) continue;  // the same for the warp
    const ObjectiveArgs &O = P.obj[k];
    const long long du = __ldg(O.dist + u);
    if (du == kDistInf) continue;
    const unsigned char *mark = markOf(P, k);
    for (int j = a + lane; j < e; j += 32) pushEdge(P, O, mark, u, du, j);
  }
}

/// The in-row chunks scanNeed listed, one per warp: the lowest tight tail
/// of each chunk lowers its vertex's parent.
__global__ void __launch_bounds__(kRecThreads) scanChunks(const __grid_constant__ EngineParams P) {
  if (launchFailed(P)) return;
  const int n = P.n;
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const long long gwarp = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  const int scans = min(__ldcg(&P.ctl->recChunks[1]), P.recChunkCap);
  for (long long i = gwarp; i < scans; i += nwarps) {
    int v, k, a, e;
    if (!chunkOf(P, 1, __ldcg(P.recChunkList + P.recChunkCap + i), v, k, a, e)) continue;
    const ObjectiveArgs &O = P.obj[k];
    const long long d = __ldg(O.dist + v);
    int best = INT_MAX;
    for (int j = a + lane; j < e; j += 32) {
      const int u = __ldg(P.inCol + j);
      if (!inRange(u, n)) continue;
      const long long du = __ldg(O.dist + u);
      if (du != kDistInf && du + __ldg(O.inW + j) == d && u < best) best = u;
    }
    best = __reduce_min_sync(kFull, best);
    if (lane == 0 && best != INT_MAX) atomicMin(O.parent + v, best);
  }
}

}  // namespace

cudaError_t launchRestrictedRecovery(const EngineParams &p, int sms, cudaStream_t s) {
  markReach<<<sms * 8, kRecThreads, 0, s>>>(p);
  markChunks<<<sms * 8, kRecThreads, 0, s>>>(p);
  scanNeed<<<sms * 8, kRecThreads, 0, s>>>(p);
  scanChunks<<<sms * 8, kRecThreads, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace mospb200
