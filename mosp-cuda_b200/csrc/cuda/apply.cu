// apply.cu - Step 1 on the GPU: apply a change batch to a device CSR graph
// (the semantics of applyChangeBatch, reference src/csrGraph.cu:727-894).
//
// Semantics, per source row u (the host restatement is applyBatchView in
// csrc/host/csrGraph.cpp):
//   * deletions first, in file order: each removes the first live edge (u,v);
//   * then insertions, in file order: an insertion (u,v) overwrites the
//     weights of the first live edge (u,v) if there is one, else appends a
//     new edge at the end of the row;
//   * the weight-increase mask of insertion i has bit k set when the final
//     weight of (u,v) exceeds the original one (first occurrence of v in the
//     original and in the updated row) in objective k.
// The sequential rules reduce to a per-(u,v) "group" computation: with c
// original occurrences of v in row u, cD deletions and cI insertions, the
// first min(c, cD) occurrences die; if c > cD and cI > 0 occurrence cD takes
// the weights of the group's last insertion; if c <= cD and cI > 0 one edge
// with those weights is appended, the appended edges of a row ordered by the
// file position of their group's first insertion; every insertion of the
// group gets the same mask (last insertion against occurrence 0, 0 if c = 0).
//
// Kernels (all plain launches on one stream; sizes that only the device
// knows are read from device counters, grids are sized by upper bounds):
//   keys -> stable LSD radix sort of (u,v) keys -> groups -> touched rows ->
//   occurrence count over the touched rows' edges -> group resolution ->
//   new degrees + scan -> appended-edge order (second radix sort) -> copy of
//   untouched rows (CTA row windows) and of touched rows (warp per row).
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <utility>

#include "engine.h"

namespace mospb200 {
namespace {

constexpr int kSortThreads = 1024;  // one item per thread, tile = 1024
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanChunk = kScanThreads * kScanItems;
constexpr int kCopyRows = 1024;  // rows per CTA window of the bulk copy
constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ bool stopped(const int *invalid) {
  return *reinterpret_cast<const volatile int *>(invalid) != 0;
}

// --- exclusive scan of int arrays: out[i] = sum(in[0..i)), out[len] = total --
__device__ int blockScanExclusive(int x, int *total) {
  __shared__ int warpSums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = x;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int o = __shfl_up_sync(kFullMask, incl, off);
    if (lane >= off) incl += o;
  }
  if (lane == 31) warpSums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    int s = lane < nw ? warpSums[lane] : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int o = __shfl_up_sync(kFullMask, s, off);
      if (lane >= off) s += o;
    }
    warpSums[lane] = s;  // inclusive over warps
  }
  __syncthreads();
  const int before = warp > 0 ? warpSums[warp - 1] : 0;
  *total = warpSums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before + incl - x;
}

__global__ void __launch_bounds__(kScanThreads) scanChunkSums(const int *in, long long len, int *aux) {
  const long long base = static_cast<long long>(blockIdx.x) * kScanChunk;
  int s = 0;
  for (int i = 0; i < kScanItems; ++i) {
    const long long j = base + static_cast<long long>(i) * kScanThreads + threadIdx.x;
    if (j < len) s += in[j];
  }
  int total;
  blockScanExclusive(s, &total);
  if (threadIdx.x == 0) aux[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) scanAux(int *aux, long long chunks, int *out, long long len) {
  int carry = 0;
  for (long long base = 0; base < chunks; base += kScanThreads) {
    const long long j = base + threadIdx.x;
    const int x = j < chunks ? aux[j] : 0;
    int total;
    const int ex = blockScanExclusive(x, &total);
    if (j < chunks) aux[j] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) out[len] = carry;
}

__global__ void __launch_bounds__(kScanThreads) scanChunks(const int *in, long long len, const int *aux,
                                                           int *out) {
  const long long base = static_cast<long long>(blockIdx.x) * kScanChunk;
  // each thread owns kScanItems consecutive items
  int v[kScanItems];
  int s = 0;
  for (int i = 0; i < kScanItems; ++i) {
    const long long j = base + static_cast<long long>(threadIdx.x) * kScanItems + i;
    v[i] = j < len ? in[j] : 0;
    s += v[i];
  }
  int total;
  int run = blockScanExclusive(s, &total) + aux[blockIdx.x];
  for (int i = 0; i < kScanItems; ++i) {
    const long long j = base + static_cast<long long>(threadIdx.x) * kScanItems + i;
    if (j < len) out[j] = run;
    run += v[i];
  }
}

cudaError_t exclusiveScan(const int *in, int *out, long long len, int *aux, cudaStream_t s) {
  const long long chunks = (len + kScanChunk - 1) / kScanChunk;
  if (chunks > 0) {
    scanChunkSums<<<static_cast<unsigned>(chunks), kScanThreads, 0, s>>>(in, len, aux);
  }
  scanAux<<<1, kScanThreads, 0, s>>>(aux, chunks, out, len);
  if (chunks > 0) {
    scanChunks<<<static_cast<unsigned>(chunks), kScanThreads, 0, s>>>(in, len, aux, out);
  }
  return cudaGetLastError();
}

// --- stable LSD radix sort of (u64 key, int value) pairs, 8-bit digits ------
__global__ void __launch_bounds__(kSortThreads) radixHistogram(const unsigned long long *keys,
                                                               const int *count, int shift,
                                                               int tiles, int *hist,
                                                               const int *invalid) {
  __shared__ int bins[256];
  if (threadIdx.x < 256) bins[threadIdx.x] = 0;
  __syncthreads();
  const int N = *count;
  const long long i = static_cast<long long>(blockIdx.x) * kSortThreads + threadIdx.x;
  if (i < N && !stopped(invalid)) atomicAdd(&bins[(keys[i] >> shift) & 255], 1);
  __syncthreads();
  if (threadIdx.x < 256) hist[static_cast<long long>(threadIdx.x) * tiles + blockIdx.x] = bins[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) radixScatter(const unsigned long long *keysIn,
                                                             const int *valsIn, const int *count,
                                                             int shift, int tiles,
                                                             const int *offsets,
                                                             unsigned long long *keysOut,
                                                             int *valsOut, const int *invalid) {
  __shared__ int warpCount[32][256];
  for (int j = threadIdx.x; j < 32 * 256; j += blockDim.x) (&warpCount[0][0])[j] = 0;
  __syncthreads();
  const int N = *count;
  const long long i = static_cast<long long>(blockIdx.x) * kSortThreads + threadIdx.x;
  const bool valid = i < N && !stopped(invalid);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long key = 0;
  int digit = 0, rankInWarp = 0;
  if (valid) {
    key = keysIn[i];
    digit = static_cast<int>((key >> shift) & 255);
    const unsigned peers = __match_any_sync(__activemask(), digit);
    rankInWarp = __popc(peers & ((1u << lane) - 1u));
    if (rankInWarp == 0) warpCount[warp][digit] = __popc(peers);
  }
  __syncthreads();
  if (threadIdx.x < 256) {
    int run = 0;
    for (int w = 0; w < 32; ++w) {
      const int c = warpCount[w][threadIdx.x];
      warpCount[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
  if (valid) {
    const int pos = offsets[static_cast<long long>(digit) * tiles + blockIdx.x] +
                    warpCount[warp][digit] + rankInWarp;
    keysOut[pos] = key;
    valsOut[pos] = valsIn[i];
  }
}

// --- the apply steps ---------------------------------------------------------
__global__ void makeKeys(ApplyParams P, unsigned long long *keys, int *vals, int *counters) {
  const long long B = static_cast<long long>(P.nDel) + P.nIns;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; j < B; j += stride) {
    int u, v;
    if (j < P.nDel) {
      u = P.delFrom[j];
      v = P.delTo[j];
    } else {
      u = P.insFrom[j - P.nDel];
      v = P.insTo[j - P.nDel];
    }
    if (u < 0 || u >= P.n || v < 0 || v >= P.n) {
      counters[kApplyInvalid] = 1;
      u = v = 0;
    }
    keys[j] = (static_cast<unsigned long long>(u) << P.vbits) | static_cast<unsigned>(v);
    vals[j] = static_cast<int>(j);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) counters[kApplyEntries] = static_cast<int>(B);
}

/// flags[j] = 1 where a new (u,v) group starts in the sorted keys.
__global__ void groupHeads(const unsigned long long *keys, long long B, int *flags, const int *invalid) {
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  const bool stop = stopped(invalid);
  for (long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; j < B; j += stride) {
    flags[j] = !stop && (j == 0 || keys[j] != keys[j - 1]) ? 1 : 0;
  }
}

__global__ void groupStarts(const int *flags, const int *pos, long long B, int *gStart, int *counters) {
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; j < B; j += stride) {
    if (flags[j]) gStart[pos[j]] = static_cast<int>(j);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int G = pos[B];
    counters[kApplyGroups] = G;
    gStart[G] = static_cast<int>(B);
  }
}

/// Per group: deletions, insertions, first and last insertion; row heads.
__global__ void groupInfo(ApplyParams P, const unsigned long long *keys, const int *vals,
                          ApplyGroups g, long long B, int *rowHead, const int *counters) {
  const int G = counters[kApplyGroups];
  const unsigned long long vmask = (1ULL << P.vbits) - 1;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; x < B; x += stride) {
    if (x >= G) {
      rowHead[x] = 0;
      continue;
    }
    const int s = g.start[x], e = g.start[x + 1];
    int cD = 0, cI = 0, firstIns = -1, lastIns = -1;
    for (int j = s; j < e; ++j) {
      const int val = vals[j];
      if (val < P.nDel) {
        ++cD;
      } else {
        ++cI;
        if (firstIns < 0) firstIns = val - P.nDel;
        lastIns = val - P.nDel;
      }
    }
    const unsigned long long key = keys[s];
    g.u[x] = static_cast<int>(key >> P.vbits);
    g.v[x] = static_cast<int>(key & vmask);
    g.cD[x] = cD;
    g.cI[x] = cI;
    g.firstIns[x] = firstIns;
    g.lastIns[x] = lastIns;
    g.occ[x] = 0;
    g.first[x] = INT_MAX;
    rowHead[x] = (x == 0 || (keys[g.start[x - 1]] >> P.vbits) != (key >> P.vbits)) ? 1 : 0;
  }
}

/// Touched rows: row id, first group, degree (for the slot scan).
__global__ void touchedRows(ApplyParams P, ApplyGroups g, long long B, const int *rowHead,
                            const int *rowPos, ApplyRows r, unsigned char *touched, int *counters) {
  const int G = counters[kApplyGroups];
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; x < B; x += stride) {
    // entries beyond the touched rows contribute nothing to the slot scan
    if (x >= rowPos[B]) r.deg[x] = 0;
    if (x < G && rowHead[x]) {
      const int k = rowPos[x];
      const int u = g.u[x];
      r.row[k] = u;
      r.gs[k] = static_cast<int>(x);
      r.deg[k] = P.row[u + 1] - P.row[u];
      touched[u] = 1;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int R = rowPos[B];
    counters[kApplyRows] = R;
    r.gs[R] = G;
  }
}

__device__ __forceinline__ int upperBound(const int *a, int n, long long x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] <= x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int findGroup(const int *gv, int lo, int hi, int v) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (gv[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/// Occurrences of each group's head in its original row, and the first one.
__global__ void countOccurrences(ApplyParams P, ApplyGroups g, ApplyRows r, const int *counters) {
  if (stopped(counters + kApplyInvalid)) return;
  const int R = counters[kApplyRows];
  const long long S = r.off[R];
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < S; t += stride) {
    const int k = upperBound(r.off, R, t) - 1;
    const int u = r.row[k];
    const int e = P.row[u] + static_cast<int>(t - r.off[k]);
    const int v = P.col[e];
    const int gs = r.gs[k], ge = r.gs[k + 1];
    const int x = findGroup(g.v, gs, ge, v);
    if (x < ge && g.v[x] == v) {
      atomicAdd(&g.occ[x], 1);
      atomicMin(&g.first[x], e);
    }
  }
}

/// Dead and overwritten original edges, per-row removed/appended counts,
/// appended groups and the weight-increase mask.
__global__ void resolveGroups(ApplyParams P, ApplyGroups g, long long B, unsigned char *slot,
                              int *removed, int *appended, int *appFlag, const int *counters) {
  const int G = counters[kApplyGroups];
  const bool stop = stopped(counters + kApplyInvalid);
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; x < B; x += stride) {
    if (x >= G || stop) {
      appFlag[x] = 0;
      continue;
    }
    const int c = g.occ[x], cD = g.cD[x], cI = g.cI[x];
    const int u = g.u[x], v = g.v[x];
    if (c == 1) {
      if (cD >= 1) slot[g.first[x]] = 1;
      else if (cI > 0) slot[g.first[x]] = 2;
    } else if (c > 1) {
      // repeated edge (u,v): walk the row in order
      int occ = 0;
      for (int e = g.first[x]; e < P.row[u + 1] && occ <= cD; ++e) {
        if (P.col[e] != v) continue;
        if (occ < cD) slot[e] = 1;
        else if (cI > 0) slot[e] = 2;
        ++occ;
      }
    }
    const int rem = c < cD ? c : cD;
    const int app = (c <= cD && cI > 0) ? 1 : 0;
    if (rem > 0) atomicAdd(&removed[u], rem);
    if (app) atomicAdd(&appended[u], 1);
    appFlag[x] = app;
    if (cI > 0) {
      unsigned bits = 0;
      if (c >= 1) {
        const int *wn = P.insW + static_cast<long long>(g.lastIns[x]) * P.K;
        const int *wo = P.w + static_cast<long long>(g.first[x]) * P.K;
        for (int k = 0; k < P.K; ++k) bits |= (wn[k] > wo[k] ? 1u : 0u) << k;
      }
      // every insertion of the group gets the same mask
      for (int j = g.start[x]; j < g.start[x + 1]; ++j) {
        const int val = P.sortedVals[j];
        if (val >= P.nDel) P.mask[val - P.nDel] = bits;
      }
    }
  }
}

/// Keys of the appended groups: (row, file position of the first insertion).
__global__ void appendKeys(ApplyParams P, ApplyGroups g, long long B, const int *appFlag,
                           const int *appPos, unsigned long long *keys, int *vals, int *counters) {
  const int G = counters[kApplyGroups];
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; x < B; x += stride) {
    if (x < G && appFlag[x]) {
      const int a = appPos[x];
      keys[a] = (static_cast<unsigned long long>(g.u[x]) << P.ibits) |
                static_cast<unsigned>(g.firstIns[x]);
      vals[a] = static_cast<int>(x);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) counters[kApplyAppended] = appPos[B];
}

/// Rank of each appended group among its row's appended groups.
__global__ void appendRanks(ApplyParams P, const unsigned long long *keys, const int *vals,
                            long long B, int *rank, const int *counters) {
  const int A = counters[kApplyAppended];
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long a = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; a < A; a += stride) {
    const unsigned long long rowKey = keys[a] >> P.ibits;
    int lo = 0, hi = static_cast<int>(a);
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((keys[mid] >> P.ibits) < rowKey) lo = mid + 1; else hi = mid;
    }
    rank[vals[a]] = static_cast<int>(a) - lo;
  }
}

__global__ void newDegrees(ApplyParams P, const int *removed, const int *appended, int *deg,
                           const int *counters) {
  const bool stop = stopped(counters + kApplyInvalid);
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long u = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; u < P.n; u += stride) {
    deg[u] = stop ? 0 : P.row[u + 1] - P.row[u] - removed[u] + appended[u];
  }
}

/// Untouched rows keep their edges: CTA windows of kCopyRows rows, threads
/// stride over the window's edges and find their row in shared memory.
__global__ void __launch_bounds__(256) copyUntouched(ApplyParams P, const unsigned char *touched,
                                                     const int *counters) {
  if (stopped(counters + kApplyInvalid)) return;
  __shared__ int sRow[kCopyRows + 1];
  __shared__ int sNew[kCopyRows];
  const int K = P.K;
  for (long long r0 = static_cast<long long>(blockIdx.x) * kCopyRows; r0 < P.n;
       r0 += static_cast<long long>(gridDim.x) * kCopyRows) {
    const int rows = static_cast<int>(P.n - r0 < kCopyRows ? P.n - r0 : kCopyRows);
    for (int i = threadIdx.x; i <= rows; i += blockDim.x) sRow[i] = P.row[r0 + i];
    for (int i = threadIdx.x; i < rows; i += blockDim.x) {
      sNew[i] = touched[r0 + i] ? -1 : P.newRow[r0 + i];
    }
    __syncthreads();
    const int e0 = sRow[0], e1 = sRow[rows];
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
      int lo = 0, hi = rows;  // last row with sRow[row] <= e
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (sRow[mid] <= e) lo = mid; else hi = mid;
      }
      const int base = sNew[lo];
      if (base < 0) continue;
      const int out = base + (e - sRow[lo]);
      P.newCol[out] = P.col[e];
      for (int k = 0; k < K; ++k) {
        P.newW[static_cast<long long>(out) * K + k] = P.w[static_cast<long long>(e) * K + k];
      }
    }
    __syncthreads();
  }
}

/// Touched rows: one warp per row compacts the live edges in order (with
/// the last insertion's weights on an overwritten edge), then writes the
/// appended edges.
__global__ void copyTouched(ApplyParams P, ApplyGroups g, ApplyRows r, const unsigned char *slot,
                            const int *appFlag, const int *appRank, const int *counters) {
  if (stopped(counters + kApplyInvalid)) return;
  const int R = counters[kApplyRows];
  const int lane = threadIdx.x & 31;
  const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  const int K = P.K;
  for (long long k = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); k < R;
       k += warps) {
    const int u = r.row[k];
    const int gs = r.gs[k], ge = r.gs[k + 1];
    const int b = P.row[u], e1 = P.row[u + 1];
    int out = P.newRow[u];
    for (int c0 = b; c0 < e1; c0 += 32) {
      const int e = c0 + lane;
      const int s = e < e1 ? slot[e] : 1;
      const unsigned live = __ballot_sync(kFullMask, s != 1);
      if (s != 1) {
        const int o = out + __popc(live & ((1u << lane) - 1u));
        const int v = P.col[e];
        P.newCol[o] = v;
        const int *src = P.w + static_cast<long long>(e) * K;
        if (s == 2) {
          const int x = findGroup(g.v, gs, ge, v);
          src = P.insW + static_cast<long long>(g.lastIns[x]) * K;
        }
        for (int q = 0; q < K; ++q) P.newW[static_cast<long long>(o) * K + q] = src[q];
      }
      out += __popc(live);
    }
    // out = newRow[u] + deg - removed[u]: the appended edges follow
    for (int x = gs + lane; x < ge; x += 32) {
      if (!appFlag[x]) continue;
      const int o = out + appRank[x];
      P.newCol[o] = g.v[x];
      const int *src = P.insW + static_cast<long long>(g.lastIns[x]) * K;
      for (int q = 0; q < K; ++q) P.newW[static_cast<long long>(o) * K + q] = src[q];
    }
  }
}

/// Largest weight (original edges and insertions) and weight sum (original
/// edges) per objective (reference src/mospUpdate.cu:104-136).
__global__ void weightStats(ApplyParams P, long long *stats) {
  __shared__ long long sMax[32], sSum[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long T = static_cast<long long>(gridDim.x) * blockDim.x;
  for (int k = 0; k < P.K; ++k) {
    long long mx = 1, sum = 0;
    for (long long e = tid; e < P.m; e += T) {
      const long long w = P.w[e * P.K + k];
      mx = w > mx ? w : mx;
      sum += w;
    }
    for (long long i = tid; i < P.nIns; i += T) {
      const long long w = P.insW[i * P.K + k];
      mx = w > mx ? w : mx;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const long long om = __shfl_down_sync(kFullMask, mx, off);
      mx = om > mx ? om : mx;
      sum += __shfl_down_sync(kFullMask, sum, off);
    }
    if (lane == 0) {
      sMax[warp] = mx;
      sSum[warp] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w2 = 1; w2 < static_cast<int>(blockDim.x >> 5); ++w2) {
        mx = sMax[w2] > mx ? sMax[w2] : mx;
        sum += sSum[w2];
      }
      atomicMax(&stats[k], mx);
      atomicAdd(reinterpret_cast<unsigned long long *>(&stats[kMaxK + k]),
                static_cast<unsigned long long>(sum));
    }
    __syncthreads();
  }
}

int bitsFor(long long x) {
  int b = 1;
  while ((1LL << b) <= x) ++b;
  return b;
}

template <typename T>
T *carve(unsigned char *&p, long long count) {
  T *r = reinterpret_cast<T *>(p);
  p += (static_cast<long long>(sizeof(T)) * (count > 0 ? count : 1) + 255) / 256 * 256;
  return r;
}

struct Layout {
  unsigned long long *keysA, *keysB, *appKeysA, *appKeysB;
  int *valsA, *valsB, *appValsA, *appValsB;
  int *flags, *pos, *hist, *aux, *rowHead, *rowPos, *appFlag, *appPos, *appRank;
  int *removed, *appended, *deg;
  unsigned char *touched, *slot;
  int *counters;
  long long *stats;
  ApplyGroups g;
  ApplyRows r;
  long long tiles;
  unsigned char *end;
};

Layout layoutFor(unsigned char *base, long long n, long long m, long long B) {
  Layout L;
  unsigned char *p = base;
  const long long tiles = (B + kSortThreads - 1) / kSortThreads;
  L.tiles = tiles;
  L.counters = carve<int>(p, 64);
  L.stats = carve<long long>(p, 2 * kMaxK);
  L.keysA = carve<unsigned long long>(p, B);
  L.keysB = carve<unsigned long long>(p, B);
  L.appKeysA = carve<unsigned long long>(p, B);
  L.appKeysB = carve<unsigned long long>(p, B);
  L.valsA = carve<int>(p, B);
  L.valsB = carve<int>(p, B);
  L.appValsA = carve<int>(p, B);
  L.appValsB = carve<int>(p, B);
  L.flags = carve<int>(p, B + 1);
  L.pos = carve<int>(p, B + 1);
  L.hist = carve<int>(p, 256 * tiles + 1);
  const long long longest = 256 * tiles + 1 > n + 1 ? 256 * tiles + 1 : n + 1;
  L.aux = carve<int>(p, (longest + kScanChunk - 1) / kScanChunk + 1);
  L.rowHead = carve<int>(p, B + 1);
  L.rowPos = carve<int>(p, B + 1);
  L.appFlag = carve<int>(p, B + 1);
  L.appPos = carve<int>(p, B + 1);
  L.appRank = carve<int>(p, B + 1);
  L.g.start = carve<int>(p, B + 1);
  L.g.u = carve<int>(p, B);
  L.g.v = carve<int>(p, B);
  L.g.cD = carve<int>(p, B);
  L.g.cI = carve<int>(p, B);
  L.g.firstIns = carve<int>(p, B);
  L.g.lastIns = carve<int>(p, B);
  L.g.occ = carve<int>(p, B);
  L.g.first = carve<int>(p, B);
  L.r.row = carve<int>(p, B + 1);
  L.r.gs = carve<int>(p, B + 1);
  L.r.deg = carve<int>(p, B + 1);
  L.r.off = carve<int>(p, B + 1);
  L.removed = carve<int>(p, n);
  L.appended = carve<int>(p, n);
  L.deg = carve<int>(p, n + 1);
  L.touched = carve<unsigned char>(p, n);
  L.slot = carve<unsigned char>(p, m);
  L.end = p;
  return L;
}

/// Stable sort of `count` (<= capacity) pairs over the low `bits` key bits;
/// the result ends in (*keys, *vals) (the buffers are swapped as needed).
cudaError_t radixSort(unsigned long long *&keys, int *&vals, unsigned long long *&keysTmp,
                      int *&valsTmp, const int *count, long long capacity, int bits, int *hist,
                      int *aux, const int *invalid, cudaStream_t s) {
  const long long tiles = (capacity + kSortThreads - 1) / kSortThreads;
  if (tiles == 0) return cudaSuccess;
  for (int shift = 0; shift < bits; shift += 8) {
    radixHistogram<<<static_cast<unsigned>(tiles), kSortThreads, 0, s>>>(keys, count, shift,
                                                                        static_cast<int>(tiles), hist,
                                                                        invalid);
    cudaError_t err = exclusiveScan(hist, hist, 256 * tiles, aux, s);
    if (err != cudaSuccess) return err;
    radixScatter<<<static_cast<unsigned>(tiles), kSortThreads, 0, s>>>(
        keys, vals, count, shift, static_cast<int>(tiles), hist, keysTmp, valsTmp, invalid);
    std::swap(keys, keysTmp);
    std::swap(vals, valsTmp);
  }
  return cudaGetLastError();
}

unsigned gridFor(long long items, int threads, int sms) {
  const long long want = (items + threads - 1) / threads;
  const long long cap = static_cast<long long>(sms) * 8;
  return static_cast<unsigned>(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

size_t applyScratchBytes(long long n, long long m, long long nIns, long long nDel) {
  // lay the buffers out from a 256-aligned dummy base to measure the span
  unsigned char *base = reinterpret_cast<unsigned char *>(static_cast<uintptr_t>(256));
  Layout L = layoutFor(base, n, m, nIns + nDel);
  return static_cast<size_t>(L.end - base) + 256;
}

cudaError_t applyBatchGpu(ApplyParams P, void *scratch, int sms, cudaStream_t s, int *hostCounters,
                          long long *hostStats) {
  const long long B = static_cast<long long>(P.nDel) + P.nIns;
  Layout L = layoutFor(static_cast<unsigned char *>(scratch), P.n, P.m, B);
  P.vbits = bitsFor(P.n);
  P.ibits = bitsFor(P.nIns);
  cudaError_t err = cudaMemsetAsync(L.counters, 0, 64 * sizeof(int), s);
  if (err == cudaSuccess) err = cudaMemsetAsync(L.removed, 0, sizeof(int) * P.n, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(L.appended, 0, sizeof(int) * P.n, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(L.touched, 0, P.n, s);
  if (err == cudaSuccess && P.m > 0) err = cudaMemsetAsync(L.slot, 0, P.m, s);
  if (err != cudaSuccess) return err;
  int *invalid = L.counters + kApplyInvalid;
  const int T = 256;
  const unsigned gB = gridFor(B, T, sms);
  if (B > 0) {
    makeKeys<<<gB, T, 0, s>>>(P, L.keysA, L.valsA, L.counters);
    unsigned long long *keys = L.keysA, *keysTmp = L.keysB;
    int *vals = L.valsA, *valsTmp = L.valsB;
    if ((err = radixSort(keys, vals, keysTmp, valsTmp, L.counters + kApplyEntries, B, 2 * P.vbits,
                         L.hist, L.aux, invalid, s)) != cudaSuccess) {
      return err;
    }
    P.sortedVals = vals;
    groupHeads<<<gB, T, 0, s>>>(keys, B, L.flags, invalid);
    if ((err = exclusiveScan(L.flags, L.pos, B, L.aux, s)) != cudaSuccess) return err;
    groupStarts<<<gB, T, 0, s>>>(L.flags, L.pos, B, L.g.start, L.counters);
    groupInfo<<<gB, T, 0, s>>>(P, keys, vals, L.g, B, L.rowHead, L.counters);
    if ((err = exclusiveScan(L.rowHead, L.rowPos, B, L.aux, s)) != cudaSuccess) return err;
    touchedRows<<<gB, T, 0, s>>>(P, L.g, B, L.rowHead, L.rowPos, L.r, L.touched, L.counters);
    if ((err = exclusiveScan(L.r.deg, L.r.off, B, L.aux, s)) != cudaSuccess) return err;
    countOccurrences<<<static_cast<unsigned>(sms) * 4, T, 0, s>>>(P, L.g, L.r, L.counters);
    resolveGroups<<<gB, T, 0, s>>>(P, L.g, B, L.slot, L.removed, L.appended, L.appFlag,
                                   L.counters);
    if ((err = exclusiveScan(L.appFlag, L.appPos, B, L.aux, s)) != cudaSuccess) return err;
    appendKeys<<<gB, T, 0, s>>>(P, L.g, B, L.appFlag, L.appPos, L.appKeysA, L.appValsA,
                                L.counters);
    unsigned long long *ak = L.appKeysA, *akTmp = L.appKeysB;
    int *av = L.appValsA, *avTmp = L.appValsB;
    if ((err = radixSort(ak, av, akTmp, avTmp, L.counters + kApplyAppended, B,
                         P.vbits + P.ibits, L.hist, L.aux, invalid, s)) != cudaSuccess) {
      return err;
    }
    appendRanks<<<gB, T, 0, s>>>(P, ak, av, B, L.appRank, L.counters);
  }
  newDegrees<<<gridFor(P.n, T, sms), T, 0, s>>>(P, L.removed, L.appended, L.deg, L.counters);
  if ((err = exclusiveScan(L.deg, P.newRow, P.n, L.aux, s)) != cudaSuccess) return err;
  copyUntouched<<<gridFor(P.n, kCopyRows, sms), 256, 0, s>>>(P, L.touched, L.counters);
  if (B > 0) {
    copyTouched<<<static_cast<unsigned>(sms) * 4, 256, 0, s>>>(P, L.g, L.r, L.slot, L.appFlag,
                                                              L.appRank, L.counters);
  }
  if (hostStats != nullptr) {
    if ((err = cudaMemsetAsync(L.stats, 0, 2 * kMaxK * sizeof(long long), s)) != cudaSuccess) {
      return err;
    }
    weightStats<<<static_cast<unsigned>(sms) * 2, 512, 0, s>>>(P, L.stats);
  }
  if ((err = cudaGetLastError()) != cudaSuccess) return err;
  err = cudaMemcpyAsync(hostCounters, L.counters, kApplyCounters * sizeof(int),
                        cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess && hostStats != nullptr) {
    err = cudaMemcpyAsync(hostStats, L.stats, P.K * sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) {
      err = cudaMemcpyAsync(hostStats + P.K, L.stats + kMaxK, P.K * sizeof(long long),
                            cudaMemcpyDeviceToHost, s);
    }
  }
  if (err == cudaSuccess) {
    err = cudaMemcpyAsync(hostCounters + kApplyCounters, P.newRow + P.n, sizeof(int),
                          cudaMemcpyDeviceToHost, s);
  }
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  return err;
}

}  // namespace mospb200
