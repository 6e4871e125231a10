// server.cpp - serving loop for resident graphs (mosp_server_*, include/
// mosp_b200.h). No counterpart in the reference, which runs one update per
// process invocation.
//
// Graphs, their K SOSP trees and their combined (MOSP) tree stay in device
// memory. Clients submit change batches from any thread; worker threads
// (each with its own workspace and CUDA stream) take the pending batches of
// one graph at a time, oldest first:
//   * continuous batching: a worker picks up whatever is pending when it
//     becomes free, so requests that arrive while others run are admitted as
//     soon as a worker and device memory are free;
//   * coalescing: all pending batches of a graph go through one pass - each
//     batch is applied to the device CSR in order (Step 1 on the GPU), then
//     ONE engine update runs with the union of their change lists (every
//     deletion, every insertion whose weight-increase bit is set in its own
//     application, every insertion head). Over-invalidating is safe: the
//     update's fixed point is the canonical tree of the final graph whatever
//     set of subtrees is recomputed, so the result equals applying the
//     batches one by one;
//   * admission by free device memory: a pass starts only when the memory it
//     may allocate (CSR growth, Step 1 scratch, staging) fits in the free
//     device memory minus a reserve, unless nothing else is running;
//   * overlap on the device: with W > 1 workers each worker's persistent
//     cooperative launches (graph build, update, combined graph, costs) use
//     at most SMs / W CTAs of one SM each, so the grids of W passes fit on
//     the GPU side by side and run at the same time on disjoint SMs (each
//     grid waits at its barriers only for its own CTAs). Full-grid work
//     (adding a graph, or all passes when overlap is off) takes the engine
//     lock exclusively; passes take it shared. Host work, copies and Step 1
//     kernels of all workers overlap with the engine launches.
// A response carries the graph's combined tree after the pass that included
// the request and the version (number of batches applied to the graph) of
// that state; equal versions give equal results however the batches were
// grouped.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <atomic>
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "hostCore.h"
#include "mosp_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

constexpr long long kPassChanges = 262144;  // changes per coalesced pass (after the first request)

double usBetween(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::micro>(b - a).count();
}

/// Set of (u, v) edge keys for the merge's conflict check: open addressing
/// with linear probing in one flat array (no allocation per key; a pass can
/// insert a few hundred thousand keys). Keys are u << 32 | v with u, v
/// non-negative ints, so the all-ones word marks an empty slot.
class EdgeKeySet {
 public:
  static unsigned long long key(int u, int v) {
    return (static_cast<unsigned long long>(static_cast<unsigned>(u)) << 32) |
           static_cast<unsigned>(v);
  }
  /// Empties the set, sized for `expected` keys at a load of at most 1/2.
  void reset(size_t expected) {
    size_t cap = 64;
    while (cap < 2 * expected + 2) cap <<= 1;
    if (slots_.size() == cap) {
      std::fill(slots_.begin(), slots_.end(), kEmpty);
    } else {
      slots_.assign(cap, kEmpty);
    }
    count_ = 0;
  }
  bool empty() const { return count_ == 0; }
  void insert(unsigned long long k) {
    if (2 * (count_ + 1) > slots_.size()) rehash(2 * slots_.size());
    size_t i = slot(k);
    while (slots_[i] != kEmpty) {
      if (slots_[i] == k) return;
      i = (i + 1) & (slots_.size() - 1);
    }
    slots_[i] = k;
    ++count_;
  }
  bool contains(unsigned long long k) const {
    if (count_ == 0) return false;
    size_t i = slot(k);
    while (slots_[i] != kEmpty) {
      if (slots_[i] == k) return true;
      i = (i + 1) & (slots_.size() - 1);
    }
    return false;
  }

 private:
  static constexpr unsigned long long kEmpty = ~0ULL;
  size_t slot(unsigned long long k) const {
    // 64-bit finaliser of MurmurHash3 (public domain), to spread the ids
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return static_cast<size_t>(k) & (slots_.size() - 1);
  }
  void rehash(size_t cap) {
    std::vector<unsigned long long> old(cap, kEmpty);
    old.swap(slots_);
    count_ = 0;
    for (unsigned long long k : old) {
      if (k != kEmpty) insert(k);
    }
  }
  std::vector<unsigned long long> slots_;
  size_t count_ = 0;
};

struct Result {
  std::vector<long long> combDist;
  std::vector<int> combParent;
};

struct Request {
  long long ticket = 0;
  int graph = 0;
  std::vector<int> insFrom, insTo, insW, delFrom, delTo;
  Clock::time_point submit, start, done;
  bool finished = false;
  int status = MOSP_OK;
  std::string error;
  long long version = 0;
  int coalesced = 0;
  std::shared_ptr<Result> result;
};

/// Device memory owned by the server, freed with it.
template <typename T>
int grow(T *&ptr, long long &cap, long long need, std::string &err) {
  if (need <= cap && ptr != nullptr) return MOSP_OK;
  const long long want = std::max<long long>(need + need / 4 + 1024, 1);
  T *p = nullptr;
  if (cudaMalloc(reinterpret_cast<void **>(&p), static_cast<size_t>(want) * sizeof(T)) !=
      cudaSuccess) {
    cudaGetLastError();
    err = "device allocation of " + std::to_string(want * sizeof(T)) + " bytes failed";
    return MOSP_ERR_OOM;
  }
  if (ptr != nullptr) cudaFree(ptr);
  ptr = p;
  cap = want;
  return MOSP_OK;
}

struct Graph {
  int id = 0, n = 0, KG = 0, K = 0, source = 0;
  std::vector<int> pref;
  long long m = 0;
  // out-CSR with edge-major weights, double buffered for Step 1
  long long edgeCap = 0;
  int *row[2] = {nullptr, nullptr}, *col[2] = {nullptr, nullptr}, *w[2] = {nullptr, nullptr};
  int cur = 0;
  // derived device graph of the current CSR (weight columns, reverse CSR)
  long long derivedCap = 0;
  int *outW = nullptr, *inRow = nullptr, *inCol = nullptr, *inW = nullptr;
  long long *dist = nullptr, *combDist = nullptr;
  int *parent = nullptr, *combParent = nullptr;
  std::vector<long long> maxWeight, weightSum;
  long long version = 0;
  bool busy = false;
  bool broken = false;
  std::string brokenWhy;
  std::deque<std::shared_ptr<Request>> pending;

  void release() {
    for (int b = 0; b < 2; ++b) {
      if (row[b]) cudaFree(row[b]);
      if (col[b]) cudaFree(col[b]);
      if (w[b]) cudaFree(w[b]);
    }
    for (void *p : {static_cast<void *>(outW), static_cast<void *>(inRow),
                    static_cast<void *>(inCol), static_cast<void *>(inW),
                    static_cast<void *>(dist), static_cast<void *>(combDist),
                    static_cast<void *>(parent), static_cast<void *>(combParent)}) {
      if (p) cudaFree(p);
    }
  }
};

/// A device array that grows on demand, at least doubling (a reallocation's
/// cudaFree waits for the whole device, so it should be rare); contents are
/// not kept.
template <typename T>
struct Buf {
  T *p = nullptr;
  long long cap = 0;
  int fit(long long need, std::string &err) {
    return grow(p, cap, need <= cap ? need : std::max(need, 2 * cap), err);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

/// Per-worker device and pinned staging, grown on demand.
struct Staging {
  Buf<int> insFrom, insTo, insW, delFrom, delTo, chFrom, chTo, heads;
  Buf<unsigned> mask;
  long long hostCap = 0;
  unsigned char *host = nullptr;  // pinned

  void release() {
    for (Buf<int> *b : {&insFrom, &insTo, &insW, &delFrom, &delTo, &chFrom, &chTo, &heads}) {
      b->release();
    }
    mask.release();
    if (host) cudaFreeHost(host);
  }
  int hostBytes(long long need, std::string &err) {
    if (need <= hostCap && host != nullptr) return MOSP_OK;
    const long long want = std::max(need + need / 4, 2 * hostCap) + 4096;
    unsigned char *p = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void **>(&p), static_cast<size_t>(want), 0) != cudaSuccess) {
      cudaGetLastError();
      err = "pinned allocation failed";
      return MOSP_ERR_OOM;
    }
    if (host) cudaFreeHost(host);
    host = p;
    hostCap = want;
    return MOSP_OK;
  }
};

unsigned long long mix64(unsigned long long x) {
  x ^= x >> 31;
  x *= 0x7fb5d329728ea185ULL;
  x ^= x >> 27;
  x *= 0x81dadef4bc2dd44dULL;
  x ^= x >> 33;
  return x;
}

/// Order-independent checksum of a tree: the sum over v of a mixed hash of
/// (v, dist[v]) and of (v, parent[v]).
unsigned long long checksumOf(const long long *dist, const int *parent, int n) {
  unsigned long long h = 0;
  for (int v = 0; v < n; ++v) {
    const unsigned long long key = static_cast<unsigned long long>(v) * 0x9e3779b97f4a7c15ULL;
    h += mix64(key ^ static_cast<unsigned long long>(dist[v])) +
         mix64(~key ^ static_cast<unsigned long long>(static_cast<unsigned>(parent[v])));
  }
  return h;
}

}  // namespace

struct mosp_server {
  int device = 0;
  int maxCoalesce = 64;
  long long reserveBytes = 0;
  std::mutex mu;
  std::condition_variable workCv, doneCv;
  // shared by passes whose grids are limited to a worker's SM share,
  // exclusive for full-grid launches
  std::shared_mutex gpuLock;
  bool overlap = true;   // passes of different workers run side by side
  int workers = 1;
  // largest resident graph: every worker reserves its workspace and staging
  // for it before its next pass (reserveEpoch counts the growths), so that
  // passes allocate nothing - an allocation or free waits for the whole
  // device, including the other workers' passes
  int maxN = 0, maxK = 0;
  long long maxM = 0;
  int reserveEpoch = 0;
  std::atomic<int> enginesActive{0};
  bool stop = false;
  int running = 0;
  std::vector<std::unique_ptr<Graph>> graphs;
  std::unordered_map<long long, std::shared_ptr<Request>> tickets;
  long long nextTicket = 1;
  std::vector<std::thread> threads;
  mosp_workspace *setupWs = nullptr;
  cudaStream_t setupStream = nullptr;
  mosp_server_stats stats{};

  ~mosp_server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    workCv.notify_all();
    for (std::thread &t : threads) t.join();
    cudaSetDevice(device);
    for (auto &g : graphs) g->release();
    if (setupWs) mosp_workspace_destroy(setupWs);
    if (setupStream) cudaStreamDestroy(setupStream);
  }

  /// Bytes a pass over `reqs` of graph g may allocate.
  long long passBytes(const Graph &g, const std::deque<std::shared_ptr<Request>> &q,
                      size_t count) const {
    long long ins = 0, del = 0;
    for (size_t i = 0; i < count; ++i) {
      ins += static_cast<long long>(q[i]->insFrom.size());
      del += static_cast<long long>(q[i]->delFrom.size());
    }
    const long long b = ins + del;
    long long bytes = b * 200 + static_cast<long long>(g.n) * 16 + g.m + (4LL << 20);
    const long long edges = g.m + ins;
    if (edges > g.edgeCap) bytes += 2 * edges * (8 + 4LL * g.KG);
    if (edges > g.derivedCap) bytes += edges * (4 + 8LL * g.KG);
    return bytes;
  }

  /// The graph whose oldest pending request is the oldest, among the idle
  /// graphs whose pass fits in free memory (any, when nothing runs).
  Graph *pick() {
    Graph *best = nullptr;
    size_t freeB = 0, totalB = 0;
    bool haveInfo = cudaMemGetInfo(&freeB, &totalB) == cudaSuccess;
    if (!haveInfo) cudaGetLastError();
    for (auto &gp : graphs) {
      Graph &g = *gp;
      if (g.busy || g.pending.empty()) continue;
      if (best != nullptr && best->pending.front()->submit <= g.pending.front()->submit) continue;
      const size_t count = std::min<size_t>(g.pending.size(), static_cast<size_t>(maxCoalesce));
      const long long need = passBytes(g, g.pending, count);
      if (running > 0 && haveInfo &&
          static_cast<long long>(freeB) - reserveBytes < need) {
        ++stats.deferred;
        continue;
      }
      best = &g;
    }
    return best;
  }

  void worker(int index);
  int runPass(mosp_workspace *ws, cudaStream_t s, Staging &st, Graph &g,
              std::vector<std::shared_ptr<Request>> &group, std::string &err);
};

int mosp_server::runPass(mosp_workspace *ws, cudaStream_t s, Staging &st, Graph &g,
                         std::vector<std::shared_ptr<Request>> &group, std::string &err) {
  const int n = g.n, KG = g.KG, K = g.K;
  std::vector<std::vector<int>> chFrom(K), chTo(K);
  std::vector<int> heads;
  std::vector<unsigned> mask;
  std::vector<long long> mx(KG, 1), sum(KG, 0);
  bool firstApply = true;
  int rc = MOSP_OK;
  const Clock::time_point tStart = Clock::now();
  auto cuda = [&err](cudaError_t e, const char *what) {
    if (e == cudaSuccess) return MOSP_OK;
    cudaGetLastError();
    err = std::string("CUDA error: ") + cudaGetErrorString(e) + " (" + what + ")";
    return MOSP_ERR_CUDA;
  };
  // The group's batches merge into one batch (deletions of all, then
  // insertions of all, each in submission order) up to the first batch
  // that deletes an edge an earlier batch of the merge inserted: until
  // then, applying the merge equals applying the batches one by one
  // (later insertions win, appended edges keep their order, repeated
  // deletions take successive occurrences). A conflict starts a new merge.
  struct Merged {
    std::vector<int> insFrom, insTo, insW, delFrom, delTo;
  };
  std::vector<Merged> merges(1);
  {
    size_t groupInserts = 0;
    for (auto &q : group) groupInserts += q->insFrom.size();
    EdgeKeySet inserted;
    inserted.reset(groupInserts);
    auto key = EdgeKeySet::key;
    for (auto &q : group) {
      bool conflict = false;
      for (size_t i = 0; i < q->delFrom.size() && !conflict && !inserted.empty(); ++i) {
        conflict = inserted.contains(key(q->delFrom[i], q->delTo[i]));
      }
      if (conflict) {
        merges.emplace_back();
        inserted.reset(groupInserts);
      }
      Merged &mg = merges.back();
      mg.insFrom.insert(mg.insFrom.end(), q->insFrom.begin(), q->insFrom.end());
      mg.insTo.insert(mg.insTo.end(), q->insTo.begin(), q->insTo.end());
      mg.insW.insert(mg.insW.end(), q->insW.begin(), q->insW.end());
      mg.delFrom.insert(mg.delFrom.end(), q->delFrom.begin(), q->delFrom.end());
      mg.delTo.insert(mg.delTo.end(), q->delTo.begin(), q->delTo.end());
      for (size_t i = 0; i < q->insFrom.size(); ++i) inserted.insert(key(q->insFrom[i], q->insTo[i]));
    }
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    stats.applies += static_cast<long long>(merges.size());
  }
  for (const Merged &merged : merges) {
    const Merged *r = &merged;
    const long long nIns = static_cast<long long>(r->insFrom.size());
    const long long nDel = static_cast<long long>(r->delFrom.size());
    // stage the batch through pinned memory
    const long long hb = (3 * nIns + nIns * KG + 2 * nDel) * 4;
    if ((rc = st.hostBytes(hb, err)) != MOSP_OK) return rc;
    if ((rc = st.insFrom.fit(nIns, err)) || (rc = st.insTo.fit(nIns, err)) ||
        (rc = st.insW.fit(nIns * KG, err)) || (rc = st.delFrom.fit(nDel, err)) ||
        (rc = st.delTo.fit(nDel, err)) || (rc = st.mask.fit(nIns, err))) {
      return rc;
    }
    unsigned char *h = st.host;
    auto put = [&h](const std::vector<int> &v) {
      std::memcpy(h, v.data(), v.size() * sizeof(int));
      int *p = reinterpret_cast<int *>(h);
      h += v.size() * sizeof(int);
      return p;
    };
    int *hIf = put(r->insFrom), *hIt = put(r->insTo), *hIw = put(r->insW);
    int *hDf = put(r->delFrom), *hDt = put(r->delTo);
    if ((rc = cuda(cudaMemcpyAsync(st.insFrom.p, hIf, nIns * 4, cudaMemcpyHostToDevice, s), "upload")) ||
        (rc = cuda(cudaMemcpyAsync(st.insTo.p, hIt, nIns * 4, cudaMemcpyHostToDevice, s), "upload")) ||
        (rc = cuda(cudaMemcpyAsync(st.insW.p, hIw, nIns * KG * 4, cudaMemcpyHostToDevice, s),
                   "upload")) ||
        (rc = cuda(cudaMemcpyAsync(st.delFrom.p, hDf, nDel * 4, cudaMemcpyHostToDevice, s), "upload")) ||
        (rc = cuda(cudaMemcpyAsync(st.delTo.p, hDt, nDel * 4, cudaMemcpyHostToDevice, s), "upload"))) {
      return rc;
    }
    // room for the updated CSR in the other buffer (both grow together)
    const long long need = g.m + nIns;
    if (need > g.edgeCap) {
      long long capA = 0, capB = 0, capC = 0, capD = 0;
      int *nc = nullptr, *nw = nullptr, *oc = nullptr, *ow = nullptr;
      if ((rc = grow(nc, capA, need, err)) != MOSP_OK) return rc;
      if ((rc = grow(nw, capB, capA * KG, err)) != MOSP_OK) return rc;
      if ((rc = grow(oc, capC, capA, err)) != MOSP_OK) return rc;
      if ((rc = grow(ow, capD, capA * KG, err)) != MOSP_OK) return rc;
      if ((rc = cuda(cudaMemcpyAsync(nc, g.col[g.cur], g.m * 4, cudaMemcpyDeviceToDevice, s), "copy")) ||
          (rc = cuda(cudaMemcpyAsync(nw, g.w[g.cur], g.m * KG * 4, cudaMemcpyDeviceToDevice, s),
                     "copy")) ||
          (rc = cuda(cudaStreamSynchronize(s), "copy"))) {
        return rc;
      }
      cudaFree(g.col[g.cur]);
      cudaFree(g.w[g.cur]);
      cudaFree(g.col[1 - g.cur]);
      cudaFree(g.w[1 - g.cur]);
      g.col[g.cur] = nc;
      g.w[g.cur] = nw;
      g.col[1 - g.cur] = oc;
      g.w[1 - g.cur] = ow;
      g.edgeCap = capA;
    }
    const int o = 1 - g.cur;
    int newM = 0;
    long long amx[MOSP_MAX_OBJECTIVES], asum[MOSP_MAX_OBJECTIVES];
    rc = mosp_apply_batch_device(ws, n, KG, static_cast<int>(g.m), g.row[g.cur], g.col[g.cur],
                                 g.w[g.cur], static_cast<int>(nIns), st.insFrom.p, st.insTo.p,
                                 st.insW.p, static_cast<int>(nDel), st.delFrom.p, st.delTo.p,
                                 g.row[o], g.col[o], g.w[o], g.edgeCap, &newM, st.mask.p, amx, asum,
                                 s);
    if (rc != MOSP_OK) {
      err = mosp_last_error();
      return rc;
    }
    g.cur = o;
    g.m = newM;
    for (int k = 0; k < KG; ++k) {
      mx[k] = std::max(mx[k], amx[k]);
      if (firstApply) sum[k] = asum[k];
    }
    firstApply = false;
    mask.resize(static_cast<size_t>(nIns));
    if (nIns > 0 &&
        (rc = cuda(cudaMemcpy(mask.data(), st.mask.p, nIns * 4, cudaMemcpyDeviceToHost), "mask"))) {
      return rc;
    }
    for (int k = 0; k < K; ++k) {
      chFrom[k].insert(chFrom[k].end(), r->delFrom.begin(), r->delFrom.end());
      chTo[k].insert(chTo[k].end(), r->delTo.begin(), r->delTo.end());
      for (long long i = 0; i < nIns; ++i) {
        if (mask[i] & (1u << k)) {
          chFrom[k].push_back(r->insFrom[i]);
          chTo[k].push_back(r->insTo[i]);
        }
      }
    }
    heads.insert(heads.end(), r->insTo.begin(), r->insTo.end());
  }
  for (int k = 0; k < KG; ++k) g.maxWeight[k] = std::max(g.maxWeight[k], mx[k]);
  if (!group.empty()) g.weightSum = sum;

  // change lists and heads to the device
  std::vector<int> off(K + 1, 0), allFrom, allTo;
  for (int k = 0; k < K; ++k) {
    allFrom.insert(allFrom.end(), chFrom[k].begin(), chFrom[k].end());
    allTo.insert(allTo.end(), chTo[k].begin(), chTo[k].end());
    off[k + 1] = static_cast<int>(allFrom.size());
  }
  if ((rc = st.chFrom.fit(static_cast<long long>(allFrom.size()), err)) ||
      (rc = st.chTo.fit(static_cast<long long>(allTo.size()), err)) ||
      (rc = st.heads.fit(static_cast<long long>(heads.size()), err))) {
    return rc;
  }
  if ((rc = cuda(cudaMemcpy(st.chFrom.p, allFrom.data(), allFrom.size() * 4, cudaMemcpyHostToDevice),
                 "lists")) ||
      (rc = cuda(cudaMemcpy(st.chTo.p, allTo.data(), allTo.size() * 4, cudaMemcpyHostToDevice),
                 "lists")) ||
      (rc = cuda(cudaMemcpy(st.heads.p, heads.data(), heads.size() * 4, cudaMemcpyHostToDevice),
                 "heads"))) {
    return rc;
  }
  // derived device graph of the updated CSR
  if (g.m > g.derivedCap) {
    long long a = 0, b = 0, c = 0;
    if (g.outW) cudaFree(g.outW);
    if (g.inCol) cudaFree(g.inCol);
    if (g.inW) cudaFree(g.inW);
    g.outW = g.inCol = g.inW = nullptr;
    if ((rc = grow(g.inCol, a, g.m, err)) != MOSP_OK) return rc;
    if ((rc = grow(g.outW, b, a * KG, err)) != MOSP_OK) return rc;
    if ((rc = grow(g.inW, c, a * KG, err)) != MOSP_OK) return rc;
    g.derivedCap = a;
  }
  std::vector<long long> delta(K);
  for (int k = 0; k < K; ++k) delta[k] = mosp_default_delta(g.m, n, g.weightSum[k]);
  const Clock::time_point tEngine = Clock::now();
  {
    std::shared_lock<std::shared_mutex> shared(gpuLock, std::defer_lock);
    std::unique_lock<std::shared_mutex> whole(gpuLock, std::defer_lock);
    // with overlap, this worker's share of the SMs for its cooperative
    // grids, so that every worker's grids fit on the GPU together
    const bool side = overlap && workers > 1;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    mosp_workspace_set_grid(ws, side ? std::max(1, sms / workers) : 0, 0);
    if (side) {
      shared.lock();
    } else {
      whole.lock();
    }
    if (enginesActive.fetch_add(1) > 0) {
      std::lock_guard<std::mutex> lk(mu);
      ++stats.overlapped;
    }
    rc = mosp_build_device_graph(ws, n, static_cast<int>(g.m), KG, g.row[g.cur], g.col[g.cur],
                                 g.w[g.cur], g.outW, g.inRow, g.inCol, g.inW, s);
    if (rc == MOSP_OK) {
      rc = mosp_update_device(ws, n, static_cast<int>(g.m), K, g.row[g.cur], g.col[g.cur], g.outW,
                              g.inRow, g.inCol, g.inW, st.chFrom.p, st.chTo.p, off.data(), st.heads.p,
                              static_cast<int>(heads.size()), g.source, delta.data(),
                              g.maxWeight.data(), g.pref.empty() ? nullptr : g.pref.data(), g.dist,
                              g.parent, g.combDist, g.combParent, nullptr, nullptr, s);
    }
    enginesActive.fetch_sub(1);
  }
  if (rc != MOSP_OK) {
    err = mosp_last_error();
    return rc;
  }
  const Clock::time_point tResult = Clock::now();
  // the combined tree back to the host, through pinned staging
  auto res = std::make_shared<Result>();
  res->combDist.resize(n);
  res->combParent.resize(n);
  if ((rc = st.hostBytes(static_cast<long long>(n) * 12, err)) != MOSP_OK) return rc;
  if ((rc = cuda(cudaMemcpyAsync(st.host, g.combDist, static_cast<size_t>(n) * 8,
                                 cudaMemcpyDeviceToHost, s), "download")) ||
      (rc = cuda(cudaMemcpyAsync(st.host + static_cast<size_t>(n) * 8, g.combParent,
                                 static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, s),
                 "download")) ||
      (rc = cuda(cudaStreamSynchronize(s), "download"))) {
    return rc;
  }
  std::memcpy(res->combDist.data(), st.host, static_cast<size_t>(n) * 8);
  std::memcpy(res->combParent.data(), st.host + static_cast<size_t>(n) * 8,
              static_cast<size_t>(n) * 4);
  // (the checksum is computed by mosp_server_wait, in the client's thread)
  const Clock::time_point tDone = Clock::now();
  {
    std::lock_guard<std::mutex> lk(mu);
    stats.apply_us += usBetween(tStart, tEngine);
    stats.engine_us += usBetween(tEngine, tResult);
    stats.result_us += usBetween(tResult, tDone);
  }
  g.version += static_cast<long long>(group.size());
  for (auto &r : group) {
    r->result = res;
    r->version = g.version;
    r->coalesced = static_cast<int>(group.size());
  }
  return MOSP_OK;
}

void mosp_server::worker(int index) {
  (void)index;
  cudaSetDevice(device);
  mosp_workspace *ws = nullptr;
  cudaStream_t s = nullptr;
  Staging st;
  std::string setupErr;
  if (mosp_workspace_create(&ws) != MOSP_OK) setupErr = mosp_last_error();
  // every resident tree is this library's own output (canonical), so the
  // distance-only objectives recover parents only where a pass reaches
  if (setupErr.empty()) mosp_workspace_set_canonical_trees(ws, 1);

  if (setupErr.empty() && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    setupErr = "stream creation failed";
  }
  int reservedEpoch = 0;
  for (;;) {
    std::unique_lock<std::mutex> lk(mu);
    if (setupErr.empty() && reservedEpoch != reserveEpoch) {
      const int n = maxN, K = maxK;
      const long long m = maxM;
      reservedEpoch = reserveEpoch;
      lk.unlock();
      std::string ignored;
      // best effort: a pass that needs more still allocates what it needs
      if (mosp_workspace_reserve_graph(ws, n, m + kPassChanges, K) == MOSP_OK) {
        st.hostBytes(static_cast<long long>(n) * 12, ignored);
      }
      lk.lock();
    }
    Graph *g = nullptr;
    workCv.wait(lk, [&] {
      if (stop || reservedEpoch != reserveEpoch) return true;
      g = pick();
      return g != nullptr;
    });
    if (g == nullptr) {
      if (stop) break;
      continue;  // reserve for a larger graph first
    }
    std::vector<std::shared_ptr<Request>> group;
    // a pass takes up to maxCoalesce requests and, past its first request,
    // no more than kPassChanges changes, which bounds its duration
    long long passChanges = 0;
    while (!g->pending.empty() && static_cast<int>(group.size()) < maxCoalesce) {
      const Request &q = *g->pending.front();
      const long long c = static_cast<long long>(q.insFrom.size() + q.delFrom.size());
      if (!group.empty() && passChanges + c > kPassChanges) break;
      passChanges += c;
      group.push_back(g->pending.front());
      g->pending.pop_front();
    }
    g->busy = true;
    ++running;
    const Clock::time_point start = Clock::now();
    for (auto &r : group) r->start = start;
    const bool broken = g->broken;
    lk.unlock();

    std::string err;
    int rc = MOSP_OK;
    if (!setupErr.empty()) {
      rc = MOSP_ERR_CUDA;
      err = setupErr;
    } else if (broken) {
      rc = MOSP_ERR_INVALID;
      err = "Error: the graph is unusable after an earlier failure: " + g->brokenWhy;
    } else {
      rc = runPass(ws, s, st, *g, group, err);
    }

    lk.lock();
    const Clock::time_point done = Clock::now();
    if (rc != MOSP_OK && !g->broken) {
      g->broken = true;
      g->brokenWhy = err;
    }
    long long changes = 0;
    for (auto &r : group) {
      r->status = rc;
      r->error = err;
      r->done = done;
      r->finished = true;
      changes += static_cast<long long>(r->insFrom.size() + r->delFrom.size());
      r->insFrom.clear();
      r->insTo.clear();
      r->insW.clear();
      r->delFrom.clear();
      r->delTo.clear();
    }
    ++stats.passes;
    stats.requests += static_cast<long long>(group.size());
    stats.changes += changes;
    stats.max_coalesced = std::max<int>(stats.max_coalesced, static_cast<int>(group.size()));
    stats.busy_us += usBetween(start, done);
    g->busy = false;
    --running;
    lk.unlock();
    doneCv.notify_all();
    workCv.notify_all();
  }
  st.release();
  if (s) cudaStreamDestroy(s);
  if (ws) mosp_workspace_destroy(ws);
}

using mospb200::recordFailure;

extern "C" int mosp_server_create(int workers, long long reserve_bytes, int max_coalesce,
                                  mosp_server **out) {
  if (out == nullptr || workers < 1 || workers > 16 || reserve_bytes < 0 || max_coalesce < 1) {
    return recordFailure(MOSP_ERR_INVALID, "Error: invalid server parameters.");
  }
  *out = nullptr;
  auto srv = std::make_unique<mosp_server>();
  if (cudaGetDevice(&srv->device) != cudaSuccess) {
    cudaGetLastError();
    return recordFailure(MOSP_ERR_CUDA, "Error: no CUDA device.");
  }
  srv->reserveBytes = reserve_bytes;
  srv->maxCoalesce = max_coalesce;
  srv->workers = workers;
  if (mosp_workspace_create(&srv->setupWs) != MOSP_OK) return MOSP_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&srv->setupStream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return recordFailure(MOSP_ERR_CUDA, "Error: stream creation failed.");
  }
  for (int i = 0; i < workers; ++i) {
    mosp_server *p = srv.get();
    srv->threads.emplace_back([p, i] { p->worker(i); });
  }
  *out = srv.release();
  return MOSP_OK;
}

extern "C" void mosp_server_destroy(mosp_server *s) { delete s; }

extern "C" int mosp_server_set_overlap(mosp_server *s, int on) {
  if (s == nullptr || on < 0 || on > 1) return recordFailure(MOSP_ERR_INVALID, "Error: invalid overlap mode.");
  std::lock_guard<std::mutex> lk(s->mu);
  s->overlap = on != 0;
  return MOSP_OK;
}

extern "C" int mosp_server_add_graph(mosp_server *s, int n, int KG, int m, const int *h_row,
                                     const int *h_col, const int *h_w, int K, int source,
                                     const int *h_pref, int *graph_id) {
  if (s == nullptr || graph_id == nullptr || n <= 0 || KG < 1 || KG > MOSP_MAX_OBJECTIVES ||
      m < 0 || h_row == nullptr || (m > 0 && (h_col == nullptr || h_w == nullptr)) || K < 1 ||
      K > KG || source < 0 || source >= n || h_row[n] != m) {
    return recordFailure(MOSP_ERR_INVALID, "Error: invalid graph for the server.");
  }
  if (h_pref != nullptr && mosp_preference_scale(h_pref, K) == 0) {
    return recordFailure(MOSP_ERR_INVALID, "Error: invalid preference vector (need K values >= 1).");
  }
  cudaSetDevice(s->device);
  auto g = std::make_unique<Graph>();
  g->n = n;
  g->KG = KG;
  g->K = K;
  g->source = source;
  if (h_pref) g->pref.assign(h_pref, h_pref + K);
  g->m = m;
  g->maxWeight.assign(KG, 1);
  g->weightSum.assign(KG, 0);
  for (long long e = 0; e < m; ++e) {
    for (int k = 0; k < KG; ++k) {
      const int w = h_w[e * KG + k];
      g->maxWeight[k] = std::max<long long>(g->maxWeight[k], w);
      g->weightSum[k] += w;
    }
  }
  std::string err;
  long long rowCap = 0, capA = 0, capB = 0, capC = 0, capD = 0, capE = 0, capF = 0;
  int rc = MOSP_OK;
  auto fail = [&](int code) {
    g->release();
    return recordFailure(code, err.c_str());
  };
  for (int b = 0; b < 2; ++b) {
    rowCap = 0;
    if ((rc = grow(g->row[b], rowCap, n + 1LL, err)) != MOSP_OK) return fail(rc);
  }
  if ((rc = grow(g->col[0], capA, m, err)) != MOSP_OK) return fail(rc);
  if ((rc = grow(g->col[1], capB, capA, err)) != MOSP_OK) return fail(rc);
  if ((rc = grow(g->w[0], capC, capA * KG, err)) != MOSP_OK) return fail(rc);
  if ((rc = grow(g->w[1], capD, capA * KG, err)) != MOSP_OK) return fail(rc);
  g->edgeCap = capA;
  if ((rc = grow(g->inCol, capE, capA, err)) != MOSP_OK) return fail(rc);
  g->derivedCap = capE;
  capF = 0;
  if ((rc = grow(g->outW, capF, capA * KG, err)) != MOSP_OK) return fail(rc);
  capF = 0;
  if ((rc = grow(g->inW, capF, capA * KG, err)) != MOSP_OK) return fail(rc);
  capF = 0;
  if ((rc = grow(g->inRow, capF, n + 1LL, err)) != MOSP_OK) return fail(rc);
  capF = 0;
  if ((rc = grow(g->dist, capF, static_cast<long long>(K) * n, err)) != MOSP_OK) return fail(rc);
  capF = 0;
  if ((rc = grow(g->parent, capF, static_cast<long long>(K) * n, err)) != MOSP_OK) return fail(rc);
  capF = 0;
  if ((rc = grow(g->combDist, capF, n, err)) != MOSP_OK) return fail(rc);
  capF = 0;
  if ((rc = grow(g->combParent, capF, n, err)) != MOSP_OK) return fail(rc);
  if (cudaMemcpy(g->row[0], h_row, (n + 1LL) * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(g->col[0], h_col, static_cast<size_t>(m) * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(g->w[0], h_w, static_cast<size_t>(m) * KG * 4, cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    cudaGetLastError();
    err = "Error: graph upload failed.";
    return fail(MOSP_ERR_CUDA);
  }
  {
    // initial canonical trees and the combined tree on the GPU
    std::unique_lock<std::shared_mutex> gpu(s->gpuLock);
    rc = mosp_build_device_graph(s->setupWs, n, m, KG, g->row[0], g->col[0], g->w[0], g->outW,
                                 g->inRow, g->inCol, g->inW, s->setupStream);
    for (int k = 0; k < K && rc == MOSP_OK; ++k) {
      rc = mosp_sosp_from_scratch(s->setupWs, n, m, g->row[0], g->col[0],
                                  g->outW + static_cast<size_t>(k) * m, source,
                                  mosp_default_delta(m, n, g->weightSum[k]), g->maxWeight[k],
                                  g->dist + static_cast<size_t>(k) * n,
                                  g->parent + static_cast<size_t>(k) * n, nullptr, s->setupStream);
    }
    if (rc == MOSP_OK) {
      rc = mosp_combined_sosp(s->setupWs, n, K, g->parent, g->pref.empty() ? nullptr : g->pref.data(),
                              source, 0, g->combDist, g->combParent, nullptr, s->setupStream);
    }
  }
  if (rc != MOSP_OK) {
    err = mosp_last_error();
    return fail(rc);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  g->id = static_cast<int>(s->graphs.size());
  *graph_id = g->id;
  if (n > s->maxN || m > s->maxM || K > s->maxK) {
    s->maxN = std::max(s->maxN, n);
    s->maxM = std::max<long long>(s->maxM, m);
    s->maxK = std::max(s->maxK, K);
    ++s->reserveEpoch;
  }
  s->graphs.push_back(std::move(g));
  s->workCv.notify_all();
  return MOSP_OK;
}

extern "C" int mosp_server_submit(mosp_server *s, int graph_id, int n_ins, const int *h_ins_from,
                                  const int *h_ins_to, const int *h_ins_w, int n_del,
                                  const int *h_del_from, const int *h_del_to, long long *ticket) {
  if (s == nullptr || ticket == nullptr || n_ins < 0 || n_del < 0 ||
      (n_ins > 0 && (h_ins_from == nullptr || h_ins_to == nullptr || h_ins_w == nullptr)) ||
      (n_del > 0 && (h_del_from == nullptr || h_del_to == nullptr))) {
    return recordFailure(MOSP_ERR_INVALID, "Error: invalid request.");
  }
  auto r = std::make_shared<Request>();
  r->submit = Clock::now();
  std::unique_lock<std::mutex> lk(s->mu);
  if (graph_id < 0 || graph_id >= static_cast<int>(s->graphs.size())) {
    return recordFailure(MOSP_ERR_INVALID, "Error: unknown graph id.");
  }
  Graph &g = *s->graphs[graph_id];
  lk.unlock();
  for (int i = 0; i < n_ins; ++i) {
    if (h_ins_from[i] < 0 || h_ins_from[i] >= g.n || h_ins_to[i] < 0 || h_ins_to[i] >= g.n) {
      return recordFailure(MOSP_ERR_INVALID, "Error: inserted edge endpoint out of range.");
    }
  }
  for (int i = 0; i < n_del; ++i) {
    if (h_del_from[i] < 0 || h_del_from[i] >= g.n || h_del_to[i] < 0 || h_del_to[i] >= g.n) {
      return recordFailure(MOSP_ERR_INVALID, "Error: deleted edge endpoint out of range.");
    }
  }
  r->graph = graph_id;
  r->insFrom.assign(h_ins_from, h_ins_from + n_ins);
  r->insTo.assign(h_ins_to, h_ins_to + n_ins);
  r->insW.assign(h_ins_w, h_ins_w + static_cast<size_t>(n_ins) * g.KG);
  r->delFrom.assign(h_del_from, h_del_from + n_del);
  r->delTo.assign(h_del_to, h_del_to + n_del);
  lk.lock();
  r->ticket = s->nextTicket++;
  *ticket = r->ticket;
  s->tickets[r->ticket] = r;
  g.pending.push_back(r);
  lk.unlock();
  s->workCv.notify_one();
  return MOSP_OK;
}

extern "C" int mosp_server_wait(mosp_server *s, long long ticket, long long *h_comb_dist,
                                int *h_comb_parent, mosp_server_result *info) {
  if (s == nullptr) return recordFailure(MOSP_ERR_INVALID, "Error: null server.");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return recordFailure(MOSP_ERR_INVALID, "Error: unknown ticket.");
  std::shared_ptr<Request> r = it->second;
  s->doneCv.wait(lk, [&] { return r->finished; });
  s->tickets.erase(it);
  const int n = s->graphs[r->graph]->n;
  lk.unlock();
  if (info != nullptr) {
    info->status = r->status;
    info->graph = r->graph;
    info->version = r->version;
    info->coalesced = r->coalesced;
    info->reserved = 0;
    info->queue_us = usBetween(r->submit, r->start);
    info->latency_us = usBetween(r->submit, r->done);
    info->checksum =
        r->result ? checksumOf(r->result->combDist.data(), r->result->combParent.data(), n) : 0;
  }
  if (r->status != MOSP_OK) return recordFailure(r->status, r->error.c_str());
  if (h_comb_dist) std::memcpy(h_comb_dist, r->result->combDist.data(), static_cast<size_t>(n) * 8);
  if (h_comb_parent) {
    std::memcpy(h_comb_parent, r->result->combParent.data(), static_cast<size_t>(n) * 4);
  }
  return MOSP_OK;
}

extern "C" int mosp_server_read_graph(mosp_server *s, int graph_id, long long *version,
                                      long long *h_dist, int *h_parent, long long *h_comb_dist,
                                      int *h_comb_parent) {
  if (s == nullptr) return recordFailure(MOSP_ERR_INVALID, "Error: null server.");
  std::unique_lock<std::mutex> lk(s->mu);
  if (graph_id < 0 || graph_id >= static_cast<int>(s->graphs.size())) {
    return recordFailure(MOSP_ERR_INVALID, "Error: unknown graph id.");
  }
  Graph &g = *s->graphs[graph_id];
  // wait until no pass runs on the graph and hold it meanwhile
  s->doneCv.wait(lk, [&] { return !g.busy; });
  g.busy = true;
  lk.unlock();
  cudaSetDevice(s->device);
  const size_t kn = static_cast<size_t>(g.K) * g.n;
  cudaError_t e = cudaSuccess;
  if (h_dist) e = cudaMemcpy(h_dist, g.dist, kn * 8, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && h_parent) e = cudaMemcpy(h_parent, g.parent, kn * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && h_comb_dist) {
    e = cudaMemcpy(h_comb_dist, g.combDist, static_cast<size_t>(g.n) * 8, cudaMemcpyDeviceToHost);
  }
  if (e == cudaSuccess && h_comb_parent) {
    e = cudaMemcpy(h_comb_parent, g.combParent, static_cast<size_t>(g.n) * 4,
                   cudaMemcpyDeviceToHost);
  }
  lk.lock();
  if (version) *version = g.version;
  g.busy = false;
  lk.unlock();
  s->workCv.notify_all();
  s->doneCv.notify_all();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return recordFailure(MOSP_ERR_CUDA, "Error: reading the graph's trees failed.");
  }
  return MOSP_OK;
}

extern "C" int mosp_server_get_stats(mosp_server *s, mosp_server_stats *out) {
  if (s == nullptr || out == nullptr) return recordFailure(MOSP_ERR_INVALID, "Error: null argument.");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  return MOSP_OK;
}
