// safeFilterGpu.cpp - the `--safe` connectivity filter of the change
// generator with its reachability computed on the GPU (interface:
// include/mospGenerators.h).
//
// The host filter applies the whole batch and runs a BFS over the updated
// graph on one core in every round. Here a round is Step 1 on the GPU
// (mosp_apply_batch_device: all insertions plus the deletions kept so far,
// on unit weights) followed by a unit-weight SSSP from the source on the
// engine (mosp_sosp_from_scratch; reachable = finite distance), and only
// the distances come back. The rounds themselves are deletionFilter.h's, so
// the kept deletions are the host filter's.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "csrGraph.cuh"
#include "deletionFilter.h"
#include "mospGenerators.h"
#include "mosp_b200.h"

namespace {

/// Device arrays of one filter call, freed together.
class DeviceArrays {
public:
  ~DeviceArrays() {
    for (void *p : owned_) cudaFree(p);
  }
  template <typename T>
  T *make(size_t count) {
    void *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      ok_ = false;
      return nullptr;
    }
    owned_.push_back(p);
    return static_cast<T *>(p);
  }
  bool ok() const { return ok_; }

private:
  std::vector<void *> owned_;
  bool ok_ = true;
};

template <typename T>
bool upload(T *dst, const T *src, size_t count) {
  return count == 0 || cudaMemcpy(dst, src, count * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
}

}  // namespace

int filterUnsafeDeletionsGpu(const CsrGraph &g, int source, ChangeBatch &batch) {
  const int n = g.numberOfNodes;
  const long long m = g.numberOfEdges();
  const int nIns = batch.numberOfInserts();
  if (n <= 0 || source < 0 || source >= n || m + nIns > INT_MAX) return -1;
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
    cudaGetLastError();
    return -1;
  }
  mosp_workspace *ws = nullptr;
  if (mosp_workspace_create(&ws) != MOSP_OK) return -1;
  struct Release {
    mosp_workspace *ws;
    ~Release() { mosp_workspace_destroy(ws); }
  } release{ws};

  const size_t cap = static_cast<size_t>(m) + nIns;
  DeviceArrays dev;
  int *row = dev.make<int>(n + 1), *col = dev.make<int>(m), *ones = dev.make<int>(cap);
  int *insFrom = dev.make<int>(nIns), *insTo = dev.make<int>(nIns);
  int *delFrom = dev.make<int>(batch.numberOfDeletes()), *delTo = dev.make<int>(batch.numberOfDeletes());
  int *newRow = dev.make<int>(n + 1), *newCol = dev.make<int>(cap), *newW = dev.make<int>(cap);
  unsigned *mask = dev.make<unsigned>(nIns);
  long long *dist = dev.make<long long>(n);
  int *parent = dev.make<int>(n);
  if (!dev.ok()) return -1;
  const std::vector<int> hostOnes(cap, 1);
  if (!upload(row, g.rowPtr.data(), n + 1) || !upload(col, g.colInd.data(), m) ||
      !upload(ones, hostOnes.data(), cap) || !upload(insFrom, batch.insertFrom.data(), nIns) ||
      !upload(insTo, batch.insertTo.data(), nIns)) {
    return -1;
  }
  std::vector<long long> hostDist(n);
  // reachable from the source over the graph (r, c) with m' unit-weight edges
  auto reach = [&](const int *r, const int *c, int edges) -> std::vector<char> {
    if (mosp_sosp_from_scratch(ws, n, edges, r, c, ones, source, 1LL << 40, 1, dist, parent, nullptr,
                               nullptr) != MOSP_OK ||
        cudaMemcpy(hostDist.data(), dist, n * sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess) {
      return {};
    }
    std::vector<char> out(n);
    for (int v = 0; v < n; ++v) out[v] = hostDist[v] < MOSP_DISTANCE_INF / 2;
    return out;
  };
  const std::vector<char> before = reach(row, col, static_cast<int>(m));
  if (before.empty()) return -1;
  ChangeBatch work = batch;
  const int rounds = filterDeletionRounds(before, work, [&](const ChangeBatch &b) -> std::vector<char> {
    const int nDel = b.numberOfDeletes();
    int newM = 0;
    if (!upload(delFrom, b.deleteFrom.data(), nDel) || !upload(delTo, b.deleteTo.data(), nDel) ||
        mosp_apply_batch_device(ws, n, 1, static_cast<int>(m), row, col, ones, nIns, insFrom, insTo, ones,
                                nDel, delFrom, delTo, newRow, newCol, newW, static_cast<long long>(cap),
                                &newM, mask, nullptr, nullptr, nullptr) != MOSP_OK) {
      return {};
    }
    return reach(newRow, newCol, newM);
  });
  if (rounds < 0) return -1;
  batch.deleteFrom.swap(work.deleteFrom);
  batch.deleteTo.swap(work.deleteTo);
  return rounds;
}
