// hostCapi.cpp - C ABI of the host side (include/mosp_b200_host.h).
#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "changeGenerator.cuh"
#include "csrGraph.cuh"
#include "dijkstra.cuh"
#include "hostCore.h"
#include "mospGenerators.h"
#include "mospUpdate.cuh"
#include "mosp_b200.h"
#include "mosp_b200_host.h"

struct mosp_host_graph {
  CsrGraph g;
};
struct mosp_host_batch {
  ChangeBatch b;
};

namespace {

int wrapGraph(CsrGraph &&g, mosp_host_graph **out) {
  if (out == nullptr) return MOSP_ERR_INVALID;
  *out = new mosp_host_graph{std::move(g)};
  return MOSP_OK;
}

int wrapBatch(ChangeBatch &&b, mosp_host_batch **out) {
  if (out == nullptr) return MOSP_ERR_INVALID;
  *out = new mosp_host_batch{std::move(b)};
  return MOSP_OK;
}

/// Children lists of a parent array (source excluded).
void childrenOf(const int *parent, int n, int source, std::vector<int> &first,
                std::vector<int> &kids) {
  first.assign(static_cast<size_t>(n) + 1, 0);
  kids.assign(n, 0);
  for (int v = 0; v < n; ++v) {
    if (v != source && parent[v] >= 0) ++first[parent[v] + 1];
  }
  for (int v = 0; v < n; ++v) first[v + 1] += first[v];
  std::vector<int> fill(first.begin(), first.end() - 1);
  for (int v = 0; v < n; ++v) {
    if (v != source && parent[v] >= 0) kids[fill[parent[v]]++] = v;
  }
}

}  // namespace

extern "C" {

int mosp_graph_read(const char *prefix, const char *cache_path, mosp_host_graph **out) {
  if (prefix == nullptr || out == nullptr) return MOSP_ERR_INVALID;
  CsrGraph g;
  if (!loadCsrGraph(prefix, g, cache_path == nullptr ? "" : cache_path)) return MOSP_ERR_INVALID;
  return wrapGraph(std::move(g), out);
}

int mosp_graph_write(const mosp_host_graph *g, const char *prefix) {
  if (g == nullptr || prefix == nullptr) return MOSP_ERR_INVALID;
  return writeCsrGraph(prefix, g->g) ? MOSP_OK : MOSP_ERR_INVALID;
}

int mosp_graph_save_cache(const mosp_host_graph *g, const char *path, const char *source_prefix) {
  if (g == nullptr || path == nullptr || source_prefix == nullptr) return MOSP_ERR_INVALID;
  return saveCsrGraphBinary(path, g->g, source_prefix) ? MOSP_OK : MOSP_ERR_INVALID;
}

int mosp_graph_from_arrays(int n, int K, const int *row, const int *col, const int *w,
                           mosp_host_graph **out) {
  if (n <= 0 || K <= 0 || row == nullptr || out == nullptr) return MOSP_ERR_INVALID;
  const int m = row[n];
  if (row[0] != 0 || m < 0 || (m > 0 && (col == nullptr || w == nullptr))) return MOSP_ERR_INVALID;
  CsrGraph g;
  g.numberOfNodes = n;
  g.numberOfObjectives = K;
  g.rowPtr.assign(row, row + n + 1);
  g.colInd.assign(col, col + m);
  g.weights.assign(w, w + static_cast<size_t>(m) * K);
  for (int u = 0; u < n; ++u) {
    if (g.rowPtr[u + 1] < g.rowPtr[u]) return MOSP_ERR_INVALID;
  }
  for (int v : g.colInd) {
    if (v < 0 || v >= n) return MOSP_ERR_INVALID;
  }
  for (int x : g.weights) {
    if (x < 1) return MOSP_ERR_INVALID;
  }
  return wrapGraph(std::move(g), out);
}

int mosp_graph_grid_road(int width, int height, double keep, double shortcut_fraction, int K,
                         int wmin, int wmax, unsigned seed, mosp_host_graph **out) {
  CsrGraph g;
  if (!generateGridRoad(width, height, keep, shortcut_fraction, K, wmin, wmax, seed, g)) {
    return MOSP_ERR_INVALID;
  }
  return wrapGraph(std::move(g), out);
}

int mosp_graph_rmat(int scale, int edge_factor, double a, double b, double c, int K, int wmin,
                    int wmax, int log_uniform, unsigned seed, mosp_host_graph **out) {
  CsrGraph g;
  if (!generateRmat(scale, edge_factor, a, b, c, K, wmin, wmax, log_uniform != 0, seed, g)) {
    return MOSP_ERR_INVALID;
  }
  return wrapGraph(std::move(g), out);
}

int mosp_graph_info(const mosp_host_graph *g, int *n, int *K, long long *m) {
  if (g == nullptr) return MOSP_ERR_INVALID;
  if (n) *n = g->g.numberOfNodes;
  if (K) *K = g->g.numberOfObjectives;
  if (m) *m = g->g.numberOfEdges();
  return MOSP_OK;
}

int mosp_graph_arrays(const mosp_host_graph *g, const int **row, const int **col, const int **w) {
  if (g == nullptr) return MOSP_ERR_INVALID;
  if (row) *row = g->g.rowPtr.data();
  if (col) *col = g->g.colInd.data();
  if (w) *w = g->g.weights.data();
  return MOSP_OK;
}

void mosp_graph_free(mosp_host_graph *g) { delete g; }

int mosp_batch_generate(const mosp_host_graph *g, int n_changes, double ins_pct, int mode,
                        int local_hops, int safe, unsigned seed, int source, int wmin, int wmax,
                        mosp_host_batch **out) {
  if (g == nullptr || mode < 0 || mode > 3) return MOSP_ERR_INVALID;
  ChangeGeneratorOptions opt;
  opt.numberOfChanges = n_changes;
  opt.insertionPercentage = ins_pct;
  opt.mode = static_cast<ChangeMode>(mode);
  opt.localHops = local_hops;
  opt.safeDeletions = safe != 0;
  opt.seed = seed;
  opt.source = source;
  opt.weightMin = wmin;
  opt.weightMax = wmax;
  ChangeBatch b;
  if (!generateChangeBatch(g->g, opt, b)) return MOSP_ERR_INVALID;
  return wrapBatch(std::move(b), out);
}

int mosp_batch_near(const mosp_host_graph *g, int grid_width, int n_ins, int n_del,
                    int max_manhattan, int safe, unsigned seed, int source, int wmin, int wmax,
                    mosp_host_batch **out) {
  if (g == nullptr) return MOSP_ERR_INVALID;
  ChangeBatch b;
  if (!generateNearBatch(g->g, grid_width, n_ins, n_del, max_manhattan, safe != 0, seed, source,
                         wmin, wmax, b)) {
    return MOSP_ERR_INVALID;
  }
  return wrapBatch(std::move(b), out);
}

int mosp_batch_read(const char *insert_path, const char *delete_path, int K, int n,
                    mosp_host_batch **out) {
  if (insert_path == nullptr || delete_path == nullptr) return MOSP_ERR_INVALID;
  ChangeBatch b;
  if (!readChangeBatch(insert_path, delete_path, K, n, b)) return MOSP_ERR_INVALID;
  return wrapBatch(std::move(b), out);
}

int mosp_batch_write(const mosp_host_batch *b, const char *insert_path, const char *delete_path) {
  if (b == nullptr || insert_path == nullptr || delete_path == nullptr) return MOSP_ERR_INVALID;
  return writeChangeBatch(b->b, insert_path, delete_path) ? MOSP_OK : MOSP_ERR_INVALID;
}

int mosp_batch_from_arrays(int K, int n_ins, const int *ins_from, const int *ins_to,
                           const int *ins_w, int n_del, const int *del_from, const int *del_to,
                           mosp_host_batch **out) {
  if (K <= 0 || n_ins < 0 || n_del < 0 ||
      (n_ins > 0 && (ins_from == nullptr || ins_to == nullptr || ins_w == nullptr)) ||
      (n_del > 0 && (del_from == nullptr || del_to == nullptr))) {
    return MOSP_ERR_INVALID;
  }
  ChangeBatch b;
  b.numberOfObjectives = K;
  b.insertFrom.assign(ins_from, ins_from + n_ins);
  b.insertTo.assign(ins_to, ins_to + n_ins);
  b.insertWeights.assign(ins_w, ins_w + static_cast<size_t>(n_ins) * K);
  b.deleteFrom.assign(del_from, del_from + n_del);
  b.deleteTo.assign(del_to, del_to + n_del);
  return wrapBatch(std::move(b), out);
}

int mosp_batch_info(const mosp_host_batch *b, int *K, int *n_ins, int *n_del) {
  if (b == nullptr) return MOSP_ERR_INVALID;
  if (K) *K = b->b.numberOfObjectives;
  if (n_ins) *n_ins = b->b.numberOfInserts();
  if (n_del) *n_del = b->b.numberOfDeletes();
  return MOSP_OK;
}

int mosp_batch_arrays(const mosp_host_batch *b, const int **ins_from, const int **ins_to,
                      const int **ins_w, const int **del_from, const int **del_to,
                      const unsigned **increase_mask) {
  if (b == nullptr) return MOSP_ERR_INVALID;
  if (ins_from) *ins_from = b->b.insertFrom.data();
  if (ins_to) *ins_to = b->b.insertTo.data();
  if (ins_w) *ins_w = b->b.insertWeights.data();
  if (del_from) *del_from = b->b.deleteFrom.data();
  if (del_to) *del_to = b->b.deleteTo.data();
  if (increase_mask) *increase_mask = b->b.weightIncreaseMask.data();
  return MOSP_OK;
}

void mosp_batch_free(mosp_host_batch *b) { delete b; }

int mosp_apply_batch(const mosp_host_graph *g, mosp_host_batch *b, mosp_host_graph **updated) {
  if (g == nullptr || b == nullptr || updated == nullptr) return MOSP_ERR_INVALID;
  for (int i = 0; i < b->b.numberOfInserts(); ++i) {
    if (b->b.insertFrom[i] < 0 || b->b.insertFrom[i] >= g->g.numberOfNodes ||
        b->b.insertTo[i] < 0 || b->b.insertTo[i] >= g->g.numberOfNodes) {
      return MOSP_ERR_INVALID;
    }
  }
  for (int i = 0; i < b->b.numberOfDeletes(); ++i) {
    if (b->b.deleteFrom[i] < 0 || b->b.deleteFrom[i] >= g->g.numberOfNodes ||
        b->b.deleteTo[i] < 0 || b->b.deleteTo[i] >= g->g.numberOfNodes) {
      return MOSP_ERR_INVALID;
    }
  }
  CsrGraph u;
  if (!applyChangeBatch(g->g, b->b, u)) return MOSP_ERR_INVALID;
  return wrapGraph(std::move(u), updated);
}

int mosp_host_dijkstra(const mosp_host_graph *g, int objective, int source, long long *dist,
                       int *parent) {
  if (g == nullptr || dist == nullptr || parent == nullptr || objective < 0 ||
      objective >= g->g.numberOfObjectives || source < 0 || source >= g->g.numberOfNodes) {
    return MOSP_ERR_INVALID;
  }
  std::vector<long long> d;
  std::vector<int> p;
  dijkstraCsrGraph(g->g, objective, source, d, p);
  std::copy(d.begin(), d.end(), dist);
  std::copy(p.begin(), p.end(), parent);
  return MOSP_OK;
}

int mosp_canonicalize_tree(const mosp_host_graph *g, int objective, int source,
                           const long long *dist, int *parent) {
  if (g == nullptr || dist == nullptr || parent == nullptr || objective < 0 ||
      objective >= g->g.numberOfObjectives) {
    return MOSP_ERR_INVALID;
  }
  std::vector<long long> d(dist, dist + g->g.numberOfNodes);
  canonicalizeTree(g->g, objective, source, d, parent);
  return MOSP_OK;
}

int mosp_read_tree(const char *dist_path, const char *parent_path, int n, long long *dist,
                   int *parent) {
  if (dist_path == nullptr || parent_path == nullptr || dist == nullptr || parent == nullptr) {
    return MOSP_ERR_INVALID;
  }
  std::vector<long long> d;
  std::vector<int> p;
  if (!readDistances(dist_path, n, d) || !readParents(parent_path, n, p)) return MOSP_ERR_INVALID;
  std::copy(d.begin(), d.end(), dist);
  std::copy(p.begin(), p.end(), parent);
  return MOSP_OK;
}

int mosp_write_tree(const char *dist_path, const char *parent_path, int n, const long long *dist,
                    const int *parent) {
  if (dist_path == nullptr || parent_path == nullptr || dist == nullptr || parent == nullptr) {
    return MOSP_ERR_INVALID;
  }
  const bool ok = writeDistances(dist_path, std::vector<long long>(dist, dist + n)) &&
                  writeParents(parent_path, std::vector<int>(parent, parent + n));
  return ok ? MOSP_OK : MOSP_ERR_INVALID;
}

int mosp_algorithmic_bytes(const mosp_host_graph *g, const mosp_host_batch *b, int K, int source,
                           const long long *old_dist, const int *old_parent,
                           const long long *new_dist, const int *new_parent,
                           long long combined_edges, long long *bytes_update,
                           long long *bytes_combined, long long *invalidated_total,
                           long long *expanded_total) {
  if (g == nullptr || b == nullptr || K <= 0 || K > g->g.numberOfObjectives ||
      old_dist == nullptr || old_parent == nullptr || new_dist == nullptr ||
      new_parent == nullptr) {
    return MOSP_ERR_INVALID;
  }
  const CsrGraph &G = g->g;
  const ChangeBatch &B = b->b;
  const int n = G.numberOfNodes;
  std::vector<int> indeg(n, 0);
  for (int v : G.colInd) ++indeg[v];
  auto outdeg = [&](int u) { return static_cast<long long>(G.rowPtr[u + 1] - G.rowPtr[u]); };
  // distinct insert heads other than the source
  std::vector<char> isHead(n, 0);
  for (int v : B.insertTo) {
    if (v != source) isHead[v] = 1;
  }
  long long heads = 0;
  for (int v = 0; v < n; ++v) heads += isHead[v];
  long long total = 0, invTotal = 0, expTotal = 0;
  std::vector<int> first, kids;
  std::vector<char> inv(n);
  for (int k = 0; k < K; ++k) {
    const long long *od = old_dist + static_cast<size_t>(k) * n;
    const int *op = old_parent + static_cast<size_t>(k) * n;
    const long long *nd = new_dist + static_cast<size_t>(k) * n;
    const int *np = new_parent + static_cast<size_t>(k) * n;
    // changed edges of objective k and the roots they cut
    std::fill(inv.begin(), inv.end(), 0);
    std::vector<int> stack;
    long long changed = 0;
    auto root = [&](int u, int v) {
      ++changed;
      if (op[v] == u && !inv[v]) {
        inv[v] = 1;
        stack.push_back(v);
      }
    };
    for (int i = 0; i < B.numberOfDeletes(); ++i) root(B.deleteFrom[i], B.deleteTo[i]);
    for (int i = 0; i < B.numberOfInserts(); ++i) {
      if (!B.weightIncreaseMask.empty() && (B.weightIncreaseMask[i] & (1u << k))) {
        root(B.insertFrom[i], B.insertTo[i]);
      }
    }
    childrenOf(op, n, source, first, kids);
    while (!stack.empty()) {
      const int x = stack.back();
      stack.pop_back();
      for (int c = first[x]; c < first[x + 1]; ++c) {
        if (!inv[kids[c]]) {
          inv[kids[c]] = 1;
          stack.push_back(kids[c]);
        }
      }
    }
    long long bytes = 4LL * n + 16 * changed + 4 * heads;
    for (int v = 0; v < n; ++v) {
      const bool reach = nd[v] < DISTANCE_INF / 2;
      if (inv[v] || isHead[v]) bytes += 8 + 16 * static_cast<long long>(indeg[v]);
      const bool decreased = reach && (od[v] >= DISTANCE_INF / 2 || nd[v] < od[v]);
      if ((inv[v] && reach) || decreased) {
        bytes += 8 + 16 * outdeg(v);
        ++expTotal;
      }
      if (nd[v] != od[v] || np[v] != op[v]) bytes += 12;
      invTotal += inv[v];
    }
    total += bytes;
  }
  const long long Ec = combined_edges;
  if (bytes_update) *bytes_update = total;
  if (bytes_combined) {
    *bytes_combined = 4LL * K * n + 8LL * (n + 1) + 24 * Ec + 12LL * n;
  }
  if (invalidated_total) *invalidated_total = invTotal;
  if (expanded_total) *expanded_total = expTotal;
  return MOSP_OK;
}

}  // extern "C"
