// ref_cpu_driver.cpp - TEST INFRASTRUCTURE. A C ABI over the reference's own
// CPU code (SMShovan/MOSP-CUDA), compiled together with the reference
// sources by oracle/Makefile into oracle/_ref/libref_cpu.so. It gives the
// tests and the CPU baseline of bench.py direct access to the reference
// implementation: batch application, the change generator, host Dijkstra,
// the combined-graph reference, the MOSP path costs and the sequential SOSP
// update (the reference's CPU path). Only reference headers are included.
#include "changeGenerator.cuh"
#include "csrGraph.cuh"
#include "dijkstra.cuh"
#include "parallelCombinedGraph.cuh"
#include "sequentialSOSPUpdate.cuh"
#include "validation.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

// The compute-only variant of the sequential update: the same source
// compiled a second time under another name, with a clock read inserted at
// the start of its Phase 1 and at the start of its output stage
// (oracle/instrument_ref.py writes that copy into _ref/ at build time).
bool sequentialSOSPUpdateTimed(const std::string &, const std::string &, const std::string &,
                               const std::string &, const std::string &, int, int,
                               const std::string &, const std::string &);

namespace {

std::chrono::steady_clock::time_point g_marks[3];

CsrGraph makeGraph(int n, int K, const int *row, const int *col, const int *w) {
  CsrGraph g;
  g.numberOfNodes = n;
  g.numberOfObjectives = K;
  g.rowPtr.assign(row, row + n + 1);
  g.colInd.assign(col, col + row[n]);
  g.weights.assign(w, w + static_cast<size_t>(row[n]) * K);
  return g;
}

}  // namespace

extern "C" {

int ref_dijkstra(int n, int K, const int *row, const int *col, const int *w, int k, int source,
                 long long *dist, int *parent) {
  const CsrGraph g = makeGraph(n, K, row, col, w);
  std::vector<long long> d;
  std::vector<int> p;
  dijkstraCsrGraph(g, k, source, d, p);
  std::copy(d.begin(), d.end(), dist);
  std::copy(p.begin(), p.end(), parent);
  return 0;
}

long long ref_apply_batch(int n, int K, const int *row, const int *col, const int *w, int n_ins,
                          const int *ins_from, const int *ins_to, const int *ins_w, int n_del,
                          const int *del_from, const int *del_to, int *out_row, int *out_col,
                          int *out_w, long long cap, unsigned *mask) {
  const CsrGraph g = makeGraph(n, K, row, col, w);
  ChangeBatch b;
  b.numberOfObjectives = K;
  b.insertFrom.assign(ins_from, ins_from + n_ins);
  b.insertTo.assign(ins_to, ins_to + n_ins);
  b.insertWeights.assign(ins_w, ins_w + static_cast<size_t>(n_ins) * K);
  b.deleteFrom.assign(del_from, del_from + n_del);
  b.deleteTo.assign(del_to, del_to + n_del);
  CsrGraph u;
  if (!applyChangeBatch(g, b, u)) return -1;
  const long long m = u.numberOfEdges();
  if (m > cap) return -1;
  std::copy(u.rowPtr.begin(), u.rowPtr.end(), out_row);
  std::copy(u.colInd.begin(), u.colInd.end(), out_col);
  std::copy(u.weights.begin(), u.weights.end(), out_w);
  std::copy(b.weightIncreaseMask.begin(), b.weightIncreaseMask.end(), mask);
  return m;
}

/// generateChangeBatch; outputs need room for n_changes entries each.
int ref_generate_changes(int n, int K, const int *row, const int *col, const int *w, int n_changes,
                         double ins_pct, int mode, int local_hops, int safe, unsigned seed,
                         int source, int wmin, int wmax, int *ins_from, int *ins_to, int *ins_w,
                         int *n_ins, int *del_from, int *del_to, int *n_del) {
  const CsrGraph g = makeGraph(n, K, row, col, w);
  ChangeGeneratorOptions o;
  o.numberOfChanges = n_changes;
  o.insertionPercentage = ins_pct;
  o.mode = static_cast<ChangeMode>(mode);
  o.localHops = local_hops;
  o.safeDeletions = safe != 0;
  o.seed = seed;
  o.source = source;
  o.weightMin = wmin;
  o.weightMax = wmax;
  ChangeBatch b;
  if (!generateChangeBatch(g, o, b)) return -1;
  *n_ins = b.numberOfInserts();
  *n_del = b.numberOfDeletes();
  std::copy(b.insertFrom.begin(), b.insertFrom.end(), ins_from);
  std::copy(b.insertTo.begin(), b.insertTo.end(), ins_to);
  std::copy(b.insertWeights.begin(), b.insertWeights.end(), ins_w);
  std::copy(b.deleteFrom.begin(), b.deleteFrom.end(), del_from);
  std::copy(b.deleteTo.begin(), b.deleteTo.end(), del_to);
  return 0;
}

/// combinedGraphReference + dijkstraCsrGraph: the host reference of Steps
/// 2-3. pref: K values or NULL.
int ref_combined_dijkstra(int n, int K, const int *parents, int source, const int *pref,
                          long long *dist, int *parent, long long *edges) {
  const std::vector<int> p(parents, parents + static_cast<size_t>(n) * K);
  const std::vector<int> pv = pref == nullptr ? std::vector<int>() : std::vector<int>(pref, pref + K);
  const CsrGraph c = combinedGraphReference(p, n, K, source, pv);
  std::vector<long long> d;
  std::vector<int> q;
  dijkstraCsrGraph(c, 0, source, d, q);
  std::copy(d.begin(), d.end(), dist);
  std::copy(q.begin(), q.end(), parent);
  if (edges != nullptr) *edges = c.numberOfEdges();
  return 0;
}

int ref_path_costs(int n, int KG, const int *row, const int *col, const int *w, const int *parent,
                   int source, long long *costs) {
  const CsrGraph g = makeGraph(n, KG, row, col, w);
  std::vector<long long> c;
  if (!mospPathCosts(g, std::vector<int>(parent, parent + n), source, c)) return -1;
  std::copy(c.begin(), c.end(), costs);
  return 0;
}

/// Clock read of the instrumented copy: 1 = Phase 1 starts (input read and
/// batch applied), 2 = output stage starts (update computed).
void mosp_ref_phase_mark(int which) {
  if (which >= 0 && which < 3) g_marks[which] = std::chrono::steady_clock::now();
}

/// The reference's own text writers and reader (the formats its CPU path
/// reads and writes), so that the benchmark's reference arm needs no other
/// library for its input and output files.
int ref_write_csr(const char *prefix, int n, int K, const int *row, const int *col, const int *w) {
  return writeCsrGraph(prefix, makeGraph(n, K, row, col, w)) ? 0 : -1;
}

int ref_write_changes(const char *insert_path, const char *delete_path, int K, int n_ins,
                      const int *ins_from, const int *ins_to, const int *ins_w, int n_del,
                      const int *del_from, const int *del_to) {
  ChangeBatch b;
  b.numberOfObjectives = K;
  b.insertFrom.assign(ins_from, ins_from + n_ins);
  b.insertTo.assign(ins_to, ins_to + n_ins);
  b.insertWeights.assign(ins_w, ins_w + static_cast<size_t>(n_ins) * K);
  b.deleteFrom.assign(del_from, del_from + n_del);
  b.deleteTo.assign(del_to, del_to + n_del);
  return writeChangeBatch(b, insert_path, delete_path) ? 0 : -1;
}

int ref_write_tree(const char *dist_path, const char *tree_path, int n, const long long *dist,
                   const int *parent) {
  const bool ok = writeDistances(dist_path, std::vector<long long>(dist, dist + n)) &&
                  writeParents(tree_path, std::vector<int>(parent, parent + n));
  return ok ? 0 : -1;
}

int ref_read_parents(const char *path, int n, int *parent) {
  std::vector<int> p;
  if (!readParents(path, n, p)) return -1;
  std::copy(p.begin(), p.end(), parent);
  return 0;
}

/// The reference's CPU update path as its tests call it (file API).
int ref_sequential_update(const char *graph_prefix, const char *dist_in, const char *tree_in,
                          const char *insert_path, const char *delete_path, int objective,
                          int source, const char *dist_out, const char *tree_out) {
  return sequentialSOSPUpdate(graph_prefix, dist_in, tree_in, insert_path, delete_path, objective,
                              source, dist_out, tree_out)
             ? 0
             : -1;
}

/// The same update, from the instrumented copy: *compute_s receives the
/// time of its Phases 1-2 (roots, subtree invalidation, relaxation), without
/// the text input, the batch application and the output.
int ref_sequential_update_timed(const char *graph_prefix, const char *dist_in, const char *tree_in,
                                const char *insert_path, const char *delete_path, int objective,
                                int source, const char *dist_out, const char *tree_out,
                                double *compute_s) {
  g_marks[1] = g_marks[2] = std::chrono::steady_clock::time_point();
  const bool ok = sequentialSOSPUpdateTimed(graph_prefix, dist_in, tree_in, insert_path, delete_path,
                                            objective, source, dist_out, tree_out);
  if (compute_s != nullptr) {
    *compute_s = std::chrono::duration<double>(g_marks[2] - g_marks[1]).count();
  }
  return ok ? 0 : -1;
}

}  // extern "C"
