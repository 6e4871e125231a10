// mosp - run one MOSP update on prepared inputs (drop-in for the reference
// CLI, SMShovan/MOSP-CUDA src/mosp.cu: same flags, output files, report and
// summary line "RESULT gpu_compute_ms=<a> end_to_end_ms=<b>"; exit code 2 on
// usage errors, 1 on failures).
//
//   mosp --graph <csrPrefix> --changes <dir> --init <dir> [-k K] [--source s]
//        [--pref p1,..,pK] [--delta D] [--cache file] [--canonicalize]
//        [--out dir] [--no-output] [--validate] [--timing file.csv] [--quiet]
//
// Outputs in --out: obj<k>/distancesUpdated.txt, obj<k>/SSSPTreeUpdated.txt,
// combinedGraph/distancesCsr.txt (units of 1/L, L = lcm(Pref)),
// combinedGraph/SSSPTreeCsr.txt, combinedGraph/mospCosts.txt ("v c1 .. cKG":
// the objective values of the MOSP path to v, every objective of the graph).
#include <cuda_runtime.h>

#include <algorithm>
#include <charconv>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "csrGraph.cuh"
#include "dijkstra.cuh"
#include "hostCore.h"
#include "mospUpdate.cuh"
#include "stageTimer.cuh"
#include "validation.cuh"

namespace {

struct Options {
  std::string graph, changes, init, out = "mosp-output", timingCsv, cache;
  std::vector<int> pref;
  int K = 0;
  int source = 0;
  long long delta = 0;
  bool canonicalize = false, writeOutput = true, validate = false, quiet = false;
};

void usage() {
  std::cerr << "usage: mosp --graph <csrPrefix> --changes <dir> --init <dir>\n"
               "            [-k K] [--source s] [--pref p1,..,pK] [--delta D]\n"
               "            [--cache file] [--canonicalize] [--out dir]\n"
               "            [--no-output] [--validate] [--timing file.csv]\n"
               "            [--quiet]\n";
}

/// One command-line flag: how many values it takes and what it does with
/// its value (a false return is a usage error).
struct Flag {
  const char *name;
  bool takesValue;
  std::function<bool(Options &, const std::string &)> apply;
};

bool intInRange(const std::string &flag, const std::string &text, long long lo, long long hi,
                long long &out) {
  if (parseInteger(text, lo, hi, out)) return true;
  std::cerr << flag << ": expected an integer from " << lo << " to " << hi << ", not '" << text
            << "'\n";
  return false;
}

const std::vector<Flag> &flagTable() {
  static const std::vector<Flag> table = {
      {"--graph", true, [](Options &o, const std::string &v) { o.graph = v; return true; }},
      {"--changes", true, [](Options &o, const std::string &v) { o.changes = v; return true; }},
      {"--init", true, [](Options &o, const std::string &v) { o.init = v; return true; }},
      {"--out", true, [](Options &o, const std::string &v) { o.out = v; return true; }},
      {"--timing", true, [](Options &o, const std::string &v) { o.timingCsv = v; return true; }},
      {"--cache", true, [](Options &o, const std::string &v) { o.cache = v; return true; }},
      {"-k", true,
       [](Options &o, const std::string &v) {
         long long x = 0;
         if (!intInRange("-k", v, 0, INT_MAX, x)) return false;
         o.K = static_cast<int>(x);
         return true;
       }},
      {"--source", true,
       [](Options &o, const std::string &v) {
         long long x = 0;
         if (!intInRange("--source", v, 0, INT_MAX, x)) return false;
         o.source = static_cast<int>(x);
         return true;
       }},
      {"--delta", true,
       [](Options &o, const std::string &v) { return intInRange("--delta", v, 1, LLONG_MAX, o.delta); }},
      {"--pref", true,
       [](Options &o, const std::string &v) {
         // comma-separated preference weights, each >= 1
         size_t from = 0;
         while (from < v.size()) {
           const size_t comma = std::min(v.find(',', from), v.size());
           long long x = 0;
           if (!intInRange("--pref", v.substr(from, comma - from), 1, INT_MAX, x)) return false;
           o.pref.push_back(static_cast<int>(x));
           from = comma + 1;
         }
         return true;
       }},
      {"--canonicalize", false, [](Options &o, const std::string &) { return o.canonicalize = true; }},
      {"--no-output", false, [](Options &o, const std::string &) { o.writeOutput = false; return true; }},
      {"--validate", false, [](Options &o, const std::string &) { return o.validate = true; }},
      {"--quiet", false, [](Options &o, const std::string &) { return o.quiet = true; }},
  };
  return table;
}

bool parseOptions(int argc, char **argv, Options &o) {
  const std::vector<Flag> &table = flagTable();
  for (int i = 1; i < argc; ++i) {
    const std::string arg = argv[i];
    const auto flag = std::find_if(table.begin(), table.end(),
                                   [&](const Flag &f) { return arg == f.name; });
    if (flag == table.end()) {
      std::cerr << "mosp: no such option: " << arg << "\n";
      return false;
    }
    std::string value;
    if (flag->takesValue) {
      if (i + 1 == argc) {
        std::cerr << "mosp: " << arg << " needs a value\n";
        return false;
      }
      value = argv[++i];
    }
    if (!flag->apply(o, value)) return false;
  }
  return !o.graph.empty() && !o.changes.empty() && !o.init.empty();
}

double msSince(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

/// Objective k's part of a K * n objective-major array.
template <typename T>
std::vector<T> objectivePart(const std::vector<T> &all, int k, int n) {
  const auto first = all.begin() + static_cast<std::ptrdiff_t>(k) * n;
  return std::vector<T>(first, first + n);
}

bool writeCosts(const std::string &path, const std::vector<long long> &costs, int KG) {
  const size_t n = KG > 0 ? costs.size() / KG : 0;
  return mospb200::writeLinesParallel(path, n, [&](size_t v, std::string &out) {
    char d[24];
    out.append(d, std::to_chars(d, d + 24, v).ptr);
    for (int k = 0; k < KG; ++k) {
      const long long c = costs[v * KG + k];
      out.push_back(' ');
      if (c >= DISTANCE_INF / 2) {
        out.append("INF");
      } else {
        out.append(d, std::to_chars(d, d + 24, c).ptr);
      }
    }
    out.push_back('\n');
  });
}

/// --validate: every updated tree against host Dijkstra on the updated
/// graph (exact parents when the input trees were canonical), and the MOSP
/// tree against Dijkstra on the host combined graph of the updated trees.
/// The K + 1 checks are independent and run side by side; the report lines
/// come out in objective order.
bool validate(const CsrGraph &updated, const MospResult &r, int source, const std::vector<int> &pref,
              bool requireCanonical) {
  const int n = updated.numberOfNodes, K = r.numberOfObjectives;
  CsrGraph reverse;
  transposeCsrGraph(updated, reverse);
  std::vector<TreeCheck> checks(K + 1);
  auto checkObjective = [&](int k) {
    std::vector<long long> refDist;
    std::vector<int> refParent;
    dijkstraCsrGraph(updated, k, source, refDist, refParent);
    checks[k] = checkSospTree(reverse, k, source, objectivePart(r.distances, k, n),
                              objectivePart(r.parents, k, n), refDist,
                              requireCanonical ? &refParent : nullptr);
  };
  auto checkCombined = [&] {
    const CsrGraph combined = combinedGraphReference(r.parents, n, K, source, pref);
    CsrGraph combinedReverse;
    transposeCsrGraph(combined, combinedReverse);
    std::vector<long long> refDist;
    std::vector<int> refParent;
    dijkstraCsrGraph(combined, 0, source, refDist, refParent);
    checks[K] = checkSospTree(combinedReverse, 0, source, r.combinedDistances, r.combinedParent,
                              refDist, &refParent);
  };
  std::vector<std::thread> workers;
  for (int k = 0; k < K; ++k) workers.emplace_back(checkObjective, k);
  checkCombined();
  for (std::thread &t : workers) t.join();
  bool all = true;
  for (int k = 0; k <= K; ++k) {
    // the MOSP tree is computed from scratch, so it is always canonical
    const bool ok = checks[k].ok(k == K || requireCanonical);
    all = all && ok;
    std::cout << "VALIDATE " << (k == K ? std::string("combined") : "obj" + std::to_string(k)) << " "
              << (ok ? "PASS" : "FAIL") << " (" << checks[k].summary() << ")\n";
  }
  return all;
}

}  // namespace

int main(int argc, char **argv) {
  Options opt;
  if (!parseOptions(argc, argv, opt)) {
    usage();
    return 2;
  }
  // load every kernel when the context is created, not inside the first
  // timed update (an explicit setting in the environment wins)
  setenv("CUDA_MODULE_LOADING", "EAGER", 0);
  setInstrumentation(!opt.timingCsv.empty());
  const auto start = std::chrono::steady_clock::now();
  double contextMs = 0, loadMs = 0, canonicalizeMs = 0, writeMs = 0;
  {
    const auto t = std::chrono::steady_clock::now();
    ScopedStage stage("cuda_context_init");
    cudaFree(nullptr);
    contextMs = msSince(t);
  }
  auto t = std::chrono::steady_clock::now();
  CsrGraph original;
  ChangeBatch batch;
  {
    ScopedStage stage("read_graph");
    if (!loadCsrGraph(opt.graph, original, opt.cache)) return 1;
  }
  const int n = original.numberOfNodes, KG = original.numberOfObjectives;
  const int K = opt.K > 0 ? std::min(opt.K, KG) : KG;
  std::vector<long long> distances(static_cast<size_t>(K) * n);
  std::vector<int> parents(static_cast<size_t>(K) * n);
  {
    ScopedStage stage("read_changes_and_trees");
    std::vector<std::vector<long long>> dist(K);
    std::vector<std::vector<int>> par(K);
    std::vector<std::function<bool()>> reads{[&] {
      return readChangeBatch(opt.changes + "/insert.txt", opt.changes + "/delete.txt", KG, n, batch);
    }};
    for (int k = 0; k < K; ++k) {
      const std::string dir = opt.init + "/obj" + std::to_string(k);
      reads.push_back([&, k, dir] { return readDistances(dir + "/distancesOriginal.txt", n, dist[k]); });
      reads.push_back([&, k, dir] { return readParents(dir + "/SSSPTreeOriginal.txt", n, par[k]); });
    }
    if (!runConcurrently(reads)) return 1;
    for (int k = 0; k < K; ++k) {
      std::copy(dist[k].begin(), dist[k].end(), distances.begin() + static_cast<size_t>(k) * n);
      std::copy(par[k].begin(), par[k].end(), parents.begin() + static_cast<size_t>(k) * n);
    }
  }
  loadMs = msSince(t);
  if (opt.canonicalize) {
    const auto tc = std::chrono::steady_clock::now();
    for (int k = 0; k < K; ++k) {
      canonicalizeTree(original, k, opt.source, objectivePart(distances, k, n),
                       parents.data() + static_cast<size_t>(k) * n);
    }
    canonicalizeMs = msSince(tc);
  }

  MospOptions options;
  options.source = opt.source;
  options.numberOfObjectives = K;
  options.preferences = opt.pref;
  options.delta = opt.delta;
  // trees normalised by --canonicalize follow the lowest-id rule
  options.canonicalTrees = opt.canonicalize;
  CsrGraph updated;
  MospResult result;
  std::vector<long long> costs;
  if (!mospUpdateWithCosts(original, batch, distances, parents, options, updated, result,
                           opt.writeOutput ? &costs : nullptr)) {
    return 1;
  }

  if (opt.writeOutput) {
    const auto tw = std::chrono::steady_clock::now();
    ScopedStage stage("write_outputs");
    for (int k = 0; k < K; ++k) std::filesystem::create_directories(opt.out + "/obj" + std::to_string(k));
    std::filesystem::create_directories(opt.out + "/combinedGraph");
    std::vector<std::function<bool()>> writes;
    for (int k = 0; k < K; ++k) {
      const std::string dir = opt.out + "/obj" + std::to_string(k);
      writes.push_back([&, k, dir] {
        return writeDistances(dir + "/distancesUpdated.txt", objectivePart(result.distances, k, n));
      });
      writes.push_back([&, k, dir] {
        return writeParents(dir + "/SSSPTreeUpdated.txt", objectivePart(result.parents, k, n));
      });
    }
    const std::string comb = opt.out + "/combinedGraph";
    writes.push_back([&] { return writeDistances(comb + "/distancesCsr.txt", result.combinedDistances); });
    writes.push_back([&] { return writeParents(comb + "/SSSPTreeCsr.txt", result.combinedParent); });
    writes.push_back([&] { return writeCosts(comb + "/mospCosts.txt", costs, KG); });
    if (!runConcurrently(writes)) {
      std::cerr << "cannot write the outputs to " << opt.out << "\n";
      return 1;
    }
    writeMs = msSince(tw);
  }
  const double endToEnd = msSince(start);

  const MospTimings &tm = result.timings;
  if (!opt.quiet) {
    std::printf("graph  n=%d m=%d K=%d; batch %d inserts, %d deletes\n", n, updated.numberOfEdges(),
                K, batch.numberOfInserts(), batch.numberOfDeletes());
    std::printf("host   context %.1f ms, read inputs %.1f ms, canonicalize %.1f ms, apply batch "
                "%.1f ms, upload %.1f ms, download %.1f ms, write %.1f ms\n",
                contextMs, loadMs, canonicalizeMs, tm.applyBatch, tm.upload, tm.download, writeMs);
    for (int k = 0; k < K; ++k) {
      const SospStats &s = result.objectiveStats[k];
      std::printf("obj%d   SOSP update %.3f ms (invalidated %d, jump rounds %d, iterations %d, "
                  "epochs %d, pushes %lld)\n",
                  k, tm.objectives[k], s.invalidated, s.jumpRounds, s.iterations, s.epochs,
                  s.pushes);
    }
    const CombineStats &c = result.combineStats;
    std::printf("comb   combined graph + SOSP %.3f ms (%d edges, L=%lld, delta %lld, iterations "
                "%d, pushes %lld)\n",
                tm.combined, c.numberOfEdges, c.scale, c.delta, c.search.iterations,
                c.search.pushes);
  }
  if (!opt.timingCsv.empty()) {
    recordStage("TOTAL_end_to_end", endToEnd);
    if (!writeInstrumentationCsv(opt.timingCsv)) std::cerr << "cannot write " << opt.timingCsv << "\n";
  }
  std::printf("RESULT gpu_compute_ms=%.3f end_to_end_ms=%.3f\n", tm.gpuCompute(), endToEnd);
  std::fflush(stdout);
  if (opt.validate && !validate(updated, result, opt.source, opt.pref, opt.canonicalize)) return 1;
  return 0;
}
