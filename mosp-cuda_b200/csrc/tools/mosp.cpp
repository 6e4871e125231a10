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

bool parseOptions(int argc, char **argv, Options &o) {
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&](std::string &dst) {
      if (i + 1 >= argc) return false;
      dst = argv[++i];
      return true;
    };
    std::string v;
    long long x = 0;
    auto integer = [&](long long lo, long long hi) {
      if (!next(v)) return false;
      if (parseInteger(v, lo, hi, x)) return true;
      std::cerr << a << " needs an integer in [" << lo << ", " << hi << "], got '" << v << "'\n";
      return false;
    };
    if (a == "--graph") {
      if (!next(o.graph)) return false;
    } else if (a == "--changes") {
      if (!next(o.changes)) return false;
    } else if (a == "--init") {
      if (!next(o.init)) return false;
    } else if (a == "--out") {
      if (!next(o.out)) return false;
    } else if (a == "--timing") {
      if (!next(o.timingCsv)) return false;
    } else if (a == "--cache") {
      if (!next(o.cache)) return false;
    } else if (a == "-k") {
      if (!integer(0, INT_MAX)) return false;
      o.K = static_cast<int>(x);
    } else if (a == "--source") {
      if (!integer(0, INT_MAX)) return false;
      o.source = static_cast<int>(x);
    } else if (a == "--delta") {
      if (!integer(1, LLONG_MAX)) return false;
      o.delta = x;
    } else if (a == "--pref") {
      if (!next(v)) return false;
      std::istringstream list(v);
      std::string item;
      while (std::getline(list, item, ',')) {
        if (!parseInteger(item, 1, INT_MAX, x)) {
          std::cerr << "--pref needs integers >= 1, got '" << v << "'\n";
          return false;
        }
        o.pref.push_back(static_cast<int>(x));
      }
    } else if (a == "--canonicalize") {
      o.canonicalize = true;
    } else if (a == "--no-output") {
      o.writeOutput = false;
    } else if (a == "--validate") {
      o.validate = true;
    } else if (a == "--quiet") {
      o.quiet = true;
    } else {
      std::cerr << "unknown option: " << a << "\n";
      return false;
    }
  }
  return !o.graph.empty() && !o.changes.empty() && !o.init.empty();
}

double msSince(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

template <typename T>
std::vector<T> slice(const std::vector<T> &all, int k, int n) {
  return std::vector<T>(all.begin() + static_cast<size_t>(k) * n,
                        all.begin() + static_cast<size_t>(k + 1) * n);
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

bool validate(const CsrGraph &updated, const MospResult &r, int source, const std::vector<int> &pref,
              bool requireCanonical) {
  const int n = updated.numberOfNodes, K = r.numberOfObjectives;
  CsrGraph reverse;
  transposeCsrGraph(updated, reverse);
  bool all = true;
  for (int k = 0; k < K; ++k) {
    std::vector<long long> refDist;
    std::vector<int> refParent;
    dijkstraCsrGraph(updated, k, source, refDist, refParent);
    const TreeCheck c = checkSospTree(reverse, k, source, slice(r.distances, k, n),
                                      slice(r.parents, k, n), refDist,
                                      requireCanonical ? &refParent : nullptr);
    const bool ok = c.ok(requireCanonical);
    all = all && ok;
    std::cout << "VALIDATE obj" << k << " " << (ok ? "PASS" : "FAIL") << " (" << c.summary() << ")\n";
  }
  const CsrGraph combined = combinedGraphReference(r.parents, n, K, source, pref);
  CsrGraph combinedReverse;
  transposeCsrGraph(combined, combinedReverse);
  std::vector<long long> refDist;
  std::vector<int> refParent;
  dijkstraCsrGraph(combined, 0, source, refDist, refParent);
  const TreeCheck c = checkSospTree(combinedReverse, 0, source, r.combinedDistances,
                                    r.combinedParent, refDist, &refParent);
  const bool ok = c.ok(true);  // built from scratch: always canonical
  std::cout << "VALIDATE combined " << (ok ? "PASS" : "FAIL") << " (" << c.summary() << ")\n";
  return all && ok;
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
      canonicalizeTree(original, k, opt.source, slice(distances, k, n),
                       parents.data() + static_cast<size_t>(k) * n);
    }
    canonicalizeMs = msSince(tc);
  }

  MospOptions options;
  options.source = opt.source;
  options.numberOfObjectives = K;
  options.preferences = opt.pref;
  options.delta = opt.delta;
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
        return writeDistances(dir + "/distancesUpdated.txt", slice(result.distances, k, n));
      });
      writes.push_back([&, k, dir] {
        return writeParents(dir + "/SSSPTreeUpdated.txt", slice(result.parents, k, n));
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
