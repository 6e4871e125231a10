// mospPrep - input preparation (drop-in for the reference CLI,
// SMShovan/MOSP-CUDA src/mospPrep.cu; same subcommands, arguments, output
// files and seeded outputs), plus generators of the synthetic workloads and
// a GPU path for the initial trees.
//
//   mospPrep mtx2csr <in.mtx> <outPrefix> <K> <wmin> <wmax> <seed>
//   mospPrep widen <inPrefix> <outPrefix> <K> <wmin> <wmax> <seed>
//   mospPrep cache <csrPrefix> <binaryPath>
//   mospPrep changes <csrPrefix> <outDir> [--changes N] [--ins PCT] [--gpu]
//            [--mode uniform|targeted|reweight|increase] [--local HOPS]
//            [--safe] [--seed S] [--source s] [--wmin a] [--wmax b]
//   mospPrep init <csrPrefix> <outDir> [--source s] [--gpu]
//   mospPrep expected <csrPrefix> <changesDir> <outDir> [--source s] [--gpu]
//   mospPrep grid <outPrefix> <width> <height> <keep> <shortcut> <K> <wmin> <wmax> <seed>
//   mospPrep rmat <outPrefix> <scale> <edgeFactor> <a> <b> <c> <K> <wmin> <wmax> <log 0|1> <seed>
//   mospPrep nearchanges <csrPrefix> <outDir> <gridWidth> <inserts> <deletes> <maxManhattan>
//            [--safe] [--seed S] [--source s] [--wmin a] [--wmax b]
//
// --gpu computes the trees with the canonical SSSP engine on the GPU
// instead of host Dijkstra (identical output).
#include <algorithm>
#include <charconv>
#include <chrono>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <random>
#include <string>
#include <string_view>
#include <vector>

#include "changeGenerator.cuh"
#include "csrGraph.cuh"
#include "deviceGraph.cuh"
#include "dijkstra.cuh"
#include "mospGenerators.h"
#include "sospUpdateGpu.cuh"

namespace {

double msSince(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

int usage() {
  std::cerr
      << "usage: mospPrep mtx2csr <in.mtx> <outPrefix> <K> <wmin> <wmax> <seed>\n"
         "       mospPrep widen <inPrefix> <outPrefix> <K> <wmin> <wmax> <seed>\n"
         "       mospPrep cache <csrPrefix> <binaryPath>\n"
         "       mospPrep changes <csrPrefix> <outDir> [--changes N] [--ins PCT]\n"
         "                [--mode uniform|targeted|reweight|increase] [--local HOPS]\n"
         "                [--safe] [--seed S] [--source s] [--wmin a] [--wmax b]\n"
         "       mospPrep init <csrPrefix> <outDir> [--source s] [--gpu]\n"
         "       mospPrep expected <csrPrefix> <changesDir> <outDir> [--source s] [--gpu]\n"
         "       mospPrep grid <outPrefix> <width> <height> <keep> <shortcut> <K> <wmin> <wmax> <seed>\n"
         "       mospPrep rmat <outPrefix> <scale> <edgeFactor> <a> <b> <c> <K> <wmin> <wmax> <log> <seed>\n"
         "       mospPrep nearchanges <csrPrefix> <outDir> <gridWidth> <inserts> <deletes>\n"
         "                <maxManhattan> [--safe] [--seed S] [--source s] [--wmin a] [--wmax b]\n";
  return 2;
}

bool weightArguments(char **argv, int &K, int &wmin, int &wmax, unsigned &seed) {
  long long k = 0, lo = 0, hi = 0, s = 0;
  if (!parseInteger(argv[0], 1, 32, k)) {
    std::cerr << "K must be an integer in [1, 32]\n";
    return false;
  }
  if (!parseInteger(argv[1], 1, INT_MAX, lo) || !parseInteger(argv[2], lo, INT_MAX, hi)) {
    std::cerr << "weights need 1 <= wmin <= wmax <= " << INT_MAX << "\n";
    return false;
  }
  if (!parseInteger(argv[3], 0, UINT_MAX, s)) {
    std::cerr << "seed must be an integer in [0, " << UINT_MAX << "]\n";
    return false;
  }
  K = static_cast<int>(k);
  wmin = static_cast<int>(lo);
  wmax = static_cast<int>(hi);
  seed = static_cast<unsigned>(s);
  return true;
}

bool parseReal(const char *text, double lo, double hi, double &x) {
  char *end = nullptr;
  x = std::strtod(text, &end);
  return end != text && *end == '\0' && x >= lo && x <= hi;
}

/// Next line of `text` from `pos` (without its newline); false at the end.
bool nextLine(const std::string &text, size_t &pos, std::string_view &line) {
  if (pos >= text.size()) return false;
  const size_t eol = std::min(text.find('\n', pos), text.size());
  line = std::string_view(text).substr(pos, eol - pos);
  pos = eol + 1;
  return true;
}

/// Leading integers of a line (blanks between), at most `want` of them.
int leadingIntegers(std::string_view line, long long *out, int want) {
  int got = 0;
  const char *p = line.data(), *end = line.data() + line.size();
  while (got < want) {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    const auto r = std::from_chars(p, end, out[got]);
    if (r.ec != std::errc()) break;
    p = r.ptr;
    ++got;
  }
  return got;
}

/// Matrix Market -> CSR text: a "symmetric" file gives both directions,
/// self-loops and repeated pairs are dropped, every edge gets K weights
/// uniform in [wmin, wmax] drawn edge by edge from mt19937(seed), the draw
/// order the reference's mospPrep uses, so the same seed gives the same
/// files.
int mtxToCsr(const std::string &in, const std::string &prefix, int K, int wmin, int wmax,
             unsigned seed) {
  std::ifstream file(in, std::ios::binary);
  if (!file) {
    std::cerr << in << ": cannot open\n";
    return 1;
  }
  const std::string text((std::istreambuf_iterator<char>(file)), std::istreambuf_iterator<char>());
  size_t pos = 0;
  std::string_view line;
  if (!nextLine(text, pos, line)) {
    std::cerr << in << ": empty file\n";
    return 1;
  }
  const bool symmetric = line.find("symmetric") != std::string_view::npos;
  do {
    if (!nextLine(text, pos, line)) line = std::string_view();
  } while (!line.empty() && line.front() == '%');
  long long size[3] = {0, 0, 0};
  if (leadingIntegers(line, size, 3) != 3 || size[0] <= 0 || size[0] != size[1] ||
      size[0] > INT32_MAX) {
    std::cerr << in << ": the size line is not 'n n entries' for a square matrix\n";
    return 1;
  }
  const long long n = size[0], entries = size[2];
  std::vector<uint64_t> pairs;
  pairs.reserve(static_cast<size_t>(symmetric ? 2 * entries : entries));
  for (long long i = 0; i < entries; ++i) {
    if (!nextLine(text, pos, line)) {
      std::cerr << in << ": " << entries << " entries announced, " << i << " found\n";
      return 1;
    }
    long long ab[2] = {0, 0};
    leadingIntegers(line, ab, 2);
    const long long a = ab[0] - 1, b = ab[1] - 1;  // 1-based in the file
    if (a < 0 || b < 0 || a >= n || b >= n || a == b) continue;
    pairs.push_back(static_cast<uint64_t>(a) << 32 | static_cast<uint32_t>(b));
    if (symmetric) pairs.push_back(static_cast<uint64_t>(b) << 32 | static_cast<uint32_t>(a));
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  CsrGraph g;
  g.numberOfNodes = static_cast<int>(n);
  g.numberOfObjectives = K;
  g.rowPtr.resize(static_cast<size_t>(n) + 1);
  g.colInd.resize(pairs.size());
  size_t e = 0;
  for (int u = 0; u < g.numberOfNodes; ++u) {
    g.rowPtr[u] = static_cast<int>(e);
    for (; e < pairs.size() && (pairs[e] >> 32) == static_cast<uint64_t>(u); ++e) {
      g.colInd[e] = static_cast<int>(pairs[e] & 0xffffffffu);
    }
  }
  g.rowPtr[g.numberOfNodes] = static_cast<int>(e);
  std::mt19937 rng(seed);
  std::uniform_int_distribution<int> draw(wmin, wmax);
  g.weights.resize(pairs.size() * static_cast<size_t>(K));
  std::generate(g.weights.begin(), g.weights.end(), [&] { return draw(rng); });
  if (!writeCsrGraph(prefix, g)) return 1;
  std::cout << "mtx2csr: n=" << g.numberOfNodes << " directed edges=" << g.numberOfEdges()
            << " symmetric=" << symmetric << "\n";
  return 0;
}

/// More objectives for a CSR graph: the existing weights stay, each edge
/// gets K - K_old new ones drawn from mt19937(seed), edge by edge.
int widen(const std::string &in, const std::string &out, int K, int wmin, int wmax, unsigned seed) {
  CsrGraph g;
  if (!readCsrGraph(in, g)) return 1;
  const int had = g.numberOfObjectives;
  if (K < had) {
    std::cerr << in << " has " << had << " objectives already; widen only adds\n";
    return 1;
  }
  std::mt19937 rng(seed);
  std::uniform_int_distribution<int> draw(wmin, wmax);
  const size_t m = static_cast<size_t>(g.numberOfEdges());
  std::vector<int> wide(m * K);
  for (size_t e = 0; e < m; ++e) {
    int *dst = wide.data() + e * K;
    std::copy_n(g.weights.data() + e * had, had, dst);
    std::generate_n(dst + had, K - had, [&] { return draw(rng); });
  }
  g.weights = std::move(wide);
  g.numberOfObjectives = K;
  return writeCsrGraph(out, g) ? 0 : 1;
}

bool changeOptions(int argc, char **argv, int first, ChangeGeneratorOptions &o) {
  for (int i = first; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--safe") {
      o.safeDeletions = true;
      continue;
    }
    if (a == "--gpu") {  // the --safe filter's reachability on the GPU
      useGpuDeletionFilter(true);
      continue;
    }
    if (i + 1 >= argc) {
      std::cerr << "missing value for " << a << "\n";
      return false;
    }
    const std::string v = argv[++i];
    long long x = 0;
    auto integer = [&](long long lo, long long hi) {
      if (parseInteger(v, lo, hi, x)) return true;
      std::cerr << a << " needs an integer in [" << lo << ", " << hi << "], got '" << v << "'\n";
      return false;
    };
    if (a == "--changes") {
      if (!integer(0, INT_MAX)) return false;
      o.numberOfChanges = static_cast<int>(x);
    } else if (a == "--ins") {
      char *end = nullptr;
      o.insertionPercentage = std::strtod(v.c_str(), &end);
      if (v.empty() || *end != '\0' || !(o.insertionPercentage >= 0) || o.insertionPercentage > 100) {
        std::cerr << "--ins needs a percentage in [0, 100], got '" << v << "'\n";
        return false;
      }
    } else if (a == "--mode") {
      if (!parseChangeMode(v, o.mode)) {
        std::cerr << "unknown mode '" << v << "'\n";
        return false;
      }
    } else if (a == "--local") {
      if (!integer(0, INT_MAX)) return false;
      o.localHops = static_cast<int>(x);
    } else if (a == "--seed") {
      if (!integer(0, UINT_MAX)) return false;
      o.seed = static_cast<unsigned>(x);
    } else if (a == "--source") {
      if (!integer(0, INT_MAX)) return false;
      o.source = static_cast<int>(x);
    } else if (a == "--wmin") {
      if (!integer(1, INT_MAX)) return false;
      o.weightMin = static_cast<int>(x);
    } else if (a == "--wmax") {
      if (!integer(1, INT_MAX)) return false;
      o.weightMax = static_cast<int>(x);
    } else {
      std::cerr << "unknown option " << a << "\n";
      return false;
    }
  }
  if (o.weightMin > o.weightMax) {
    std::cerr << "--wmin must not exceed --wmax\n";
    return false;
  }
  return true;
}

/// Trailing "[--source s] [--gpu]" of init / expected.
bool treeOptions(int argc, char **argv, int first, int n, int &source, bool &gpu) {
  source = 0;
  gpu = false;
  for (int i = first; i < argc; ++i) {
    long long v = 0;
    if (std::strcmp(argv[i], "--gpu") == 0) {
      gpu = true;
      continue;
    }
    if (std::strcmp(argv[i], "--source") != 0 || i + 1 >= argc ||
        !parseInteger(argv[i + 1], 0, INT_MAX, v)) {
      std::cerr << "expected --source <vertex>\n";
      return false;
    }
    source = static_cast<int>(v);
    ++i;
  }
  if (source >= n) {
    std::cerr << "source " << source << " out of range [0, " << n << ")\n";
    return false;
  }
  return true;
}

/// Canonical trees of every objective: host Dijkstra, or the GPU engine.
int allTrees(const CsrGraph &g, int source, bool gpu, const std::string &outDir, const char *distName,
             const char *treeName) {
  DeviceGraph device;
  SospWorkspace ws;
  if (gpu && (!uploadDeviceGraph(g, device) || !ws.reserve(g.numberOfNodes))) return 1;
  for (int k = 0; k < g.numberOfObjectives; ++k) {
    const auto t = std::chrono::steady_clock::now();
    std::vector<long long> dist;
    std::vector<int> parent;
    if (gpu) {
      long long maxW = 1, sum = 0;
      for (int e = 0; e < g.numberOfEdges(); ++e) {
        maxW = std::max<long long>(maxW, g.weight(e, k));
        sum += g.weight(e, k);
      }
      DeviceArray<long long> dd(g.numberOfNodes);
      DeviceArray<int> dp(g.numberOfNodes);
      if (!sospFromScratchGpu(device.out(k), source, defaultDelta(g.numberOfEdges(), g.numberOfNodes, sum),
                              maxW, ws, dd.data(), dp.data()) ||
          !dd.download(dist) || !dp.download(parent)) {
        return 1;
      }
    } else {
      dijkstraCsrGraph(g, k, source, dist, parent);
    }
    const std::string dir = outDir + "/obj" + std::to_string(k);
    if (!writeDistances(dir + "/" + distName, dist) || !writeParents(dir + "/" + treeName, parent)) {
      return 1;
    }
    std::cout << (gpu ? "gpu sssp obj" : "dijkstra obj") << k << ": " << msSince(t) << " ms\n";
  }
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) return usage();
  const std::string cmd = argv[1];
  const auto start = std::chrono::steady_clock::now();
  int rc = 0, K = 0, wmin = 0, wmax = 0, source = 0;
  unsigned seed = 0;
  bool gpu = false;
  if (cmd == "mtx2csr" && argc == 8) {
    if (!weightArguments(argv + 4, K, wmin, wmax, seed)) return usage();
    rc = mtxToCsr(argv[2], argv[3], K, wmin, wmax, seed);
  } else if (cmd == "widen" && argc == 8) {
    if (!weightArguments(argv + 4, K, wmin, wmax, seed)) return usage();
    rc = widen(argv[2], argv[3], K, wmin, wmax, seed);
  } else if (cmd == "cache" && argc == 4) {
    CsrGraph g;
    rc = readCsrGraph(argv[2], g) && saveCsrGraphBinary(argv[3], g, argv[2]) ? 0 : 1;
  } else if (cmd == "changes" && argc >= 4) {
    ChangeGeneratorOptions o;
    if (!changeOptions(argc, argv, 4, o)) return usage();
    CsrGraph g;
    ChangeBatch b;
    std::string report;
    const std::string dir = argv[3];
    rc = readCsrGraph(argv[2], g) && generateChangeBatch(g, o, b, &report) &&
                 writeChangeBatch(b, dir + "/insert.txt", dir + "/delete.txt")
             ? 0
             : 1;
    std::cout << "changes: " << report << "\n";
    if (o.safeDeletions) std::cout << "safe filter: " << lastDeletionFilterMs() << " ms\n";
  } else if (cmd == "init" && argc >= 4) {
    CsrGraph g;
    if (!readCsrGraph(argv[2], g)) {
      rc = 1;
    } else if (!treeOptions(argc, argv, 4, g.numberOfNodes, source, gpu)) {
      return usage();
    } else {
      rc = allTrees(g, source, gpu, argv[3], "distancesOriginal.txt", "SSSPTreeOriginal.txt");
    }
  } else if (cmd == "expected" && argc >= 5) {
    CsrGraph original, updated;
    ChangeBatch b;
    const std::string changes = argv[3];
    if (!readCsrGraph(argv[2], original) ||
        !readChangeBatch(changes + "/insert.txt", changes + "/delete.txt",
                         original.numberOfObjectives, original.numberOfNodes, b) ||
        !applyChangeBatch(original, b, updated)) {
      rc = 1;
    } else if (!treeOptions(argc, argv, 5, original.numberOfNodes, source, gpu)) {
      return usage();
    } else {
      rc = allTrees(updated, source, gpu, argv[4], "distancesUpdated.txt", "SSSPTreeUpdated.txt");
    }
  } else if (cmd == "grid" && argc == 11) {
    long long w = 0, h = 0;
    double keep = 0, shortcut = 0;
    if (!parseInteger(argv[3], 1, 46340, w) || !parseInteger(argv[4], 1, 46340, h) ||
        !parseReal(argv[5], 0, 1, keep) || !parseReal(argv[6], 0, 1, shortcut) ||
        !weightArguments(argv + 7, K, wmin, wmax, seed)) {
      return usage();
    }
    CsrGraph g;
    rc = generateGridRoad(static_cast<int>(w), static_cast<int>(h), keep, shortcut, K, wmin, wmax,
                          seed, g) &&
                 writeCsrGraph(argv[2], g)
             ? 0
             : 1;
    std::cout << "grid: n=" << g.numberOfNodes << " directed edges=" << g.numberOfEdges() << "\n";
  } else if (cmd == "rmat" && argc == 13) {
    long long scale = 0, ef = 0, logw = 0;
    double a = 0, b = 0, c = 0;
    if (!parseInteger(argv[3], 1, 30, scale) || !parseInteger(argv[4], 1, 1024, ef) ||
        !parseReal(argv[5], 0, 1, a) || !parseReal(argv[6], 0, 1, b) || !parseReal(argv[7], 0, 1, c) ||
        !parseInteger(argv[11], 0, 1, logw)) {
      return usage();
    }
    char *wargs[4] = {argv[8], argv[9], argv[10], argv[12]};
    if (!weightArguments(wargs, K, wmin, wmax, seed)) return usage();
    CsrGraph g;
    rc = generateRmat(static_cast<int>(scale), static_cast<int>(ef), a, b, c, K, wmin, wmax,
                      logw != 0, seed, g) &&
                 writeCsrGraph(argv[2], g)
             ? 0
             : 1;
    std::cout << "rmat: n=" << g.numberOfNodes << " directed edges=" << g.numberOfEdges() << "\n";
  } else if (cmd == "nearchanges" && argc >= 8) {
    long long width = 0, ins = 0, del = 0, dist = 0;
    if (!parseInteger(argv[4], 1, INT_MAX, width) || !parseInteger(argv[5], 0, INT_MAX, ins) ||
        !parseInteger(argv[6], 0, INT_MAX, del) || !parseInteger(argv[7], 1, 1024, dist)) {
      return usage();
    }
    ChangeGeneratorOptions o;
    if (!changeOptions(argc, argv, 8, o)) return usage();
    CsrGraph g;
    ChangeBatch b;
    const std::string dir = argv[3];
    rc = readCsrGraph(argv[2], g) &&
                 generateNearBatch(g, static_cast<int>(width), static_cast<int>(ins),
                                   static_cast<int>(del), static_cast<int>(dist), o.safeDeletions,
                                   o.seed, o.source, o.weightMin, o.weightMax, b) &&
                 writeChangeBatch(b, dir + "/insert.txt", dir + "/delete.txt")
             ? 0
             : 1;
    std::cout << "nearchanges: inserts=" << b.numberOfInserts() << " deletes=" << b.numberOfDeletes()
              << "\n";
  } else {
    return usage();
  }
  std::cout << cmd << " done in " << msSince(start) << " ms (rc=" << rc << ")\n";
  return rc;
}
