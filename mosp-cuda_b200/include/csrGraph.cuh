#ifndef MOSP_B200_CSR_GRAPH_CUH
#define MOSP_B200_CSR_GRAPH_CUH

// Host data model and file formats of the MOSP update path. Declarations
// match the reference interface (SMShovan/MOSP-CUDA headers/csrGraph.cuh:
// 18-185) so that code written against it compiles unchanged; the
// implementation is this library's (src: csrc/host/csrGraph.cpp).

#include <functional>
#include <string>
#include <vector>

/// Directed multi-objective graph, CSR by source vertex. Objective k of
/// edge e is weights[e * numberOfObjectives + k] (edge-major, the layout of
/// the Values text file).
struct CsrGraph {
  int numberOfNodes = 0;
  int numberOfObjectives = 0;
  std::vector<int> rowPtr;  ///< numberOfNodes + 1 offsets
  std::vector<int> colInd;  ///< head of every edge
  std::vector<int> weights; ///< numberOfObjectives weights per edge

  int numberOfEdges() const { return rowPtr.empty() ? 0 : rowPtr.back(); }
  int weight(int edge, int objective) const {
    return weights[static_cast<size_t>(edge) * numberOfObjectives + objective];
  }
};

/// One batch of edge changes (insert.txt / delete.txt). insertWeights holds
/// numberOfObjectives weights per insertion. applyChangeBatch() fills
/// weightIncreaseMask: bit k of entry i is set when insertion i overwrote an
/// edge of the original graph and raised its objective-k weight.
struct ChangeBatch {
  int numberOfObjectives = 0;
  std::vector<int> insertFrom, insertTo;
  std::vector<int> insertWeights;
  std::vector<int> deleteFrom, deleteTo;
  std::vector<unsigned int> weightIncreaseMask;

  int numberOfInserts() const { return static_cast<int>(insertFrom.size()); }
  int numberOfDeletes() const { return static_cast<int>(deleteFrom.size()); }
};

/// Read <prefix>RowPtr.txt, <prefix>ColInd.txt and <prefix>Values.txt.
/// Rejects offsets that do not start at 0 or decrease, column ids outside
/// [0, n), values above INT_MAX and weights outside [1, INT_MAX]; the
/// message names the file and line.
bool readCsrGraph(const std::string &prefix, CsrGraph &graph);

/// Write a graph in the same three-file text format.
bool writeCsrGraph(const std::string &prefix, const CsrGraph &graph);

/// Save a graph as a binary cache (format MOSPCSR2) of the text graph at
/// sourcePrefix, recording the canonical prefix and the size and mtime of
/// the three text files.
bool saveCsrGraphBinary(const std::string &path, const CsrGraph &graph,
                        const std::string &sourcePrefix);

/// Load a cache written by saveCsrGraphBinary(); fails silently when the
/// file is missing, truncated, of another format, made from other text
/// files (prefix, size or mtime differ) or holds an invalid CSR.
bool loadCsrGraphBinary(const std::string &path, CsrGraph &graph,
                        const std::string &sourcePrefix);

/// Load a text graph, through the binary cache when cachePath is set and
/// the cache matches; otherwise parse the text and (re)write the cache.
bool loadCsrGraph(const std::string &prefix, CsrGraph &graph,
                  const std::string &cachePath = "");

/// Read insert.txt ("u v w1 .. wK") and delete.txt ("u v"); endpoints in
/// [0, numberOfNodes), inserted weights in [1, INT_MAX].
bool readChangeBatch(const std::string &insertPath,
                     const std::string &deletePath, int numberOfObjectives,
                     int numberOfNodes, ChangeBatch &batch);

/// Apply a batch: every deletion removes the first remaining (u,v) edge,
/// then insertions in file order overwrite the weights of an existing
/// (u,v) edge or append a new one (the last insertion of a pair wins).
/// Surviving edges keep their order. Fills batch.weightIncreaseMask.
bool applyChangeBatch(const CsrGraph &original, ChangeBatch &batch,
                      CsrGraph &updated);

/// Reverse graph: row v lists u for every edge u -> v.
void transposeCsrGraph(const CsrGraph &graph, CsrGraph &reverse);

/// Read a distance file ("v d" or "v INF"): every vertex exactly once,
/// no negative distance.
bool readDistances(const std::string &path, int numberOfNodes,
                   std::vector<long long> &distances);

/// Read a parent file ("v p", p = -1 for none): every vertex exactly once,
/// p in [-1, numberOfNodes).
bool readParents(const std::string &path, int numberOfNodes,
                 std::vector<int> &parent);

/// Write distances; values >= DISTANCE_INF / 2 are written as INF.
bool writeDistances(const std::string &path,
                    const std::vector<long long> &distances);

/// Write a parent array.
bool writeParents(const std::string &path, const std::vector<int> &parent);

/// Run independent jobs concurrently; true if every job returned true.
bool runConcurrently(const std::vector<std::function<bool()>> &jobs);

/// Parse a whole decimal integer in [minimum, maximum] (no sign '+', no
/// blanks, no trailing characters).
bool parseInteger(const std::string &text, long long minimum,
                  long long maximum, long long &value);

/// Distance sentinel; values >= DISTANCE_INF / 2 mean unreachable.
constexpr long long DISTANCE_INF = 0x7fffffffffffffffLL / 4;

#endif // MOSP_B200_CSR_GRAPH_CUH
