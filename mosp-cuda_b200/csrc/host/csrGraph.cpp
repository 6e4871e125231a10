// csrGraph.cpp - host data model, text and binary formats, batch
// application (interface: include/csrGraph.cuh; formats and semantics of
// SMShovan/MOSP-CUDA src/csrGraph.cu:405-1064).
#include "csrGraph.cuh"
#include "hostCore.h"

#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <chrono>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <functional>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

namespace {

namespace fs = std::filesystem;

bool slurp(const std::string &path, std::string &text) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (f == nullptr) return false;
  struct stat st;
  if (fstat(fileno(f), &st) != 0) {
    std::fclose(f);
    return false;
  }
  text.resize(static_cast<size_t>(st.st_size));
  const size_t got = text.empty() ? 0 : std::fread(&text[0], 1, text.size(), f);
  std::fclose(f);
  return got == text.size();
}

void makeParentDir(const std::string &path) {
  const fs::path parent = fs::path(path).parent_path();
  if (!parent.empty()) {
    std::error_code ec;
    fs::create_directories(parent, ec);
  }
}

/// Buffered writer of decimal integers and short strings.
class Writer {
public:
  explicit Writer(const std::string &path) {
    makeParentDir(path);
    file_ = std::fopen(path.c_str(), "wb");
    buf_.reserve(kChunk + 64);
  }
  ~Writer() { close(); }
  bool ok() const { return file_ != nullptr && good_; }
  void num(long long v) {
    char d[24];
    const auto r = std::to_chars(d, d + sizeof(d), v);
    buf_.append(d, r.ptr);
    spill();
  }
  void str(const char *s) {
    buf_.append(s);
    spill();
  }
  void ch(char c) {
    buf_.push_back(c);
    spill();
  }
  bool close() {
    if (file_ == nullptr) return good_;
    flush();
    if (std::fclose(file_) != 0) good_ = false;
    file_ = nullptr;
    return good_;
  }

private:
  static constexpr size_t kChunk = 1u << 22;
  void spill() {
    if (buf_.size() >= kChunk) flush();
  }
  void flush() {
    if (file_ != nullptr && !buf_.empty() &&
        std::fwrite(buf_.data(), 1, buf_.size(), file_) != buf_.size()) {
      good_ = false;
    }
    buf_.clear();
  }
  FILE *file_ = nullptr;
  std::string buf_;
  bool good_ = true;
};

/// Cursor over an in-memory text file.
class Cursor {
public:
  explicit Cursor(const std::string &t) : begin_(t.data()), p_(t.data()), end_(t.data() + t.size()) {}
  /// Bytes [from, to) of t; line numbers still count from the start of t.
  Cursor(const std::string &t, size_t from, size_t to)
      : begin_(t.data()), p_(t.data() + from), end_(t.data() + to) {}
  size_t offset() const { return static_cast<size_t>(p_ - begin_); }
  void blanks() {
    while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\r')) ++p_;
  }
  void space() {
    while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\r' || *p_ == '\n')) ++p_;
  }
  bool done() const { return p_ >= end_; }
  bool eol() const { return p_ < end_ && *p_ == '\n'; }
  void next() { ++p_; }
  bool literal(const char *w) {
    const size_t len = std::strlen(w);
    if (static_cast<size_t>(end_ - p_) >= len && std::memcmp(p_, w, len) == 0) {
      p_ += len;
      return true;
    }
    return false;
  }
  bool integer(long long &v) {
    const auto r = std::from_chars(p_, end_, v);
    if (r.ec != std::errc()) return false;
    p_ = r.ptr;
    return true;
  }
  long long line() const { return 1 + static_cast<long long>(std::count(begin_, p_, '\n')); }

private:
  const char *begin_, *p_, *end_;
};

std::string at(const std::string &path, long long line) { return path + ":" + std::to_string(line); }

[[gnu::cold, gnu::noinline]] bool errorAt(const char *what, const std::string &path, long long line) {
  std::cout << "Error: " << what << " at " << at(path, line) << ".\n";
  return false;
}

bool validWeight(long long w) { return w >= 1 && w <= INT_MAX; }

// --- parallel text I/O --------------------------------------------------------
// Text files are parsed and formatted in chunks on all host cores: a chunk
// boundary is moved to the next line start, every chunk is parsed on its
// own, and the first error in file order is reported (the one a sequential
// parse stops at). Formatting writes each chunk to its own buffer and the
// buffers to the file in order, so the bytes equal a sequential writer's.

int ioParts(size_t bytes) {
  unsigned hc = std::thread::hardware_concurrency();
  if (hc == 0) hc = 4;
  const size_t byMb = std::max<size_t>(1, bytes >> 20);
  return static_cast<int>(std::min<size_t>(std::min<unsigned>(hc, 64u), byMb));
}

/// parts + 1 offsets into text, each after a newline (or 0 / size).
std::vector<size_t> lineChunks(const std::string &text, int parts) {
  std::vector<size_t> b(static_cast<size_t>(parts) + 1, text.size());
  b[0] = 0;
  for (int i = 1; i < parts; ++i) {
    size_t pos = std::max(b[i - 1], text.size() / parts * i);
    while (pos < text.size() && pos > 0 && text[pos - 1] != '\n') ++pos;
    b[i] = pos;
  }
  return b;
}

void parallelRun(int parts, const std::function<void(int)> &fn) {
  if (parts <= 1) {
    fn(0);
    return;
  }
  std::vector<std::thread> threads;
  threads.reserve(parts);
  for (int i = 0; i < parts; ++i) threads.emplace_back([&fn, i] { fn(i); });
  for (auto &t : threads) t.join();
}

/// First error of a chunked parse: byte offset (SIZE_MAX: none) and message
/// builder given the line number.
struct ChunkError {
  size_t pos = SIZE_MAX;
  std::function<std::string(long long)> message;
  void set(size_t at, std::function<std::string(long long)> m) {
    if (at < pos) {
      pos = at;
      message = std::move(m);
    }
  }
};

long long lineOf(const std::string &text, size_t pos) {
  return 1 + static_cast<long long>(std::count(text.begin(), text.begin() + pos, '\n'));
}

/// Whitespace-separated tokens in text[from, to).
size_t countTokens(const std::string &text, size_t from, size_t to) {
  size_t tokens = 0;
  bool inToken = false;
  const char *p = text.data();
  for (size_t i = from; i < to; ++i) {
    const char ch = p[i];
    const bool blank = ch == ' ' || ch == '\n' || ch == '\t' || ch == '\r';
    tokens += (!blank && !inToken) ? 1 : 0;
    inToken = !blank;
  }
  return tokens;
}

/// Exclusive prefix of per-chunk token counts (counted in parallel).
std::vector<size_t> tokenOffsets(const std::string &text, const std::vector<size_t> &b) {
  const int parts = static_cast<int>(b.size()) - 1;
  std::vector<size_t> at(static_cast<size_t>(parts) + 1, 0);
  parallelRun(parts, [&](int i) { at[i + 1] = countTokens(text, b[i], b[i + 1]); });
  for (int i = 0; i < parts; ++i) at[i + 1] += at[i];
  return at;
}

/// Whitespace-separated integers in [0, INT_MAX] (ids and offsets).
bool parseIds(const std::string &path, std::vector<int> &out, std::string &err) {
  std::string text;
  if (!slurp(path, text)) {
    err = "could not read " + path;
    return false;
  }
  const int parts = ioParts(text.size());
  const std::vector<size_t> b = lineChunks(text, parts);
  // count the tokens first so that every chunk parses straight into place
  const std::vector<size_t> start = tokenOffsets(text, b);
  out.assign(start[parts], 0);
  std::vector<ChunkError> errs(parts);
  parallelRun(parts, [&](int i) {
    Cursor c(text, b[i], b[i + 1]);
    int *o = out.data() + start[i];
    long long v = 0;
    c.space();
    while (!c.done()) {
      const size_t pos = c.offset();
      if (!c.integer(v)) {
        errs[i].set(pos, [path](long long line) { return "invalid token at " + path + ":" + std::to_string(line); });
        return;
      }
      if (v < 0 || v > INT_MAX) {
        errs[i].set(pos, [path, v](long long line) {
          return "value " + std::to_string(v) + " out of range [0, " + std::to_string(INT_MAX) + "] at " +
                 path + ":" + std::to_string(line);
        });
        return;
      }
      *o++ = static_cast<int>(v);
      c.space();
    }
  });
  for (int i = 0; i < parts; ++i) {
    if (errs[i].pos != SIZE_MAX) {
      err = errs[i].message(lineOf(text, errs[i].pos));
      return false;
    }
  }
  return true;
}

/// Values file: one line of K weights per edge (K taken from the first
/// line that has any).
bool parseValues(const std::string &path, std::vector<int> &w, int &K, long long &lines,
                 std::string &err) {
  std::string text;
  if (!slurp(path, text)) {
    err = "Could not read CSR values file " + path + ".";
    return false;
  }
  const int parts = ioParts(text.size());
  const std::vector<size_t> b = lineChunks(text, parts);
  const std::vector<size_t> start = tokenOffsets(text, b);
  w.assign(start[parts], 0);
  std::vector<ChunkError> errs(parts);
  std::vector<int> chunkK(parts, 0);
  std::vector<size_t> firstLine(parts, SIZE_MAX);
  std::vector<long long> chunkLines(parts, 0);
  parallelRun(parts, [&](int i) {
    Cursor c(text, b[i], b[i + 1]);
    int *o = w.data() + start[i];
    for (;;) {
      c.blanks();
      const size_t lineStart = c.offset();
      int count = 0;
      long long v = 0;
      while (!c.done() && !c.eol()) {
        const size_t at = c.offset();
        if (!c.integer(v)) {
          errs[i].set(at, [path](long long line) {
            return "Invalid token in CSR values file at " + path + ":" + std::to_string(line) + ".";
          });
          return;
        }
        if (!validWeight(v)) {
          errs[i].set(at, [path, v](long long line) {
            return "CSR weight " + std::to_string(v) + " out of range [1, " + std::to_string(INT_MAX) +
                   "] at " + path + ":" + std::to_string(line) + ".";
          });
          return;
        }
        *o++ = static_cast<int>(v);
        ++count;
        c.blanks();
      }
      if (count > 0) {
        if (chunkK[i] == 0) {
          chunkK[i] = count;
          firstLine[i] = lineStart;
        } else if (count != chunkK[i]) {
          errs[i].set(c.offset(), [path](long long line) {
            return "Inconsistent number of objectives at " + path + ":" + std::to_string(line) + ".";
          });
          return;
        }
        ++chunkLines[i];
      }
      if (c.done()) break;
      c.next();
    }
  });
  K = 0;
  lines = 0;
  for (int i = 0; i < parts; ++i) {
    // a chunk whose lines have another width than the file's first line
    // fails at its own first line, before any error inside the chunk
    if (chunkK[i] != 0 && K != 0 && chunkK[i] != K) {
      err = "Inconsistent number of objectives at " + path + ":" +
            std::to_string(lineOf(text, firstLine[i])) + ".";
      return false;
    }
    if (errs[i].pos != SIZE_MAX) {
      err = errs[i].message(lineOf(text, errs[i].pos));
      return false;
    }
    if (K == 0) K = chunkK[i];
    lines += chunkLines[i];
  }
  return true;
}

constexpr char kMagic[8] = {'M', 'O', 'S', 'P', 'C', 'S', 'R', '2'};

/// Where a binary cache came from: canonical text prefix, sizes and mtimes
/// (ns) of the three text files.
struct Origin {
  std::string prefix;
  int64_t size[3] = {0, 0, 0};
  int64_t mtime[3] = {0, 0, 0};
  bool operator==(const Origin &o) const {
    return prefix == o.prefix && std::equal(size, size + 3, o.size) &&
           std::equal(mtime, mtime + 3, o.mtime);
  }
};

bool originOf(const std::string &prefix, Origin &o) {
  std::error_code ec;
  const fs::path canon = fs::weakly_canonical(prefix, ec);
  if (ec) return false;
  o.prefix = canon.string();
  const char *suffix[3] = {"RowPtr.txt", "ColInd.txt", "Values.txt"};
  for (int i = 0; i < 3; ++i) {
    const std::string file = prefix + suffix[i];
    const auto sz = fs::file_size(file, ec);
    if (ec) return false;
    const auto t = fs::last_write_time(file, ec);
    if (ec) return false;
    o.size[i] = static_cast<int64_t>(sz);
    o.mtime[i] = static_cast<int64_t>(
        std::chrono::duration_cast<std::chrono::nanoseconds>(t.time_since_epoch()).count());
  }
  return true;
}

/// CSR invariants of arrays read from a cache, checked in parallel chunks.
bool csrArraysValid(const CsrGraph &g) {
  const int n = g.numberOfNodes;
  const size_t m = g.colInd.size();
  if (g.rowPtr.size() != static_cast<size_t>(n) + 1 || g.rowPtr[0] != 0 ||
      static_cast<size_t>(g.rowPtr[n]) != m ||
      g.weights.size() != m * static_cast<size_t>(g.numberOfObjectives)) {
    return false;
  }
  constexpr int kParts = 16;
  std::vector<std::function<bool()>> jobs;
  for (int j = 0; j < kParts; ++j) {
    jobs.push_back([&g, j, n, m] {
      auto part = [](size_t size, int i) { return size * i / kParts; };
      const size_t r = g.rowPtr.size(), w = g.weights.size();
      for (size_t i = std::max<size_t>(part(r, j), 1); i < part(r, j + 1); ++i) {
        if (g.rowPtr[i] < g.rowPtr[i - 1]) return false;
      }
      for (size_t i = part(m, j); i < part(m, j + 1); ++i) {
        if (g.colInd[i] < 0 || g.colInd[i] >= n) return false;
      }
      for (size_t i = part(w, j); i < part(w, j + 1); ++i) {
        if (g.weights[i] < 1) return false;
      }
      return true;
    });
  }
  return runConcurrently(jobs);
}

}  // namespace

// ---------------------------------------------------------------------------

namespace mospb200 {

bool writeLinesParallel(const std::string &path, size_t count,
                        const std::function<void(size_t, std::string &)> &line) {
  makeParentDir(path);
  FILE *f = std::fopen(path.c_str(), "wb");
  if (f == nullptr) return false;
  // chunks of about 64K lines, formatted in waves of one chunk per core
  const int parts = static_cast<int>(std::max<size_t>(1, (count + 65535) >> 16));
  std::vector<std::string> bufs(parts);
  bool ok = true;
  const int wave = ioParts(count * 8);
  for (int w0 = 0; w0 < parts && ok; w0 += wave) {
    const int w1 = std::min(parts, w0 + wave);
    parallelRun(w1 - w0, [&](int j) {
      const int i = w0 + j;
      const size_t a = count * static_cast<size_t>(i) / parts;
      const size_t z = count * static_cast<size_t>(i + 1) / parts;
      std::string &out = bufs[i];
      out.reserve((z - a) * 12);
      for (size_t x = a; x < z; ++x) line(x, out);
    });
    for (int i = w0; i < w1 && ok; ++i) {
      ok = std::fwrite(bufs[i].data(), 1, bufs[i].size(), f) == bufs[i].size();
      std::string().swap(bufs[i]);
    }
  }
  return (std::fclose(f) == 0) && ok;
}

}  // namespace mospb200

using mospb200::writeLinesParallel;

bool runConcurrently(const std::vector<std::function<bool()>> &jobs) {
  std::vector<char> ok(jobs.size(), 0);
  std::vector<std::thread> threads;
  threads.reserve(jobs.size());
  for (size_t i = 0; i < jobs.size(); ++i) {
    threads.emplace_back([&, i] { ok[i] = jobs[i]() ? 1 : 0; });
  }
  for (auto &t : threads) t.join();
  return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
}

bool parseInteger(const std::string &text, long long minimum, long long maximum,
                  long long &value) {
  if (text.empty() || std::isspace(static_cast<unsigned char>(text[0])) || text[0] == '+') {
    return false;
  }
  char *end = nullptr;
  errno = 0;
  value = std::strtoll(text.c_str(), &end, 10);
  return errno == 0 && *end == '\0' && value >= minimum && value <= maximum;
}

bool readCsrGraph(const std::string &prefix, CsrGraph &graph) {
  graph = CsrGraph();
  bool rowsOk = false, colsOk = false, valsOk = false;
  int K = 0;
  long long lines = 0;
  std::string rowsErr, colsErr, valsErr;
  runConcurrently({
      [&] { return rowsOk = parseIds(prefix + "RowPtr.txt", graph.rowPtr, rowsErr); },
      [&] { return colsOk = parseIds(prefix + "ColInd.txt", graph.colInd, colsErr); },
      [&] { return valsOk = parseValues(prefix + "Values.txt", graph.weights, K, lines, valsErr); },
  });
  if (!rowsOk) {
    std::cout << "Error: CSR row pointers: " << rowsErr << "\n";
    return false;
  }
  if (graph.rowPtr.size() < 2) {
    std::cout << "Error: Could not read CSR row pointers: " << prefix << "RowPtr.txt\n";
    return false;
  }
  graph.numberOfNodes = static_cast<int>(graph.rowPtr.size()) - 1;
  const int m = graph.rowPtr.back();
  if (graph.rowPtr[0] != 0) {
    std::cout << "Error: CSR row pointers must start at 0.\n";
    return false;
  }
  for (int i = 0; i < graph.numberOfNodes; ++i) {
    if (graph.rowPtr[i + 1] < graph.rowPtr[i]) {
      std::cout << "Error: CSR row pointers are not monotone.\n";
      return false;
    }
  }
  if (!colsOk) {
    std::cout << "Error: CSR column indices: " << colsErr << "\n";
    return false;
  }
  if (static_cast<long long>(graph.colInd.size()) != m) {
    std::cout << "Error: CSR column index file missing or size mismatch.\n";
    return false;
  }
  for (int v : graph.colInd) {
    if (v >= graph.numberOfNodes) {
      std::cout << "Error: CSR column index out of range.\n";
      return false;
    }
  }
  if (!valsOk) {
    std::cout << "Error: " << valsErr << "\n";
    return false;
  }
  if (lines != m) {
    std::cout << "Error: values size mismatch.\n";
    return false;
  }
  graph.numberOfObjectives = K;
  return true;
}

bool writeCsrGraph(const std::string &prefix, const CsrGraph &graph) {
  const int K = graph.numberOfObjectives;
  bool okRows = false, okCols = false, okVals = false;
  auto num = [](std::string &out, long long x) {
    char d[24];
    out.append(d, std::to_chars(d, d + sizeof(d), x).ptr);
  };
  runConcurrently({
      [&] {
        return okRows = writeLinesParallel(prefix + "RowPtr.txt", graph.rowPtr.size(),
                                           [&](size_t i, std::string &out) {
                                             num(out, graph.rowPtr[i]);
                                             out.push_back('\n');
                                           });
      },
      [&] {
        return okCols = writeLinesParallel(prefix + "ColInd.txt", graph.colInd.size(),
                                           [&](size_t i, std::string &out) {
                                             num(out, graph.colInd[i]);
                                             out.push_back('\n');
                                           });
      },
      [&] {
        return okVals = writeLinesParallel(
                   prefix + "Values.txt", static_cast<size_t>(graph.numberOfEdges()),
                   [&](size_t e, std::string &out) {
                     for (int k = 0; k < K; ++k) {
                       num(out, graph.weight(static_cast<int>(e), k));
                       if (k + 1 < K) out.push_back(' ');
                     }
                     out.push_back('\n');
                   });
      },
  });
  if (!okRows || !okCols || !okVals) {
    std::cout << "Error: Could not write CSR files: " << prefix << "\n";
    return false;
  }
  return true;
}

bool saveCsrGraphBinary(const std::string &path, const CsrGraph &graph,
                        const std::string &sourcePrefix) {
  Origin o;
  if (!originOf(sourcePrefix, o)) return false;
  makeParentDir(path);
  FILE *f = std::fopen(path.c_str(), "wb");
  if (f == nullptr) return false;
  const int32_t header[2] = {graph.numberOfNodes, graph.numberOfObjectives};
  const int64_t m = graph.numberOfEdges();
  const int64_t plen = static_cast<int64_t>(o.prefix.size());
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(&plen, sizeof(plen), 1, f) == 1 &&
            std::fwrite(o.prefix.data(), 1, o.prefix.size(), f) == o.prefix.size() &&
            std::fwrite(o.size, sizeof(o.size), 1, f) == 1 &&
            std::fwrite(o.mtime, sizeof(o.mtime), 1, f) == 1 &&
            std::fwrite(header, sizeof(header), 1, f) == 1 && std::fwrite(&m, sizeof(m), 1, f) == 1 &&
            std::fwrite(graph.rowPtr.data(), sizeof(int), graph.rowPtr.size(), f) == graph.rowPtr.size() &&
            std::fwrite(graph.colInd.data(), sizeof(int), graph.colInd.size(), f) == graph.colInd.size() &&
            std::fwrite(graph.weights.data(), sizeof(int), graph.weights.size(), f) == graph.weights.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    std::error_code ec;
    fs::remove(path, ec);
  }
  return ok;
}

bool loadCsrGraphBinary(const std::string &path, CsrGraph &graph, const std::string &sourcePrefix) {
  Origin expected, recorded;
  if (!originOf(sourcePrefix, expected)) return false;
  FILE *f = std::fopen(path.c_str(), "rb");
  if (f == nullptr) return false;
  char magic[8];
  int32_t header[2] = {0, 0};
  int64_t m = 0, plen = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 &&
            std::fread(&plen, sizeof(plen), 1, f) == 1 && plen >= 0 && plen <= (1 << 16);
  if (ok) {
    recorded.prefix.resize(static_cast<size_t>(plen));
    ok = std::fread(&recorded.prefix[0], 1, recorded.prefix.size(), f) == recorded.prefix.size() &&
         std::fread(recorded.size, sizeof(recorded.size), 1, f) == 1 &&
         std::fread(recorded.mtime, sizeof(recorded.mtime), 1, f) == 1 && recorded == expected;
  }
  ok = ok && std::fread(header, sizeof(header), 1, f) == 1 && std::fread(&m, sizeof(m), 1, f) == 1 &&
       header[0] > 0 && header[1] > 0 && header[1] <= 32 && m >= 0 && m <= INT_MAX;
  if (ok) {
    // the header must agree with the file length before anything is allocated
    std::error_code ec;
    const uintmax_t fileSize = fs::file_size(path, ec);
    const long pos = std::ftell(f);
    const uint64_t bytes = sizeof(int) * (static_cast<uint64_t>(header[0]) + 1 +
                                          static_cast<uint64_t>(m) * (1 + header[1]));
    ok = !ec && pos >= 0 && fileSize == static_cast<uintmax_t>(pos) + bytes;
  }
  if (ok) {
    graph.numberOfNodes = header[0];
    graph.numberOfObjectives = header[1];
    graph.rowPtr.resize(static_cast<size_t>(header[0]) + 1);
    graph.colInd.resize(static_cast<size_t>(m));
    graph.weights.resize(static_cast<size_t>(m) * header[1]);
    ok = std::fread(graph.rowPtr.data(), sizeof(int), graph.rowPtr.size(), f) == graph.rowPtr.size() &&
         std::fread(graph.colInd.data(), sizeof(int), graph.colInd.size(), f) == graph.colInd.size() &&
         std::fread(graph.weights.data(), sizeof(int), graph.weights.size(), f) == graph.weights.size() &&
         std::fgetc(f) == EOF && csrArraysValid(graph);
  }
  std::fclose(f);
  if (!ok) graph = CsrGraph();
  return ok;
}

bool loadCsrGraph(const std::string &prefix, CsrGraph &graph, const std::string &cachePath) {
  if (!cachePath.empty()) {
    if (loadCsrGraphBinary(cachePath, graph, prefix)) return true;
    std::error_code ec;
    if (fs::exists(cachePath, ec)) {
      std::cout << "Note: binary cache " << cachePath << " does not match the text graph " << prefix
                << " (another graph, changed files or an old format); rebuilding it.\n";
    }
  }
  if (!readCsrGraph(prefix, graph)) return false;
  if (!cachePath.empty() && !saveCsrGraphBinary(cachePath, graph, prefix)) {
    std::cout << "Warning: could not write binary cache " << cachePath << "\n";
  }
  return true;
}

bool readChangeBatch(const std::string &insertPath, const std::string &deletePath,
                     int numberOfObjectives, int numberOfNodes, ChangeBatch &batch) {
  batch = ChangeBatch();
  batch.numberOfObjectives = numberOfObjectives;
  auto inRange = [&](long long x) { return x >= 0 && x < numberOfNodes; };
  std::string text;
  if (!slurp(insertPath, text)) {
    std::cout << "Error: Could not open insert file: " << insertPath << "\n";
    return false;
  }
  {
    Cursor c(text);
    std::vector<long long> tok;
    for (;;) {
      c.blanks();
      tok.clear();
      long long v = 0;
      while (!c.done() && !c.eol()) {
        if (!c.integer(v)) return errorAt("Invalid insert line", insertPath, c.line());
        tok.push_back(v);
        c.blanks();
      }
      if (!tok.empty()) {
        if (static_cast<int>(tok.size()) < 2 + numberOfObjectives) {
          return errorAt("Invalid insert line", insertPath, c.line());
        }
        if (!inRange(tok[0]) || !inRange(tok[1])) {
          return errorAt("Inserted edge endpoint out of range", insertPath, c.line());
        }
        for (int k = 0; k < numberOfObjectives; ++k) {
          if (!validWeight(tok[2 + k])) {
            std::cout << "Error: Inserted edge weight " << tok[2 + k] << " out of range [1, "
                      << INT_MAX << "] at " << at(insertPath, c.line()) << ".\n";
            return false;
          }
        }
        batch.insertFrom.push_back(static_cast<int>(tok[0]));
        batch.insertTo.push_back(static_cast<int>(tok[1]));
        for (int k = 0; k < numberOfObjectives; ++k) {
          batch.insertWeights.push_back(static_cast<int>(tok[2 + k]));
        }
      }
      if (c.done()) break;
      c.next();
    }
  }
  if (!slurp(deletePath, text)) {
    std::cout << "Error: Could not open delete file: " << deletePath << "\n";
    return false;
  }
  Cursor c(text);
  for (;;) {
    c.blanks();
    long long pair[2] = {0, 0};
    int count = 0;
    long long v = 0;
    while (!c.done() && !c.eol()) {
      if (!c.integer(v)) return errorAt("Invalid delete line", deletePath, c.line());
      if (count < 2) pair[count] = v;
      ++count;
      c.blanks();
    }
    if (count >= 2) {  // lines with fewer than two values are skipped
      if (!inRange(pair[0]) || !inRange(pair[1])) {
        return errorAt("Deleted edge endpoint out of range", deletePath, c.line());
      }
      batch.deleteFrom.push_back(static_cast<int>(pair[0]));
      batch.deleteTo.push_back(static_cast<int>(pair[1]));
    }
    if (c.done()) break;
    c.next();
  }
  return true;
}

bool applyChangeBatch(const CsrGraph &original, ChangeBatch &batch, CsrGraph &updated) {
  return mospb200::applyBatchView(mospb200::viewOf(original), mospb200::viewOf(batch), updated,
                                  batch.weightIncreaseMask);
}

namespace mospb200 {

bool applyBatchView(const GraphView &g, const BatchView &b, CsrGraph &updated,
                    std::vector<unsigned> &mask) {
  const int n = g.n;
  const int K = g.K;
  if (b.K != K) {
    std::cout << "Error: change batch has " << b.K << " objectives, graph has " << K << ".\n";
    return false;
  }
  if (K > 32) {
    std::cout << "Error: at most 32 objectives are supported.\n";
    return false;
  }
  const int nIns = b.nIns, nDel = b.nDel;
  // Bucket the changes by source row (stable: file order within a row).
  std::vector<int> delStart(static_cast<size_t>(n) + 1, 0), insStart(static_cast<size_t>(n) + 1, 0);
  for (int i = 0; i < nDel; ++i) ++delStart[b.delFrom[i] + 1];
  for (int i = 0; i < nIns; ++i) ++insStart[b.insFrom[i] + 1];
  for (int u = 0; u < n; ++u) {
    delStart[u + 1] += delStart[u];
    insStart[u + 1] += insStart[u];
  }
  std::vector<int> delOf(nDel), insOf(nIns);
  {
    std::vector<int> fill(delStart.begin(), delStart.end() - 1);
    for (int i = 0; i < nDel; ++i) delOf[fill[b.delFrom[i]]++] = i;
    fill.assign(insStart.begin(), insStart.end() - 1);
    for (int i = 0; i < nIns; ++i) insOf[fill[b.insFrom[i]]++] = i;
  }
  // A changed row is a list of (head, source of its weights): source >= 0
  // is an original edge, source < 0 insertion -source-1; dead entries are
  // deletions.
  struct Slot {
    int head;
    long long from;
    bool live;
  };
  std::vector<int> rowOf(n, -1);
  std::vector<std::vector<Slot>> rows;
  for (int u = 0; u < n; ++u) {
    if (delStart[u] == delStart[u + 1] && insStart[u] == insStart[u + 1]) continue;
    std::vector<Slot> row;
    row.reserve(g.row[u + 1] - g.row[u] + (insStart[u + 1] - insStart[u]));
    for (int e = g.row[u]; e < g.row[u + 1]; ++e) row.push_back({g.col[e], e, true});
    for (int j = delStart[u]; j < delStart[u + 1]; ++j) {
      const int v = b.delTo[delOf[j]];
      for (Slot &s : row) {
        if (s.live && s.head == v) {
          s.live = false;
          break;
        }
      }
    }
    for (int j = insStart[u]; j < insStart[u + 1]; ++j) {
      const int i = insOf[j];
      const int v = b.insTo[i];
      bool hit = false;
      for (Slot &s : row) {
        if (s.live && s.head == v) {
          s.from = -static_cast<long long>(i) - 1;
          hit = true;
          break;
        }
      }
      if (!hit) row.push_back({v, -static_cast<long long>(i) - 1, true});
    }
    rowOf[u] = static_cast<int>(rows.size());
    rows.push_back(std::move(row));
  }
  updated = CsrGraph();
  updated.numberOfNodes = n;
  updated.numberOfObjectives = K;
  updated.rowPtr.assign(static_cast<size_t>(n) + 1, 0);
  for (int u = 0; u < n; ++u) {
    int deg = g.row[u + 1] - g.row[u];
    if (rowOf[u] >= 0) {
      deg = 0;
      for (const Slot &s : rows[rowOf[u]]) deg += s.live ? 1 : 0;
    }
    updated.rowPtr[u + 1] = updated.rowPtr[u] + deg;
  }
  const size_t m = static_cast<size_t>(updated.rowPtr[n]);
  updated.colInd.resize(m);
  updated.weights.resize(m * K);
  for (int u = 0; u < n; ++u) {
    int out = updated.rowPtr[u];
    if (rowOf[u] < 0) {
      const int lo = g.row[u], hi = g.row[u + 1];
      std::copy(g.col + lo, g.col + hi, updated.colInd.begin() + out);
      std::copy(g.w + static_cast<size_t>(lo) * K, g.w + static_cast<size_t>(hi) * K,
                updated.weights.begin() + static_cast<size_t>(out) * K);
      continue;
    }
    for (const Slot &s : rows[rowOf[u]]) {
      if (!s.live) continue;
      updated.colInd[out] = s.head;
      const int *w = s.from >= 0 ? g.w + static_cast<size_t>(s.from) * K
                                 : b.insW + static_cast<size_t>(-s.from - 1) * K;
      std::copy(w, w + K, updated.weights.begin() + static_cast<size_t>(out) * K);
      ++out;
    }
  }
  // Weight increases: final weights of (u,v) against the original edge
  // (first occurrence of v in row u on both sides).
  mask.assign(nIns, 0u);
  for (int i = 0; i < nIns; ++i) {
    const int u = b.insFrom[i], v = b.insTo[i];
    int before = -1, after = -1;
    for (int e = g.row[u]; e < g.row[u + 1]; ++e) {
      if (g.col[e] == v) {
        before = e;
        break;
      }
    }
    if (before < 0) continue;
    for (int e = updated.rowPtr[u]; e < updated.rowPtr[u + 1]; ++e) {
      if (updated.colInd[e] == v) {
        after = e;
        break;
      }
    }
    if (after < 0) continue;
    unsigned bits = 0;
    for (int k = 0; k < K; ++k) {
      if (updated.weight(after, k) > g.weight(before, k)) bits |= 1u << k;
    }
    mask[i] = bits;
  }
  return true;
}

}  // namespace mospb200

void transposeCsrGraph(const CsrGraph &graph, CsrGraph &reverse) {
  const int n = graph.numberOfNodes, K = graph.numberOfObjectives;
  const size_t m = static_cast<size_t>(graph.numberOfEdges());
  reverse = CsrGraph();
  reverse.numberOfNodes = n;
  reverse.numberOfObjectives = K;
  reverse.rowPtr.assign(static_cast<size_t>(n) + 1, 0);
  for (size_t e = 0; e < m; ++e) ++reverse.rowPtr[graph.colInd[e] + 1];
  for (int v = 0; v < n; ++v) reverse.rowPtr[v + 1] += reverse.rowPtr[v];
  reverse.colInd.resize(m);
  reverse.weights.resize(m * K);
  std::vector<int> fill(reverse.rowPtr.begin(), reverse.rowPtr.end() - 1);
  for (int u = 0; u < n; ++u) {
    for (int e = graph.rowPtr[u]; e < graph.rowPtr[u + 1]; ++e) {
      const int pos = fill[graph.colInd[e]]++;
      reverse.colInd[pos] = u;
      for (int k = 0; k < K; ++k) {
        reverse.weights[static_cast<size_t>(pos) * K + k] = graph.weight(e, k);
      }
    }
  }
}

namespace {

/// Chunked parse of "v x" lines (x an integer, or INF when allowInf): calls
/// store(v, x) for every line (lines of a chunk in order, chunks in
/// parallel, so store must tolerate concurrent calls for distinct v) and
/// returns the number of lines; on the first bad line in file order prints
/// the message of `errorOf(kind)` and returns -1.
template <typename Store>
long long parseVertexLines(const std::string &text, const std::string &path, bool allowInf,
                           long long minX, int numberOfNodes, const char *badLine,
                           const char *badVertex, const char *badValue, Store store) {
  const int parts = ioParts(text.size());
  const std::vector<size_t> b = lineChunks(text, parts);
  std::vector<long long> listed(parts, 0);
  std::vector<size_t> errPos(parts, SIZE_MAX);
  std::vector<const char *> errWhat(parts, nullptr);
  parallelRun(parts, [&](int i) {
    Cursor c(text, b[i], b[i + 1]);
    auto fail = [&](const char *what) {
      errPos[i] = c.offset();
      errWhat[i] = what;
    };
    for (;;) {
      c.space();
      if (c.done()) break;
      long long v = 0, x = 0;
      if (!c.integer(v)) return fail(badLine);
      c.blanks();
      if (allowInf && c.literal("INF")) {
        x = DISTANCE_INF;
      } else if (!c.integer(x)) {
        return fail(badLine);
      }
      if (v < 0 || v >= numberOfNodes || (!allowInf && (x < minX || x >= numberOfNodes))) {
        return fail(badVertex);
      }
      if (allowInf && x < minX) return fail(badValue);
      ++listed[i];
      store(v, x);
    }
  });
  long long total = 0;
  for (int i = 0; i < parts; ++i) {
    if (errPos[i] != SIZE_MAX) {
      errorAt(errWhat[i], path, lineOf(text, errPos[i]));
      return -1;
    }
    total += listed[i];
  }
  return total;
}

}  // namespace

bool readDistances(const std::string &path, int numberOfNodes, std::vector<long long> &distances) {
  std::string text;
  if (!slurp(path, text)) {
    std::cout << "Error: Could not open distances file: " << path << "\n";
    return false;
  }
  distances.assign(numberOfNodes, -1);  // -1: not listed yet
  long long *d = distances.data();
  const long long listed = parseVertexLines(
      text, path, true, 0, numberOfNodes, "Invalid line in distances file",
      "Vertex ID out of range in distances file", "Negative distance",
      [d](long long v, long long x) { __atomic_store_n(d + v, x, __ATOMIC_RELAXED); });
  if (listed < 0) return false;
  if (listed != numberOfNodes ||
      std::find(distances.begin(), distances.end(), -1LL) != distances.end()) {
    std::cout << "Error: " << path << " must list each of the " << numberOfNodes
              << " vertices exactly once (" << listed << " lines).\n";
    return false;
  }
  return true;
}

bool readParents(const std::string &path, int numberOfNodes, std::vector<int> &parent) {
  std::string text;
  if (!slurp(path, text)) {
    std::cout << "Error: Could not open SSSP tree file: " << path << "\n";
    return false;
  }
  parent.assign(numberOfNodes, -2);  // -2: not listed yet
  int *p = parent.data();
  const long long listed = parseVertexLines(
      text, path, false, -1, numberOfNodes, "Invalid line in SSSP tree file",
      "Vertex ID out of range in SSSP tree file", "Vertex ID out of range in SSSP tree file",
      [p](long long v, long long x) { __atomic_store_n(p + v, static_cast<int>(x), __ATOMIC_RELAXED); });
  if (listed < 0) return false;
  if (listed != numberOfNodes || std::find(parent.begin(), parent.end(), -2) != parent.end()) {
    std::cout << "Error: " << path << " must list each of the " << numberOfNodes
              << " vertices exactly once (" << listed << " lines).\n";
    return false;
  }
  return true;
}

bool writeDistances(const std::string &path, const std::vector<long long> &distances) {
  const bool ok = writeLinesParallel(path, distances.size(), [&](size_t v, std::string &out) {
    char d[24];
    out.append(d, std::to_chars(d, d + sizeof(d), static_cast<long long>(v)).ptr);
    out.push_back(' ');
    if (distances[v] >= DISTANCE_INF / 2) {
      out.append("INF");
    } else {
      out.append(d, std::to_chars(d, d + sizeof(d), distances[v]).ptr);
    }
    out.push_back('\n');
  });
  if (!ok) std::cout << "Error: Could not write distances file: " << path << "\n";
  return ok;
}

bool writeParents(const std::string &path, const std::vector<int> &parent) {
  const bool ok = writeLinesParallel(path, parent.size(), [&](size_t v, std::string &out) {
    char d[24];
    out.append(d, std::to_chars(d, d + sizeof(d), static_cast<long long>(v)).ptr);
    out.push_back(' ');
    out.append(d, std::to_chars(d, d + sizeof(d), parent[v]).ptr);
    out.push_back('\n');
  });
  if (!ok) std::cout << "Error: Could not write SSSP tree file: " << path << "\n";
  return ok;
}
