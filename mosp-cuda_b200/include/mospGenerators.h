#ifndef MOSP_B200_GENERATORS_H
#define MOSP_B200_GENERATORS_H

// Seeded synthetic inputs of the benchmark workloads. The reference measures
// on SuiteSparse road and geometric graphs (bench/prepare.sh); these
// generators produce graphs of the same shape in the reference's CSR format
// (`mospPrep grid|rmat|nearchanges`). No counterpart in the reference.

struct CsrGraph;
struct ChangeBatch;

/// Road-network shape: a width x height grid whose undirected edges are
/// kept with probability keep, plus one diagonal shortcut on a
/// shortcutFraction of the vertices; the largest connected component is
/// kept and renumbered in row-major order; rows are sorted by head; every
/// directed edge gets K weights uniform in [wmin, wmax].
bool generateGridRoad(int width, int height, double keep, double shortcutFraction, int K, int wmin,
                      int wmax, unsigned seed, CsrGraph &graph);

/// R-MAT: edgeFactor * 2^scale / 2 vertex pairs drawn with quadrant
/// probabilities a, b, c, d = 1 - a - b - c, symmetrised, self-loops and
/// duplicates removed (about edgeFactor * 2^scale directed edges); K
/// weights per directed edge, uniform or log-uniform in [wmin, wmax].
bool generateRmat(int scale, int edgeFactor, double a, double b, double c, int K, int wmin,
                  int wmax, bool logUniform, unsigned seed, CsrGraph &graph);

/// Batch on a grid graph with row-major ids (width gridWidth): nIns
/// insertions of distinct non-edges (u, v) with 1 <= |dx| + |dy| <=
/// maxManhattan on the grid and weights uniform in [wmin, wmax]; nDel
/// deletions of distinct existing edges; with safe, deletions that would
/// disconnect a vertex from source are dropped.
bool generateNearBatch(const CsrGraph &graph, int gridWidth, int nIns, int nDel, int maxManhattan,
                       bool safe, unsigned seed, int source, int wmin, int wmax,
                       ChangeBatch &batch);

/// Remove deletions that would cut a vertex reachable from source off
/// (the connectivity filter of `mospPrep changes --safe`); returns the
/// number of filter rounds.
int filterUnsafeDeletions(const CsrGraph &graph, int source, ChangeBatch &batch);

/// The same filter with reachability computed on the current GPU: each
/// round applies the batch with Step 1 (mosp_apply_batch_device) and runs a
/// unit-weight SSSP from the source on the engine. Same rounds and the
/// same kept deletions as the host filter. Returns the rounds, or -1 if a
/// GPU step failed (the batch is then unchanged).
int filterUnsafeDeletionsGpu(const CsrGraph &graph, int source, ChangeBatch &batch);

/// Route filterUnsafeDeletions (and so `--safe` batches of
/// generateChangeBatch) to the GPU path; it falls back to the host when a
/// GPU step fails.
void useGpuDeletionFilter(bool on);

/// Wall time (ms) of the last filterUnsafeDeletions call.
double lastDeletionFilterMs();

#endif // MOSP_B200_GENERATORS_H
