/*
 * mosp_b200_host.h - C ABI of the host side of the MOSP update path:
 * graph and change-batch files, batch application, input generators and
 * the host checks that `mospPrep` and `mosp --validate` use. Together with
 * mosp_b200.h it lets a caller without C++ (ctypes, cgo, JNI) drive the
 * whole path. Host memory only; status codes as in mosp_b200.h.
 *
 * Graph and batch handles own their arrays; pointers returned by the
 * *_arrays calls stay valid until the handle is freed.
 */
#ifndef MOSP_B200_HOST_H
#define MOSP_B200_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mosp_host_graph mosp_host_graph;
typedef struct mosp_host_batch mosp_host_batch;

/* Change modes of mosp_batch_generate (reference ChangeMode,
 * headers/changeGenerator.cuh:28). */
#define MOSP_MODE_UNIFORM 0
#define MOSP_MODE_TARGETED 1
#define MOSP_MODE_REWEIGHT 2
#define MOSP_MODE_INCREASE 3

/* --- graphs ------------------------------------------------------------- */

/* Text CSR <prefix>{RowPtr,ColInd,Values}.txt, through the binary cache
 * when cache_path is non-NULL (reference loadCsrGraph,
 * src/csrGraph.cu:600-620). */
int mosp_graph_read(const char *prefix, const char *cache_path,
                    mosp_host_graph **out);
/* Reference writeCsrGraph (src/csrGraph.cu:474-501). */
int mosp_graph_write(const mosp_host_graph *g, const char *prefix);
/* Binary cache of the text graph at source_prefix (reference
 * saveCsrGraphBinary, src/csrGraph.cu:503-536). */
int mosp_graph_save_cache(const mosp_host_graph *g, const char *path,
                          const char *source_prefix);
/* Copy of caller arrays: row[n+1], col[m], w[m*K] edge-major. */
int mosp_graph_from_arrays(int n, int K, const int *row, const int *col,
                           const int *w, mosp_host_graph **out);
/* Road-network shape: width x height grid, each undirected grid edge kept
 * with probability keep, shortcut_fraction of the vertices get one
 * diagonal shortcut (both directions), largest connected component kept
 * and renumbered in row-major order; K weights per directed edge, uniform
 * in [wmin, wmax]. No counterpart in the reference (its inputs are
 * SuiteSparse files, bench/prepare.sh). */
int mosp_graph_grid_road(int width, int height, double keep,
                         double shortcut_fraction, int K, int wmin, int wmax,
                         unsigned seed, mosp_host_graph **out);
/* R-MAT graph: 2^scale vertices, edge_factor * 2^scale draws with
 * quadrant probabilities a, b, c (d = 1 - a - b - c), symmetrised, no
 * self-loops or duplicates; K weights per edge, uniform in [wmin, wmax]
 * or (log_uniform != 0) log-uniform. No counterpart in the reference. */
int mosp_graph_rmat(int scale, int edge_factor, double a, double b, double c,
                    int K, int wmin, int wmax, int log_uniform, unsigned seed,
                    mosp_host_graph **out);
int mosp_graph_info(const mosp_host_graph *g, int *n, int *K, long long *m);
int mosp_graph_arrays(const mosp_host_graph *g, const int **row,
                      const int **col, const int **w);
void mosp_graph_free(mosp_host_graph *g);

/* --- change batches ------------------------------------------------------ */

/* Reference generateChangeBatch (src/changeGenerator.cu:133-344): same
 * batch for the same graph, options and seed. */
int mosp_batch_generate(const mosp_host_graph *g, int n_changes,
                        double ins_pct, int mode, int local_hops, int safe,
                        unsigned seed, int source, int wmin, int wmax,
                        mosp_host_batch **out);
/* Batch for a grid graph of the given width (row-major ids): n_ins
 * insertions of non-edges (u, v) within Manhattan distance max_manhattan
 * on the grid, n_del deletions of distinct existing edges (safe != 0:
 * minus those that would disconnect a vertex from source). No counterpart
 * in the reference. */
int mosp_batch_near(const mosp_host_graph *g, int grid_width, int n_ins,
                    int n_del, int max_manhattan, int safe, unsigned seed,
                    int source, int wmin, int wmax, mosp_host_batch **out);
/* Reference readChangeBatch (src/csrGraph.cu:626-725). */
int mosp_batch_read(const char *insert_path, const char *delete_path, int K,
                    int n, mosp_host_batch **out);
/* Reference writeChangeBatch (src/changeGenerator.cu:346-371). */
int mosp_batch_write(const mosp_host_batch *b, const char *insert_path,
                     const char *delete_path);
int mosp_batch_from_arrays(int K, int n_ins, const int *ins_from,
                           const int *ins_to, const int *ins_w, int n_del,
                           const int *del_from, const int *del_to,
                           mosp_host_batch **out);
int mosp_batch_info(const mosp_host_batch *b, int *K, int *n_ins, int *n_del);
/* increase_mask is filled by mosp_apply_batch. */
int mosp_batch_arrays(const mosp_host_batch *b, const int **ins_from,
                      const int **ins_to, const int **ins_w,
                      const int **del_from, const int **del_to,
                      const unsigned **increase_mask);
void mosp_batch_free(mosp_host_batch *b);

/* --- host algorithms ------------------------------------------------------ */

/* Reference applyChangeBatch (src/csrGraph.cu:727-894); fills the
 * batch's weight-increase masks. */
int mosp_apply_batch(const mosp_host_graph *g, mosp_host_batch *b,
                     mosp_host_graph **updated);
/* Reference dijkstraCsrGraph (src/Dijkstra.cu:239-272): lowest-id ties. */
int mosp_host_dijkstra(const mosp_host_graph *g, int objective, int source,
                       long long *dist, int *parent);
/* Reference canonicalizeTree (src/mospUpdate.cu:40-55). */
int mosp_canonicalize_tree(const mosp_host_graph *g, int objective,
                           int source, const long long *dist, int *parent);
/* Reference readDistances / readParents (src/csrGraph.cu:943-1030). */
int mosp_read_tree(const char *dist_path, const char *parent_path, int n,
                   long long *dist, int *parent);
/* Reference writeDistances / writeParents (src/csrGraph.cu:1032-1064). */
int mosp_write_tree(const char *dist_path, const char *parent_path, int n,
                    const long long *dist, const int *parent);

/* Bytes one MOSP update must move at least (the roofline numerator),
 * from the old and new trees (K*n each, objective-major) of the updated
 * graph g and the applied batch b (with its increase masks). Per
 * objective k with invalidated set I, insert heads H, changed edges C,
 * S = I plus the vertices whose distance decreased and W the vertices
 * whose (distance, parent) changed:
 *   4n + 16|C| + 4|H| + sum_{v in I+H} (8 + 16 indeg v)
 *      + sum_{u in S} (8 + 16 outdeg u) + 12|W|;
 * combined step with E_c edges: 4Kn + 8(n+1) + 24 E_c + 12n.
 * Also returns the counts it used. No counterpart in the reference. */
int mosp_algorithmic_bytes(const mosp_host_graph *g, const mosp_host_batch *b,
                           int K, int source, const long long *old_dist,
                           const int *old_parent, const long long *new_dist,
                           const int *new_parent, long long combined_edges,
                           long long *bytes_update, long long *bytes_combined,
                           long long *invalidated_total,
                           long long *expanded_total);

#ifdef __cplusplus
}
#endif

#endif /* MOSP_B200_HOST_H */
