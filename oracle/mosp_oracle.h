/*
 * mosp_oracle.h - TEST INFRASTRUCTURE. CPU restatement of the reference
 * algorithms of the DynaMOSP update path (SMShovan/MOSP-CUDA), used only as
 * the checker by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py. Nothing in the product links or calls it.
 *
 * Parity pins: the restatement is checked against the reference's golden
 * vectors (the worked example of src/mospTest.cu:454-542) and against the
 * reference's own code compiled into oracle/_ref (tests/test_oracle*.py).
 *
 * Conventions: int32 ids/offsets/weights, int64 distances, edge-major
 * weights w[e*K+k], objective-major trees x[k*n+v], ORACLE_INF for
 * unreachable (values >= ORACLE_INF/2 mean INF), parent -1 for none.
 */
#ifndef MOSP_ORACLE_H
#define MOSP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_INF (0x7fffffffffffffffLL / 4)

/* Reference applyChangeBatch (src/csrGraph.cu:727-894): deletions first
 * (first remaining (u,v) each), then insertions in order (overwrite the
 * first live (u,v) or append). Writes the updated CSR (out_row[n+1],
 * out_col/out_w with room for cap_edges edges) and the weight-increase
 * masks (n_ins). Returns the new edge count, or -1 if cap_edges is too
 * small or an endpoint is out of range. */
long long oracle_apply_batch(int n, int K, const int *row, const int *col,
                             const int *w, int n_ins, const int *ins_from,
                             const int *ins_to, const int *ins_w, int n_del,
                             const int *del_from, const int *del_to,
                             int *out_row, int *out_col, int *out_w,
                             long long cap_edges, unsigned *mask);

/* Reverse CSR (rows by head, tails in increasing order), edge-major
 * weights (reference transposeCsrGraph, src/csrGraph.cu:896-922). */
void oracle_transpose(int n, int K, const int *row, const int *col,
                      const int *w, int *rrow, int *rcol, int *rw);

/* Binary-heap Dijkstra of objective k; among equal distances the lowest
 * parent id wins (reference dijkstraCsrGraph, src/Dijkstra.cu:239-272). */
void oracle_dijkstra(int n, int K, const int *row, const int *col,
                     const int *w, int k, int source, long long *dist,
                     int *parent);

/* Sequential SOSP update of objective k (reference sequentialSOSPUpdate,
 * Phases 1-2, src/sequentialSOSPUpdate.cu:456-612) on the UPDATED graph
 * (out-CSR row/col/w and in-CSR rrow/rcol/rw, K weights per edge): roots
 * are the heads v of changed edges (u,v) with parent[v] == u; their
 * subtrees are invalidated; invalidated vertices and insert heads are
 * re-evaluated over all in-edges; then out-neighbours of every vertex
 * whose distance decreased are re-evaluated until nothing changes.
 * dist/parent: old tree in, new tree out. Returns the number of
 * propagation rounds. */
int oracle_sequential_update(int n, int K, int k, int source, const int *row,
                             const int *col, const int *w, const int *rrow,
                             const int *rcol, const int *rw, int n_changed,
                             const int *changed_from, const int *changed_to,
                             int n_heads, const int *heads, long long *dist,
                             int *parent);

/* L = lcm(Pref) (<= 2^20), 0 if invalid; pref NULL = all 1s
 * (reference preferenceScale, src/combinedGraphGpu.cu:129-147). */
long long oracle_preference_scale(const int *pref, int K);

/* Combined graph of K trees (reference combinedGraphReference,
 * src/validation.cu:88-125): edge (p,v) iff p = Parent_i[v] for some i,
 * weight L*(K+1) - sum_{i: Parent_i[v]==p} L/Pref_i; rows in vertex order,
 * edges of a row in the order of their heads v, then of the first tree.
 * crow[n+1], ccol/cw with room for K*n. Returns the edge count, -1 on an
 * invalid preference vector. */
long long oracle_combined_graph(int n, int K, const int *parents, int source,
                                const int *pref, int *crow, int *ccol,
                                int *cw);

/* MOSP path costs (reference mospPathCosts, src/combinedGraphGpu.cu:
 * 161-208): costs[v*KG+k] = objective-k length of the tree path
 * source -> v using the first (p,v) edge of row p; ORACLE_INF if v is not
 * reached. Returns 0, or -1 if a tree edge is missing. */
int oracle_path_costs(int n, int KG, const int *row, const int *col,
                      const int *w, const int *parent, int source,
                      long long *costs);

/* Reference checkSospTree (src/validation.cu:28-86): counts[0..3] =
 * distance mismatches, inconsistent parents, non-canonical parents,
 * parent mismatches (ref_parent may be NULL). rrow/rcol/rw: in-CSR. */
void oracle_check_tree(int n, int K, int k, int source, const int *rrow,
                       const int *rcol, const int *rw, const long long *dist,
                       const int *parent, const long long *ref_dist,
                       const int *ref_parent, long long counts[4]);

#ifdef __cplusplus
}
#endif

#endif /* MOSP_ORACLE_H */
