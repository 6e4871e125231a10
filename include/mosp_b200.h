/*
 * mosp_b200.h - C ABI of the B200 (sm_100a) DynaMOSP update engine.
 *
 * Every entry point takes plain pointers and sizes and returns an int
 * status (MOSP_OK on success). Device pointers are named d_*; host arrays
 * are named h_* or are documented as host memory. `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream).
 *
 * Each function names the reference interface it replaces
 * (SMShovan/MOSP-CUDA, file:line). The C++ API of the reference
 * (sospUpdateGpu, sospFromScratchGpu, combinedGraphSospGpu,
 * uploadDeviceGraph, mospUpdate) is rebuilt on top of these calls by the
 * C++ layer of this library, with the reference's declarations kept.
 *
 * Conventions shared with the reference:
 *   - vertex ids and CSR offsets are int32, weights int32 in [1, INT_MAX],
 *     distances int64, parents int32 (-1 = none);
 *   - unreachable vertices get MOSP_DISTANCE_INF and parent -1;
 *   - parent ties are broken by the lowest parent id (canonical trees);
 *   - multi-objective arrays are objective-major: x[k * n + v].
 *
 * Calls on one workspace must not overlap; a workspace is bound to the
 * device that was current when it was created, and every call that takes
 * it makes that device current for the calling thread.
 */
#ifndef MOSP_B200_H
#define MOSP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define MOSP_ABI_VERSION 1

/* Status codes. */
#define MOSP_OK 0
#define MOSP_ERR_INVALID 1     /* bad argument or malformed input */
#define MOSP_ERR_OVERFLOW 2    /* distances do not fit the packed words */
#define MOSP_ERR_OOM 3         /* device or pinned allocation failed */
#define MOSP_ERR_CUDA 4        /* a CUDA runtime call failed */
#define MOSP_ERR_TIMEOUT 5     /* a bounded device-side wait ran out */
#define MOSP_ERR_UNSUPPORTED 6 /* device lacks a required feature */

/* Distance sentinel (same value as the reference's DISTANCE_INF,
 * headers/csrGraph.cuh:185). Values >= MOSP_DISTANCE_INF / 2 mean INF. */
#define MOSP_DISTANCE_INF (0x7fffffffffffffffLL / 4)

/* Largest number of objectives of one fused call and of the combined
 * graph (the reference's limit, src/combinedGraphGpu.cu:259). */
#define MOSP_MAX_OBJECTIVES 32

typedef struct mosp_workspace mosp_workspace;

/* Counters of one SOSP update (reference SospStats,
 * headers/sospUpdateGpu.cuh:35-45). */
typedef struct mosp_sosp_stats {
  int invalidated;    /* vertices in invalidated subtrees */
  int jump_rounds;    /* pointer-jumping rounds */
  int iterations;     /* near-far push iterations */
  int epochs;         /* far-pile threshold increases */
  long long pushes;   /* vertex expansions */
  int packed_parents; /* 1: (distance, parent) words; 0: distance-only */
  int reserved;
} mosp_sosp_stats;

/* Counters of the combined-graph step (reference CombineStats,
 * headers/combinedGraphGpu.cuh:17-23). */
typedef struct mosp_combine_stats {
  int edges;          /* edges of the combined graph */
  int reserved;
  long long scale;    /* L = lcm(Pref): distances are in units of 1/L */
  long long delta;    /* near-far bucket width used for Step 3 */
  mosp_sosp_stats search;
} mosp_combine_stats;

/* Stage times of mosp_update_host, milliseconds (reference MospTimings,
 * headers/mospUpdate.cuh:35-46). */
typedef struct mosp_timings {
  double apply_batch;  /* GPU: apply the batch (Step 1), masks, change lists */
  double upload;       /* graph, trees and batch to the GPU */
  double objectives;   /* GPU: the K SOSP updates (one fused launch) */
  double combined;     /* GPU: combined graph + its SOSP tree */
  double costs;        /* GPU: MOSP path costs */
  double download;     /* results back to the host */
} mosp_timings;

/* ---------------------------------------------------------------------- */
/* Library and helpers                                                      */
/* ---------------------------------------------------------------------- */

/* MOSP_ABI_VERSION of the loaded library. */
int mosp_abi_version(void);

/* Message of the last failing call on this host thread ("" if none). */
const char *mosp_last_error(void);

/* Short name of a status code. */
const char *mosp_status_name(int status);

/* Default near-far bucket width max(1, 32 * avgWeight / avgOutDegree).
 * Replaces defaultDelta (src/sospUpdateGpu.cu:607-616). */
long long mosp_default_delta(long long num_edges, int num_nodes,
                             long long weight_sum);

/* Packing of (distance, parent) words for n vertices and weights up to
 * max_weight: *parent_bits = bits of the parent field, or 0 when the bound
 * (n - 1) * max_weight does not fit next to it (distance-only words with
 * parent recovery); *max_distance = that bound. MOSP_ERR_OVERFLOW if the
 * bound does not fit in 62 bits. Replaces choosePacking / makePacking
 * (src/sospUpdateGpu.cu:133-143, 670-681). */
int mosp_choose_packing(int n, long long max_weight, int *parent_bits,
                        unsigned long long *max_distance);

/* L = lcm(Pref) of the combined graph, 0 if invalid (a value < 1, K values
 * expected, or L > 2^20). h_pref may be NULL (all 1s). Replaces
 * preferenceScale (src/combinedGraphGpu.cu:129-147). */
long long mosp_preference_scale(const int *h_pref, int K);

/* ---------------------------------------------------------------------- */
/* Workspace (device scratch reused by every call; replaces SospWorkspace,  */
/* headers/sospUpdateGpu.cuh:53-79, and CombineWorkspace,                   */
/* headers/combinedGraphGpu.cuh:28-50)                                      */
/* ---------------------------------------------------------------------- */

int mosp_workspace_create(mosp_workspace **out);
void mosp_workspace_destroy(mosp_workspace *ws);

/* Reserve scratch for K objectives of graphs with up to n vertices
 * (no-op if large enough). */
int mosp_workspace_reserve(mosp_workspace *ws, int n, int K);

/* mosp_workspace_reserve plus everything the near-far loops of graphs with
 * up to m edges need (near lists, the asynchronous near queue), so that
 * later calls on such graphs allocate nothing in the workspace (e.g. a
 * serving loop reserves before its first request). */
int mosp_workspace_reserve_graph(mosp_workspace *ws, int n, long long m, int K);

/* Batched instances: many independent graphs stored as one disjoint union
 * (vertex ids offset per instance) are updated by single launches when the
 * workspace knows every instance's root. After this call every entry point
 * that takes a `source` treats all `count` distinct vertices as roots
 * (distance 0, parent -1; the `source` argument must be one of them), so
 * each instance's trees, combined graph and costs are its own. count <= 1
 * returns to single-source runs. No counterpart in the reference, which
 * runs one instance per call. */
int mosp_workspace_set_sources(mosp_workspace *ws, const int *h_sources,
                               int count);

/* Near-far bucket width of the combined-graph step run by
 * mosp_update_device, mosp_update_host and mosp_combined_sosp called with
 * delta <= 0 (0 = the default heuristic of the reference,
 * src/combinedGraphGpu.cu:310-312). Results do not depend on it; the
 * autotuner (mosp_autotune_update) picks it. */
int mosp_workspace_set_combined_delta(mosp_workspace *ws, long long delta);

/* CTA-local expansion rounds of the near-far loop (0..16) for update
 * launches (default 0) and for from-scratch and combined-graph launches
 * (default 2): after its share of an iteration, each CTA expands the near
 * entries it has just produced itself up to this many times before the grid
 * barrier, so a frontier advances several hops per barrier (it pays on
 * deep, sparse graphs such as the combined graph). Results do not depend on
 * it; the autotuner picks both. No counterpart in the reference. */
int mosp_workspace_set_local_rounds(mosp_workspace *ws, int update_rounds,
                                    int scratch_rounds);

/* Narrow iterations: a near-far iteration with at most max_items items
 * (default 512; 0 = never) runs on one CTA, which then expands what it
 * produces for up to `rounds` CTA-local rounds (default 64) before the grid
 * barrier - thin wavefronts of deep graphs and the tails of epochs then
 * cost a CTA barrier per hop instead of a grid barrier. Results do not
 * depend on it. No counterpart in the reference. */
int mosp_workspace_set_narrow(mosp_workspace *ws, int max_items, int rounds);

/* Near-far loop of the persistent launches: on = 1 (default) runs it
 * asynchronously - after each far-pile split every warp claims entries of
 * a sharded near queue, expands them and pushes what improves, with no grid
 * barrier until the phase has run dry - where the graph has no rows of more
 * than 2,048 edges; 0 runs the bulk-synchronous loop (one grid barrier per
 * iteration, the reference's schedule, src/sospUpdateGpu.cu:385-476) for
 * every graph. queue_slots bounds the near queue (8 bytes a slot; 0 = one
 * slot per vertex and objective plus n, at least 2^20) and the bulk loop's
 * near lists (entries per objective; 0 = min(n + m, max(2n, 2^20))):
 * entries that find them full go to the far pile and are taken up in the
 * next phase or split. Results do not depend on either. */
int mosp_workspace_set_async(mosp_workspace *ws, int on, long long queue_slots);

/* Declares that the input trees of this workspace's update calls follow the
 * lowest-id tie rule (every tree this library returns does, and so does a
 * tree from the reference's mospPrep init or canonicalizeTree). An
 * objective that runs on distances alone (more than 64 bits per packed
 * word) then recovers its parents only at the vertices the batch can reach
 * (the vertices whose distance, parent distance or in-edges changed, and
 * the out-neighbours of the vertices whose distance changed) instead of
 * over every edge; for such input trees the result is the same. Off by
 * default: the reference rebuilds every parent of such an objective
 * (src/sospUpdateGpu.cu:491-512), which also normalises input trees that
 * break ties differently. */
int mosp_workspace_set_canonical_trees(mosp_workspace *ws, int on);

/* When on, mosp_update_device records its launch sequence (control-block
 * clears, the update and combined launches, the status readback) as one
 * CUDA graph and replays it while the launch parameters stay the same; it
 * is captured again when they change. Per-launch timing
 * (mosp_workspace_enable_timing) is not recorded in this mode.
 * mosp_workspace_graph_launches counts the graph launches so far. No
 * counterpart in the reference. */
int mosp_workspace_use_graphs(mosp_workspace *ws, int on);
int mosp_workspace_graph_launches(mosp_workspace *ws, int *count);

/* Bound on every device-side wait of the persistent kernels (default
 * 10000 ms). A run that exceeds it stops and returns MOSP_ERR_TIMEOUT. */
int mosp_workspace_set_timeout_ms(mosp_workspace *ws, long long ms);

/* Launch shape of the persistent kernels: CTAs per SM (0 = as many as
 * fit). Results do not depend on it. */
int mosp_workspace_set_ctas_per_sm(mosp_workspace *ws, int ctas_per_sm);

/* Grid and hub threshold of the persistent engine launches. ctas = 0 uses
 * one 1,024-thread CTA per SM on every SM (the occupancy-sized grid of the
 * reference, src/sospUpdateGpu.cu:553-595); a smaller count launches fewer
 * CTAs (cheaper grid barriers, fewer warps). hub_edges (0 = 2,048, else at
 * least 64): rows with more edges are expanded and reduced by a whole CTA,
 * and a graph with such rows runs the bulk near-far loop. Results do not
 * depend on either; mosp_autotune_update picks both. No counterpart in the
 * reference. */
int mosp_workspace_set_grid(mosp_workspace *ws, int ctas, int hub_edges);

/* The workspace's current engine settings: grid CTAs, hub threshold and
 * near-far loop (1 asynchronous, 0 bulk), e.g. after mosp_autotune_update. */
int mosp_workspace_tuning(mosp_workspace *ws, int *ctas, int *hub_edges, int *async_on);

/* Grid size (CTAs) the persistent kernels use on this device. */
int mosp_workspace_grid(mosp_workspace *ws, int *ctas);

/* Per-launch timing: when on, the engine records CUDA events around each
 * persistent launch on the caller's stream; mosp_workspace_last_timing
 * returns the durations (ms) of the last SOSP-update launch and the last
 * combined-graph launch (after the call that ran them returned). */
int mosp_workspace_enable_timing(mosp_workspace *ws, int on);
int mosp_workspace_last_timing(mosp_workspace *ws, float *update_ms,
                               float *combined_ms);

/* Device clock (%globaltimer, ns) at the 8 phase boundaries of the last
 * SOSP-update launch (which = 0) or combined-graph launch (which = 1):
 * start, trees packed / graph built, roots marked, subtrees flagged,
 * candidates listed, pull pass done, near-far loop done, results written
 * (0 for phases a launch does not have). */
int mosp_workspace_last_phases(mosp_workspace *ws, int which,
                               unsigned long long *ns);

/* Near-far loop profile of the last update (which = 0) or combined (1)
 * launch: time (ns), iterations and list items of the iterations that split
 * a far pile (index 0) and of the pure push iterations (index 1); ns[2..6]
 * (ns has 7 entries) split the push iterations of CTA 0 into decision step,
 * own items, wait for the CTA's other warps, list flush and grid barrier. */
int mosp_workspace_loop_profile(mosp_workspace *ws, int which,
                                unsigned long long *ns, long long *iters,
                                long long *items);

/* Device buffer number `slot` (0..31) of the workspace, grown to at least
 * `bytes` (contents kept only while it does not grow); freed with the
 * workspace. Lets a caller keep its graph and trees on the device between
 * calls without managing allocations. No counterpart in the reference. */
int mosp_workspace_buffer(mosp_workspace *ws, int slot, unsigned long long bytes,
                          void **d_ptr);

/* ---------------------------------------------------------------------- */
/* Device graph                                                             */
/* ---------------------------------------------------------------------- */

/* From the out-edge CSR (d_out_row[n+1], d_out_col[m]) and edge-major
 * weights (d_edge_major_w[e*K+k]) build on the GPU the objective-major
 * weight columns d_out_w[k*m+e] and the reverse CSR d_in_row[n+1],
 * d_in_col[m], d_in_w[k*m+e]. Also checks that the CSR is well formed
 * (offsets monotone from 0 to m, ids in [0, n)). Replaces the GPU part
 * of uploadDeviceGraph (src/deviceGraph.cu:87-135). */
int mosp_build_device_graph(mosp_workspace *ws, int n, int m, int K,
                            const int *d_out_row, const int *d_out_col,
                            const int *d_edge_major_w, int *d_out_w,
                            int *d_in_row, int *d_in_col, int *d_in_w,
                            void *stream);

/* ---------------------------------------------------------------------- */
/* SOSP update engine                                                       */
/* ---------------------------------------------------------------------- */

/* Incremental SOSP update of one objective, in place: on entry
 * d_dist[n] / d_parent[n] hold the tree of the old graph, on return the
 * tree of the graph whose out- and in-edges are given (with canonical
 * input trees the result is the canonical tree). changed_from/to
 * (n_changed entries, device) are the deleted or weight-increased edges,
 * insert_heads (n_heads, device) the heads of all inserted edges.
 * delta > 0 is the near-far bucket width, max_weight the largest weight.
 * Synchronous; stats may be NULL. Replaces sospUpdateGpu
 * (headers/sospUpdateGpu.cuh:98-102, src/sospUpdateGpu.cu:685-717). */
int mosp_sosp_update(mosp_workspace *ws, int n, int m, const int *d_out_row,
                     const int *d_out_col, const int *d_out_w,
                     const int *d_in_row, const int *d_in_col,
                     const int *d_in_w, const int *d_changed_from,
                     const int *d_changed_to, int n_changed,
                     const int *d_insert_heads, int n_heads, int source,
                     long long delta, long long max_weight, long long *d_dist,
                     int *d_parent, mosp_sosp_stats *stats, void *stream);

/* The K (<= 32) SOSP updates of one MOSP update in ONE persistent launch:
 * the objectives share the topology and the insert heads and run their
 * near-far loops side by side behind the same grid barriers. Every
 * h_-prefixed array has K entries in host memory; the pointers in them
 * are device pointers. stats (K entries) may be NULL. The per-objective
 * results equal K calls of mosp_sosp_update. Replaces the K calls of
 * sospUpdateGpu in mospUpdate (src/mospUpdate.cu:167-194). */
int mosp_sosp_update_multi(
    mosp_workspace *ws, int n, int m, int K, const int *d_out_row,
    const int *d_out_col, const int *const *h_out_w, const int *d_in_row,
    const int *d_in_col, const int *const *h_in_w,
    const int *const *h_changed_from, const int *const *h_changed_to,
    const int *h_n_changed, const int *d_insert_heads, int n_heads,
    int source, const long long *h_delta, const long long *h_max_weight,
    long long *const *h_dist, int *const *h_parent, mosp_sosp_stats *stats,
    void *stream);

/* Step 1 on the GPU: applies a change batch to a device out-CSR (edge-major
 * weights w[e*K+k], as in the reference's host CsrGraph) and writes the
 * updated out-CSR, which needs room for m + n_ins edges (new_capacity), and
 * the weight-increase mask of every insertion. *new_m receives the updated
 * edge count. Deletions come first (each removes the first live (u,v) in
 * its row, in file order), then insertions (each overwrites the first live
 * (u,v) or appends at the end of its row); the result equals the host
 * applyChangeBatch edge for edge. When h_max_weight / h_weight_sum are
 * non-NULL they receive (K entries each) the largest weight of the original
 * edges and insertions (at least 1) and the weight sum of the original
 * edges, the inputs of the default delta. Replaces applyChangeBatch
 * (src/csrGraph.cu:727-894) and the per-objective statistics of mospUpdate
 * (src/mospUpdate.cu:104-136). */
int mosp_apply_batch_device(mosp_workspace *ws, int n, int K, int m,
                            const int *d_row, const int *d_col, const int *d_w,
                            int n_ins, const int *d_ins_from,
                            const int *d_ins_to, const int *d_ins_w, int n_del,
                            const int *d_del_from, const int *d_del_to,
                            int *d_new_row, int *d_new_col, int *d_new_w,
                            long long new_capacity, int *new_m,
                            unsigned *d_mask, long long *h_max_weight,
                            long long *h_weight_sum, void *stream);

/* Canonical single-source shortest paths from scratch. Replaces
 * sospFromScratchGpu (headers/sospUpdateGpu.cuh:107-110,
 * src/sospUpdateGpu.cu:719-745). */
int mosp_sosp_from_scratch(mosp_workspace *ws, int n, int m,
                           const int *d_out_row, const int *d_out_col,
                           const int *d_out_w, int source, long long delta,
                           long long max_weight, long long *d_dist,
                           int *d_parent, mosp_sosp_stats *stats,
                           void *stream);

/* Limits of mosp_sosp_from_scratch_static: its scratch is a fixed device
 * array of about 10 MB sized for these. */
#define MOSP_STATIC_MAX_VERTICES 65536
#define MOSP_STATIC_MAX_EDGES 262144

/* mosp_sosp_from_scratch without a workspace and without any device or
 * pinned allocation, for callers that cannot allocate during a call (device
 * memory owned by another allocator or a fixed budget; latency-critical
 * handlers, where an allocation may synchronize the device; plugin hosts
 * that forbid it). The engine's scratch is a file-scope __device__ array
 * reserved when the library's module is loaded, one per device; results
 * equal mosp_sosp_from_scratch's. This entry point has no counterpart in
 * the reference.
 *   - n <= MOSP_STATIC_MAX_VERTICES and m <= MOSP_STATIC_MAX_EDGES; larger
 *     graphs are rejected with MOSP_ERR_INVALID and a message.
 *   - The CSR is checked on the device before it is used (row offsets
 *     monotone from 0 to m, columns in [0, n)); a malformed graph returns
 *     MOSP_ERR_INVALID.
 *   - Runs on the current device. The first call on a device does the
 *     setup (module load, launch-shape query); make it before any stream
 *     capture on that device. Every call looks up the array's device
 *     address with that device current, so a device reset does not leave
 *     a stale address behind.
 *   - The call clears the scratch regions that must start at zero (control
 *     block, stamp generation, stamps, in-far flags) in `stream` before the
 *     launch, so an aborted call leaves nothing behind.
 *   - Calls on one device share the scratch: calls that overlap in time
 *     (two host threads, or unordered streams) race and must be serialized
 *     by the caller. A call returns after its result is complete. */
int mosp_sosp_from_scratch_static(int n, int m, const int *d_out_row,
                                  const int *d_out_col, const int *d_out_w,
                                  int source, long long delta,
                                  long long max_weight, long long *d_dist,
                                  int *d_parent, mosp_sosp_stats *stats,
                                  void *stream);

/* Steps 2-3 of the MOSP update in one persistent launch: build the
 * combined graph of the K trees d_parents[k*n+v] (edge (p,v) iff p is the
 * parent of v in some tree; weight L*(K+1) - sum_{i: Parent_i[v]==p}
 * L/Pref_i) and its canonical SSSP tree from source (distances in units
 * of 1/L). h_pref: K host values or NULL (all 1s). delta <= 0 selects the
 * default width of the combined graph. Replaces combinedGraphSospGpu
 * (headers/combinedGraphGpu.cuh:65-69, src/combinedGraphGpu.cu:251-317). */
int mosp_combined_sosp(mosp_workspace *ws, int n, int K, const int *d_parents,
                       const int *h_pref, int source, long long delta,
                       long long *d_dist, int *d_parent,
                       mosp_combine_stats *stats, void *stream);

/* MOSP path costs on the GPU: d_costs[v*KG+k] = objective-k length of the
 * tree path source -> v in the graph (d_out_row, d_out_col, objective-major
 * d_out_w with KG columns), where edge (p,v) is the first occurrence of v
 * in row p; MOSP_DISTANCE_INF if v is unreachable. MOSP_ERR_INVALID if a
 * tree edge is not in the graph. Replaces the host mospPathCosts
 * (src/combinedGraphGpu.cu:161-208). */
int mosp_path_costs(mosp_workspace *ws, int n, int m, int KG,
                    const int *d_out_row, const int *d_out_col,
                    const int *d_out_w, const int *d_parent, int source,
                    long long *d_costs, void *stream);

/* The device part of one MOSP update: K fused SOSP updates (as
 * mosp_sosp_update_multi, with the objective-major weight columns
 * d_out_w / d_in_w of K objectives starting at column 0), then Steps 2-3
 * (mosp_combined_sosp) on the updated trees, queued back to back with one
 * synchronization at the end. d_dist/d_parent hold the K trees
 * (objective-major), d_changed_from/to the concatenated per-objective
 * change lists with h_changed_offset[K+1] (host) delimiting them.
 * Replaces the GPU stages of mospUpdate (src/mospUpdate.cu:167-209). */
int mosp_update_device(mosp_workspace *ws, int n, int m, int K,
                       const int *d_out_row, const int *d_out_col,
                       const int *d_out_w, const int *d_in_row,
                       const int *d_in_col, const int *d_in_w,
                       const int *d_changed_from, const int *d_changed_to,
                       const int *h_changed_offset, const int *d_insert_heads,
                       int n_heads, int source, const long long *h_delta,
                       const long long *h_max_weight, const int *h_pref,
                       long long *d_dist, int *d_parent,
                       long long *d_comb_dist, int *d_comb_parent,
                       mosp_sosp_stats *stats, mosp_combine_stats *cstats,
                       void *stream);

/* Autotuner of the near-far widths and local rounds: runs
 * mosp_update_device on the given inputs with the update width scaled by
 * 1/4 .. 8 around h_delta and 0..2 local rounds, and the combined-graph
 * width scaled by 1 .. 32 around its default with 0..4 local rounds,
 * timing each launch with CUDA events (median of three runs), and returns the
 * fastest per-objective widths (h_best_delta, K entries), the fastest
 * combined width (*h_best_comb_delta, for
 * mosp_workspace_set_combined_delta), the fastest local rounds
 * (h_best_rounds[0] update, [1] combined, for
 * mosp_workspace_set_local_rounds; may be NULL) and their summed launch
 * time (*h_best_ms, may be NULL). The trees d_dist /
 * d_parent are restored to their input values before returning; results of
 * later updates do not depend on the widths chosen. With the best widths
 * it then times the near-far loop (asynchronous or bulk), two smaller grids
 * (3/4 and 1/2 of the CTAs) and, when the graph has hub rows, hub
 * thresholds of 16,384 and 2^20 edges, and leaves the fastest of those set
 * on the workspace (mosp_workspace_tuning reads them). It allocates a copy
 * of the trees for the duration of the call. No counterpart in the
 * reference (its width is the fixed heuristic of defaultDelta and its grid
 * the occupancy-sized one). */
int mosp_autotune_update(mosp_workspace *ws, int n, int m, int K,
                         const int *d_out_row, const int *d_out_col,
                         const int *d_out_w, const int *d_in_row,
                         const int *d_in_col, const int *d_in_w,
                         const int *d_changed_from, const int *d_changed_to,
                         const int *h_changed_offset,
                         const int *d_insert_heads, int n_heads, int source,
                         const long long *h_delta,
                         const long long *h_max_weight, const int *h_pref,
                         long long *d_dist, int *d_parent,
                         long long *d_comb_dist, int *d_comb_parent,
                         long long *h_best_delta, long long *h_best_comb_delta,
                         int *h_best_rounds, float *h_best_ms, void *stream);

/* ---------------------------------------------------------------------- */
/* Whole MOSP update from host memory (the reference's in-memory pipeline)  */
/* ---------------------------------------------------------------------- */

/* One MOSP update with host inputs and outputs: apply the batch to the
 * graph (n vertices, KG objectives, m edges; h_w edge-major e*KG+k),
 * upload, run the first K objectives (K <= KG; 0 = all) and Steps 2-3 on
 * the GPU, download, and (if h_costs != NULL) compute the MOSP path costs
 * (n*KG) on the GPU. Inputs: inserts "u v w1..wKG" (h_ins_w insertion-
 * major), deletes "u v", initial trees h_init_dist/h_init_parent (K*n,
 * rooted at source). h_pref: K values or NULL; delta <= 0: default per
 * objective. Outputs: h_dist/h_parent (K*n), h_comb_dist/h_comb_parent
 * (n). timings may be NULL. Replaces mospUpdate
 * (headers/mospUpdate.cuh:69-73, src/mospUpdate.cu:57-225). */
int mosp_update_host(mosp_workspace *ws, int n, int KG, int m,
                     const int *h_row, const int *h_col, const int *h_w,
                     int n_ins, const int *h_ins_from, const int *h_ins_to,
                     const int *h_ins_w, int n_del, const int *h_del_from,
                     const int *h_del_to, const long long *h_init_dist,
                     const int *h_init_parent, int K, int source,
                     const int *h_pref, long long delta, long long *h_dist,
                     int *h_parent, long long *h_comb_dist,
                     int *h_comb_parent, long long *h_costs,
                     mosp_timings *timings);

/* ---------------------------------------------------------------------- */
/* Failure-path check                                                       */
/* ---------------------------------------------------------------------- */

/* Runs a grid barrier that one CTA never reaches, bounded by timeout_ms
 * (<= 10000); *device_status receives the status the kernel reported
 * (MOSP_ERR_TIMEOUT when the bounded wait works). The workspace stays
 * usable afterwards. No counterpart in the reference (whose grid barriers
 * are unbounded, src/sospUpdateGpu.cu:644-649). */
int mosp_debug_barrier_timeout(mosp_workspace *ws, long long timeout_ms,
                               int *device_status);

/* Device time per grid barrier of the persistent kernels' launch shape
 * (`rounds` barriers; with `reads` != 0 each round also reads two control
 * words per CTA, as a near-far iteration does). For tuning the launch
 * shape. No counterpart in the reference. */
int mosp_debug_barrier_cost(mosp_workspace *ws, int rounds, int reads,
                            double *ns_per_round);

/* ---------------------------------------------------------------------- */
/* Serving: resident graphs, change batches from many clients                */
/* ---------------------------------------------------------------------- */

/* A server keeps graphs, their K SOSP trees and their combined (MOSP) tree
 * in device memory and applies change batches that clients submit from any
 * thread. Worker threads take the pending batches of one graph at a time
 * (oldest first): batches that arrive while others run are picked up as
 * soon as a worker and device memory are free; the pending batches of one
 * graph are coalesced into one pass of at most max_coalesce requests and
 * 262,144 changes past its first request (merged into one batch up to the
 * first batch that deletes an edge an earlier one inserted, then one
 * engine update with the union of their change lists, which gives the
 * same trees as applying them one by one); a pass starts only when the memory it may
 * allocate fits in the free device memory minus `reserve_bytes` (unless no
 * pass is running). With W > 1 workers each worker's persistent launches
 * use 1/W of the SMs, so the passes of different workers run on the device
 * at the same time (mosp_server_set_overlap turns this off: one pass's
 * launches at a time, each on the whole GPU); copies and host work overlap
 * in both modes. No counterpart in the reference, which runs one update per
 * invocation. */
typedef struct mosp_server mosp_server;

typedef struct mosp_server_result {
  int status;          /* MOSP_OK or the pass's error */
  int graph;
  long long version;   /* batches applied to the graph in the returned state */
  int coalesced;       /* requests in the pass that served this one */
  int reserved;
  double queue_us;     /* submit -> pass start */
  double latency_us;   /* submit -> result in host memory */
  unsigned long long checksum; /* order-independent hash of the returned tree,
                                  computed by mosp_server_wait */
} mosp_server_result;

typedef struct mosp_server_stats {
  long long requests;  /* requests served */
  long long passes;    /* GPU passes (a pass serves >= 1 request) */
  long long changes;   /* changes applied */
  long long deferred;  /* times a graph's pass waited for device memory */
  long long applies;   /* Step 1 runs (merged batches; > passes on conflicts) */
  int max_coalesced;
  int overlapped;      /* passes whose engine launches ran while another
                          pass's did (on disjoint SMs) */
  double busy_us;      /* summed pass durations over the workers */
  double apply_us;     /* of which: uploads, Step 1, change lists */
  double engine_us;    /* graph build + update + combined (incl. lock wait) */
  double result_us;    /* combined tree download and checksum */
} mosp_server_stats;

/* workers: 1..16 threads; max_coalesce: most requests per pass. */
int mosp_server_create(int workers, long long reserve_bytes, int max_coalesce,
                       mosp_server **out);
void mosp_server_destroy(mosp_server *server);

/* Upload a graph (host CSR, edge-major weights h_w[e*KG+k]) and compute its
 * K canonical trees from `source` and its combined tree (Pref h_pref, K
 * values or NULL) on the GPU; *graph_id identifies it. */
int mosp_server_add_graph(mosp_server *server, int n, int KG, int m,
                          const int *h_row, const int *h_col, const int *h_w,
                          int K, int source, const int *h_pref, int *graph_id);

/* Queue a change batch (host arrays, copied before returning) for a graph;
 * *ticket identifies the request. Batches of one graph are applied in
 * submission order. */
int mosp_server_submit(mosp_server *server, int graph_id, int n_ins,
                       const int *h_ins_from, const int *h_ins_to,
                       const int *h_ins_w, int n_del, const int *h_del_from,
                       const int *h_del_to, long long *ticket);

/* Wait for a request: the graph's combined distances and parents (n each,
 * either may be NULL) after the pass that served it, and its record. */
int mosp_server_wait(mosp_server *server, long long ticket,
                     long long *h_comb_dist, int *h_comb_parent,
                     mosp_server_result *info);

/* The graph's current state (after any running pass): its version, the K
 * trees (K*n, objective-major) and the combined tree; any output may be
 * NULL. */
int mosp_server_read_graph(mosp_server *server, int graph_id,
                           long long *version, long long *h_dist,
                           int *h_parent, long long *h_comb_dist,
                           int *h_comb_parent);

int mosp_server_get_stats(mosp_server *server, mosp_server_stats *out);

/* on = 1 (default): passes of different workers share the device (1/W of
 * the SMs each); 0: one pass's launches at a time on the whole GPU. Set it
 * before submitting work. */
int mosp_server_set_overlap(mosp_server *server, int on);

#ifdef __cplusplus
}
#endif

#endif /* MOSP_B200_H */
