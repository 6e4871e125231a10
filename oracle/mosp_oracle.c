/*
 * mosp_oracle.c - TEST INFRASTRUCTURE: CPU restatement of the reference
 * algorithms (see mosp_oracle.h). Used only as the checker; the product
 * never calls it.
 */
#include "mosp_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* batch application: src/csrGraph.cu:727-894                               */
/* ------------------------------------------------------------------------ */
long long oracle_apply_batch(int n, int K, const int *row, const int *col,
                             const int *w, int n_ins, const int *ins_from,
                             const int *ins_to, const int *ins_w, int n_del,
                             const int *del_from, const int *del_to,
                             int *out_row, int *out_col, int *out_w,
                             long long cap_edges, unsigned *mask) {
  /* Per vertex: a dynamic list of (head, weight source) entries. Weight
   * source >= 0: original edge; < 0: insertion -src-1. */
  typedef struct {
    int head;
    long long src;
    int live;
  } entry;
  long long total = 0;
  int i, u;
  for (i = 0; i < n_ins; ++i)
    if (ins_from[i] < 0 || ins_from[i] >= n || ins_to[i] < 0 || ins_to[i] >= n) return -1;
  for (i = 0; i < n_del; ++i)
    if (del_from[i] < 0 || del_from[i] >= n || del_to[i] < 0 || del_to[i] >= n) return -1;
  entry **lists = (entry **)calloc((size_t)n, sizeof(entry *));
  int *len = (int *)calloc((size_t)n, sizeof(int));
  int *cap = (int *)calloc((size_t)n, sizeof(int));
  char *touched = (char *)calloc((size_t)n, 1);
  /* rows with changes get an explicit list; file order is kept because the
   * changes are replayed in file order below */
  for (i = 0; i < n_del; ++i) touched[del_from[i]] = 1;
  for (i = 0; i < n_ins; ++i) touched[ins_from[i]] = 1;
  for (u = 0; u < n; ++u) {
    if (!touched[u]) continue;
    int deg = row[u + 1] - row[u];
    cap[u] = deg + 4;
    lists[u] = (entry *)malloc((size_t)cap[u] * sizeof(entry));
    for (int e = row[u]; e < row[u + 1]; ++e) {
      lists[u][len[u]].head = col[e];
      lists[u][len[u]].src = e;
      lists[u][len[u]].live = 1;
      ++len[u];
    }
  }
  for (i = 0; i < n_del; ++i) {
    u = del_from[i];
    for (int j = 0; j < len[u]; ++j) {
      if (lists[u][j].live && lists[u][j].head == del_to[i]) {
        lists[u][j].live = 0;
        break;
      }
    }
  }
  for (i = 0; i < n_ins; ++i) {
    u = ins_from[i];
    int hit = 0;
    for (int j = 0; j < len[u]; ++j) {
      if (lists[u][j].live && lists[u][j].head == ins_to[i]) {
        lists[u][j].src = -(long long)i - 1;
        hit = 1;
        break;
      }
    }
    if (!hit) {
      if (len[u] == cap[u]) {
        cap[u] *= 2;
        lists[u] = (entry *)realloc(lists[u], (size_t)cap[u] * sizeof(entry));
      }
      lists[u][len[u]].head = ins_to[i];
      lists[u][len[u]].src = -(long long)i - 1;
      lists[u][len[u]].live = 1;
      ++len[u];
    }
  }
  out_row[0] = 0;
  for (u = 0; u < n; ++u) {
    long long deg = row[u + 1] - row[u];
    if (touched[u]) {
      deg = 0;
      for (int j = 0; j < len[u]; ++j) deg += lists[u][j].live;
    }
    total += deg;
    out_row[u + 1] = (int)total;
  }
  if (total <= cap_edges) {
    for (u = 0; u < n; ++u) {
      long long o = out_row[u];
      if (!touched[u]) {
        for (int e = row[u]; e < row[u + 1]; ++e, ++o) {
          out_col[o] = col[e];
          memcpy(out_w + o * K, w + (long long)e * K, sizeof(int) * (size_t)K);
        }
        continue;
      }
      for (int j = 0; j < len[u]; ++j) {
        if (!lists[u][j].live) continue;
        out_col[o] = lists[u][j].head;
        const int *src = lists[u][j].src >= 0 ? w + lists[u][j].src * K
                                              : ins_w + (-lists[u][j].src - 1) * K;
        memcpy(out_w + o * K, src, sizeof(int) * (size_t)K);
        ++o;
      }
    }
    /* weight increases: first (u,v) of the original row against the first
     * (u,v) of the updated row */
    for (i = 0; i < n_ins; ++i) {
      int a = -1, b = -1, v = ins_to[i];
      u = ins_from[i];
      mask[i] = 0;
      for (int e = row[u]; e < row[u + 1]; ++e)
        if (col[e] == v) { a = e; break; }
      if (a < 0) continue;
      for (int e = out_row[u]; e < out_row[u + 1]; ++e)
        if (out_col[e] == v) { b = e; break; }
      if (b < 0) continue;
      for (int k = 0; k < K; ++k)
        if (out_w[(long long)b * K + k] > w[(long long)a * K + k]) mask[i] |= 1u << k;
    }
  }
  for (u = 0; u < n; ++u) free(lists[u]);
  free(lists);
  free(len);
  free(cap);
  free(touched);
  return total <= cap_edges ? total : -1;
}

void oracle_transpose(int n, int K, const int *row, const int *col,
                      const int *w, int *rrow, int *rcol, int *rw) {
  long long m = row[n];
  int *fill = (int *)malloc(sizeof(int) * (size_t)(n + 1));
  memset(rrow, 0, sizeof(int) * (size_t)(n + 1));
  for (long long e = 0; e < m; ++e) ++rrow[col[e] + 1];
  for (int v = 0; v < n; ++v) rrow[v + 1] += rrow[v];
  memcpy(fill, rrow, sizeof(int) * (size_t)n);
  for (int u = 0; u < n; ++u) {
    for (int e = row[u]; e < row[u + 1]; ++e) {
      int pos = fill[col[e]]++;
      rcol[pos] = u;
      memcpy(rw + (long long)pos * K, w + (long long)e * K, sizeof(int) * (size_t)K);
    }
  }
  free(fill);
}

/* ------------------------------------------------------------------------ */
/* Dijkstra: src/Dijkstra.cu:239-272                                        */
/* ------------------------------------------------------------------------ */
typedef struct {
  long long d;
  int v;
} item;

static void heap_push(item *h, long long *size, item x) {
  long long i = (*size)++;
  while (i > 0) {
    long long p = (i - 1) / 2;
    if (h[p].d < x.d || (h[p].d == x.d && h[p].v <= x.v)) break;
    h[i] = h[p];
    i = p;
  }
  h[i] = x;
}

static item heap_pop(item *h, long long *size) {
  item top = h[0], last = h[--(*size)];
  long long i = 0;
  for (;;) {
    long long c = 2 * i + 1;
    if (c >= *size) break;
    if (c + 1 < *size && (h[c + 1].d < h[c].d || (h[c + 1].d == h[c].d && h[c + 1].v < h[c].v))) ++c;
    if (last.d < h[c].d || (last.d == h[c].d && last.v <= h[c].v)) break;
    h[i] = h[c];
    i = c;
  }
  if (*size > 0) h[i] = last;
  return top;
}

void oracle_dijkstra(int n, int K, const int *row, const int *col,
                     const int *w, int k, int source, long long *dist,
                     int *parent) {
  for (int v = 0; v < n; ++v) {
    dist[v] = ORACLE_INF;
    parent[v] = -1;
  }
  if (source < 0 || source >= n) return;
  long long cap = (long long)row[n] + 2, size = 0;
  item *heap = (item *)malloc(sizeof(item) * (size_t)cap);
  dist[source] = 0;
  item s = {0, source};
  heap_push(heap, &size, s);
  while (size > 0) {
    item t = heap_pop(heap, &size);
    if (t.d != dist[t.v]) continue;
    for (int e = row[t.v]; e < row[t.v + 1]; ++e) {
      int v = col[e];
      long long c = t.d + w[(long long)e * K + k];
      if (c < dist[v]) {
        dist[v] = c;
        parent[v] = t.v;
        if (size == cap) {
          cap *= 2;
          heap = (item *)realloc(heap, sizeof(item) * (size_t)cap);
        }
        item x = {c, v};
        heap_push(heap, &size, x);
      } else if (c == dist[v] && v != source && t.v < parent[v]) {
        parent[v] = t.v; /* equal distance: lowest parent id */
      }
    }
  }
  free(heap);
}

/* ------------------------------------------------------------------------ */
/* sequential update: src/sequentialSOSPUpdate.cu:456-612                   */
/* ------------------------------------------------------------------------ */
/* best (distance, lowest id) over the in-edges of v; returns 1 and writes
 * the new pair if it is strictly better, *decreased if the distance fell */
static int relax_vertex(int v, int K, int k, const int *rrow, const int *rcol,
                        const int *rw, long long *dist, int *parent,
                        int *decreased) {
  long long best = ORACLE_INF;
  int bp = -1;
  for (int e = rrow[v]; e < rrow[v + 1]; ++e) {
    int u = rcol[e];
    if (dist[u] >= ORACLE_INF / 2) continue;
    long long c = dist[u] + rw[(long long)e * K + k];
    if (c < best || (c == best && u < bp)) {
      best = c;
      bp = u;
    }
  }
  int better = best < dist[v] || (best == dist[v] && bp >= 0 && bp < parent[v]);
  *decreased = best < dist[v];
  if (better) {
    dist[v] = best;
    parent[v] = bp;
  }
  return better;
}

int oracle_sequential_update(int n, int K, int k, int source, const int *row,
                             const int *col, const int *w, const int *rrow,
                             const int *rcol, const int *rw, int n_changed,
                             const int *changed_from, const int *changed_to,
                             int n_heads, const int *heads, long long *dist,
                             int *parent) {
  (void)w;
  char *invalid = (char *)calloc((size_t)n, 1);
  char *affected = (char *)calloc((size_t)n, 1);
  char *candidate = (char *)calloc((size_t)n, 1);
  int *queue = (int *)malloc(sizeof(int) * (size_t)n);
  int *aff = (int *)malloc(sizeof(int) * (size_t)n);
  int *cand = (int *)malloc(sizeof(int) * (size_t)n);
  int *first = (int *)calloc((size_t)n + 1, sizeof(int));
  int *kids = (int *)malloc(sizeof(int) * (size_t)n);
  long long qn = 0, an = 0;
  int rounds = 0, dec;
  /* roots */
  for (int i = 0; i < n_changed; ++i) {
    int u = changed_from[i], v = changed_to[i];
    if (parent[v] == u && !invalid[v]) {
      invalid[v] = 1;
      queue[qn++] = v;
    }
  }
  /* subtrees of the roots (children lists of the old tree) */
  for (int v = 0; v < n; ++v)
    if (v != source && parent[v] >= 0) ++first[parent[v] + 1];
  for (int v = 0; v < n; ++v) first[v + 1] += first[v];
  {
    int *fill = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    memcpy(fill, first, sizeof(int) * (size_t)n);
    for (int v = 0; v < n; ++v)
      if (v != source && parent[v] >= 0) kids[fill[parent[v]]++] = v;
    free(fill);
  }
  for (long long i = 0; i < qn; ++i) {
    int x = queue[i];
    for (int c = first[x]; c < first[x + 1]; ++c) {
      if (!invalid[kids[c]]) {
        invalid[kids[c]] = 1;
        queue[qn++] = kids[c];
      }
    }
  }
  for (long long i = 0; i < qn; ++i) {
    dist[queue[i]] = ORACLE_INF;
    parent[queue[i]] = -1;
  }
  /* first re-evaluation: invalidated vertices, then insert heads */
  for (long long i = 0; i < qn; ++i) {
    int v = queue[i];
    relax_vertex(v, K, k, rrow, rcol, rw, dist, parent, &dec);
    if (dec && !affected[v]) {
      affected[v] = 1;
      aff[an++] = v;
    }
  }
  for (int i = 0; i < n_heads; ++i) {
    int v = heads[i];
    if (v == source) continue;
    relax_vertex(v, K, k, rrow, rcol, rw, dist, parent, &dec);
    if (dec && !affected[v]) {
      affected[v] = 1;
      aff[an++] = v;
    }
  }
  /* propagation: re-evaluate the out-neighbours of every vertex whose
   * distance decreased */
  while (an > 0) {
    long long cn = 0;
    ++rounds;
    for (long long i = 0; i < an; ++i) {
      int x = aff[i];
      affected[x] = 0;
      for (int e = row[x]; e < row[x + 1]; ++e) {
        int y = col[e];
        if (y == source || candidate[y]) continue;
        candidate[y] = 1;
        cand[cn++] = y;
      }
    }
    an = 0;
    for (long long i = 0; i < cn; ++i) {
      int y = cand[i];
      candidate[y] = 0;
      relax_vertex(y, K, k, rrow, rcol, rw, dist, parent, &dec);
      if (dec && !affected[y]) {
        affected[y] = 1;
        aff[an++] = y;
      }
    }
  }
  free(invalid);
  free(affected);
  free(candidate);
  free(queue);
  free(aff);
  free(cand);
  free(first);
  free(kids);
  return rounds;
}

/* ------------------------------------------------------------------------ */
/* combined graph: src/validation.cu:88-125, src/combinedGraphGpu.cu:129-159 */
/* ------------------------------------------------------------------------ */
static long long gcd_ll(long long a, long long b) {
  while (b != 0) {
    long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

long long oracle_preference_scale(const int *pref, int K) {
  if (pref == NULL) return 1;
  long long L = 1;
  for (int i = 0; i < K; ++i) {
    if (pref[i] < 1) return 0;
    L = L / gcd_ll(L, pref[i]) * pref[i];
    if (L > (1LL << 20)) return 0;
  }
  return L;
}

long long oracle_combined_graph(int n, int K, const int *parents, int source,
                                const int *pref, int *crow, int *ccol,
                                int *cw) {
  long long L = oracle_preference_scale(pref, K), m = 0;
  if (L == 0) return -1;
  /* count, then fill rows in order of heads (row p gets its edges in the
   * order the heads v are visited) */
  memset(crow, 0, sizeof(int) * (size_t)(n + 1));
  for (int pass = 0; pass < 2; ++pass) {
    int *fill = NULL;
    if (pass == 1) {
      for (int u = 0; u < n; ++u) crow[u + 1] += crow[u];
      fill = (int *)malloc(sizeof(int) * (size_t)(n + 1));
      memcpy(fill, crow, sizeof(int) * (size_t)(n + 1));
    }
    for (int v = 0; v < n; ++v) {
      if (v == source) continue;
      for (int k = 0; k < K; ++k) {
        int p = parents[(long long)k * n + v], seen = p < 0;
        for (int j = 0; j < k && !seen; ++j) seen = parents[(long long)j * n + v] == p;
        if (seen) continue;
        if (pass == 0) {
          ++crow[p + 1];
          continue;
        }
        long long weight = L * (K + 1);
        for (int j = 0; j < K; ++j)
          if (parents[(long long)j * n + v] == p) weight -= pref == NULL ? L : L / pref[j];
        int pos = fill[p]++;
        ccol[pos] = v;
        cw[pos] = (int)weight;
        ++m;
      }
    }
    free(fill);
  }
  return m;
}

/* ------------------------------------------------------------------------ */
/* path costs: src/combinedGraphGpu.cu:161-208                              */
/* ------------------------------------------------------------------------ */
int oracle_path_costs(int n, int KG, const int *row, const int *col,
                      const int *w, const int *parent, int source,
                      long long *costs) {
  int *first = (int *)calloc((size_t)n + 1, sizeof(int));
  int *kids = (int *)malloc(sizeof(int) * (size_t)n);
  int *fill = (int *)malloc(sizeof(int) * (size_t)(n + 1));
  int *queue = (int *)malloc(sizeof(int) * (size_t)n);
  long long qn = 0;
  int ok = 0;
  for (long long i = 0; i < (long long)n * KG; ++i) costs[i] = ORACLE_INF;
  for (int v = 0; v < n; ++v)
    if (v != source && parent[v] >= 0) ++first[parent[v] + 1];
  for (int v = 0; v < n; ++v) first[v + 1] += first[v];
  memcpy(fill, first, sizeof(int) * (size_t)n);
  for (int v = 0; v < n; ++v)
    if (v != source && parent[v] >= 0) kids[fill[parent[v]]++] = v;
  for (int k = 0; k < KG; ++k) costs[(long long)source * KG + k] = 0;
  queue[qn++] = source;
  for (long long i = 0; i < qn && ok == 0; ++i) {
    int p = queue[i];
    for (int c = first[p]; c < first[p + 1]; ++c) {
      int v = kids[c], edge = -1;
      for (int e = row[p]; e < row[p + 1]; ++e)
        if (col[e] == v) { edge = e; break; }
      if (edge < 0) { ok = -1; break; }
      for (int k = 0; k < KG; ++k)
        costs[(long long)v * KG + k] = costs[(long long)p * KG + k] + w[(long long)edge * KG + k];
      queue[qn++] = v;
    }
  }
  free(first);
  free(kids);
  free(fill);
  free(queue);
  return ok;
}

/* ------------------------------------------------------------------------ */
/* tree check: src/validation.cu:28-86                                      */
/* ------------------------------------------------------------------------ */
void oracle_check_tree(int n, int K, int k, int source, const int *rrow,
                       const int *rcol, const int *rw, const long long *dist,
                       const int *parent, const long long *ref_dist,
                       const int *ref_parent, long long counts[4]) {
  counts[0] = counts[1] = counts[2] = counts[3] = 0;
  for (int v = 0; v < n; ++v) {
    long long dv = dist[v];
    int reach = dv < ORACLE_INF / 2;
    if (reach != (ref_dist[v] < ORACLE_INF / 2) || (reach && dv != ref_dist[v])) ++counts[0];
    if (ref_parent != NULL && parent[v] != ref_parent[v]) ++counts[3];
    if (v == source) {
      if (parent[v] != -1 || dv != 0) ++counts[1];
      continue;
    }
    if (!reach) {
      if (parent[v] != -1) ++counts[1];
      continue;
    }
    int p = parent[v], tight = 0, lowest = -1;
    for (int e = rrow[v]; e < rrow[v + 1]; ++e) {
      int u = rcol[e];
      if (dist[u] >= ORACLE_INF / 2 || dist[u] + rw[(long long)e * K + k] != dv) continue;
      if (u == p) tight = 1;
      if (lowest < 0 || u < lowest) lowest = u;
    }
    if (!tight) ++counts[1];
    else if (p != lowest) ++counts[2];
  }
}
