"""The rule behind the restricted parent recovery, checked on the host.

For a distance-only objective the library recovers the lowest-id tight
parent of every reachable vertex after the update. When the input tree
already follows that rule, the restricted form (mosp_workspace_set_canonical_trees)
keeps the input parent at every vertex v except where
  (a) v's distance changed, (b) the distance of v's input parent changed,
  (c) an edge into v was inserted or lowered, (d) the edge from v's input
      parent was deleted or raised;
those vertices take the lowest tight tail of their in-row, and every
reachable vertex whose distance changed pushes itself (atomicMin) into the
other vertices along its tight out-edges. This test applies that rule with
numpy to the oracle's canonical trees before and after random batches of
every kind, on graphs with weights in 1..3 (ties everywhere), and requires
the result to be the oracle's canonical tree of the updated graph, i.e. the
full recovery's. It checks the rule, not the kernels: the GPU tests
(tests/test_gpu_recovery.py) compare the kernels with both."""
import numpy as np
import pytest

import mosp_b200 as mb
import oracle as orc
from conftest import grid_graph, random_graph

BATCHES = [dict(mode="uniform", ins_pct=50, safe=True), dict(mode="uniform", ins_pct=50),
           dict(mode="uniform", ins_pct=0), dict(mode="uniform", ins_pct=100), dict(mode="increase"),
           dict(mode="reweight"), dict(mode="targeted", ins_pct=30)]


def restricted_parents(urow, ucol, uw, k, d0, p0, d1, heads, ch_from, ch_to, source=0):
    """Parents of the updated tree by the restricted rule, from the input
    tree (d0, p0) and the new distances d1 of objective k."""
    n = len(urow) - 1
    inf = orc.INF
    w = uw[:, k].astype(np.int64)
    tails = np.repeat(np.arange(n, dtype=np.int64), np.diff(urow))
    heads_of_edges = ucol.astype(np.int64)
    reach = d1 < inf
    changed = d1 != d0
    need = changed.copy()
    valid_p = p0 >= 0
    need[valid_p] |= changed[p0[valid_p]]                       # (b)
    need[heads] = True                                          # (c)
    need[ch_to[p0[ch_to] == ch_from]] = True                    # (d)
    tight = reach[tails] & (d1[tails] + w == d1[heads_of_edges])
    parent = np.where(reach, p0, -1).astype(np.int64)
    parent[source] = -1
    scan = need & reach
    scan[source] = False
    big = np.iinfo(np.int64).max
    parent[scan] = big
    sel = tight & scan[heads_of_edges]                          # rescans of the need rows
    np.minimum.at(parent, heads_of_edges[sel], tails[sel])
    sel = tight & changed[tails] & ~need[heads_of_edges] & (heads_of_edges != source)
    np.minimum.at(parent, heads_of_edges[sel], tails[sel])      # pushes from changed vertices
    parent[parent == big] = np.iinfo(np.int32).max              # no tight in-edge (as the full rebuild)
    return parent.astype(np.int32)


def check_rule(row, col, w, spec, seed, K):
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, max(8, len(col) // 20), seed=seed, wmax=3, **spec)
    upd = mb.apply_batch(g, b)
    ba = b.arrays()
    urow, ucol, uw = upd.arrays()
    ch = mb.changed_lists(ba, K)
    heads = np.asarray(ba["ins_to"], np.int64)
    for k in range(K):
        d0, p0 = orc.dijkstra(row, col, w, k, 0)
        d1, p1 = orc.dijkstra(urow, ucol, uw, k, 0)
        got = restricted_parents(urow, ucol, uw, k, d0, p0.astype(np.int64), d1, heads,
                                 ch[k][0].astype(np.int64), ch[k][1].astype(np.int64))
        assert np.array_equal(got, p1), f"objective {k}: {np.count_nonzero(got != p1)} parents differ"


@pytest.mark.parametrize("spec", BATCHES, ids=[f"{s['mode']}-{s.get('ins_pct', '')}" for s in BATCHES])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_restricted_rule_on_grids(spec, seed):
    row, col, w = grid_graph(30, 24, 2, 3, 0.25, 400 + seed)
    check_rule(row, col, w, spec, 500 + seed, 2)


@pytest.mark.parametrize("spec", BATCHES, ids=[f"{s['mode']}-{s.get('ins_pct', '')}" for s in BATCHES])
def test_restricted_rule_on_random_graphs(spec):
    row, col, w = random_graph(900, 3600, 2, 3, 77)
    check_rule(row, col, w, spec, 78, 2)
