"""GPU parity of the restricted parent recovery (mosp_workspace_set_canonical_trees).

An objective whose packed word would need more than 64 bits runs on
distances alone; afterwards every reachable vertex takes the lowest-id tail
of a tight in-edge. By default the library does that over every edge, as
the reference does (src/sospUpdateGpu.cu:491-512). With the input trees
declared canonical it does it only where the batch can change a parent:
vertices whose distance, parent distance or in-edges changed scan their
in-rows, and vertices whose distance changed push along their out-edges.
For canonical input trees (the oracle's lowest-id Dijkstra trees here) both
must give the oracle's trees bit for bit. The weight bound passed to the
library is raised so that every objective runs distance-only, and weights
in 1..3 make ties everywhere. Covered: every batch kind, both near-far
loops, rows of more than 64 edges in both directions (the listed rows,
handled in 128-edge chunks, one warp per chunk), batched roots, repeated
updates and an empty batch."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
from conftest import grid_graph  # noqa: E402
from gpu_util import assert_matches_oracle, run_update_device  # noqa: E402

KEYS = ("dist", "parent", "comb_dist", "comb_parent", "costs")


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")


def distance_only_bound(n):
    """A weight bound for which (n - 1) * bound does not fit next to the
    parent field (distance-only words) but stays below 2^59."""
    bound = (1 << 59) // max(n, 2)
    assert mb.choose_packing(n, bound)[0] == 0
    return bound


def both(g, b, async_on=True, **kw):
    """(full recovery, restricted recovery) of the same update."""
    out = []
    for canonical in (False, True):
        ws = mb.Workspace(timeout_ms=20000)
        ws.set_async(async_on)
        ws.set_canonical_trees(canonical)
        res = run_update_device(ws, g, b, max_weight=distance_only_bound(g.n), **kw)
        ws.close()
        assert all(s.packed_parents == 0 for s in res["stats"])
        out.append(res)
    for key in KEYS:
        assert np.array_equal(out[0][key], out[1][key]), key
    return out[1]


BATCHES = [dict(mode="uniform", ins_pct=50, safe=True), dict(mode="uniform", ins_pct=50),
           dict(mode="uniform", ins_pct=0), dict(mode="uniform", ins_pct=100), dict(mode="increase"),
           dict(mode="reweight"), dict(mode="targeted", ins_pct=30)]


@pytest.mark.parametrize("spec", BATCHES, ids=[f"{b['mode']}-{b.get('ins_pct', '')}" for b in BATCHES])
@pytest.mark.parametrize("async_on", [True, False], ids=["async", "bulk"])
def test_restricted_recovery_ties(gpu, spec, async_on):
    row, col, w = grid_graph(70, 60, 3, 3, 0.3, 81)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 900, seed=82, wmax=3, **spec)
    assert_matches_oracle(both(g, b, async_on), g, b)


def hub_graph(seed, K=2):
    """Chain 0 -> 1 -> ... -> n-1 with weights 1..3, vertex 100 with 2,000
    out-edges, vertex 4000 with ~2,000 in-edges, and random arcs; the only
    edges into vertex 100 come from 99 and 4999, so deleting 99 -> 100
    moves vertex 100 (and its long out-row pushes)."""
    n = 5000
    rng = np.random.default_rng(seed)
    edges = {(i, i + 1) for i in range(n - 1)}
    edges |= {(100, v) for v in range(1000, 3000)}
    edges |= {(u, 4000) for u in range(0, 2000)}
    edges.add((4999, 100))
    while len(edges) < 2 * (n - 1) + 4000 + 10000:
        u, v = (int(x) for x in rng.integers(0, n, 2))
        if u != v and v != 100:
            edges.add((u, v))
    edges = sorted(edges)
    row = np.zeros(n + 1, np.int64)
    for u, _ in edges:
        row[u + 1] += 1
    row = np.cumsum(row).astype(np.int32)
    col = np.array([v for _, v in edges], np.int32)
    w = rng.integers(1, 4, (len(edges), K)).astype(np.int32)
    return mb.HostGraph.from_arrays(row, col, w)


@pytest.mark.parametrize("async_on", [True, False], ids=["async", "bulk"])
def test_restricted_recovery_long_rows(gpu, async_on):
    g = hub_graph(83)
    gen = mb.HostBatch.generate(g, 600, seed=84, wmax=3, mode="targeted", ins_pct=30).arrays()
    K = g.K
    # the chain edge into the hub, and an insertion into the in-hub
    ins_from = np.concatenate([gen["ins_from"], [2500]]).astype(np.int32)
    ins_to = np.concatenate([gen["ins_to"], [4000]]).astype(np.int32)
    ins_w = np.concatenate([gen["ins_w"].reshape(-1, K), [[1] * K]]).astype(np.int32)
    del_from = np.concatenate([gen["del_from"], [99]]).astype(np.int32)
    del_to = np.concatenate([gen["del_to"], [100]]).astype(np.int32)
    keep = ~((del_from == 99) & (del_to == 100))
    keep[-1] = True
    b = mb.HostBatch.from_arrays(K, ins_from, ins_to, ins_w, del_from[keep], del_to[keep])
    assert_matches_oracle(both(g, b, async_on), g, b)


def test_restricted_recovery_empty_batch(gpu):
    row, col, w = grid_graph(40, 40, 2, 3, 0.2, 85)
    g = mb.HostGraph.from_arrays(row, col, w)
    z = np.zeros(0, np.int32)
    b = mb.HostBatch.from_arrays(2, z, z, np.zeros((0, 2), np.int32), z, z)
    assert_matches_oracle(both(g, b), g, b)


def test_restricted_recovery_repeated(gpu):
    """Trees the library returned are canonical: a second update on them
    with the restricted recovery equals the oracle on the twice-updated
    graph."""
    row, col, w = grid_graph(60, 60, 2, 3, 0.25, 86)
    g = mb.HostGraph.from_arrays(row, col, w)
    b1 = mb.HostBatch.generate(g, 700, seed=87, wmax=3, mode="targeted", ins_pct=40)
    ws = mb.Workspace(timeout_ms=20000)
    ws.set_canonical_trees(True)
    bound = distance_only_bound(g.n)
    r1 = run_update_device(ws, g, b1, max_weight=bound)
    assert_matches_oracle(r1, g, b1)
    g2 = mb.apply_batch(g, b1)
    b2 = mb.HostBatch.generate(g2, 700, seed=88, wmax=3, mode="uniform", ins_pct=50)
    r2 = run_update_device(ws, g2, b2, init=(r1["dist"], r1["parent"]), max_weight=bound)
    ws.close()
    assert_matches_oracle(r2, g2, b2)


def test_restricted_recovery_batched_roots(gpu):
    """Disjoint union of instances, one root each (mosp_workspace_set_sources);
    each instance gets its own batch, so the union stays disjoint."""
    import oracle as orc
    K = 2
    parts = [grid_graph(25 + 4 * i, 20 + 3 * i, K, 3, 0.2, 90 + i) for i in range(4)]
    rows, cols, wts, roots, bases = [np.zeros(1, np.int64)], [], [], [], []
    batch = {k: [] for k in ("ins_from", "ins_to", "ins_w", "del_from", "del_to")}
    base = 0
    for i, (row, col, w) in enumerate(parts):
        rows.append(row[1:].astype(np.int64) + rows[-1][-1])
        cols.append(col + base)
        wts.append(w)
        roots.append(base + 5)
        bases.append(base)
        pb = mb.HostBatch.generate(mb.HostGraph.from_arrays(row, col, w), 150, seed=95 + i, wmax=3,
                                   mode="targeted", ins_pct=30).arrays()
        for key in ("ins_from", "ins_to", "del_from", "del_to"):
            batch[key].append(pb[key] + base)
        batch["ins_w"].append(pb["ins_w"].reshape(-1, K))
        base += len(row) - 1
    g = mb.HostGraph.from_arrays(np.concatenate(rows).astype(np.int32), np.concatenate(cols).astype(np.int32),
                                 np.concatenate(wts).astype(np.int32))
    b = mb.HostBatch.from_arrays(K, *(np.concatenate(batch[key]).astype(np.int32)
                                      for key in ("ins_from", "ins_to", "ins_w", "del_from", "del_to")))
    ba = b.arrays()
    d0 = np.empty((K, g.n), np.int64)
    p0 = np.empty((K, g.n), np.int32)
    de = np.empty((K, g.n), np.int64)
    pe = np.empty((K, g.n), np.int32)
    for (row, col, w), r, off in zip(parts, roots, bases):
        pn = len(row) - 1
        sel_i = (ba["ins_from"] >= off) & (ba["ins_from"] < off + pn)
        sel_d = (ba["del_from"] >= off) & (ba["del_from"] < off + pn)
        upd = orc.apply_batch(row, col, w, ba["ins_from"][sel_i] - off, ba["ins_to"][sel_i] - off,
                              ba["ins_w"].reshape(-1, K)[sel_i], ba["del_from"][sel_d] - off,
                              ba["del_to"][sel_d] - off)
        for k in range(K):
            for (gr, gc, gw), dd, pp in (((row, col, w), d0, p0), (upd[:3], de, pe)):
                d, p = orc.dijkstra(gr, gc, gw, k, r - off)
                dd[k, off:off + pn] = d
                pp[k, off:off + pn] = np.where(p >= 0, p + off, p)
    for canonical in (False, True):
        ws = mb.Workspace(timeout_ms=20000)
        ws.set_sources(roots)
        ws.set_canonical_trees(canonical)
        res = run_update_device(ws, g, b, source=roots[0], init=(d0, p0), max_weight=distance_only_bound(g.n))
        ws.close()
        assert np.array_equal(res["dist"], de) and np.array_equal(res["parent"], pe), canonical
