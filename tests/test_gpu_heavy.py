"""Hub rows: rows of more than 2,048 edges are expanded (push) and reduced
(pull) by a whole CTA through a per-CTA queue of 64 rows; rows beyond the
queue stay with their warp. The graphs here have 100 hubs of 2,100-6,000
edges each (the source among them, so the combined graph's source row is a
hub too), enough to fill and overflow the queues. Every result must equal
the oracle: the update with the staged pull (K = 3) and the unstaged pull
(K = 12), the SSSP from scratch at several bucket widths, and the
distance-only fallback."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402
from gpu_util import assert_matches_oracle, run_update_device  # noqa: E402


@pytest.fixture(scope="module")
def ws():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    w = mb.Workspace(timeout_ms=30000)
    yield w
    w.close()


def hub_graph(n, hubs, K, wmin, wmax, seed):
    """Undirected graph stored as directed CSR: a chain 0-1-...-(n-1), `hubs`
    hub vertices (0 first) joined to 2,100-6,000 random vertices each, and n
    random extra links; K weights per direction drawn uniformly."""
    rng = np.random.default_rng(seed)
    hub_ids = np.concatenate([[0], rng.choice(np.arange(1, n), hubs - 1, replace=False)])
    us = [np.arange(n - 1)]
    vs = [np.arange(1, n)]
    for h in hub_ids:
        d = int(rng.integers(2100, 6001))
        us.append(np.full(d, h))
        vs.append(rng.integers(0, n, d))
    us.append(rng.integers(0, n, n))
    vs.append(rng.integers(0, n, n))
    u = np.concatenate(us).astype(np.int64)
    v = np.concatenate(vs).astype(np.int64)
    keep = u != v
    u, v = u[keep], v[keep]
    a, b = np.concatenate([u, v]), np.concatenate([v, u])
    key = np.unique(a * n + b)
    src, dst = key // n, key % n
    row = np.zeros(n + 1, np.int64)
    np.add.at(row, src + 1, 1)
    row = np.cumsum(row).astype(np.int32)
    w = rng.integers(wmin, wmax + 1, (len(dst), K), dtype=np.int64).astype(np.int32)
    return row, dst.astype(np.int32), w


def test_hub_graph_has_heavy_rows():
    row, _, _ = hub_graph(12000, 100, 1, 1, 100, 1)
    deg = np.diff(row)
    assert (deg > 2048).sum() >= 90 and deg.max() > 4000


@pytest.mark.parametrize("K", [3, 12])
def test_update_with_hubs(ws, K):
    row, col, w = hub_graph(12000, 100, K, 1, 1000, 7 + K)
    g = mb.HostGraph.from_arrays(row, col, w)
    for mode, seed in (("targeted", 11), ("uniform", 12)):
        b = mb.HostBatch.generate(g, 4000, 40.0, mode, 0, False, seed, 0, 1, 1000)
        pref = list(range(1, K + 1)) if K <= 5 else None
        res = run_update_device(ws, g, b, pref=pref)
        assert_matches_oracle(res, g, b, pref=pref)


def test_from_scratch_with_hubs(ws):
    row, col, w = hub_graph(12000, 100, 1, 1, 1000, 21)
    g = mb.HostGraph.from_arrays(row, col, w)
    dg = mb.DeviceGraph.upload(ws, g)
    d = torch.empty(g.n, dtype=torch.int64, device="cuda")
    p = torch.empty(g.n, dtype=torch.int32, device="cuda")
    de, pe = orc.dijkstra(row, col, w, 0, 0)
    for delta in (1, 300, 10 ** 9):
        ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w, 0, delta, int(w.max()), d, p)
        assert np.array_equal(d.cpu().numpy(), de), delta
        assert np.array_equal(p.cpu().numpy(), pe), delta


def test_fallback_with_hubs(ws):
    """Weights up to 2^31 - 1 on 80,000 vertices: the packed word cannot
    hold (n - 1) * maxWeight next to 17 parent bits, so distances only, then
    the lowest-id parent recovery."""
    n, W = 80000, 2_147_483_647
    row, col, w = hub_graph(n, 100, 2, 1, W, 31)
    assert mb.choose_packing(n, W)[0] == 0
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 3000, 30.0, "targeted", 0, False, 32, 0, 1, W)
    res = run_update_device(ws, g, b)
    assert all(s.packed_parents == 0 for s in res["stats"])
    assert_matches_oracle(res, g, b)


def test_from_scratch_fallback_with_hubs(ws):
    """SSSP from scratch with distance-only words: the lowest-id parent
    recovery inside the launch (update launches run it as a kernel of its
    own) on a graph with hub rows."""
    n, W = 80000, 2_147_483_647
    row, col, w = hub_graph(n, 100, 1, 1, W, 41)
    assert mb.choose_packing(n, W)[0] == 0
    g = mb.HostGraph.from_arrays(row, col, w)
    dg = mb.DeviceGraph.upload(ws, g)
    d = torch.empty(n, dtype=torch.int64, device="cuda")
    p = torch.empty(n, dtype=torch.int32, device="cuda")
    st = ws.sosp_from_scratch(n, g.m, dg.out_row, dg.out_col, dg.out_w, 0, 10 ** 12, W, d, p)
    assert st.packed_parents == 0
    de, pe = orc.dijkstra(row, col, w, 0, 0)
    assert np.array_equal(d.cpu().numpy(), de)
    assert np.array_equal(p.cpu().numpy(), pe)
