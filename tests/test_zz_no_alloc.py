"""mosp_sosp_from_scratch_static: SSSP from scratch with its scratch in a
fixed device array, through the C ABI. Its results must equal the workspace
entry point mosp_sosp_from_scratch's (and the oracle's) on consecutive calls,
it must reject graphs beyond its limits, and repeated calls must not take
device memory. The file name sorts last so that the suite also runs it after
every other GPU test."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402
from conftest import grid_graph, random_graph  # noqa: E402

MAX_N = 65536
MAX_M = 262144


@pytest.fixture(scope="module")
def ws():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    w = mb.Workspace(timeout_ms=20000)
    yield w
    w.close()


def static_call(n, m, dg, source, delta, max_weight, dist, parent):
    st = mb.SospStats()
    rc = mb.lib().mosp_sosp_from_scratch_static(
        n, m, dg.out_row.data_ptr(), dg.out_col.data_ptr(), dg.out_w.data_ptr(), source, int(delta),
        int(max_weight), dist.data_ptr(), parent.data_ptr(), C.byref(st), None)
    return rc, st


def upload(ws, row, col, w):
    g = mb.HostGraph.from_arrays(row, col, w)
    return g, mb.DeviceGraph.upload(ws, g)


def workspace_tree(ws, g, dg, source, delta, max_weight):
    d = torch.empty(g.n, dtype=torch.int64, device="cuda")
    p = torch.empty(g.n, dtype=torch.int32, device="cuda")
    st = ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w, source, delta, max_weight, d, p)
    return d.cpu().numpy(), p.cpu().numpy(), st


def static_tree(g, dg, source, delta, max_weight):
    # outputs start as garbage so that a missed write shows
    d = torch.full((g.n,), -7, dtype=torch.int64, device="cuda")
    p = torch.full((g.n,), -7, dtype=torch.int32, device="cuda")
    rc, st = static_call(g.n, g.m, dg, source, delta, max_weight, d, p)
    assert rc == mb.OK, mb.lib().mosp_last_error().decode()
    return d.cpu().numpy(), p.cpu().numpy(), st


def test_static_equals_workspace_on_consecutive_calls(ws):
    cases = [
        (grid_graph(120, 120, 1, 100, 0.25, 21), 0, 40),
        (random_graph(3000, 12000, 1, 1000, 22), 5, 500),
        (grid_graph(120, 120, 1, 100, 0.25, 21), 77, 1),
    ]
    uploaded = [(upload(ws, *graph), source, delta) for graph, source, delta in cases]
    # the static calls back to back, then the workspace calls
    static_results = [static_tree(g, dg, s, delta, int(g.arrays()[2].max()))
                      for (g, dg), s, delta in uploaded]
    for ((g, dg), s, delta), (graph, _, _), (ds, ps, sts) in zip(uploaded, cases, static_results):
        dw, pw, stw = workspace_tree(ws, g, dg, s, delta, int(graph[2].max()))
        assert np.array_equal(ds, dw) and np.array_equal(ps, pw)
        # the trees are schedule independent; iteration and push counts are not
        assert sts.packed_parents == stw.packed_parents and sts.iterations > 0
        de, pe = orc.dijkstra(*graph, 0, s)
        assert np.array_equal(ds, de) and np.array_equal(ps, pe)


def test_static_at_its_limits(ws):
    # 256 x 256 grid without drops: n = 65536, m = 261120 <= 262144
    row, col, w = grid_graph(256, 256, 1, 1000, 0.0, 23)
    assert len(row) - 1 == MAX_N and len(col) <= MAX_M
    g, dg = upload(ws, row, col, w)
    for _ in range(2):
        ds, ps, _ = static_tree(g, dg, 1234, 2000, int(w.max()))
        dw, pw, _ = workspace_tree(ws, g, dg, 1234, 2000, int(w.max()))
        assert np.array_equal(ds, dw) and np.array_equal(ps, pw)


def test_static_rejects_graphs_beyond_its_limits(ws):
    row, col, w = grid_graph(20, 20, 1, 10, 0.1, 24)
    g, dg = upload(ws, row, col, w)
    d = torch.empty(MAX_N + 1, dtype=torch.int64, device="cuda")
    p = torch.empty(MAX_N + 1, dtype=torch.int32, device="cuda")
    rc, _ = static_call(MAX_N + 1, g.m, dg, 0, 10, 10, d, p)
    assert rc == mb.ERR_INVALID
    assert b"65536" in mb.lib().mosp_last_error()
    rc, _ = static_call(g.n, MAX_M + 1, dg, 0, 10, 10, d, p)
    assert rc == mb.ERR_INVALID
    assert b"262144" in mb.lib().mosp_last_error()
    # the entry point still works after a rejection
    ds, ps, _ = static_tree(g, dg, 0, 10, int(w.max()))
    de, pe = orc.dijkstra(row, col, w, 0, 0)
    assert np.array_equal(ds, de) and np.array_equal(ps, pe)


def test_static_calls_take_no_device_memory(ws):
    row, col, w = random_graph(5000, 20000, 1, 100, 25)
    g, dg = upload(ws, row, col, w)
    d = torch.empty(g.n, dtype=torch.int64, device="cuda")
    p = torch.empty(g.n, dtype=torch.int32, device="cuda")
    assert static_call(g.n, g.m, dg, 0, 50, int(w.max()), d, p)[0] == mb.OK
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for s in (1, 2, 3):
        assert static_call(g.n, g.m, dg, s, 50, int(w.max()), d, p)[0] == mb.OK
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_static_distance_only_words(ws):
    """A declared weight bound so large that (n - 1) * max_weight does not
    fit next to the parent field (within the static limits no int32 weight
    gets there): distance-only words and the in-launch lowest-id parent
    recovery, through the static scratch, with tied distances."""
    row, col, w = grid_graph(60, 60, 1, 4, 0.1, 26)
    g, dg = upload(ws, row, col, w)
    bound = 10 ** 13
    for _ in range(2):
        ds, ps, st = static_tree(g, dg, 5, 3, bound)
        assert st.packed_parents == 0
        dw, pw, _ = workspace_tree(ws, g, dg, 5, 3, bound)
        assert np.array_equal(ds, dw) and np.array_equal(ps, pw)
    de, pe = orc.dijkstra(row, col, w, 0, 5)
    assert np.array_equal(ds, de) and np.array_equal(ps, pe)


def test_static_hub_row(ws):
    """A star hub of 3,000 edges (more than the 2,048 a warp expands alone):
    the CTA-wide hub queue runs on the static scratch too."""
    n = 6000
    rng = np.random.default_rng(27)
    edges = {(i, i + 1) for i in range(n - 1)} | {(0, v) for v in range(2, 3002)}
    while len(edges) < n - 1 + 3000 + 6000:
        u, v = rng.integers(0, n, 2)
        if u != v:
            edges.add((int(u), int(v)))
    edges = sorted(edges)
    row = np.zeros(n + 1, np.int32)
    for u, _ in edges:
        row[u + 1] += 1
    row = np.cumsum(row).astype(np.int32)
    col = np.array([v for _, v in edges], np.int32)
    w = rng.integers(1, 500, (len(edges), 1)).astype(np.int32)
    assert row[1] - row[0] > 2048
    g, dg = upload(ws, row, col, w)
    for _ in range(2):
        ds, ps, _ = static_tree(g, dg, 0, 100, int(w.max()))
        dw, pw, _ = workspace_tree(ws, g, dg, 0, 100, int(w.max()))
        assert np.array_equal(ds, dw) and np.array_equal(ps, pw)
    de, pe = orc.dijkstra(row, col, w, 0, 0)
    assert np.array_equal(ds, de) and np.array_equal(ps, pe)


def test_static_rejects_malformed_csr(ws):
    """A CSR whose last offset exceeds the edge count, or with a column out
    of range, is rejected on the device before any relaxation (small graph,
    so even an access past the check stays inside the scratch)."""
    row, col, w = grid_graph(20, 20, 1, 10, 0.0, 28)
    g = mb.HostGraph.from_arrays(row, col, w)
    n, m = g.n, g.m
    d = torch.empty(n, dtype=torch.int64, device="cuda")
    p = torch.empty(n, dtype=torch.int32, device="cuda")
    bad_row = row.copy()
    bad_row[-1] = m + 1
    col_t = torch.from_numpy(np.concatenate([col, [0]]).astype(np.int32)).cuda()
    w_t = torch.from_numpy(np.concatenate([w[:, 0], [1]]).astype(np.int32)).cuda()
    row_t = torch.from_numpy(bad_row.astype(np.int32)).cuda()
    st = mb.SospStats()
    rc = mb.lib().mosp_sosp_from_scratch_static(n, m, row_t.data_ptr(), col_t.data_ptr(), w_t.data_ptr(), 0, 10,
                                                10, d.data_ptr(), p.data_ptr(), C.byref(st), None)
    assert rc == mb.ERR_INVALID
    bad_col = col.copy()
    bad_col[7] = n + 5
    row_t = torch.from_numpy(row.astype(np.int32)).cuda()
    col_t = torch.from_numpy(bad_col.astype(np.int32)).cuda()
    rc = mb.lib().mosp_sosp_from_scratch_static(n, m, row_t.data_ptr(), col_t.data_ptr(), w_t.data_ptr(), 0, 10,
                                                10, d.data_ptr(), p.data_ptr(), C.byref(st), None)
    assert rc == mb.ERR_INVALID
    assert b"malformed CSR" in mb.lib().mosp_last_error()
    # still usable afterwards
    g2, dg2 = upload(ws, row, col, w)
    ds, ps, _ = static_tree(g2, dg2, 0, 10, int(w.max()))
    de, pe = orc.dijkstra(row, col, w, 0, 0)
    assert np.array_equal(ds, de) and np.array_equal(ps, pe)
