"""GPU parity of the asynchronous near-far loop (mosp_workspace_set_async).

The asynchronous loop replaces the engine's bulk-synchronous near-far
iterations by phases in which every warp expands entries of a sharded near
queue as they arrive. The relaxations are the same monotone packed-word
atomicMin, so every output must equal the bulk loop's and the oracle's bit
for bit: updated trees, combined tree, MOSP costs; from-scratch trees; the
distance-only fallback; batched roots; a queue so small that most entries
overflow to the far pile; and graphs with hub rows, where the launch falls
back to the bulk loop."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402
from conftest import grid_graph, random_graph  # noqa: E402
from gpu_util import assert_matches_oracle, run_update_device  # noqa: E402

KEYS = ("dist", "parent", "comb_dist", "comb_parent", "costs")


def workspace(async_on, queue_slots=0):
    w = mb.Workspace(timeout_ms=20000)
    w.set_async(async_on, queue_slots)
    return w


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")


BATCHES = [dict(mode="uniform", ins_pct=50, safe=True), dict(mode="uniform", ins_pct=50),
           dict(mode="uniform", ins_pct=0), dict(mode="uniform", ins_pct=100), dict(mode="increase"),
           dict(mode="reweight"), dict(mode="targeted", ins_pct=30)]


@pytest.mark.parametrize("spec", BATCHES, ids=[f"{b['mode']}-{b.get('ins_pct', '')}" for b in BATCHES])
def test_async_equals_bulk_and_oracle(gpu, spec):
    row, col, w = grid_graph(60, 50, 3, 100, 0.3, 31)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 800, seed=32, wmax=100, **spec)
    outs = []
    for on in (True, False):
        ws = workspace(on)
        outs.append(run_update_device(ws, g, b))
        ws.close()
    for key in KEYS:
        assert np.array_equal(outs[0][key], outs[1][key]), key
    assert_matches_oracle(outs[0], g, b)


def test_async_small_queue_overflows_to_far(gpu):
    """32 slots per shard: most near entries find their shard full and go to
    the far pile; the results stay exact."""
    row, col, w = random_graph(4000, 16000, 3, 1000, 33)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 1500, seed=34, wmax=1000)
    ws = workspace(True, queue_slots=1024)
    small = run_update_device(ws, g, b)
    ws.close()
    assert_matches_oracle(small, g, b)
    ws = workspace(True)
    big = run_update_device(ws, g, b)
    ws.close()
    for key in KEYS:
        assert np.array_equal(small[key], big[key]), key
    # overflow costs phases, not correctness
    assert small["stats"][0].iterations >= big["stats"][0].iterations


@pytest.mark.parametrize("delta", [1, 37, 10 ** 9])
def test_async_from_scratch(gpu, delta):
    row, col, w = grid_graph(90, 70, 1, 100, 0.2, 35)
    g = mb.HostGraph.from_arrays(row, col, w)
    res = []
    for on in (True, False):
        ws = workspace(on)
        dg = mb.DeviceGraph.upload(ws, g)
        d = torch.empty(g.n, dtype=torch.int64, device="cuda")
        p = torch.empty(g.n, dtype=torch.int32, device="cuda")
        ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w, 17, delta, int(w.max()), d, p)
        res.append((d.cpu().numpy(), p.cpu().numpy()))
        ws.close()
    de, pe = orc.dijkstra(row, col, w, 0, 17)
    for d, p in res:
        assert np.array_equal(d, de) and np.array_equal(p, pe)


def test_async_distance_only_fallback(gpu):
    """Weights near INT_MAX: distance-only words (the tag saturates) and the
    lowest-id parent recovery after the loop."""
    # (n - 1) * maxWeight must exceed the 47 bits left next to a 17-bit
    # parent field: 330 x 330 vertices with weights near INT_MAX
    row, col, w = grid_graph(330, 330, 2, 2 * 10 ** 9, 0.1, 36, wmin=10 ** 9)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 300, seed=37, wmax=2 * 10 ** 9)
    ws = workspace(True)
    res = run_update_device(ws, g, b)
    ws.close()
    assert res["stats"][0].packed_parents == 0
    assert_matches_oracle(res, g, b)


def test_async_ties(gpu):
    """Every weight equal: many equal-distance parents, lowest id wins."""
    row, col, _ = grid_graph(50, 50, 2, 2, 0.0, 38)
    w = np.full((len(col), 2), 7, np.int32)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 400, seed=39, wmax=7)
    ws = workspace(True)
    res = run_update_device(ws, g, b)
    ws.close()
    assert_matches_oracle(res, g, b)


def test_async_hub_rows_fall_back(gpu):
    """A graph with rows of more than 2,048 edges runs the bulk loop (the
    asynchronous one hands no row to a whole CTA); the next launch of the
    same workspace goes to the bulk loop directly. Results are exact."""
    n = 6000
    rng = np.random.default_rng(40)
    edges = {(i, i + 1) for i in range(n - 1)} | {(0, v) for v in range(1, 3000)}
    while len(edges) < n - 1 + 3000 + 8000:
        u, v = rng.integers(0, n, 2)
        if u != v:
            edges.add((int(u), int(v)))
    edges = sorted(edges)
    row = np.zeros(n + 1, np.int32)
    for u, _ in edges:
        row[u + 1] += 1
    row = np.cumsum(row).astype(np.int32)
    col = np.array([v for _, v in edges], np.int32)
    w = rng.integers(1, 100, (len(edges), 2)).astype(np.int32)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 500, seed=41, wmax=100)
    ws = workspace(True)
    for _ in range(2):
        res = run_update_device(ws, g, b)
        assert_matches_oracle(res, g, b)
    ws.close()


def test_async_batched_roots(gpu):
    """Disjoint union of instances with one root each."""
    parts = [grid_graph(20 + 5 * i, 15 + 3 * i, 2, 50, 0.2, 50 + i) for i in range(5)]
    rows, cols, ws_, roots, base = [np.zeros(1, np.int64)], [], [], [], 0
    for row, col, w in parts:
        rows.append(row[1:].astype(np.int64) + rows[-1][-1])
        cols.append(col + base)
        ws_.append(w)
        roots.append(base + 3)
        base += len(row) - 1
    row = np.concatenate(rows).astype(np.int32)
    col = np.concatenate(cols).astype(np.int32)
    w = np.concatenate(ws_)
    res = []
    for on in (True, False):
        ws = workspace(on)
        ws.set_sources(roots)
        dg = mb.DeviceGraph.upload(ws, mb.HostGraph.from_arrays(row, col, w))
        n, m = len(row) - 1, len(col)
        d = torch.empty(n, dtype=torch.int64, device="cuda")
        p = torch.empty(n, dtype=torch.int32, device="cuda")
        ws.sosp_from_scratch(n, m, dg.out_row, dg.out_col, dg.out_w[:m], roots[0], 40, int(w.max()), d, p)
        res.append((d.cpu().numpy(), p.cpu().numpy()))
        ws.close()
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
    off = 0
    for (prow, pcol, pw), r in zip(parts, roots):
        pn = len(prow) - 1
        de, pe = orc.dijkstra(prow, pcol, pw, 0, r - off)
        assert np.array_equal(res[0][0][off:off + pn], de)
        pe = np.where(pe >= 0, pe + off, pe)
        assert np.array_equal(res[0][1][off:off + pn], pe)
        off += pn


def test_async_local_continuation_option(gpu, tmp_path):
    """The opt-in warp-local continuation (engine switch 16, read from
    MOSP_ENGINE_FLAGS when the library loads) reaches the same trees: run in
    a fresh process with the switch set."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = """
import sys
sys.path[:0] = [{t!r}, {m!r}, {o!r}]
import numpy as np
import mosp_b200 as mb
from conftest import grid_graph
from gpu_util import assert_matches_oracle, run_update_device
row, col, w = grid_graph(80, 70, 3, 100, 0.3, 77)
g = mb.HostGraph.from_arrays(row, col, w)
b = mb.HostBatch.generate(g, 1500, seed=78, wmax=100)
ws = mb.Workspace(timeout_ms=20000)
res = run_update_device(ws, g, b)
assert_matches_oracle(res, g, b)
print("LOCAL_OK")
""".format(t=os.path.join(root, "tests"), m=os.path.join(root, "mosp-cuda_b200"), o=os.path.join(root, "oracle"))
    env = dict(os.environ, MOSP_ENGINE_FLAGS="16")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0 and "LOCAL_OK" in out.stdout, out.stderr[-3000:]


def test_bulk_small_near_lists_overflow_to_far(gpu):
    """The bulk loop with near lists of 1,024 entries per objective: appends
    past them go to the far pile and come back at the next split; results
    stay exact, for an update and from scratch."""
    row, col, w = random_graph(4000, 16000, 3, 1000, 43)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 1500, seed=44, wmax=1000)
    ws = workspace(False, queue_slots=1024)
    res = run_update_device(ws, g, b)
    assert_matches_oracle(res, g, b)
    dg = mb.DeviceGraph.upload(ws, g)
    d = torch.empty(g.n, dtype=torch.int64, device="cuda")
    p = torch.empty(g.n, dtype=torch.int32, device="cuda")
    ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w[:g.m], 3, 50, int(w.max()), d, p)
    ws.close()
    de, pe = orc.dijkstra(row, col, w, 0, 3)
    assert np.array_equal(d.cpu().numpy(), de) and np.array_equal(p.cpu().numpy(), pe)
