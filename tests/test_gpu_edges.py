"""Edge cases through the C ABI, against the oracle: the largest fused
objective count (K = 32, the reference's limit), an empty batch, a graph of
one vertex, a batch whose deletions and re-insertions hit the same edges,
a source other than vertex 0, and the whole host pipeline
(mosp_update_host) on the same cases."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402
from conftest import grid_graph, random_graph  # noqa: E402
from gpu_util import assert_matches_oracle, initial_trees, run_update_device  # noqa: E402


@pytest.fixture(scope="module")
def ws():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    w = mb.Workspace(timeout_ms=20000)
    yield w
    w.close()


def host_pipeline(ws, g, b, K, source=0, pref=None):
    ga, ba = g.arrays(), b.arrays()
    d0, p0 = initial_trees(ga, K, source)
    dist, par, cd, cp, costs, _ = ws.update_host(ga, ba, d0, p0, K, source, pref=pref, costs=True)
    exp = orc.expected_update(ga, ba, K, source, pref)
    assert np.array_equal(dist, exp["dist"]) and np.array_equal(par, exp["parent"])
    assert np.array_equal(cd, exp["comb_dist"]) and np.array_equal(cp, exp["comb_parent"])
    assert np.array_equal(costs, exp["costs"])


def test_thirty_two_objectives(ws):
    row, col, w = grid_graph(30, 25, 32, 100, 0.2, 71)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 120, seed=72, wmax=100)
    assert_matches_oracle(run_update_device(ws, g, b), g, b)
    host_pipeline(ws, g, b, 32)


def test_empty_batch(ws):
    row, col, w = random_graph(500, 1500, 3, 100, 73)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.from_arrays(3, np.zeros(0), np.zeros(0), np.zeros((0, 3)), np.zeros(0), np.zeros(0))
    assert_matches_oracle(run_update_device(ws, g, b), g, b)
    host_pipeline(ws, g, b, 3)


def test_single_vertex(ws):
    row, col, w = np.array([0, 0], np.int32), np.zeros(0, np.int32), np.zeros((0, 2), np.int32)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.from_arrays(2, np.zeros(0), np.zeros(0), np.zeros((0, 2)), np.zeros(0), np.zeros(0))
    host_pipeline(ws, g, b, 2)


def test_delete_and_reinsert_same_edges(ws):
    row, col, w = grid_graph(40, 40, 3, 100, 0.1, 74)
    src = np.repeat(np.arange(len(row) - 1), np.diff(row))
    rng = np.random.default_rng(75)
    pick = rng.choice(len(col), 300, replace=False)
    u, v = src[pick].astype(np.int32), col[pick].astype(np.int32)
    # delete every picked edge, re-insert half of them heavier, half lighter
    ins_w = np.where(rng.random((300, 3)) < 0.5, w[pick] + 50, np.maximum(1, w[pick] - 10)).astype(np.int32)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.from_arrays(3, u, v, ins_w, u, v)
    assert_matches_oracle(run_update_device(ws, g, b), g, b)
    host_pipeline(ws, g, b, 3)


def test_other_source(ws):
    row, col, w = grid_graph(35, 30, 3, 100, 0.2, 76)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 200, seed=77, wmax=100, source=517)
    assert_matches_oracle(run_update_device(ws, g, b, source=517), g, b, source=517)
    host_pipeline(ws, g, b, 3, source=517, pref=[3, 1, 2])
