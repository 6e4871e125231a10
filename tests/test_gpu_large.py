"""Full-size parity: the road-network update (1404 x 1404 grid, K = 3,
50,000 safe changes) and the power-law update with the distance-only
fallback (R-MAT scale 22, edge factor 16, K = 5, log-uniform weights in
[1, 10^6], Pref = (1..5), 100,000 changes: 30% insertions, 70% deletions
aimed at tree edges, not connectivity-safe). Both run through the whole
host pipeline (mosp_update_host: Step 1 on the GPU, the K updates, the
combined graph, its SSSP and the MOSP costs) and must equal the oracle."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402


@pytest.fixture(scope="module")
def ws():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    w = mb.Workspace(timeout_ms=60000)
    yield w
    w.close()


def initial_trees_gpu(ws, g, K):
    row, col, w = g.arrays()
    dg = mb.DeviceGraph.upload(ws, g)
    d = torch.empty((K, g.n), dtype=torch.int64, device="cuda")
    p = torch.empty((K, g.n), dtype=torch.int32, device="cuda")
    for k in range(K):
        ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w_col(k), 0,
                             mb.default_delta(g.m, g.n, int(w[:, k].astype(np.int64).sum())), int(w[:, k].max()),
                             d[k], p[k])
    return d.cpu().numpy(), p.cpu().numpy()


def check_full(ws, g, batch, K, pref, exp=None):
    d0, p0 = initial_trees_gpu(ws, g, K)
    garr = g.arrays()
    ba = batch.arrays()
    dist, par, cd, cp, costs, _ = ws.update_host(garr, ba, d0, p0, K, 0, pref=pref, costs=True)
    if exp is None:
        exp = orc.expected_update(garr, ba, K, 0, pref)
    for k in range(K):
        assert np.array_equal(dist[k], exp["dist"][k]), k
        assert np.array_equal(par[k], exp["parent"][k]), k
    assert np.array_equal(cd, exp["comb_dist"])
    assert np.array_equal(cp, exp["comb_parent"])
    assert np.array_equal(costs, exp["costs"])
    return exp


def test_road_network_full_size(ws):
    g = mb.HostGraph.grid_road(1404, 1404, 0.70, 0.01, 3, 1, 100, 12345)
    b = mb.HostBatch.generate(g, 50000, 50.0, "uniform", 0, True, 777, 0, 1, 100)
    assert g.n > 1_900_000
    check_full(ws, g, b, 3, None)


def test_power_law_fallback_full_size(ws):
    g = mb.HostGraph.rmat(22, 16, 0.57, 0.19, 0.19, 5, 1, 1_000_000, True, 12345)
    b = mb.HostBatch.generate(g, 100000, 30.0, "targeted", 0, False, 777, 0, 1, 1_000_000)
    assert g.n == 4_194_304 and g.m > 60_000_000
    # (n - 1) * maxWeight does not fit next to 23 parent bits: the
    # distance-only words with lowest-id parent recovery run
    assert mb.choose_packing(g.n, 1_000_000)[0] == 0
    exp = check_full(ws, g, b, 5, [1, 2, 3, 4, 5])
    # the initial trees are the library's own (canonical): the recovery
    # restricted to what the batch reaches gives the same trees
    ws.set_canonical_trees(True)
    try:
        check_full(ws, g, b, 5, [1, 2, 3, 4, 5], exp=exp)
    finally:
        ws.set_canonical_trees(False)
