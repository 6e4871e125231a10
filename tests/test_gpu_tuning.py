"""The autotuner and CUDA-graph replay of mosp_update_device: neither may
change a result. The autotuner must leave the trees as it found them and
its widths must reproduce the oracle; graph replays must reproduce it on
every call, and a parameter change must re-capture."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402
from conftest import grid_graph  # noqa: E402
from gpu_util import dev, initial_trees  # noqa: E402


@pytest.fixture(scope="module")
def ws():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    w = mb.Workspace(timeout_ms=20000)
    yield w
    w.close()


@pytest.fixture(scope="module")
def case():
    K = 3
    g0 = grid_graph(160, 160, K, 100, 0.25, 51)
    g = mb.HostGraph.from_arrays(*g0)
    b = mb.HostBatch.generate(g, 3000, 50.0, "uniform", 0, False, 52, 0, 1, 100)
    upd = mb.apply_batch(g, b)
    ba = b.arrays()
    exp = orc.expected_update(g0, ba, K, 0)
    d0, p0 = initial_trees(g0, K)
    return K, g0, g, b, upd, ba, exp, d0, p0


def args_for(ws, case):
    K, g0, g, b, upd, ba, exp, d0, p0 = case
    dg = mb.DeviceGraph.upload(ws, upd)
    ch = mb.changed_lists(ba, K)
    cf = dev(np.concatenate([c[0] for c in ch]).astype(np.int32))
    ct = dev(np.concatenate([c[1] for c in ch]).astype(np.int32))
    off = np.concatenate([[0], np.cumsum([len(c[0]) for c in ch])]).astype(np.int32)
    w = g0[2]
    maxw = [max(int(w[:, k].max()), int(ba["ins_w"][:, k].max())) for k in range(K)]
    deltas = [mb.default_delta(g.m, g.n, int(w[:, k].sum())) for k in range(K)]
    heads = dev(ba["ins_to"].astype(np.int32))
    return dg, cf, ct, off, heads, maxw, deltas


def run(ws, case, dg, cf, ct, off, heads, maxw, deltas, dist, par, cd, cp):
    K, _, _, _, upd, ba, _, _, _ = case
    return ws.update_device(upd.n, upd.m, K, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w, cf,
                            ct, off, heads, len(ba["ins_to"]), 0, deltas, maxw, None, dist, par, cd, cp)


def check(exp, dist, par, cd, cp):
    assert np.array_equal(dist.cpu().numpy(), exp["dist"])
    assert np.array_equal(par.cpu().numpy(), exp["parent"])
    assert np.array_equal(cd.cpu().numpy(), exp["comb_dist"])
    assert np.array_equal(cp.cpu().numpy(), exp["comb_parent"])


def test_autotuner_keeps_trees_and_results(ws, case):
    K, g0, g, b, upd, ba, exp, d0, p0 = case
    dg, cf, ct, off, heads, maxw, deltas = args_for(ws, case)
    dist, par = dev(d0), dev(p0)
    cd = torch.empty(upd.n, dtype=torch.int64, device="cuda")
    cp = torch.empty(upd.n, dtype=torch.int32, device="cuda")
    best, comb, ms, rounds = ws.autotune_update(upd.n, upd.m, K, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col,
                                        dg.in_w, cf, ct, off, heads, len(ba["ins_to"]), 0, deltas, maxw, None,
                                        dist, par, cd, cp)
    assert len(best) == K and all(x >= 1 for x in best) and comb >= 1 and ms > 0
    assert np.array_equal(dist.cpu().numpy(), d0) and np.array_equal(par.cpu().numpy(), p0)
    assert all(0 <= r <= 4 for r in rounds)
    ws.set_combined_delta(comb)
    ws.set_local_rounds(*rounds)
    try:
        _, cst = run(ws, case, dg, cf, ct, off, heads, maxw, best, dist, par, cd, cp)
        assert cst.delta == comb
        check(exp, dist, par, cd, cp)
    finally:
        ws.set_combined_delta(0)
        ws.set_local_rounds(0, 2)


@pytest.mark.parametrize("rounds", [(0, 0), (1, 3), (4, 6)])
def test_local_rounds_keep_results(ws, case, rounds):
    K, g0, g, b, upd, ba, exp, d0, p0 = case
    dg, cf, ct, off, heads, maxw, deltas = args_for(ws, case)
    dist, par = dev(d0), dev(p0)
    cd = torch.empty(upd.n, dtype=torch.int64, device="cuda")
    cp = torch.empty(upd.n, dtype=torch.int32, device="cuda")
    ws.set_local_rounds(*rounds)
    try:
        run(ws, case, dg, cf, ct, off, heads, maxw, deltas, dist, par, cd, cp)
        check(exp, dist, par, cd, cp)
    finally:
        ws.set_local_rounds(0, 2)


def test_graph_replay(ws, case):
    K, g0, g, b, upd, ba, exp, d0, p0 = case
    dg, cf, ct, off, heads, maxw, deltas = args_for(ws, case)
    dist, par = dev(d0), dev(p0)
    cd = torch.empty(upd.n, dtype=torch.int64, device="cuda")
    cp = torch.empty(upd.n, dtype=torch.int32, device="cuda")
    ws.use_graphs(True)
    try:
        start = ws.graph_launches()
        for rep in range(3):
            dist.copy_(dev(d0))
            par.copy_(dev(p0))
            run(ws, case, dg, cf, ct, off, heads, maxw, deltas, dist, par, cd, cp)
            check(exp, dist, par, cd, cp)
        # another width: new parameters, captured again, same results
        dist.copy_(dev(d0))
        par.copy_(dev(p0))
        run(ws, case, dg, cf, ct, off, heads, maxw, [2 * d for d in deltas], dist, par, cd, cp)
        check(exp, dist, par, cd, cp)
        assert ws.graph_launches() - start == 4
    finally:
        ws.use_graphs(False)


@pytest.mark.parametrize("loop", [True, False])
@pytest.mark.parametrize("ctas,hub", [(0, 0), (37, 0), (74, 64), (1, 0), (0, 1 << 20)])
def test_grid_and_hub_threshold_keep_results(case, loop, ctas, hub):
    """Every engine knob the autotuner searches (near-far loop, grid CTAs,
    hub-row threshold, incl. a grid of one CTA and a threshold so low that
    every longer row goes to the CTA-wide path) leaves the results equal to
    the oracle."""
    K, g0, g, b, upd, ba, exp, d0, p0 = case
    w = mb.Workspace(timeout_ms=20000)
    try:
        w.set_async(loop)
        w.set_grid(ctas, hub)
        dg, cf, ct, off, heads, maxw, deltas = args_for(w, case)
        dist, par = dev(d0), dev(p0)
        cd = torch.empty(upd.n, dtype=torch.int64, device="cuda")
        cp = torch.empty(upd.n, dtype=torch.int32, device="cuda")
        run(w, case, dg, cf, ct, off, heads, maxw, deltas, dist, par, cd, cp)
        check(exp, dist, par, cd, cp)
        got = w.tuning()
        assert got[2] == loop and (ctas == 0 or got[0] == ctas)
    finally:
        w.close()


def test_autotuner_leaves_engine_settings_consistent(case):
    """After the autotuner the workspace holds its choice of loop, grid and
    hub threshold, and an update with them reproduces the oracle."""
    K, g0, g, b, upd, ba, exp, d0, p0 = case
    w = mb.Workspace(timeout_ms=20000)
    try:
        dg, cf, ct, off, heads, maxw, deltas = args_for(w, case)
        dist, par = dev(d0), dev(p0)
        cd = torch.empty(upd.n, dtype=torch.int64, device="cuda")
        cp = torch.empty(upd.n, dtype=torch.int32, device="cuda")
        best, comb, _, rounds = w.autotune_update(upd.n, upd.m, K, dg.out_row, dg.out_col, dg.out_w, dg.in_row,
                                                  dg.in_col, dg.in_w, cf, ct, off, heads, len(ba["ins_to"]), 0,
                                                  deltas, maxw, None, dist, par, cd, cp)
        ctas, hub, loop = w.tuning()
        assert ctas >= 1 and hub >= 64
        w.set_combined_delta(comb)
        w.set_local_rounds(*rounds)
        run(w, case, dg, cf, ct, off, heads, maxw, best, dist, par, cd, cp)
        check(exp, dist, par, cd, cp)
    finally:
        w.close()
