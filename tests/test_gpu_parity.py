"""GPU parity of the sm_100a engine with the oracle, through the C ABI.

Every result must equal the oracle bit for bit (integer path): the K updated
trees (distances and canonical parents), the combined graph's tree and the
MOSP path costs. Cases follow the reference test suite (src/mospTest.cu):
the worked example, every batch kind on random and grid graphs, the
distance-only fallback (random weights and all-equal weights), the packed
word at its limit, from-scratch searches, determinism and error paths."""
import json
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402
from conftest import grid_graph, random_graph  # noqa: E402
from gpu_util import assert_matches_oracle, dev, initial_trees, run_update_device  # noqa: E402


@pytest.fixture(scope="module")
def ws():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    w = mb.Workspace(timeout_ms=20000)
    yield w
    w.close()


def test_thesis_example(ws, golden_dir):
    spec = json.load(open(os.path.join(golden_dir, "thesis_example.json")))
    edges = sorted(spec["edges"], key=lambda e: e[0])
    n = spec["n"]
    row = np.zeros(n + 1, np.int32)
    for e in edges:
        row[e[0] + 1] += 1
    row = np.cumsum(row).astype(np.int32)
    g = mb.HostGraph.from_arrays(row, [e[1] for e in edges], [e[2:] for e in edges])
    ins, dele = np.array(spec["insert"]), np.array(spec["delete"])
    b = mb.HostBatch.from_arrays(3, ins[:, 0], ins[:, 1], ins[:, 2:], dele[:, 0], dele[:, 1])
    for case in spec["mosp"]:
        res = run_update_device(ws, g, b, pref=case["pref"])
        for k in range(3):
            assert res["parent"][k].tolist() == spec["updated_trees"][k]
        path = [6]
        while res["comb_parent"][path[-1]] >= 0:
            path.append(int(res["comb_parent"][path[-1]]))
        assert path == case["path_to_u7"]
        assert res["costs"][6].tolist() == case["cost_of_u7"]
        assert_matches_oracle(res, g, b, pref=case["pref"])


KINDS = [("uniform-safe", dict(mode="uniform", ins_pct=50, safe=True)),
         ("uniform-unsafe", dict(mode="uniform", ins_pct=50)),
         ("deletions-only", dict(mode="uniform", ins_pct=0)),
         ("insertions-only", dict(mode="uniform", ins_pct=100)),
         ("increase", dict(mode="increase")),
         ("reweight", dict(mode="reweight")),
         ("targeted", dict(mode="targeted", ins_pct=50)),
         ("local", dict(mode="uniform", ins_pct=50, local=4)),
         ("local-reweight", dict(mode="reweight", local=4))]


@pytest.mark.parametrize("kind,opts", KINDS, ids=[k for k, _ in KINDS])
@pytest.mark.parametrize("shape", ["random", "grid"])
def test_batch_kinds(ws, kind, opts, shape):
    for rep in range(2):
        seed = 1000 * rep + len(kind) + (7 if shape == "grid" else 0)
        if shape == "random":
            row, col, w = random_graph(300, 900, 3, 50, seed)
        else:
            row, col, w = grid_graph(24, 18, 3, 50, 0.15, seed)
        g = mb.HostGraph.from_arrays(row, col, w)
        b = mb.HostBatch.generate(g, 80, seed=seed + 1, wmax=50, **opts)
        pref = None if rep == 0 else [1, 2, 2]
        assert_matches_oracle(run_update_device(ws, g, b, pref=pref), g, b, pref=pref)


def test_disconnecting_batch(ws):
    """Delete every in-edge of some vertices: they and what hangs below
    them become unreachable (INF, parent -1)."""
    row, col, w = grid_graph(20, 20, 2, 30, 0.1, 3)
    n = len(row) - 1
    g = mb.HostGraph.from_arrays(row, col, w)
    src = np.repeat(np.arange(n), np.diff(row))
    victims = np.random.default_rng(4).integers(1, n, n // 50)
    sel = np.isin(col, victims)
    b = mb.HostBatch.from_arrays(2, [], [], np.zeros((0, 2)), src[sel], col[sel])
    res = run_update_device(ws, g, b)
    exp = assert_matches_oracle(res, g, b)
    assert (exp["dist"] >= orc.INF // 2).any()


@pytest.mark.parametrize("case", ["c1", "c1_unsafe"])
def test_reference_fixtures_host_abi(ws, golden_dir, case):
    """mosp_update_host (host buffers in and out) reproduces the outputs the
    reference computed for the config-1 fixtures."""
    base = os.path.join(golden_dir, case)
    g = mb.HostGraph.read(os.path.join(base, "graph", "graphCsr"))
    b = mb.HostBatch.read(os.path.join(base, "changes", "insert.txt"), os.path.join(base, "changes", "delete.txt"),
                          g.K, g.n)
    pref_text = open(os.path.join(base, "pref.txt")).read().strip()
    pref = [int(x) for x in pref_text.split(",")] if pref_text else None
    d0 = np.empty((g.K, g.n), np.int64)
    p0 = np.empty((g.K, g.n), np.int32)
    for k in range(g.K):
        ob = os.path.join(base, "init", f"obj{k}")
        mb.check(mb.lib().mosp_read_tree(os.path.join(ob, "distancesOriginal.txt").encode(),
                                         os.path.join(ob, "SSSPTreeOriginal.txt").encode(), g.n,
                                         d0[k].ctypes.data, p0[k].ctypes.data))
    dist, par, cd, cp, costs, _ = ws.update_host(g.arrays(), b.arrays(), d0, p0, g.K, 0, pref)
    for k in range(g.K):
        ob = os.path.join(base, "expected", f"obj{k}")
        ed = np.empty(g.n, np.int64)
        ep = np.empty(g.n, np.int32)
        mb.check(mb.lib().mosp_read_tree(os.path.join(ob, "distancesUpdated.txt").encode(),
                                         os.path.join(ob, "SSSPTreeUpdated.txt").encode(), g.n,
                                         ed.ctypes.data, ep.ctypes.data))
        assert np.array_equal(dist[k], ed) and np.array_equal(par[k], ep)
    cb = os.path.join(base, "expected", "combinedGraph")
    ed = np.empty(g.n, np.int64)
    ep = np.empty(g.n, np.int32)
    mb.check(mb.lib().mosp_read_tree(os.path.join(cb, "distancesCsr.txt").encode(),
                                     os.path.join(cb, "SSSPTreeCsr.txt").encode(), g.n, ed.ctypes.data,
                                     ep.ctypes.data))
    assert np.array_equal(cd, ed) and np.array_equal(cp, ep)
    rows = [[orc.INF if x == "INF" else int(x) for x in line.split()[1:]]
            for line in open(os.path.join(cb, "mospCosts.txt"))]
    assert np.array_equal(costs, np.array(rows, np.int64))


def test_fused_equals_single_objective(ws):
    """K objectives in one launch == K single-objective launches."""
    row, col, w = grid_graph(30, 25, 4, 60, 0.2, 8)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 150, seed=9, wmax=60)
    upd = mb.apply_batch(g, b)
    ba = b.arrays()
    dg = mb.DeviceGraph.upload(ws, upd)
    d0, p0 = initial_trees(g.arrays(), 4)
    ch = mb.changed_lists(ba, 4)
    heads = dev(ba["ins_to"])
    maxw = [100] * 4
    deltas = [50] * 4
    dd = [dev(d0[k].copy()) for k in range(4)]
    pp = [dev(p0[k].copy()) for k in range(4)]
    cfs = [dev(c[0]) for c in ch]
    cts = [dev(c[1]) for c in ch]
    ws.sosp_update_multi(upd.n, upd.m, 4, dg.out_row, dg.out_col, [dg.out_w_col(k) for k in range(4)], dg.in_row,
                         dg.in_col, [dg.in_w_col(k) for k in range(4)], cfs, cts, [len(c[0]) for c in ch], heads,
                         len(ba["ins_to"]), 0, deltas, maxw, dd, pp)
    for k in range(4):
        d1 = dev(d0[k].copy())
        p1 = dev(p0[k].copy())
        ws.sosp_update(upd.n, upd.m, dg.out_row, dg.out_col, dg.out_w_col(k), dg.in_row, dg.in_col, dg.in_w_col(k),
                       cfs[k], cts[k], len(ch[k][0]), heads, len(ba["ins_to"]), 0, 37, 100, d1, p1)
        assert torch.equal(d1, dd[k]) and torch.equal(p1, pp[k])


def test_from_scratch_equals_dijkstra(ws):
    for seed, (row, col, w) in enumerate([grid_graph(40, 40, 1, 100, 0.25, 1), random_graph(2000, 8000, 1, 1000, 2)]):
        g = mb.HostGraph.from_arrays(row, col, w)
        dg = mb.DeviceGraph.upload(ws, g)
        d = torch.empty(g.n, dtype=torch.int64, device="cuda")
        p = torch.empty(g.n, dtype=torch.int32, device="cuda")
        for delta in (1, 50, 10 ** 9):
            ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w, 0, delta, int(w.max()), d, p)
            de, pe = orc.dijkstra(row, col, w, 0, 0)
            assert np.array_equal(d.cpu().numpy(), de) and np.array_equal(p.cpu().numpy(), pe)


@pytest.mark.parametrize("ties", [False, True])
def test_distance_only_fallback(ws, ties):
    """(n - 1) * maxWeight does not fit next to the parent ids: distances
    only, then lowest-id parent recovery (reference src/mospTest.cu:601-700).
    With all weights 2e9 most vertices have two tight parents."""
    W = 2_000_000_000
    # 320 x 320: 17 parent bits leave 47 for distances < (n - 1) * maxWeight
    row, col, w = grid_graph(320, 320, 2, W if ties else 2_147_483_647, 0.1, 5, wmin=W if ties else 1)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 2000, seed=6, wmin=W if ties else 1, wmax=W if ties else 2_147_483_647)
    res = run_update_device(ws, g, b)
    assert all(s.packed_parents == 0 for s in res["stats"])
    assert_matches_oracle(res, g, b)


def test_packing_boundary(ws):
    """n = 2^17 - 1 path with W = 2^30 + 2^14: (n-1)W still fits the packed
    word but a candidate n*W does not and must be dropped, in the pull pass,
    the push loop and from scratch (reference src/mospTest.cu:723-815)."""
    n = (1 << 17) - 1
    W = (1 << 30) + (1 << 14)
    for name, back, ins in [("pull", False, (n - 1, 1, W)), ("push", True, (n - 2, n - 1, W - 1)),
                            ("scratch", True, None)]:
        row = np.arange(n + 1, dtype=np.int32)
        row[n] = n - 1 + (1 if back else 0)
        col = np.arange(1, n + 1, dtype=np.int32)
        col[n - 1] = 1
        col = col[: row[n]]
        w = np.full((len(col), 1), W, np.int32)
        g = mb.HostGraph.from_arrays(row, col, w)
        d0, p0 = orc.dijkstra(row, col, w, 0, 0)
        if ins is None:
            dg = mb.DeviceGraph.upload(ws, g)
            d = torch.empty(n, dtype=torch.int64, device="cuda")
            p = torch.empty(n, dtype=torch.int32, device="cuda")
            st = ws.sosp_from_scratch(n, g.m, dg.out_row, dg.out_col, dg.out_w, 0, 10 ** 12, W, d, p)
            exp_d, exp_p = d0, p0
        else:
            b = mb.HostBatch.from_arrays(1, [ins[0]], [ins[1]], [[ins[2]]], [], [])
            upd = mb.apply_batch(g, b)
            ur, uc, uw = upd.arrays()
            dg = mb.DeviceGraph.upload(ws, upd)
            d, p = dev(d0), dev(p0)
            none = torch.zeros(1, dtype=torch.int32, device="cuda")
            st = ws.sosp_update(n, upd.m, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w, none, none,
                                0, dev(np.array([ins[1]], np.int32)), 1, 0, 10 ** 12, W, d, p)
            exp_d, exp_p = orc.dijkstra(ur, uc, uw, 0, 0)
        assert st.packed_parents == 1, name
        assert np.array_equal(d.cpu().numpy(), exp_d), name
        assert np.array_equal(p.cpu().numpy(), exp_p), name


def test_rmat_hubs(ws):
    """Power-law graph: rows far longer than a warp are expanded by the
    whole warp (push, pull and parent recovery)."""
    g = mb.HostGraph.rmat(12, 16, 0.57, 0.19, 0.19, 3, 1, 1_000_000, True, 42)
    b = mb.HostBatch.generate(g, 2000, ins_pct=30, seed=43, wmax=1_000_000)
    assert_matches_oracle(run_update_device(ws, g, b, pref=[1, 2, 3]), g, b, pref=[1, 2, 3])


def test_deterministic_across_launch_shapes():
    """The fixed point does not depend on the grid size, the bucket width or
    the run: identical outputs."""
    row, col, w = grid_graph(50, 40, 3, 100, 0.3, 12)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 500, seed=13, wmax=100)
    outs = []
    for ctas, delta in [(0, None), (1, 1), (1, 10 ** 6), (0, 7), (0, None)]:
        w_ = mb.Workspace(ctas_per_sm=ctas)
        res = run_update_device(w_, g, b, delta=delta)
        outs.append(res)
        w_.close()
    for r in outs[1:]:
        for key in ("dist", "parent", "comb_dist", "comb_parent", "costs"):
            assert np.array_equal(r[key], outs[0][key]), key


def test_overflow_and_invalid_inputs(ws):
    row, col, w = grid_graph(10, 10, 1, 10, 0.0, 1)
    g = mb.HostGraph.from_arrays(row, col, w)
    dg = mb.DeviceGraph.upload(ws, g)
    d0, p0 = orc.dijkstra(row, col, w, 0, 0)
    none = torch.zeros(1, dtype=torch.int32, device="cuda")
    bad = d0.copy()
    bad[5] = 10 ** 6  # larger than (n - 1) * maxWeight
    with pytest.raises(mb.MospError) as e:
        ws.sosp_update(g.n, g.m, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w, none, none, 0,
                       none, 0, 0, 10, 10, dev(bad), dev(p0))
    assert e.value.status == mb.ERR_OVERFLOW
    badp = p0.copy()
    badp[7] = g.n + 3  # parent out of range
    with pytest.raises(mb.MospError) as e:
        ws.sosp_update(g.n, g.m, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w, none, none, 0,
                       none, 0, 0, 10, 10, dev(d0), dev(badp))
    assert e.value.status == mb.ERR_INVALID
    # the workspace stays usable
    d, p = dev(d0), dev(p0)
    ws.sosp_update(g.n, g.m, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w, none, none, 0, none,
                   0, 0, 10, 10, d, p)
    assert np.array_equal(d.cpu().numpy(), d0)


def test_barrier_wait_is_bounded(ws):
    """A grid barrier that one CTA never reaches ends with a timeout status
    after its bound instead of hanging; the workspace stays usable."""
    assert ws.barrier_timeout_probe(200) == mb.ERR_TIMEOUT
    row, col, w = grid_graph(8, 8, 1, 10, 0.0, 2)
    g = mb.HostGraph.from_arrays(row, col, w)
    dg = mb.DeviceGraph.upload(ws, g)
    d = torch.empty(g.n, dtype=torch.int64, device="cuda")
    p = torch.empty(g.n, dtype=torch.int32, device="cuda")
    ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w, 0, 5, 10, d, p)
    de, pe = orc.dijkstra(row, col, w, 0, 0)
    assert np.array_equal(d.cpu().numpy(), de) and np.array_equal(p.cpu().numpy(), pe)


def test_malformed_device_graph_rejected(ws):
    row = np.array([0, 2, 3], np.int32)
    col = np.array([1, 5, 0], np.int32)  # 5 is out of range
    w = np.ones((3, 1), np.int32)
    t = lambda a: dev(a)  # noqa: E731
    out_w = torch.empty(3, dtype=torch.int32, device="cuda")
    in_row = torch.empty(3, dtype=torch.int32, device="cuda")
    in_col = torch.empty(3, dtype=torch.int32, device="cuda")
    in_w = torch.empty(3, dtype=torch.int32, device="cuda")
    with pytest.raises(mb.MospError) as e:
        ws.build_device_graph(2, 3, 1, t(row), t(col), t(w.reshape(-1)), out_w, in_row, in_col, in_w)
    assert e.value.status == mb.ERR_INVALID
