"""Batched instances (many graphs as one disjoint union, one launch per
engine step): every instance's trees, combined tree and MOSP costs must
equal the oracle's for that instance alone."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402
from conftest import grid_graph, random_graph  # noqa: E402
from gpu_util import dev  # noqa: E402
from mosp_b200 import batched as bt  # noqa: E402


@pytest.fixture(scope="module")
def ws():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    w = mb.Workspace(timeout_ms=20000)
    yield w
    w.close()


def instances(count, seed, K=3):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        if i % 3 == 2:
            g = random_graph(int(rng.integers(200, 3000)), int(rng.integers(500, 9000)), K, 100, seed * 1000 + i)
        else:
            side = int(rng.integers(8, 60))
            g = grid_graph(side, side + int(rng.integers(0, 9)), K, 100, 0.2, seed * 1000 + i)
        hg = mb.HostGraph.from_arrays(*g)
        mode = ["uniform", "targeted", "increase", "reweight"][i % 4]
        count_changes = max(2, int(len(g[1]) * rng.uniform(0.01, 0.10)))
        try:
            b = mb.HostBatch.generate(hg, count_changes, 50.0, mode, 0, False, seed * 1000 + i, 0, 1, 100)
        except mb.MospError:  # a mode without candidate edges on this graph
            b = mb.HostBatch.generate(hg, count_changes, 50.0, "uniform", 0, False, seed * 1000 + i, 0, 1, 100)
        ba = b.arrays()
        out.append((g, {k: ba[k] for k in ("ins_from", "ins_to", "ins_w", "del_from", "del_to")}))
    return out


def run_union(ws, insts, K=3):
    graphs = [g for g, _ in insts]
    row, col, w, off = bt.union_graphs(graphs)
    ub = bt.union_batches([b for _, b in insts], off)
    roots = off[:-1].astype(np.int32)
    init = [[orc.dijkstra(*g, k, 0) for k in range(K)] for g in graphs]
    d0, p0 = bt.union_trees([np.stack([x[0] for x in t]) for t in init],
                            [np.stack([x[1] for x in t]) for t in init], off)
    g = mb.HostGraph.from_arrays(row, col, w)
    batch = mb.HostBatch.from_arrays(K, ub["ins_from"], ub["ins_to"], ub["ins_w"], ub["del_from"], ub["del_to"])
    upd = mb.apply_batch(g, batch)
    ba = batch.arrays()
    dg = mb.DeviceGraph.upload(ws, upd)
    n, m = upd.n, upd.m
    ch = mb.changed_lists(ba, K)
    cf = dev(np.concatenate([c[0] for c in ch]).astype(np.int32))
    ct = dev(np.concatenate([c[1] for c in ch]).astype(np.int32))
    offs = np.concatenate([[0], np.cumsum([len(c[0]) for c in ch])]).astype(np.int32)
    maxw = [max(int(w[:, k].max()), int(ba["ins_w"][:, k].max()) if len(ba["ins_w"]) else 1) for k in range(K)]
    deltas = [mb.default_delta(g.m, g.n, int(w[:, k].sum())) for k in range(K)]
    dist, par = dev(d0), dev(p0)
    cd = torch.empty(n, dtype=torch.int64, device="cuda")
    cp = torch.empty(n, dtype=torch.int32, device="cuda")
    heads = dev(ba["ins_to"].astype(np.int32)) if len(ba["ins_to"]) else torch.zeros(1, dtype=torch.int32,
                                                                                    device="cuda")
    ws.set_sources(roots)
    try:
        stats, cst = ws.update_device(n, m, K, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w,
                                      cf, ct, offs, heads, len(ba["ins_to"]), int(roots[0]), deltas, maxw, None,
                                      dist, par, cd, cp)
        costs = torch.empty(n * K, dtype=torch.int64, device="cuda")
        ws.path_costs(n, m, K, dg.out_row, dg.out_col, dg.out_w, cp, int(roots[0]), costs)
    finally:
        ws.set_sources([])
    return off, dist.cpu().numpy(), par.cpu().numpy(), cd.cpu().numpy(), cp.cpu().numpy(), \
        costs.cpu().numpy().reshape(n, K), cst


@pytest.mark.parametrize("count,seed", [(2, 41), (12, 42), (40, 43)])
def test_batched_update_equals_each_instance(ws, count, seed):
    check_each_instance(ws, instances(count, seed))


def test_batched_workload_full_size(ws):
    """The benchmark's batched workload at full size: 256 grid-road
    instances of 1,000 to 200,000 vertices, each with its own batch of 1-10%
    of its edges in one of four modes, in one union; every instance equals
    the oracle run on that instance alone."""
    import bench
    insts = []
    for g, b, _ in bench.make_batched_workload(256):
        ba = b.arrays()
        insts.append((g.arrays(), {k: ba[k] for k in ("ins_from", "ins_to", "ins_w", "del_from", "del_to")}))
    assert len(insts) == 256
    check_each_instance(ws, insts)


def check_each_instance(ws, insts):
    off, dist, par, cd, cp, costs, cst = run_union(ws, insts)
    edges = 0
    for i, (g, b) in enumerate(insts):
        exp = orc.expected_update(g, b, 3, 0)
        assert np.array_equal(bt.split_vertices(dist, off, i), exp["dist"]), i
        assert np.array_equal(bt.split_vertices(par, off, i, parents=True), exp["parent"]), i
        assert np.array_equal(bt.split_vertices(cd, off, i), exp["comb_dist"]), i
        assert np.array_equal(bt.split_vertices(cp, off, i, parents=True), exp["comb_parent"]), i
        assert np.array_equal(costs[off[i]:off[i + 1]], exp["costs"]), i
        edges += exp["comb_edges"]
    assert cst.edges == edges


def test_batched_from_scratch(ws):
    graphs = [g for g, _ in instances(10, 44)]
    row, col, w, off = bt.union_graphs(graphs)
    g = mb.HostGraph.from_arrays(row, col, w)
    dg = mb.DeviceGraph.upload(ws, g)
    d = torch.empty(g.n, dtype=torch.int64, device="cuda")
    p = torch.empty(g.n, dtype=torch.int32, device="cuda")
    ws.set_sources(off[:-1])
    try:
        for k in range(3):
            ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w_col(k), 0, 60, int(w.max()), d, p)
            dd, pp = d.cpu().numpy(), p.cpu().numpy()
            for i, gi in enumerate(graphs):
                de, pe = orc.dijkstra(*gi, k, 0)
                assert np.array_equal(bt.split_vertices(dd, off, i), de)
                assert np.array_equal(bt.split_vertices(pp, off, i, parents=True), pe)
    finally:
        ws.set_sources([])


def test_roots_are_checked(ws):
    graphs = [g for g, _ in instances(3, 45)]
    row, col, w, off = bt.union_graphs(graphs)
    g = mb.HostGraph.from_arrays(row, col, w)
    dg = mb.DeviceGraph.upload(ws, g)
    d = torch.empty(g.n, dtype=torch.int64, device="cuda")
    p = torch.empty(g.n, dtype=torch.int32, device="cuda")
    with pytest.raises(mb.MospError):
        ws.set_sources([0, 0])
    ws.set_sources(off[:-1])
    try:
        with pytest.raises(mb.MospError):
            ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w_col(0), 1, 60, int(w.max()), d, p)
    finally:
        ws.set_sources([])
    # single-source runs again
    ws.sosp_from_scratch(g.n, g.m, dg.out_row, dg.out_col, dg.out_w_col(0), 0, 60, int(w.max()), d, p)
    de, pe = orc.dijkstra(row, col, w, 0, 0)
    assert np.array_equal(d.cpu().numpy(), de) and np.array_equal(p.cpu().numpy(), pe)
