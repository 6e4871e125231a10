"""The oracle (C restatement) pinned against the reference: the worked
example of the reference test suite (golden vectors), the committed
config-1 fixtures made by the reference's own code, and - where the
reference was compiled into oracle/_ref - the reference functions directly
on seeded inputs. CPU only."""
import json
import os

import numpy as np
import pytest

import oracle as orc
from conftest import grid_graph, random_graph

needs_ref = pytest.mark.skipif(not orc.have_ref(), reason="oracle/_ref not built (reference sources absent)")


def thesis_graph(golden_dir):
    spec = json.load(open(os.path.join(golden_dir, "thesis_example.json")))
    edges = sorted(spec["edges"], key=lambda e: e[0])  # stable: row order
    n, K = spec["n"], spec["K"]
    row = np.zeros(n + 1, np.int32)
    for e in edges:
        row[e[0] + 1] += 1
    row = np.cumsum(row).astype(np.int32)
    col = np.array([e[1] for e in edges], np.int32)
    w = np.array([e[2:] for e in edges], np.int32)
    ins = np.array(spec["insert"], np.int32)
    dele = np.array(spec["delete"], np.int32)
    batch = {"ins_from": ins[:, 0], "ins_to": ins[:, 1], "ins_w": ins[:, 2:], "del_from": dele[:, 0],
             "del_to": dele[:, 1]}
    return spec, (row, col, w), batch


def test_thesis_trees_paths_costs(golden_dir):
    spec, g, batch = thesis_graph(golden_dir)
    n, K = spec["n"], spec["K"]
    exp = orc.expected_update(g, batch, K)
    for k in range(K):
        assert exp["parent"][k].tolist() == spec["updated_trees"][k]
    for case in spec["mosp"]:
        crow, ccol, cw = orc.combined_graph(exp["parent"], n, K, 0, case["pref"])
        _, cp = orc.dijkstra(crow, ccol, cw, 0, 0)
        path = [6]
        while cp[path[-1]] >= 0:
            path.append(int(cp[path[-1]]))
        assert path == case["path_to_u7"]
        costs = orc.path_costs(*exp["updated"], cp, 0)
        assert costs[6].tolist() == case["cost_of_u7"]


def test_thesis_sequential_update(golden_dir):
    """The sequential update restatement reproduces the updated trees."""
    spec, (row, col, w), batch = thesis_graph(golden_dir)
    urow, ucol, uw, mask = orc.apply_batch(row, col, w, batch["ins_from"], batch["ins_to"],
                                           batch["ins_w"], batch["del_from"], batch["del_to"])
    for k in range(spec["K"]):
        d0, p0 = orc.dijkstra(row, col, w, k, 0)
        sel = ((mask >> k) & 1).astype(bool)
        cf = np.concatenate([batch["del_from"], batch["ins_from"][sel]])
        ct = np.concatenate([batch["del_to"], batch["ins_to"][sel]])
        d, p = orc.sequential_update(urow, ucol, uw, k, 0, cf, ct, batch["ins_to"], d0, p0)
        assert p.tolist() == spec["updated_trees"][k]
        de, _ = orc.dijkstra(urow, ucol, uw, k, 0)
        assert d.tolist() == de.tolist()


def read_pairs(path, n):
    out = np.full(n, -7, np.int64)
    for line in open(path):
        v, x = line.split()
        out[int(v)] = orc.INF if x == "INF" else int(x)
    return out


@pytest.mark.parametrize("case", ["c1", "c1_unsafe"])
def test_fixture_from_reference(golden_dir, case):
    """The oracle reproduces the committed outputs of the reference."""
    import mosp_b200 as mb
    base = os.path.join(golden_dir, case)
    g = mb.HostGraph.read(os.path.join(base, "graph", "graphCsr"))
    b = mb.HostBatch.read(os.path.join(base, "changes", "insert.txt"), os.path.join(base, "changes", "delete.txt"),
                          g.K, g.n)
    pref_text = open(os.path.join(base, "pref.txt")).read().strip()
    pref = [int(x) for x in pref_text.split(",")] if pref_text else None
    exp = orc.expected_update(g.arrays(), b.arrays(), g.K, 0, pref)
    for k in range(g.K):
        ob = os.path.join(base, "expected", f"obj{k}")
        assert np.array_equal(read_pairs(os.path.join(ob, "distancesUpdated.txt"), g.n), exp["dist"][k])
        assert np.array_equal(read_pairs(os.path.join(ob, "SSSPTreeUpdated.txt"), g.n), exp["parent"][k])
    cb = os.path.join(base, "expected", "combinedGraph")
    assert np.array_equal(read_pairs(os.path.join(cb, "distancesCsr.txt"), g.n), exp["comb_dist"])
    assert np.array_equal(read_pairs(os.path.join(cb, "SSSPTreeCsr.txt"), g.n), exp["comb_parent"])
    costs = [[orc.INF if x == "INF" else int(x) for x in line.split()[1:]]
             for line in open(os.path.join(cb, "mospCosts.txt"))]
    assert np.array_equal(np.array(costs, np.int64), exp["costs"])


def test_sequential_update_matches_dijkstra_random():
    """Sequential update (restated) == Dijkstra of the updated graph on
    random graphs and mixed batches, including disconnecting ones."""
    rng = np.random.default_rng(5)
    for rep in range(30):
        n = int(rng.integers(5, 60))
        row, col, w = random_graph(n, int(rng.integers(0, 3 * n)), 2, 20, 100 + rep)
        m = len(col)
        dels = rng.integers(0, m, int(rng.integers(0, m // 2 + 1)))
        ins_n = int(rng.integers(0, n))
        ins_from = rng.integers(0, n, ins_n)
        ins_to = rng.integers(0, n, ins_n)
        keep = ins_from != ins_to
        ins_from, ins_to = ins_from[keep], ins_to[keep]
        ins_w = rng.integers(1, 21, (len(ins_from), 2))
        src_of = np.repeat(np.arange(n), np.diff(row))
        urow, ucol, uw, mask = orc.apply_batch(row, col, w, ins_from, ins_to, ins_w, src_of[dels], col[dels])
        for k in range(2):
            d0, p0 = orc.dijkstra(row, col, w, k, 0)
            sel = ((mask >> k) & 1).astype(bool)
            cf = np.concatenate([src_of[dels], ins_from[sel]])
            ct = np.concatenate([col[dels], ins_to[sel]])
            d, p = orc.sequential_update(urow, ucol, uw, k, 0, cf, ct, ins_to, d0, p0)
            de, pe = orc.dijkstra(urow, ucol, uw, k, 0)
            assert np.array_equal(d, de) and np.array_equal(p, pe)


@needs_ref
def test_oracle_equals_reference_code():
    """Dijkstra, batch application, combined graph and costs of the oracle
    equal the reference's own functions (oracle/_ref/libref_cpu.so)."""
    for seed in range(6):
        row, col, w = grid_graph(9, 7, 3, 5 if seed % 2 else 60, 0.15, seed)
        n = len(row) - 1
        batch = orc.ref_generate_changes(row, col, w, 40, 50.0, seed % 4, 0, seed % 2 == 0, 11 + seed, 0, 1,
                                         5 if seed % 2 else 60)
        a = orc.apply_batch(row, col, w, batch["ins_from"], batch["ins_to"], batch["ins_w"], batch["del_from"],
                            batch["del_to"])
        r = orc.ref_apply_batch(row, col, w, batch["ins_from"], batch["ins_to"], batch["ins_w"],
                                batch["del_from"], batch["del_to"])
        for x, y in zip(a, r):
            assert np.array_equal(x, y)
        urow, ucol, uw, _ = a
        parents = []
        for k in range(3):
            do, po = orc.dijkstra(urow, ucol, uw, k, 0)
            dr, pr = orc.ref_dijkstra(urow, ucol, uw, k, 0)
            assert np.array_equal(do, dr) and np.array_equal(po, pr)
            parents.append(po)
        pref = [1, 2, 3] if seed % 3 == 0 else None
        crow, ccol, cw = orc.combined_graph(np.stack(parents), n, 3, 0, pref)
        cd, cp = orc.dijkstra(crow, ccol, cw, 0, 0)
        rd, rp, re = orc.ref_combined_dijkstra(np.stack(parents), n, 3, 0, pref)
        assert re == len(ccol) and np.array_equal(cd, rd) and np.array_equal(cp, rp)
        assert np.array_equal(orc.path_costs(urow, ucol, uw, cp, 0), orc.ref_path_costs(urow, ucol, uw, cp, 0))


@needs_ref
def test_oracle_sequential_equals_reference_file_api(tmp_path):
    """The restated sequential update writes what the reference's
    sequentialSOSPUpdate writes (file API, the reference CPU path)."""
    import mosp_b200 as mb
    row, col, w = grid_graph(12, 10, 2, 30, 0.1, 3)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.generate(g, 60, 50.0, "uniform", 0, False, 9, 0, 1, 30)
    prefix = str(tmp_path / "g" / "graphCsr")
    g.write(prefix)
    ins, dele = str(tmp_path / "insert.txt"), str(tmp_path / "delete.txt")
    b.write(ins, dele)
    ba = b.arrays()
    urow, ucol, uw, mask = orc.apply_batch(row, col, w, ba["ins_from"], ba["ins_to"], ba["ins_w"],
                                           ba["del_from"], ba["del_to"])
    for k in range(2):
        d0, p0 = orc.dijkstra(row, col, w, k, 0)
        din, tin = str(tmp_path / f"d{k}.txt"), str(tmp_path / f"t{k}.txt")
        mb.check(mb.lib().mosp_write_tree(din.encode(), tin.encode(), len(d0), d0.ctypes.data, p0.ctypes.data))
        dout, tout = str(tmp_path / f"od{k}.txt"), str(tmp_path / f"ot{k}.txt")
        assert orc.ref_sequential_update(prefix, din, tin, ins, dele, k, 0, dout, tout)
        sel = ((mask >> k) & 1).astype(bool)
        cf = np.concatenate([ba["del_from"], ba["ins_from"][sel]])
        ct = np.concatenate([ba["del_to"], ba["ins_to"][sel]])
        d, p = orc.sequential_update(urow, ucol, uw, k, 0, cf, ct, ba["ins_to"], d0, p0)
        assert np.array_equal(read_pairs(dout, g.n), d)
        assert np.array_equal(read_pairs(tout, g.n), p)
