"""Generate the config-1 golden fixtures with the reference's own code.

Inputs come from this library's generators (30x30 4-neighbour grid, K=3,
weights U[1,100] seed 12345; 250 insertions of non-edges within Manhattan
distance 3 plus 250 connectivity-safe deletions, seed 777; and a second,
disconnecting batch from the reference-compatible uniform generator).
Expected outputs come from the reference compiled into oracle/_ref
(libref_cpu.so: host Dijkstra, applyChangeBatch, combinedGraphReference +
Dijkstra, mospPathCosts). Files use the reference's text formats.

Run from the repository root after `python -c "import __graft_entry__ as g;
g.build()"` (needs the reference sources at build time):
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "mosp-cuda_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")


def write_trees(d, p, dist_path, tree_path):
    os.makedirs(os.path.dirname(dist_path), exist_ok=True)
    mb.check(mb.lib().mosp_write_tree(dist_path.encode(), tree_path.encode(), len(d),
                                      np.ascontiguousarray(d, np.int64).ctypes.data,
                                      np.ascontiguousarray(p, np.int32).ctypes.data))


def write_costs(path, costs):
    with open(path, "w") as f:
        for v, row in enumerate(costs):
            f.write(str(v) + "".join(" INF" if c >= orc.INF // 2 else f" {c}" for c in row) + "\n")


def make_case(name, g, batch, pref):
    base = os.path.join(OUT, name)
    g.write(os.path.join(base, "graph", "graphCsr"))
    batch.write(os.path.join(base, "changes", "insert.txt"), os.path.join(base, "changes", "delete.txt"))
    row, col, w = g.arrays()
    K = g.K
    init = []
    for k in range(K):
        d, p = orc.ref_dijkstra(row, col, w, k, 0)
        init.append((d, p))
        ob = os.path.join(base, "init", f"obj{k}")
        write_trees(d, p, os.path.join(ob, "distancesOriginal.txt"), os.path.join(ob, "SSSPTreeOriginal.txt"))
    b = batch.arrays()
    urow, ucol, uw, _ = orc.ref_apply_batch(row, col, w, b["ins_from"], b["ins_to"], b["ins_w"],
                                            b["del_from"], b["del_to"])
    parents = []
    for k in range(K):
        d, p = orc.ref_dijkstra(urow, ucol, uw, k, 0)
        parents.append(p)
        ob = os.path.join(base, "expected", f"obj{k}")
        write_trees(d, p, os.path.join(ob, "distancesUpdated.txt"), os.path.join(ob, "SSSPTreeUpdated.txt"))
    cd, cp, _ = orc.ref_combined_dijkstra(np.stack(parents), g.n, K, 0, pref)
    cb = os.path.join(base, "expected", "combinedGraph")
    write_trees(cd, cp, os.path.join(cb, "distancesCsr.txt"), os.path.join(cb, "SSSPTreeCsr.txt"))
    write_costs(os.path.join(cb, "mospCosts.txt"), orc.ref_path_costs(urow, ucol, uw, cp, 0))
    with open(os.path.join(base, "pref.txt"), "w") as f:
        f.write(",".join(map(str, pref)) if pref else "")


def main():
    if not orc.have_ref():
        sys.exit("oracle/_ref/libref_cpu.so is missing (build with the reference sources present)")
    g = mb.HostGraph.grid_road(30, 30, 1.0, 0.0, 3, 1, 100, 12345)
    make_case("c1", g, mb.HostBatch.near(g, 30, 250, 250, 3, True, 777, 0, 1, 100), None)
    make_case("c1_unsafe", g, mb.HostBatch.generate(g, 500, 30.0, "uniform", 0, False, 778, 0, 1, 100),
              [1, 2, 3])


if __name__ == "__main__":
    main()
