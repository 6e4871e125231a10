"""bench.py's workload builders on CPU: the road-network and power-law
configurations have the objective count, preferences, sizes and change
batches their descriptions state, and the power-law options used for
profiling captures change only the scale and the weight range."""
import argparse

import bench
import mosp_b200 as mb


def args(**kw):
    base = dict(workload="road", width=40, changes=500, rmat_scale=22, rmat_wmax=1_000_000)
    base.update(kw)
    return argparse.Namespace(**base)


def test_road_workload_shape():
    g, b, K, pref, desc = bench.make_workload(args())
    assert K == 3 and pref is None and desc == bench.WORKLOAD
    assert g.K == 3 and 0 < g.n <= 40 * 40
    row, col, w = g.arrays()
    assert len(row) == g.n + 1 and len(col) == g.m and w.shape == (g.m, 3)
    assert w.min() >= 1 and w.max() <= 100
    assert b.n_ins + b.n_del <= 500 and b.n_ins > 0 and b.n_del > 0


def test_powerlaw_workload_options():
    g, b, K, pref, desc = bench.make_workload(args(workload="powerlaw", rmat_scale=10, rmat_wmax=10_000_000))
    assert K == 5 and pref == [1, 2, 3, 4, 5]
    assert g.n == 1 << 10 and g.K == 5
    _, _, w = g.arrays()
    assert w.min() >= 1 and w.max() <= 10_000_000
    assert "R-MAT scale 10" in desc and "[1,10000000]" in desc
    assert "R-MAT scale 22" not in desc
    ba = b.arrays()
    assert len(ba["ins_to"]) == b.n_ins and b.n_ins + b.n_del > 0
    # the full-size configuration keeps its own description
    assert "R-MAT scale 22" in bench.POWERLAW and "[1,1e6]" in bench.POWERLAW


def test_powerlaw_full_size_takes_the_fallback():
    """The configuration's sizes put every objective on the distance-only
    words: (n - 1) * 10^6 does not fit next to the parent bits of 2^22
    vertices."""
    assert mb.choose_packing(1 << 22, 1_000_000)[0] == 0
    assert mb.choose_packing(1 << 20, 10_000_000)[0] == 0
    assert mb.choose_packing(1 << 20, 1_000_000)[0] > 0
