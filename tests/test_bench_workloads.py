"""bench.py's workload builders on CPU: the road-network and power-law
configurations have the objective count, preferences, sizes and change
batches their descriptions state, and the power-law options used for
profiling captures change only the scale and the weight range."""
import argparse
import json

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


def test_reference_arm_builds_the_same_workload():
    """The reference arm builds its input from oracle/ alone (the standalone
    generator library and the reference's own change generator); graph and
    batch equal the library arm's, for both configurations."""
    import numpy as np
    import oracle as orc
    if not orc.have_ref():
        import pytest
        pytest.skip("oracle/_ref not built")
    for a in (args(), args(workload="powerlaw", rmat_scale=10, rmat_wmax=10_000_000)):
        g, b, K, pref, desc = bench.make_workload(a)
        row, col, w, batch, K2, pref2, desc2 = bench.reference_workload(a)
        grow, gcol, gw = g.arrays()
        assert np.array_equal(row, grow) and np.array_equal(col, gcol) and np.array_equal(w, gw)
        ba = b.arrays()
        for key in ("ins_from", "ins_to", "ins_w", "del_from", "del_to"):
            assert np.array_equal(np.asarray(batch[key]).reshape(np.asarray(ba[key]).shape), ba[key]), key
        assert (K2, pref2, desc2) == (K, pref, desc)


def test_reference_arm_loads_no_library_code():
    """`bench.py --impl reference` maps only oracle/ libraries: none of this
    library's shared objects is loaded in its process."""
    import os
    import subprocess
    import sys
    import oracle as orc
    if not orc.have_ref():
        import pytest
        pytest.skip("oracle/_ref not built")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, argparse, bench\n"
            "a = argparse.Namespace(workload='road', width=40, changes=200, rmat_scale=22, rmat_wmax=10**6, "
            "steps=3, warmup=1, gpus=1)\n"
            "bench.run_reference(a)\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('LIBRARY_MAPPED' if 'libmosp_b200' in maps else 'CLEAN', 'mosp_b200' in sys.modules)\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    last = out.stdout.strip().splitlines()[-1]
    assert last == "CLEAN False", last
    assert '"impl": "reference"' in out.stdout
    line = json.loads([x for x in out.stdout.splitlines() if x.startswith("{")][-1])
    # the reference's GPU binary ran on the same files, or says why not
    gpu = line["reference_gpu"]
    assert ("unavailable" in gpu) or (gpu["runs"] == 5 and gpu["gpu_compute_ms"] > 0), gpu
