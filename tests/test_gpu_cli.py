"""End-to-end contract of the drop-in CLIs on the GPU, following the
reference's scripts/endToEndTest.sh: mospPrep prepares a 30x30 road-like
grid with extra arcs, mosp --validate runs safe, disconnecting and targeted
batches and must equal `mospPrep expected` byte for byte; mospCosts has one
"v c1 .. cK" line per vertex and equals the oracle; --canonicalize fixes
initial trees with other tie rules; -k/--pref with --cache (written, then
read) equals the text graph; trees of another source are rejected. Where
the reference's own bin/mosp was built for sm_100a (oracle/_ref/mosp_ref),
every output file must be byte-identical to it."""
import filecmp
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402
from test_cli_host import write_mtx  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "mosp-cuda_b200", "bin")
MOSP, PREP = os.path.join(BIN, "mosp"), os.path.join(BIN, "mospPrep")
MOSP_REF = os.path.join(ROOT, "oracle", "_ref", "mosp_ref")


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")


def run(cmd, cwd, ok=True):
    r = subprocess.run([str(c) for c in cmd], cwd=cwd, capture_output=True, text=True, timeout=900)
    if ok:
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r


def validated(out):
    lines = [x for x in out.splitlines() if x.startswith("VALIDATE")]
    assert any(x.startswith("VALIDATE combined PASS") for x in lines), out
    assert not any(" FAIL" in x for x in lines), out


@pytest.fixture(scope="module")
def prepared(tmp_path_factory):
    t = tmp_path_factory.mktemp("e2e")
    write_mtx(t / "graph.mtx", 7)
    g = t / "g"
    run([PREP, "mtx2csr", t / "graph.mtx", g / "csr/graphCsr", 3, 1, 20, 7], t)
    run([PREP, "init", g / "csr/graphCsr", g / "init"], t)
    run([PREP, "changes", g / "csr/graphCsr", g / "safe", "--changes", 400, "--ins", 50, "--seed", 7, "--safe"], t)
    run([PREP, "changes", g / "csr/graphCsr", g / "unsafe", "--changes", 1500, "--ins", 20, "--seed", 7], t)
    run([PREP, "changes", g / "csr/graphCsr", g / "targeted", "--changes", 200, "--mode", "targeted", "--seed", 7], t)
    return t


@pytest.mark.parametrize("batch", ["safe", "unsafe", "targeted"])
def test_validate_and_expected(prepared, batch):
    t, g = prepared, prepared / "g"
    out = t / f"out-{batch}"
    r = run([MOSP, "--graph", g / "csr/graphCsr", "--init", g / "init", "--quiet", "--changes", g / batch,
             "--out", out, "--validate"], t)
    validated(r.stdout)
    assert "RESULT gpu_compute_ms=" in r.stdout
    run([PREP, "expected", g / "csr/graphCsr", g / batch, t / f"exp-{batch}"], t)
    for k in range(3):
        for f in ("distancesUpdated.txt", "SSSPTreeUpdated.txt"):
            assert filecmp.cmp(out / f"obj{k}" / f, t / f"exp-{batch}" / f"obj{k}" / f, shallow=False), (k, f)
    # mospCosts: n lines "v c1 c2 c3", equal to the oracle's costs
    gr = mb.HostGraph.read(str(g / "csr/graphCsr"))
    lines = open(out / "combinedGraph" / "mospCosts.txt").read().splitlines()
    assert len(lines) == gr.n and all(len(x.split()) == 4 for x in lines)
    b = mb.HostBatch.read(str(g / batch / "insert.txt"), str(g / batch / "delete.txt"), 3, gr.n)
    exp = orc.expected_update(gr.arrays(), b.arrays(), 3)
    costs = np.array([[orc.INF if x == "INF" else int(x) for x in line.split()[1:]] for line in lines])
    assert np.array_equal(costs, exp["costs"])


def test_canonicalize_highest_id_trees(prepared):
    t = prepared
    ti = t / "ties"
    run([PREP, "mtx2csr", t / "graph.mtx", ti / "csr/graphCsr", 2, 1, 2, 7], t)
    run([PREP, "init", ti / "csr/graphCsr", ti / "init"], t)
    run([PREP, "changes", ti / "csr/graphCsr", ti / "changes", "--changes", 400, "--ins", 50, "--seed", 7,
         "--wmin", 1, "--wmax", 2], t)
    g = mb.HostGraph.read(str(ti / "csr/graphCsr"))
    row, col, w = g.arrays()
    changed = False
    for k in range(2):
        d, p = orc.dijkstra(row, col, w, k, 0)
        high = np.full(g.n, -1, np.int32)
        for u in range(g.n):
            if d[u] >= orc.INF // 2:
                continue
            for e in range(row[u], row[u + 1]):
                v = col[e]
                if d[v] < orc.INF // 2 and d[u] + w[e, k] == d[v] and u > high[v]:
                    high[v] = u
        high[0] = -1
        changed |= not np.array_equal(high, p)
        ob = ti / "init-high" / f"obj{k}"
        os.makedirs(ob, exist_ok=True)
        mb.check(mb.lib().mosp_write_tree(str(ob / "distancesOriginal.txt").encode(),
                                          str(ob / "SSSPTreeOriginal.txt").encode(), g.n, d.ctypes.data,
                                          high.ctypes.data))
    assert changed
    r = run([MOSP, "--graph", ti / "csr/graphCsr", "--changes", ti / "changes", "--init", ti / "init-high",
             "--out", t / "out-ties", "--canonicalize", "--quiet", "--validate"], t)
    validated(r.stdout)
    run([PREP, "expected", ti / "csr/graphCsr", ti / "changes", t / "exp-ties"], t)
    for k in range(2):
        for f in ("distancesUpdated.txt", "SSSPTreeUpdated.txt"):
            assert filecmp.cmp(t / "out-ties" / f"obj{k}" / f, t / "exp-ties" / f"obj{k}" / f, shallow=False)


def test_cache_k_pref_and_wrong_source(prepared):
    t, g = prepared, prepared / "g"
    base = [MOSP, "--graph", g / "csr/graphCsr", "--init", g / "init", "--quiet", "--changes", g / "unsafe",
            "-k", 2, "--pref", "2,1"]
    cache = t / "graph.bin"
    stamp = None
    for p in ("write", "read"):
        r = run(base + ["--cache", cache, "--out", t / f"out-cache-{p}", "--validate"], t)
        validated(r.stdout)
        assert cache.exists()
        if p == "write":
            stamp = os.stat(cache).st_mtime_ns
        else:
            assert os.stat(cache).st_mtime_ns == stamp and "Note" not in r.stdout
    r = run(base + ["--out", t / "out-text", "--validate"], t)
    validated(r.stdout)
    for p in ("write", "read"):
        cmp = filecmp.dircmp(t / "out-text", t / f"out-cache-{p}")
        assert not cmp.diff_files and not cmp.left_only and not cmp.right_only
    r = run([MOSP, "--graph", g / "csr/graphCsr", "--init", g / "init", "--quiet", "--changes", g / "safe",
             "--source", 5, "--no-output"], t, ok=False)
    assert r.returncode != 0


@pytest.mark.skipif(not os.path.exists(MOSP_REF), reason="reference bin/mosp not built")
@pytest.mark.parametrize("batch", ["safe", "unsafe", "targeted"])
def test_byte_identical_to_reference_binary(prepared, batch):
    """Same inputs through the reference's own bin/mosp (built for sm_100a)
    and through this library: every output file byte-identical."""
    t, g = prepared, prepared / "g"
    for tool, tag in ((MOSP, "ours"), (MOSP_REF, "ref")):
        run([tool, "--graph", g / "csr/graphCsr", "--init", g / "init", "--quiet", "--changes", g / batch,
             "--pref", "1,2,3", "--out", t / f"cmp-{batch}-{tag}"], t)
    a, b = t / f"cmp-{batch}-ours", t / f"cmp-{batch}-ref"
    files = [p.relative_to(b) for p in b.rglob("*.txt")]
    assert len(files) == 3 * 2 + 3
    for rel in files:
        assert filecmp.cmp(a / rel, b / rel, shallow=False), str(rel)


PREP_REF = os.path.join(ROOT, "oracle", "_ref", "mospPrep_ref")


@pytest.mark.parametrize("source", [0, 17])
def test_mosp_prep_gpu_trees_equal_host_and_reference(prepared, tmp_path, source):
    """`mospPrep init --gpu` and `expected --gpu` (the canonical GPU SSSP for
    every objective, one workspace reused across objectives) write the same
    files byte for byte as the host Dijkstra path and, where it was built,
    the reference's own mospPrep (src/mospPrep.cu:350-375)."""
    g = prepared / "g"
    csr = g / "csr/graphCsr"
    outs = {}
    for name, tool, extra in [("host", PREP, []), ("gpu", PREP, ["--gpu"]), ("ref", PREP_REF, [])]:
        if name == "ref" and not os.path.exists(PREP_REF):
            continue
        d = tmp_path / name
        run([tool, "init", csr, d / "init", "--source", source] + extra, prepared)
        run([tool, "expected", csr, g / "unsafe", d / "expected", "--source", source] + extra, prepared)
        outs[name] = d
    files = [f"{stage}/obj{k}/{kind}" for k in range(3)
             for stage, kind in (("init", "distancesOriginal.txt"), ("init", "SSSPTreeOriginal.txt"),
                                 ("expected", "distancesUpdated.txt"), ("expected", "SSSPTreeUpdated.txt"))]
    for f in files:
        for name in outs:
            if name != "host":
                assert filecmp.cmp(outs["host"] / f, outs[name] / f, shallow=False), (name, f)


@pytest.mark.parametrize("width,changes,extra", [(120, 4000, []), (200, 20000, ["--mode", "targeted"]),
                                                 (90, 3000, ["--local", "6"])])
def test_safe_filter_on_gpu_equals_host_and_reference(tmp_path, width, changes, extra):
    """`mospPrep changes --safe --gpu` (the connectivity filter's rounds with
    reachability from Step 1 and a unit-weight SSSP on the GPU) writes the
    same insert.txt / delete.txt as the host filter and as the reference's
    own mospPrep (src/changeGenerator.cu:78-114)."""
    csr = tmp_path / "csr/graphCsr"
    run([PREP, "grid", csr, width, width, "0.7", "0.01", 2, 1, 50, 12345], tmp_path)
    outs = {}
    for name, tool, flag in [("host", PREP, []), ("gpu", PREP, ["--gpu"]), ("ref", PREP_REF, [])]:
        if name == "ref" and not os.path.exists(PREP_REF):
            continue
        d = tmp_path / name
        r = run([tool, "changes", csr, d, "--changes", changes, "--seed", 777, "--safe"] + extra + flag, tmp_path)
        if name != "ref":
            assert "safe filter:" in r.stdout
        outs[name] = d
    for f in ("insert.txt", "delete.txt"):
        for name in outs:
            assert filecmp.cmp(outs["host"] / f, outs[name] / f, shallow=False), (name, f)
    # the filter dropped something, so the rounds ran
    full = tmp_path / "unsafe"
    run([PREP, "changes", csr, full, "--changes", changes, "--seed", 777] + extra, tmp_path)
    assert os.path.getsize(full / "delete.txt") >= os.path.getsize(outs["gpu"] / "delete.txt")
