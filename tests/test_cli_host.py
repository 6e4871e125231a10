"""CLI and host-side contract on CPU: `mospPrep` subcommands write the
reference's formats and - where the reference was compiled into
oracle/_ref - byte-identical files to the reference's own mospPrep for the
same arguments and seeds; the binary cache round trip; the C ABI library
loads and exports every entry point its headers declare."""
import filecmp
import os
import re
import subprocess

import numpy as np
import pytest

import mosp_b200 as mb
import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PREP = os.path.join(ROOT, "mosp-cuda_b200", "bin", "mospPrep")
PREP_REF = os.path.join(ROOT, "oracle", "_ref", "mospPrep_ref")


def declared_functions():
    names = []
    for h in ("mosp_b200.h", "mosp_b200_host.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(mosp_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_function():
    lib = mb.lib()
    names = declared_functions()
    assert len(names) >= 40
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(mb.exported_names())
    assert lib.mosp_abi_version() == 1


def test_host_helpers():
    assert mb.default_delta(0, 5, 0) == 1
    assert mb.default_delta(5_530_000, 1_970_000, 5_530_000 * 50) == int(32.0 * 50 / (5_530_000 / 1_970_000))
    assert mb.choose_packing(900, 100)[0] == 10
    bits, maxd = mb.choose_packing((1 << 17) - 1, (1 << 30) + (1 << 14))
    assert bits == 17 and maxd == ((1 << 17) - 2) * ((1 << 30) + (1 << 14))
    assert mb.choose_packing(4_194_304, 1_000_000)[0] == 0  # distance-only fallback
    assert mb.preference_scale([1, 2, 3, 4, 5], 5) == 60
    assert mb.preference_scale([0, 1], 2) == 0
    assert mb.preference_scale(None, 3) == 1


def run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def write_mtx(path, seed):
    rng = np.random.default_rng(seed)
    W = H = 20
    lines = []
    for y in range(H):
        for x in range(W):
            u = y * W + x + 1
            if x + 1 < W and rng.random() >= 0.05:
                lines += [f"{u} {u + 1}", f"{u + 1} {u}"]
            if y + 1 < H and rng.random() >= 0.05:
                lines += [f"{u} {u + W}", f"{u + W} {u}"]
    for _ in range(150):
        a, b = rng.integers(1, W * H + 1, 2)
        if a != b:
            lines.append(f"{a} {b}")
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n")
        f.write(f"{W * H} {W * H} {len(lines)}\n" + "\n".join(lines) + "\n")


def same_tree(a, b):
    return filecmp.cmp(a, b, shallow=False)


@pytest.mark.skipif(not os.path.exists(PREP_REF), reason="reference mospPrep not built")
def test_mosprep_byte_identical_to_reference(tmp_path):
    write_mtx(tmp_path / "g.mtx", 3)
    for tool, tag in ((PREP, "ours"), (PREP_REF, "ref")):
        d = tmp_path / tag
        run([tool, "mtx2csr", str(tmp_path / "g.mtx"), str(d / "csr/graphCsr"), "3", "1", "20", "5"], tmp_path)
        run([tool, "widen", str(d / "csr/graphCsr"), str(d / "w/graphCsr"), "4", "1", "20", "6"], tmp_path)
        run([tool, "init", str(d / "csr/graphCsr"), str(d / "init")], tmp_path)
        for name, extra in (("safe", ["--changes", "300", "--ins", "50", "--safe"]),
                            ("unsafe", ["--changes", "500", "--ins", "20"]),
                            ("targeted", ["--changes", "200", "--mode", "targeted"]),
                            ("reweight", ["--changes", "100", "--mode", "reweight"]),
                            ("increase", ["--changes", "100", "--mode", "increase"]),
                            ("local", ["--changes", "100", "--local", "5"])):
            run([tool, "changes", str(d / "csr/graphCsr"), str(d / name), "--seed", "9"] + extra, tmp_path)
            run([tool, "expected", str(d / "csr/graphCsr"), str(d / name), str(d / ("exp-" + name))], tmp_path)
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    files = [p.relative_to(ref) for p in ref.rglob("*.txt")]
    assert len(files) > 30
    for rel in files:
        assert same_tree(ours / rel, ref / rel), str(rel)


@pytest.mark.skipif(not os.path.exists(PREP_REF), reason="the reference's mospPrep was not built")
def test_mosprep_multichunk_files_byte_identical(tmp_path):
    """Files of several MB, which the readers and writers split into
    line-aligned chunks parsed and formatted on all host cores: every file
    equals the reference's sequential output byte for byte."""
    rng = np.random.default_rng(5)
    W = H = 400
    u = np.arange(W * H).reshape(H, W) + 1
    e = np.concatenate([np.stack([u[:, :-1].ravel(), u[:, 1:].ravel()], 1),
                        np.stack([u[:-1, :].ravel(), u[1:, :].ravel()], 1)])
    e = e[rng.random(len(e)) >= 0.05]
    e = np.concatenate([e, e[:, ::-1]])
    with open(tmp_path / "g.mtx", "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate pattern general\n{W * H} {W * H} {len(e)}\n")
        f.write("\n".join(f"{a} {b}" for a, b in e) + "\n")
    for tool, tag in ((PREP, "ours"), (PREP_REF, "ref")):
        d = tmp_path / tag
        run([tool, "mtx2csr", str(tmp_path / "g.mtx"), str(d / "csr/graphCsr"), "3", "1", "100", "5"], tmp_path)
        run([tool, "init", str(d / "csr/graphCsr"), str(d / "init")], tmp_path)
        run([tool, "changes", str(d / "csr/graphCsr"), str(d / "ch"), "--seed", "9", "--changes", "2000",
             "--ins", "50"], tmp_path)
        run([tool, "expected", str(d / "csr/graphCsr"), str(d / "ch"), str(d / "exp")], tmp_path)
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    assert os.path.getsize(ref / "csr/graphCsrColInd.txt") > 3 << 20
    files = [p.relative_to(ref) for p in ref.rglob("*.txt")]
    assert len(files) >= 15
    for rel in files:
        assert same_tree(ours / rel, ref / rel), str(rel)


def test_mosprep_init_matches_oracle(tmp_path):
    run([PREP, "grid", str(tmp_path / "g/graphCsr"), "25", "20", "0.8", "0.02", "2", "1", "50", "4"], tmp_path)
    run([PREP, "init", str(tmp_path / "g/graphCsr"), str(tmp_path / "init")], tmp_path)
    g = mb.HostGraph.read(str(tmp_path / "g/graphCsr"))
    row, col, w = g.arrays()
    for k in range(2):
        d = np.empty(g.n, np.int64)
        p = np.empty(g.n, np.int32)
        ob = tmp_path / "init" / f"obj{k}"
        mb.check(mb.lib().mosp_read_tree(str(ob / "distancesOriginal.txt").encode(),
                                         str(ob / "SSSPTreeOriginal.txt").encode(), g.n, d.ctypes.data,
                                         p.ctypes.data))
        de, pe = orc.dijkstra(row, col, w, k, 0)
        assert np.array_equal(d, de) and np.array_equal(p, pe)


def test_binary_cache_round_trip(tmp_path):
    g = mb.HostGraph.grid_road(30, 20, 0.7, 0.01, 3, 1, 100, 1)
    prefix = str(tmp_path / "g/graphCsr")
    g.write(prefix)
    cache = str(tmp_path / "g.bin")
    a = mb.HostGraph.read(prefix, cache)  # writes the cache
    assert os.path.exists(cache)
    b = mb.HostGraph.read(prefix, cache)  # reads it
    for x, y in zip(a.arrays(), b.arrays()):
        assert np.array_equal(x, y)
    for x, y in zip(g.arrays(), b.arrays()):
        assert np.array_equal(x, y)


def test_apply_batch_matches_oracle():
    g = mb.HostGraph.grid_road(40, 40, 0.7, 0.01, 3, 1, 100, 2)
    for mode in ("uniform", "reweight", "increase", "targeted"):
        b = mb.HostBatch.generate(g, 300, mode=mode, seed=3)
        u = mb.apply_batch(g, b)
        ba = b.arrays()
        orow, ocol, ow, mask = orc.apply_batch(*g.arrays(), ba["ins_from"], ba["ins_to"], ba["ins_w"],
                                               ba["del_from"], ba["del_to"])
        r, c, w = u.arrays()
        assert np.array_equal(r, orow) and np.array_equal(c, ocol) and np.array_equal(w, ow)
        assert np.array_equal(ba["mask"], mask)


@pytest.mark.skipif(not orc.have_ref(), reason="oracle/_ref not built")
def test_generator_matches_reference():
    """Same graph, options and seed: the same batch as the reference's
    generateChangeBatch, for every mode, local and safe batches."""
    g = mb.HostGraph.grid_road(30, 30, 0.75, 0.01, 3, 1, 100, 5)
    row, col, w = g.arrays()
    for mode_name, mode in mb.MODES.items():
        for local, safe in ((0, False), (0, True), (6, False)):
            ours = mb.HostBatch.generate(g, 250, 40.0, mode_name, local, safe, 17, 0, 1, 100).arrays()
            ref = orc.ref_generate_changes(row, col, w, 250, 40.0, mode, local, safe, 17, 0, 1, 100)
            for key in ("ins_from", "ins_to", "ins_w", "del_from", "del_to"):
                assert np.array_equal(ours[key], ref[key]), (mode_name, local, safe, key)


def test_invalid_inputs_rejected(tmp_path):
    """Readers reject what the reference rejects (src/mospTest.cu:827-919)."""
    def graph_ok(rows, values):
        p = tmp_path / f"g{len(list(tmp_path.iterdir()))}"
        p.mkdir()
        (p / "gRowPtr.txt").write_text(rows)
        (p / "gColInd.txt").write_text("1\n2\n")
        (p / "gValues.txt").write_text(values)
        try:
            mb.HostGraph.read(str(p / "g"))
            return True
        except mb.MospError:
            return False
    rows = "0\n1\n2\n2\n"
    assert graph_ok(rows, "4 5\n2147483647 7\n")
    for values in ("0 5\n2 7\n", "4 5\n-3 7\n", "4294967297 5\n2 7\n", "4 5\n2147483648 7\n"):
        assert not graph_ok(rows, values)
    assert not graph_ok("0\n1\n4294967298\n2\n", "4 5\n2 7\n")
    d = tmp_path / "c"
    d.mkdir()
    (d / "delete.txt").write_text("0 1\n")
    for insert, ok in (("2 0 1 2147483647\n", True), ("2 0 0 3\n", False), ("2 0 -5 3\n", False),
                       ("2 0 4294967297 3\n", False), ("2 3 1 1\n", False)):
        (d / "insert.txt").write_text(insert)
        try:
            mb.HostBatch.read(str(d / "insert.txt"), str(d / "delete.txt"), 2, 3)
            accepted = True
        except mb.MospError:
            accepted = False
        assert accepted == ok, insert
    for text, ok in (("0 0\n1 4\n2 INF\n", True), ("0 0\n1 4\n", False), ("0 0\n1 4\n1 4\n2 6\n", False),
                     ("0 0\n1 -4\n2 6\n", False)):
        (tmp_path / "d.txt").write_text(text)
        (tmp_path / "p.txt").write_text("0 -1\n1 0\n2 -1\n")
        dd = np.empty(3, np.int64)
        pp = np.empty(3, np.int32)
        st = mb.lib().mosp_read_tree(str(tmp_path / "d.txt").encode(), str(tmp_path / "p.txt").encode(), 3,
                                     dd.ctypes.data, pp.ctypes.data)
        assert (st == 0) == ok, text
