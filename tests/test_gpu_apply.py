"""Step 1 on the GPU (mosp_apply_batch_device) against the host batch
application (the reference's applyChangeBatch, src/csrGraph.cu:727-894):
the updated CSR edge for edge, the weight-increase masks and the
per-objective weight statistics (src/mospUpdate.cu:104-136). Cases cover
repeated (u,v) entries in a batch, deletions of missing edges, insert after
delete of the same edge, parallel edges in the original graph, hub rows,
and empty, deletion-only and insertion-only batches."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
from conftest import grid_graph, random_graph  # noqa: E402


@pytest.fixture(scope="module")
def ws():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    w = mb.Workspace(timeout_ms=20000)
    yield w
    w.close()


def dev(a, dtype=np.int32):
    a = np.ascontiguousarray(np.asarray(a, dtype))
    if a.size == 0:
        return torch.zeros(1, dtype=torch.int32, device="cuda")[:0]
    return torch.from_numpy(a).cuda()


def gpu_apply(ws, row, col, w, ins_from, ins_to, ins_w, del_from, del_to):
    n, K, m = len(row) - 1, w.shape[1], len(col)
    cap = m + len(ins_from)
    new_row = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    new_col = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
    new_w = torch.empty(max(cap, 1) * K, dtype=torch.int32, device="cuda")
    mask = torch.zeros(max(len(ins_from), 1), dtype=torch.int32, device="cuda")
    nm, mx, sm = ws.apply_batch_device(n, K, m, dev(row), dev(col), dev(w.reshape(-1)), dev(ins_from), dev(ins_to),
                                       dev(np.asarray(ins_w).reshape(-1)), dev(del_from), dev(del_to), new_row,
                                       new_col[:cap] if cap else new_col[:0], new_w, mask)
    return (new_row.cpu().numpy(), new_col.cpu().numpy()[:nm], new_w.cpu().numpy()[: nm * K].reshape(nm, K),
            mask.cpu().numpy()[: len(ins_from)].astype(np.uint32), mx, sm)


def check_case(ws, row, col, w, ins_from, ins_to, ins_w, del_from, del_to):
    K = w.shape[1]
    ins_w = np.asarray(ins_w, np.int32).reshape(-1, K)
    g = mb.HostGraph.from_arrays(row, col, w)
    b = mb.HostBatch.from_arrays(K, ins_from, ins_to, ins_w, del_from, del_to)
    upd = mb.apply_batch(g, b)
    er, ec, ew = upd.arrays()
    emask = b.arrays()["mask"].astype(np.uint32)
    r, c, ww, mask, mx, sm = gpu_apply(ws, row, col, w, ins_from, ins_to, ins_w, del_from, del_to)
    assert np.array_equal(r, er)
    assert np.array_equal(c, ec)
    assert np.array_equal(ww, ew)
    assert np.array_equal(mask, emask)
    emx = [max(1, int(w[:, k].max()) if len(w) else 1, int(ins_w[:, k].max()) if len(ins_w) else 1)
           for k in range(K)]
    esm = [int(w[:, k].astype(np.int64).sum()) for k in range(K)]
    assert mx == emx and sm == esm


def random_batch(rng, n, row, col, n_ins, n_del, K, wmax=100, local_pairs=None):
    m = len(col)
    src = np.repeat(np.arange(n), np.diff(row))
    # deletions: mostly existing edges, some missing ones, some repeated
    pick = rng.integers(0, m, n_del)
    del_from, del_to = src[pick].copy(), col[pick].copy()
    miss = rng.random(n_del) < 0.2
    del_to[miss] = rng.integers(0, n, miss.sum())
    rep = rng.random(n_del) < 0.1
    if n_del > 1:
        j = rng.integers(0, n_del, rep.sum())
        del_from[rep], del_to[rep] = del_from[j], del_to[j]
    # insertions: existing edges (overwrite), deleted edges (re-insert),
    # new edges and repeats of earlier insertions
    ins_from = rng.integers(0, n, n_ins)
    ins_to = rng.integers(0, n, n_ins)
    ex = rng.random(n_ins) < 0.35
    pe = rng.integers(0, m, ex.sum())
    ins_from[ex], ins_to[ex] = src[pe], col[pe]
    rd = rng.random(n_ins) < 0.15
    if n_del > 0:
        j = rng.integers(0, n_del, rd.sum())
        ins_from[rd], ins_to[rd] = del_from[j], del_to[j]
    rp = rng.random(n_ins) < 0.1
    if n_ins > 1:
        j = rng.integers(0, n_ins, rp.sum())
        ins_from[rp], ins_to[rp] = ins_from[j], ins_to[j]
    ins_w = rng.integers(1, wmax + 1, (n_ins, K))
    return ins_from, ins_to, ins_w, del_from, del_to


@pytest.mark.parametrize("shape", ["grid", "random"])
@pytest.mark.parametrize("sizes", [(500, 500), (3000, 0), (0, 3000), (0, 0), (20000, 20000)])
def test_apply_matches_host(ws, shape, sizes):
    if shape == "grid":
        row, col, w = grid_graph(150, 150, 3, 100, 0.2, 31)
    else:
        row, col, w = random_graph(20000, 60000, 3, 100, 32)
    n = len(row) - 1
    rng = np.random.default_rng(hash((shape, sizes)) % 2**32)
    batch = random_batch(rng, n, row, col, sizes[0], sizes[1], 3)
    check_case(ws, row, col, w, *batch)


def test_apply_parallel_edges_and_hubs(ws):
    """Original rows with repeated heads (parallel edges) and two hub rows
    receiving thousands of changes."""
    rng = np.random.default_rng(33)
    n = 5000
    rows = [list(rng.integers(0, n, rng.integers(0, 6))) for _ in range(n)]
    rows[7] = list(rng.integers(0, n, 40000))           # hub with many repeats
    rows[4000] = list(rng.integers(0, 50, 3000))         # hub of parallel edges
    for u in range(0, n, 3):
        if rows[u]:
            rows[u] += rows[u][:2]                       # duplicate heads
    row = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    col = np.concatenate([np.asarray(r, np.int32) for r in rows])
    w = rng.integers(1, 1000, (len(col), 2)).astype(np.int32)
    ins_from, ins_to, ins_w, del_from, del_to = random_batch(rng, n, row, col, 6000, 6000, 2, 1000)
    hub = rng.random(6000) < 0.3
    ins_from[hub] = 7
    del_from[rng.random(6000) < 0.3] = 4000
    del_to[del_from == 4000] = rng.integers(0, 50, (del_from == 4000).sum())
    check_case(ws, row, col, w, ins_from, ins_to, ins_w, del_from, del_to)


def test_apply_rejects_out_of_range(ws):
    row, col, w = grid_graph(10, 10, 1, 10, 0.0, 34)
    with pytest.raises(mb.MospError):
        gpu_apply(ws, row, col, w, np.array([0]), np.array([100]), np.array([[5]]), np.zeros(0), np.zeros(0))
    # still usable afterwards
    check_case(ws, row, col, w, np.array([0, 1]), np.array([5, 2]), np.array([[5], [7]]), np.array([0]),
               np.array([1]))
