"""TEST INFRASTRUCTURE: ctypes access to the parity checker.

* ``oracle`` functions wrap libmosp_oracle.so, the C restatement of the
  reference algorithms (mosp_oracle.c);
* ``ref`` functions wrap oracle/_ref/libref_cpu.so, the reference's own CPU
  code compiled from its sources (present only where the reference sources
  were available at build time; ``have_ref()`` says whether it is).

* ``workload_*`` functions build the seeded benchmark graphs from
  oracle/_gen/libworkload.so (the library's generators compiled on their
  own), for the benchmark's reference arm.

Only tests/, __graft_entry__.smoke() and the cpu_baseline and reference
legs of bench.py use this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "libmosp_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_cpu.so")
REF_DIR = os.path.join(HERE, "_ref")
INF = 0x7FFFFFFFFFFFFFFF // 4

_p = C.c_void_p
_i = C.c_int
_ll = C.c_longlong

_ORACLE_SIGS = {
    "oracle_apply_batch": (_ll, [_i, _i, _p, _p, _p, _i, _p, _p, _p, _i, _p, _p, _p, _p, _p, _ll, _p]),
    "oracle_transpose": (None, [_i, _i, _p, _p, _p, _p, _p, _p]),
    "oracle_dijkstra": (None, [_i, _i, _p, _p, _p, _i, _i, _p, _p]),
    "oracle_sequential_update": (_i, [_i, _i, _i, _i, _p, _p, _p, _p, _p, _p, _i, _p, _p, _i, _p, _p, _p]),
    "oracle_preference_scale": (_ll, [_p, _i]),
    "oracle_combined_graph": (_ll, [_i, _i, _p, _i, _p, _p, _p, _p]),
    "oracle_path_costs": (_i, [_i, _i, _p, _p, _p, _p, _i, _p]),
    "oracle_check_tree": (None, [_i, _i, _i, _i, _p, _p, _p, _p, _p, _p, _p, _p]),
}
_REF_SIGS = {
    "ref_dijkstra": (_i, [_i, _i, _p, _p, _p, _i, _i, _p, _p]),
    "ref_apply_batch": (_ll, [_i, _i, _p, _p, _p, _i, _p, _p, _p, _i, _p, _p, _p, _p, _p, _ll, _p]),
    "ref_generate_changes": (_i, [_i, _i, _p, _p, _p, _i, C.c_double, _i, _i, _i, C.c_uint, _i, _i, _i,
                                  _p, _p, _p, _p, _p, _p, _p]),
    "ref_combined_dijkstra": (_i, [_i, _i, _p, _i, _p, _p, _p, _p]),
    "ref_path_costs": (_i, [_i, _i, _p, _p, _p, _p, _i, _p]),
    "ref_sequential_update": (_i, [C.c_char_p] * 5 + [_i, _i, C.c_char_p, C.c_char_p]),
    "ref_sequential_update_timed": (_i, [C.c_char_p] * 5 + [_i, _i, C.c_char_p, C.c_char_p, _p]),
    "ref_write_csr": (_i, [C.c_char_p, _i, _i, _p, _p, _p]),
    "ref_write_changes": (_i, [C.c_char_p, C.c_char_p, _i, _i, _p, _p, _p, _i, _p, _p]),
    "ref_write_tree": (_i, [C.c_char_p, C.c_char_p, _i, _p, _p]),
    "ref_read_parents": (_i, [C.c_char_p, _i, _p]),
}
_WORKLOAD_SIGS = {
    "wl_grid_road": (_p, [_i, _i, C.c_double, C.c_double, _i, _i, _i, C.c_uint, _p, _p]),
    "wl_rmat": (_p, [_i, _i, C.c_double, C.c_double, C.c_double, _i, _i, _i, _i, C.c_uint, _p, _p]),
    "wl_copy": (None, [_p, _p, _p, _p]),
    "wl_free": (None, [_p]),
}
WORKLOAD_LIB = os.path.join(HERE, "_gen", "libworkload.so")

_olib = None
_rlib = None
_wlib = None


def _load(path, sigs):
    handle = C.CDLL(path)
    for name, (res, args) in sigs.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    return handle


def olib():
    global _olib
    if _olib is None:
        _olib = _load(ORACLE_LIB, _ORACLE_SIGS)
    return _olib


def have_ref() -> bool:
    return os.path.exists(REF_LIB)


def rlib():
    global _rlib
    if _rlib is None:
        _rlib = _load(REF_LIB, _REF_SIGS)
    return _rlib


def wlib():
    global _wlib
    if _wlib is None:
        _wlib = _load(WORKLOAD_LIB, _WORKLOAD_SIGS)
    return _wlib


def _a(x, dt):
    return np.ascontiguousarray(x, dtype=dt)


def P(x):
    return None if x is None else x.ctypes.data


# ---------------------------------------------------------------------------
# C restatement
# ---------------------------------------------------------------------------
def apply_batch(row, col, w, ins_from, ins_to, ins_w, del_from, del_to):
    """Updated (row, col, w[m,K]) and the weight-increase masks."""
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    n = len(row) - 1
    K = w.shape[1]
    ins_from, ins_to, ins_w = _a(ins_from, np.int32), _a(ins_to, np.int32), _a(ins_w, np.int32)
    del_from, del_to = _a(del_from, np.int32), _a(del_to, np.int32)
    cap = len(col) + len(ins_from)
    orow = np.empty(n + 1, np.int32)
    ocol = np.empty(max(cap, 1), np.int32)
    ow = np.empty((max(cap, 1), K), np.int32)
    mask = np.zeros(max(len(ins_from), 1), np.uint32)
    m = olib().oracle_apply_batch(n, K, P(row), P(col), P(w), len(ins_from), P(ins_from), P(ins_to), P(ins_w),
                                  len(del_from), P(del_from), P(del_to), P(orow), P(ocol), P(ow), cap, P(mask))
    if m < 0:
        raise ValueError("oracle_apply_batch failed")
    return orow, ocol[:m].copy(), ow[:m].copy(), mask[: len(ins_from)].copy()


def transpose(row, col, w):
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    n = len(row) - 1
    K = w.shape[1]
    m = len(col)
    rrow = np.empty(n + 1, np.int32)
    rcol = np.empty(max(m, 1), np.int32)
    rw = np.empty((max(m, 1), K), np.int32)
    olib().oracle_transpose(n, K, P(row), P(col), P(w), P(rrow), P(rcol), P(rw))
    return rrow, rcol[:m], rw[:m]


def dijkstra(row, col, w, k, source):
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    n = len(row) - 1
    d = np.empty(n, np.int64)
    p = np.empty(n, np.int32)
    olib().oracle_dijkstra(n, w.shape[1], P(row), P(col), P(w), k, source, P(d), P(p))
    return d, p


def sequential_update(row, col, w, k, source, changed_from, changed_to, heads, dist, parent):
    """The reference's sequential update on the updated graph; returns the
    new (dist, parent)."""
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    rrow, rcol, rw = transpose(row, col, w)
    n = len(row) - 1
    d = _a(dist, np.int64).copy()
    p = _a(parent, np.int32).copy()
    cf, ct, h = _a(changed_from, np.int32), _a(changed_to, np.int32), _a(heads, np.int32)
    olib().oracle_sequential_update(n, w.shape[1], k, source, P(row), P(col), P(w), P(rrow), P(rcol), P(rw),
                                    len(cf), P(cf), P(ct), len(h), P(h), P(d), P(p))
    return d, p


def preference_scale(pref, K):
    arr = None if pref is None else _a(pref, np.int32)
    return int(olib().oracle_preference_scale(P(arr), K))


def combined_graph(parents, n, K, source, pref=None):
    par = _a(parents, np.int32).reshape(-1)
    crow = np.empty(n + 1, np.int32)
    ccol = np.empty(max(K * n, 1), np.int32)
    cw = np.empty(max(K * n, 1), np.int32)
    pa = None if pref is None else _a(pref, np.int32)
    m = olib().oracle_combined_graph(n, K, P(par), source, P(pa), P(crow), P(ccol), P(cw))
    if m < 0:
        raise ValueError("invalid preference vector")
    return crow, ccol[:m].copy(), cw[:m].reshape(-1, 1).copy()


def path_costs(row, col, w, parent, source):
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    n = len(row) - 1
    KG = w.shape[1]
    costs = np.empty(n * KG, np.int64)
    par = _a(parent, np.int32)
    if olib().oracle_path_costs(n, KG, P(row), P(col), P(w), P(par), source, P(costs)) != 0:
        raise ValueError("a tree edge is missing from the graph")
    return costs.reshape(n, KG)


def check_tree(rrow, rcol, rw, k, source, dist, parent, ref_dist, ref_parent=None):
    rrow, rcol, rw = _a(rrow, np.int32), _a(rcol, np.int32), _a(rw, np.int32)
    counts = np.zeros(4, np.int64)
    d, p, rd = _a(dist, np.int64), _a(parent, np.int32), _a(ref_dist, np.int64)
    rp = None if ref_parent is None else _a(ref_parent, np.int32)
    olib().oracle_check_tree(len(rrow) - 1, rw.shape[1], k, source, P(rrow), P(rcol), P(rw), P(d), P(p),
                             P(rd), P(rp), P(counts))
    return counts


def expected_update(graph, batch, K, source=0, pref=None, init=None):
    """Expected outputs of one MOSP update from the C restatement:
    canonical Dijkstra trees of the updated graph, the combined graph's
    Dijkstra tree and the MOSP path costs. graph = (row, col, w[m, KG]);
    batch = dict(ins_from, ins_to, ins_w, del_from, del_to)."""
    row, col, w = graph
    urow, ucol, uw, mask = apply_batch(row, col, w, batch["ins_from"], batch["ins_to"], batch["ins_w"],
                                       batch["del_from"], batch["del_to"])
    n = len(row) - 1
    dist = np.empty((K, n), np.int64)
    par = np.empty((K, n), np.int32)
    for k in range(K):
        dist[k], par[k] = dijkstra(urow, ucol, uw, k, source)
    crow, ccol, cw = combined_graph(par, n, K, source, pref)
    cd, cp = dijkstra(crow, ccol, cw, 0, source)
    costs = path_costs(urow, ucol, uw, cp, source)
    return {"updated": (urow, ucol, uw), "mask": mask, "dist": dist, "parent": par, "comb_dist": cd,
            "comb_parent": cp, "comb_edges": len(ccol), "costs": costs}


# ---------------------------------------------------------------------------
# The reference's own code (oracle/_ref/libref_cpu.so)
# ---------------------------------------------------------------------------
def ref_dijkstra(row, col, w, k, source):
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    n = len(row) - 1
    d = np.empty(n, np.int64)
    p = np.empty(n, np.int32)
    rlib().ref_dijkstra(n, w.shape[1], P(row), P(col), P(w), k, source, P(d), P(p))
    return d, p


def ref_apply_batch(row, col, w, ins_from, ins_to, ins_w, del_from, del_to):
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    n = len(row) - 1
    K = w.shape[1]
    ins_from, ins_to, ins_w = _a(ins_from, np.int32), _a(ins_to, np.int32), _a(ins_w, np.int32)
    del_from, del_to = _a(del_from, np.int32), _a(del_to, np.int32)
    cap = len(col) + len(ins_from)
    orow = np.empty(n + 1, np.int32)
    ocol = np.empty(max(cap, 1), np.int32)
    ow = np.empty((max(cap, 1), K), np.int32)
    mask = np.zeros(max(len(ins_from), 1), np.uint32)
    m = rlib().ref_apply_batch(n, K, P(row), P(col), P(w), len(ins_from), P(ins_from), P(ins_to), P(ins_w),
                               len(del_from), P(del_from), P(del_to), P(orow), P(ocol), P(ow), cap, P(mask))
    if m < 0:
        raise ValueError("ref_apply_batch failed")
    return orow, ocol[:m].copy(), ow[:m].copy(), mask[: len(ins_from)].copy()


def ref_generate_changes(row, col, w, changes, ins_pct=50.0, mode=0, local=0, safe=False, seed=1, source=0,
                         wmin=1, wmax=100):
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    n = len(row) - 1
    K = w.shape[1]
    cap = max(changes, 1)
    ifr, ito = np.empty(cap, np.int32), np.empty(cap, np.int32)
    iw = np.empty(cap * K, np.int32)
    dfr, dto = np.empty(cap, np.int32), np.empty(cap, np.int32)
    ni, nd = C.c_int(), C.c_int()
    rc = rlib().ref_generate_changes(n, K, P(row), P(col), P(w), changes, ins_pct, mode, local, int(safe), seed,
                                     source, wmin, wmax, P(ifr), P(ito), P(iw), C.addressof(ni), P(dfr), P(dto),
                                     C.addressof(nd))
    if rc != 0:
        raise ValueError("ref_generate_changes failed")
    a, b = ni.value, nd.value
    return {"ins_from": ifr[:a].copy(), "ins_to": ito[:a].copy(), "ins_w": iw[: a * K].reshape(a, K).copy(),
            "del_from": dfr[:b].copy(), "del_to": dto[:b].copy()}


def ref_combined_dijkstra(parents, n, K, source, pref=None):
    par = _a(parents, np.int32).reshape(-1)
    d = np.empty(n, np.int64)
    p = np.empty(n, np.int32)
    e = C.c_longlong()
    pa = None if pref is None else _a(pref, np.int32)
    rlib().ref_combined_dijkstra(n, K, P(par), source, P(pa), P(d), P(p), C.addressof(e))
    return d, p, e.value


def ref_path_costs(row, col, w, parent, source):
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    n = len(row) - 1
    KG = w.shape[1]
    costs = np.empty(n * KG, np.int64)
    par = _a(parent, np.int32)
    if rlib().ref_path_costs(n, KG, P(row), P(col), P(w), P(par), source, P(costs)) != 0:
        raise ValueError("a tree edge is missing from the graph")
    return costs.reshape(n, KG)


def ref_sequential_update(graph_prefix, dist_in, tree_in, insert_path, delete_path, k, source, dist_out,
                          tree_out):
    e = lambda s: s.encode()  # noqa: E731
    return rlib().ref_sequential_update(e(graph_prefix), e(dist_in), e(tree_in), e(insert_path),
                                        e(delete_path), k, source, e(dist_out), e(tree_out)) == 0


def ref_sequential_update_timed(graph_prefix, dist_in, tree_in, insert_path, delete_path, k, source, dist_out,
                                tree_out):
    """The same call through the instrumented copy: (ok, seconds of its
    Phases 1-2, the update computation alone)."""
    e = lambda s: s.encode()  # noqa: E731
    secs = C.c_double()
    rc = rlib().ref_sequential_update_timed(e(graph_prefix), e(dist_in), e(tree_in), e(insert_path),
                                            e(delete_path), k, source, e(dist_out), e(tree_out),
                                            C.addressof(secs))
    return rc == 0, secs.value


def ref_write_csr(prefix, row, col, w):
    row, col, w = _a(row, np.int32), _a(col, np.int32), _a(w, np.int32)
    if rlib().ref_write_csr(prefix.encode(), len(row) - 1, w.shape[1], P(row), P(col), P(w)) != 0:
        raise OSError(f"ref_write_csr failed for {prefix}")


def ref_write_changes(insert_path, delete_path, K, batch):
    ifr, ito = _a(batch["ins_from"], np.int32), _a(batch["ins_to"], np.int32)
    iw = _a(batch["ins_w"], np.int32)
    dfr, dto = _a(batch["del_from"], np.int32), _a(batch["del_to"], np.int32)
    if rlib().ref_write_changes(insert_path.encode(), delete_path.encode(), K, len(ifr), P(ifr), P(ito), P(iw),
                                len(dfr), P(dfr), P(dto)) != 0:
        raise OSError("ref_write_changes failed")


def ref_write_tree(dist_path, tree_path, dist, parent):
    d, p = _a(dist, np.int64), _a(parent, np.int32)
    if rlib().ref_write_tree(dist_path.encode(), tree_path.encode(), len(d), P(d), P(p)) != 0:
        raise OSError("ref_write_tree failed")


def ref_read_parents(path, n):
    p = np.empty(n, np.int32)
    if rlib().ref_read_parents(path.encode(), n, P(p)) != 0:
        raise OSError(f"ref_read_parents failed for {path}")
    return p


# ---------------------------------------------------------------------------
# Seeded benchmark graphs (oracle/_gen/libworkload.so: the library's own
# generators, built without the library)
# ---------------------------------------------------------------------------
def _workload(handle, n, m, K):
    if not handle:
        raise ValueError("invalid workload parameters")
    row = np.empty(n.value + 1, np.int32)
    col = np.empty(max(m.value, 1), np.int32)
    w = np.empty((max(m.value, 1), K), np.int32)
    wlib().wl_copy(handle, P(row), P(col), P(w))
    wlib().wl_free(handle)
    return row, col[: m.value], w[: m.value]


def workload_grid_road(width, height, keep, shortcut, K, wmin, wmax, seed):
    n, m = C.c_int(), C.c_longlong()
    h = wlib().wl_grid_road(width, height, keep, shortcut, K, wmin, wmax, seed, C.addressof(n), C.addressof(m))
    return _workload(h, n, m, K)


def workload_rmat(scale, edge_factor, a, b, c, K, wmin, wmax, log_uniform, seed):
    n, m = C.c_int(), C.c_longlong()
    h = wlib().wl_rmat(scale, edge_factor, a, b, c, K, wmin, wmax, int(log_uniform), seed, C.addressof(n),
                       C.addressof(m))
    return _workload(h, n, m, K)
