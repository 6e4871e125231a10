"""Helpers of the GPU tests: run the library's C ABI on torch device memory
and compare with the oracle."""
import numpy as np
import torch

import mosp_b200 as mb
import oracle as orc


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def initial_trees(graph_arrays, K, source=0):
    row, col, w = graph_arrays
    n = len(row) - 1
    d = np.empty((K, n), np.int64)
    p = np.empty((K, n), np.int32)
    for k in range(K):
        d[k], p[k] = orc.dijkstra(row, col, w, k, source)
    return d, p


def run_update_device(ws, g, batch, K=None, source=0, pref=None, init=None, delta=None, max_weight=None):
    """One MOSP update through mosp_update_device: the batch is applied by
    the library (host), the updated graph uploaded, the K fused updates and
    Steps 2-3 run on the GPU. Returns numpy results and the stats.
    max_weight overrides the per-objective weight bound (a larger bound
    makes the objectives run distance-only)."""
    K = K or g.K
    ga = g.arrays()
    d0, p0 = init if init is not None else initial_trees(ga, K, source)
    upd = mb.apply_batch(g, batch)
    ba = batch.arrays()
    dg = mb.DeviceGraph.upload(ws, upd)
    n, m = upd.n, upd.m
    ch = mb.changed_lists(ba, K)
    ch_from = np.concatenate([c[0] for c in ch]) if ch else np.zeros(0, np.int32)
    ch_to = np.concatenate([c[1] for c in ch]) if ch else np.zeros(0, np.int32)
    off = np.concatenate([[0], np.cumsum([len(c[0]) for c in ch])]).astype(np.int32)
    orig_w = ga[2]
    maxw = [max(1, int(orig_w[:, k].max()) if len(orig_w) else 1,
                int(ba["ins_w"][:, k].max()) if len(ba["ins_w"]) else 1) for k in range(K)]
    if max_weight is not None:
        maxw = [int(max_weight)] * K
    if delta is None:
        deltas = [mb.default_delta(max(g.m, 1), g.n, int(orig_w[:, k].sum())) for k in range(K)]
    else:
        deltas = [delta] * K
    dist = dev(d0[:K].copy())
    par = dev(p0[:K].copy())
    cd = torch.empty(n, dtype=torch.int64, device="cuda")
    cp = torch.empty(n, dtype=torch.int32, device="cuda")
    heads = dev(ba["ins_to"].astype(np.int32)) if len(ba["ins_to"]) else torch.zeros(1, dtype=torch.int32,
                                                                                    device="cuda")
    cf = dev(ch_from) if len(ch_from) else torch.zeros(1, dtype=torch.int32, device="cuda")
    ct = dev(ch_to) if len(ch_to) else torch.zeros(1, dtype=torch.int32, device="cuda")
    stats, cst = ws.update_device(n, m, K, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w, cf, ct,
                                  off, heads, len(ba["ins_to"]), source, deltas, maxw, pref, dist, par, cd, cp)
    costs = torch.empty(n * upd.K, dtype=torch.int64, device="cuda")
    ws.path_costs(n, m, upd.K, dg.out_row, dg.out_col, dg.out_w, cp, source, costs)
    return {"dist": dist.cpu().numpy(), "parent": par.cpu().numpy(), "comb_dist": cd.cpu().numpy(),
            "comb_parent": cp.cpu().numpy(), "costs": costs.cpu().numpy().reshape(n, upd.K), "stats": stats,
            "cstats": cst}


def assert_matches_oracle(res, g, batch, K=None, source=0, pref=None):
    K = K or g.K
    exp = orc.expected_update(g.arrays(), batch.arrays(), K, source, pref)
    for k in range(K):
        assert np.array_equal(res["dist"][k], exp["dist"][k]), f"objective {k} distances differ"
        assert np.array_equal(res["parent"][k], exp["parent"][k]), f"objective {k} parents differ"
    assert np.array_equal(res["comb_dist"], exp["comb_dist"]), "combined distances differ"
    assert np.array_equal(res["comb_parent"], exp["comb_parent"]), "combined parents differ"
    assert np.array_equal(res["costs"], exp["costs"]), "MOSP costs differ"
    assert res["cstats"].edges == exp["comb_edges"]
    return exp
