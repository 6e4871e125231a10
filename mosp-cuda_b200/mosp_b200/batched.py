"""Batched instances: many independent graphs and change batches stored as
one disjoint union, so that one launch of each engine step updates all of
them (mosp_workspace_set_sources gives the engine every instance's root).

Vertex v of instance i is union vertex offsets[i] + v; instance i's edges
keep their row order, so the union's results sliced back per instance equal
the per-instance results exactly."""
import numpy as np


def union_graphs(graphs):
    """graphs: list of (row[n_i+1], col[m_i], w[m_i, K]). Returns (row, col,
    w, offsets[len+1]) of the disjoint union."""
    ns = [len(r) - 1 for r, _, _ in graphs]
    offsets = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    ms = [len(c) for _, c, _ in graphs]
    eoff = np.concatenate([[0], np.cumsum(ms)]).astype(np.int64)
    if offsets[-1] >= 2**31 or eoff[-1] >= 2**31:
        raise ValueError("the union exceeds int32 vertex or edge ids")
    row = np.empty(offsets[-1] + 1, np.int32)
    for i, (r, _, _) in enumerate(graphs):
        row[offsets[i]:offsets[i + 1]] = np.asarray(r[:-1], np.int64) + eoff[i]
    row[-1] = eoff[-1]
    col = np.concatenate([np.asarray(c, np.int64) + offsets[i] for i, (_, c, _) in enumerate(graphs)]
                         ).astype(np.int32) if graphs else np.zeros(0, np.int32)
    w = np.concatenate([np.asarray(x, np.int32) for _, _, x in graphs]) if graphs else np.zeros((0, 1), np.int32)
    return row, col, w, offsets


def union_batches(batches, offsets):
    """batches: list of dicts (ins_from, ins_to, ins_w, del_from, del_to) in
    instance ids. Returns one batch in union ids (instance order, each
    instance's file order kept)."""
    def cat(key, shift):
        parts = [np.asarray(b[key], np.int64) + (offsets[i] if shift else 0) for i, b in enumerate(batches)]
        return np.concatenate(parts).astype(np.int32) if parts else np.zeros(0, np.int32)
    K = next((np.asarray(b["ins_w"]).shape[1] for b in batches if len(b["ins_w"])), 1)
    ins_w = [np.asarray(b["ins_w"], np.int32).reshape(-1, K) for b in batches]
    return {"ins_from": cat("ins_from", True), "ins_to": cat("ins_to", True),
            "ins_w": np.concatenate(ins_w) if ins_w else np.zeros((0, K), np.int32),
            "del_from": cat("del_from", True), "del_to": cat("del_to", True)}


def union_trees(dists, parents, offsets):
    """Per-instance trees (K x n_i) in instance ids -> union trees (K x N)."""
    d = np.concatenate(dists, axis=1)
    p = np.concatenate([np.where(np.asarray(pp) >= 0, np.asarray(pp, np.int64) + offsets[i], -1)
                        for i, pp in enumerate(parents)], axis=1).astype(np.int32)
    return d, p


def split_vertices(arr, offsets, i, parents=False):
    """Instance i's slice of a per-vertex union array (last axis); parent
    ids are shifted back to instance ids."""
    a = np.asarray(arr)[..., offsets[i]:offsets[i + 1]]
    if parents:
        a = np.where(a >= 0, a - offsets[i], -1).astype(np.int32)
    return a
