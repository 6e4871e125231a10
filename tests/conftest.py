"""Shared test setup: import paths, the `gpu` marker and small fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "mosp-cuda_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")


def grid_graph(width, height, K, wmax, drop, seed, wmin=1):
    """Road-like grid (both directions, a fraction of links dropped) with K
    random weights per edge; returns (row, col, w[m, K])."""
    rng = np.random.default_rng(seed)
    rows = [[] for _ in range(width * height)]
    for y in range(height):
        for x in range(width):
            u = y * width + x
            for dx, dy in ((1, 0), (0, 1)):
                nx, ny = x + dx, y + dy
                if nx >= width or ny >= height or rng.random() < drop:
                    continue
                v = ny * width + nx
                rows[u].append((v, rng.integers(wmin, wmax + 1, K)))
                rows[v].append((u, rng.integers(wmin, wmax + 1, K)))
    row = np.zeros(width * height + 1, np.int32)
    col, w = [], []
    for u, r in enumerate(rows):
        row[u + 1] = row[u] + len(r)
        for v, ws in r:
            col.append(v)
            w.append(ws)
    return row, np.array(col, np.int32), np.array(w, np.int32).reshape(-1, K)


def random_graph(n, extra, K, wmax, seed):
    """Spanning chain 0 -> 1 -> ... -> n-1 plus random distinct arcs."""
    rng = np.random.default_rng(seed)
    edges = {(i, i + 1) for i in range(n - 1)}
    while len(edges) < n - 1 + extra:
        u, v = rng.integers(0, n, 2)
        if u != v:
            edges.add((int(u), int(v)))
    edges = sorted(edges)
    row = np.zeros(n + 1, np.int32)
    for u, _ in edges:
        row[u + 1] += 1
    row = np.cumsum(row).astype(np.int32)
    col = np.array([v for _, v in edges], np.int32)
    w = rng.integers(1, wmax + 1, (len(edges), K)).astype(np.int32)
    return row, col, w
