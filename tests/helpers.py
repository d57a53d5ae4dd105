"""Shared helpers for the parity tests (graph fixtures and canonical forms)."""
import numpy as np

import gpu_heipa as H
import oracle as O


def to_oracle(g):
    return O.Graph(g.xadj, g.adj, g.ew, g.vw)


def sorted_rows(xadj, adj, ew):
    """Canonical CSR: rows sorted by neighbour id (weights follow)."""
    xadj = np.asarray(xadj, np.int64)
    n = len(xadj) - 1
    rows = np.repeat(np.arange(n), np.diff(xadj))
    order = np.lexsort((adj, rows))
    return np.asarray(xadj, np.uint32), np.asarray(adj)[order], (None if ew is None else np.asarray(ew)[order])


def small_graphs():
    """(name, graph) pairs covering the three generators at test sizes."""
    return [
        ("grid64", H.Graph.grid(64, 64)),
        ("grid_w", H.Graph.grid(48, 80, 1, 10, seed=3)),
        ("rmat12", H.Graph.rmat(12, 8, seed=5)),
        ("rmat14", H.Graph.rmat(14, 16, seed=7)),
        ("rgg", H.Graph.rgg3d(20000, 10.0, 1, 100, seed=11)),
    ]


def block_partition_grid(w, h, bx, by):
    """Labels of a w x h grid cut into bx x by rectangles (id = row*bx + col)."""
    ys, xs = np.divmod(np.arange(w * h), w)
    return ((ys * by // h) * bx + (xs * bx // w)).astype(np.uint32)


def perturb(part, k, frac, seed):
    rng = np.random.default_rng(seed)
    p = part.copy()
    idx = rng.choice(len(p), int(frac * len(p)), replace=False)
    p[idx] = rng.integers(0, k, len(idx)).astype(np.uint32)
    return p


def star(n_leaves):
    n = n_leaves + 1
    xadj = [0, n_leaves]
    adj = list(range(1, n))
    for i in range(1, n):
        adj.append(0)
        xadj.append(len(adj))
    return H.Graph(np.array(xadj), np.array(adj))


def k2n(n):
    """Two hubs {0,1} connected to leaves 2..n+1 (leaves are twins)."""
    rows = [list(range(2, n + 2)), list(range(2, n + 2))] + [[0, 1] for _ in range(n)]
    xadj = np.cumsum([0] + [len(r) for r in rows])
    return H.Graph(xadj, np.concatenate([np.array(r) for r in rows]))


def isolated_plus_path(n_iso, n_path):
    """n_iso isolated vertices followed by a path of n_path vertices."""
    rows = [[] for _ in range(n_iso)]
    for i in range(n_path):
        r = []
        if i > 0:
            r.append(n_iso + i - 1)
        if i + 1 < n_path:
            r.append(n_iso + i + 1)
        rows.append(r)
    xadj = np.cumsum([0] + [len(r) for r in rows])
    adj = np.concatenate([np.array(r, dtype=np.uint32) for r in rows]) if xadj[-1] else np.zeros(0, np.uint32)
    return H.Graph(xadj, adj)
