"""Parity of the CUDA path with the CPU oracle on the full-size benchmark
configurations (through the C ABI with host buffers, as a user calls it):

* R-MAT scale 22, edge factor 16, (0.57, 0.19, 0.19, 0.05), edge weights
  U[1, 10], k = 64, eps = 0.03, config default;
* 3D random geometric graph, 8,388,608 points, mean degree 14, edge weights
  U[1, 100], explicit unit vertex weights, hierarchy 4:8:6, distance
  1:10:100, eps = 0.03, configs HM and IM.

Every check is exact: identical labels and identical int64 objectives, every
block at most L_max = ceil((1 + eps) W / k), and the edge cut / J recomputed
here in int64 from the returned labels (independently of both
implementations). The oracle runs on all host threads; each case takes tens
of seconds of CPU time.
"""
import numpy as np
import pytest

import gpu_heipa as H
import oracle as O

pytestmark = pytest.mark.gpu

EPS = 0.03


def int64_objective(g, part, hier=None, dist=None):
    """Edge cut (undirected, each edge once) or J (over directed entries, as
    the reference reports it) in int64, computed in chunks of rows."""
    xadj = np.asarray(g.xadj, np.int64)
    part = np.asarray(part, np.int64)
    if hier is not None:
        k = int(np.prod(hier))
        ids = np.arange(k)
        D = np.zeros((k, k), np.int64)
        group = 1
        same_before = np.zeros((k, k), bool)
        for a, d in zip(hier, dist):
            group *= a
            same = (ids[:, None] // group) == (ids[None, :] // group)
            D[same & ~same_before] = d
            same_before |= same
        np.fill_diagonal(D, 0)
    total = 0
    step = 1 << 20
    for lo in range(0, g.n, step):
        hi = min(g.n, lo + step)
        a, b = int(xadj[lo]), int(xadj[hi])
        src = np.repeat(part[lo:hi], np.diff(xadj[lo:hi + 1]))
        dst = part[np.asarray(g.adj[a:b], np.int64)]
        w = np.ones(b - a, np.int64) if g.ew is None else np.asarray(g.ew[a:b], np.int64)
        if hier is None:
            total += int((w * (src != dst)).sum())
        else:
            total += int((w * D[src, dst]).sum())
    return total // 2 if hier is None else total


def check_balance(g, part, k):
    assert int(part.max()) < k
    bw = np.bincount(part, weights=(None if g.vw is None else g.vw), minlength=k)
    assert bw.max() <= O.lmax(g.total_weight(), k, EPS)


def context_for(g, scale):
    return H.Context(0, scale * H.arena_estimate(g.n, g.m, g.ew is not None, g.vw is not None))


def test_rmat22_k64_default_full_size():
    g = H.Graph.rmat(22, 16, 0.57, 0.19, 0.19, 1, 10, 1)
    assert g.n == 1 << 22
    with context_for(g, 1) as ctx:
        part, cut = ctx.partition(g, 64, EPS, "default", 1)
    opart, ocut = O.partition(O.Graph(g.xadj, g.adj, g.ew, g.vw), 64, EPS, False, 1)
    assert cut == ocut
    np.testing.assert_array_equal(part, opart)
    check_balance(g, part, 64)
    assert int64_objective(g, part) == cut


@pytest.fixture(scope="module")
def rgg23():
    return H.Graph.rgg3d(8388608, 14.0, 1, 100, 1, True)


@pytest.mark.parametrize("mode", ["HM", "IM"])
def test_rgg23_mapping_full_size(rgg23, mode):
    g = rgg23
    hier, dist = [4, 8, 6], [1, 10, 100]
    with context_for(g, 2) as ctx:
        part, J = ctx.process_map(g, hier, dist, EPS, mode, 1)
    og = O.Graph(g.xadj, g.adj, g.ew, g.vw)
    if mode == "IM":
        opart, oJ = O.map_im(og, hier, dist, EPS, 1)
    else:
        opart, oJ = O.map_hm(og, hier, dist, EPS, False, 1)
    assert J == oJ
    np.testing.assert_array_equal(part, opart)
    check_balance(g, part, 192)
    assert int64_objective(g, part, hier, dist) == J
    assert J > 2 ** 31  # the int32 accumulator of the reference would overflow here
