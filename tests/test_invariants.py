"""Structural invariants of graphs and partitions, after the reference's
checker list (src/utility/asserts.h:36-166: ids in range, no self loops, no
parallel edges, positive edge weights, block ids < k, block weights equal to
the recomputed sums), plus the conservation laws of contraction (total vertex
weight; edge weight between clusters) and symmetry of every level. Applied on
the CPU to the generators, to every level of the oracle's coarsening and to
the oracle's partitions and mappings (the CUDA path is compared with those
results bit for bit by the GPU tests)."""
import numpy as np
import pytest

import gpu_heipa as H
import oracle as O
from helpers import small_graphs, to_oracle


def edge_list(xadj, adj, ew):
    xadj = np.asarray(xadj, np.int64)
    n = len(xadj) - 1
    u = np.repeat(np.arange(n, dtype=np.int64), np.diff(xadj))
    v = np.asarray(adj, np.int64)
    w = np.ones(len(v), np.int64) if ew is None else np.asarray(ew, np.int64)
    return n, u, v, w


def check_graph(xadj, adj, ew, vw):
    """asserts.h:36-86 (ids < n, no loops, no double edges, positive weights)
    and symmetry with equal weights in both directions."""
    n, u, v, w = edge_list(xadj, adj, ew)
    assert np.all(np.diff(np.asarray(xadj, np.int64)) >= 0), "offsets not monotone"
    assert len(v) == int(xadj[-1])
    if len(v):
        assert v.max() < n, "neighbour id out of range"
        assert np.all(u != v), "self loop"
        key = u * n + v
        assert len(np.unique(key)) == len(key), "parallel edges"
        assert w.min() > 0, "non-positive edge weight"
        order = np.argsort(key)
        rkey = v * n + u
        pos = np.searchsorted(key[order], rkey)
        assert np.all(pos < len(key)) and np.all(key[order][np.minimum(pos, len(key) - 1)] == rkey), "asymmetric"
        assert np.array_equal(w[order][pos], w), "asymmetric weight"
    if vw is not None:
        assert np.asarray(vw).min(initial=1) > 0, "non-positive vertex weight"


def check_contraction(fine, mapping, nc, coarse):
    """Coarse vertex weights are the member sums; the coarse edge weight
    between two clusters is the fine weight between them (graph.h:127-390)."""
    fx, fa, fe, fv = fine
    cx, ca, ce, cv = coarse
    n, u, v, w = edge_list(fx, fa, fe)
    mp = np.asarray(mapping, np.int64)
    assert mp.min(initial=0) >= 0 and mp.max(initial=-1) < nc
    fvw = np.ones(n, np.int64) if fv is None else np.asarray(fv, np.int64)
    cvw = np.ones(nc, np.int64) if cv is None else np.asarray(cv, np.int64)
    assert np.array_equal(np.bincount(mp, weights=fvw, minlength=nc).astype(np.int64), cvw)
    cu, cvv = mp[u], mp[v]
    cross = cu != cvv
    want = {}
    for a, b, x in zip(cu[cross].tolist(), cvv[cross].tolist(), w[cross].tolist()):
        want[(a, b)] = want.get((a, b), 0) + x
    _, u2, v2, w2 = edge_list(cx, ca, ce)
    got = dict(zip(zip(u2.tolist(), v2.tolist()), w2.tolist()))
    assert got == want


def check_partition(xadj, adj, ew, vw, part, k, lmax=None):
    """asserts.h:111-141: every block id < k; block weights; the balance bound."""
    part = np.asarray(part, np.int64)
    assert part.min(initial=0) >= 0 and part.max(initial=-1) < k
    n = len(xadj) - 1
    wv = np.ones(n, np.int64) if vw is None else np.asarray(vw, np.int64)
    bw = np.bincount(part, weights=wv, minlength=k).astype(np.int64)
    assert bw.sum() == wv.sum()
    if lmax is not None:
        assert bw.max(initial=0) <= lmax
    return bw


GRAPHS = small_graphs()


@pytest.mark.parametrize("name,g", GRAPHS, ids=[x[0] for x in GRAPHS])
def test_every_oracle_level_is_a_simple_symmetric_graph(name, g):
    check_graph(g.xadj, g.adj, g.ew, g.vw)
    og = to_oracle(g)
    for _ in range(12):
        if og.n <= 64:
            break
        mp, nc = O.match(og)
        oc = O.contract(og, mp, nc)
        fine, coarse = og.arrays(), oc.arrays()
        check_graph(*coarse)
        check_contraction(fine, mp, nc, coarse)
        if oc.n == og.n:
            break
        og = oc


@pytest.mark.parametrize("name,g,k", [("grid96", H.Graph.grid(96, 96), 16), ("rmat13", H.Graph.rmat(13, 8, seed=4), 32),
                                      ("rgg", H.Graph.rgg3d(12000, 12.0, 1, 50, seed=6, explicit_vw=True), 8)],
                         ids=["grid96", "rmat13", "rgg"])
def test_oracle_partitions_are_valid(name, g, k):
    og = to_oracle(g)
    for ultra in (False, True):
        part, cut = O.partition(og, k, 0.03, ultra, 3)
        check_partition(g.xadj, g.adj, g.ew, g.vw, part, k, O.lmax(g.total_weight(), k, 0.03))
        assert cut == O.edge_cut(og, part)


def test_oracle_mappings_are_valid():
    g = H.Graph.rgg3d(15000, 14.0, 1, 100, seed=8, explicit_vw=True)
    og = to_oracle(g)
    hier, dist = [2, 4, 3], [1, 10, 100]
    for part, J in (O.map_im(og, hier, dist, 0.03, 3), O.map_hm(og, hier, dist, 0.03, False, 3)):
        check_partition(g.xadj, g.adj, g.ew, g.vw, part, 24)
        assert J == O.comm_cost(og, part, hier, dist)


def test_checkers_catch_violations():
    # a planted mistake of each kind on a small graph must be reported
    g = H.Graph.grid(4, 4, 1, 5, seed=1)
    x, a, e = g.xadj.copy(), g.adj.copy(), g.ew.copy()
    bad = [(x, np.where(np.arange(len(a)) == 0, 16, a), e),       # id out of range
           (x, np.where(np.arange(len(a)) == 0, 0, a), e),        # self loop at vertex 0
           (x, a, np.where(np.arange(len(e)) == 0, 0, e)),        # zero weight
           (x, a, np.where(np.arange(len(e)) == 0, e[0] + 1, e))]  # asymmetric weight
    for xx, aa, ee in bad:
        with pytest.raises(AssertionError):
            check_graph(xx, aa, ee, None)
    with pytest.raises(AssertionError):
        check_partition(x, a, e, None, np.full(16, 4), 4)
