"""The host initial partitioner against the reference's own code.

The reference's METIS-derived k-way partitioner (GPU_HeiPa::ModifiedMetis,
src/initial_partitioning/kway_partitioner/kway_core.h) is plain C++; it is
compiled from the reference's unmodified sources by oracle/build_ref.py into
oracle/_ref/libkway_ref.so. The product restates it (host/metis_kway.cpp,
reached through the C ABI's hp_initial_partition). On the same graph (same
vertex and row order), k, imbalance and seed the two partitions must be
identical, label for label. This pins every initial partition the product
computes, and with it the oracle pipelines' first step (which call the
reference library directly when it is built).
"""
import importlib.util
import os

import numpy as np
import pytest

import gpu_heipa as H
import oracle as O

_spec = importlib.util.spec_from_file_location(
    "oracle_build_ref", os.path.join(os.path.dirname(O.__file__), "build_ref.py"))
_build_ref = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_build_ref)

pytestmark = pytest.mark.skipif(O.ref_lib() is None, reason="oracle/_ref/libkway_ref.so is not built")


def test_reference_library_is_built_where_its_sources_are():
    # wherever the reference sources exist, the recipe must have built the
    # library (so that this module's tests never skip silently there)
    if os.path.isdir(os.path.join(_build_ref.REF, _build_ref.KWAY_DIR)):
        assert os.path.exists(_build_ref.LIB)
    assert O.uses_reference_kway()


def _both(g, k, imb, seed):
    vw = np.ones(g.n, np.int32) if g.vw is None else g.vw
    ew = np.ones(g.m, np.int32) if g.ew is None else g.ew
    want = O.ref_kway(g.xadj, g.adj, vw, ew, k, imb, seed)
    got = H.initial_partition(g, k, imb, seed)
    return got, want


def _random_graph(rng, n, deg, unit, isolated=0):
    pairs = set()
    for _ in range(n * deg // 2):
        a, b = (int(x) for x in rng.integers(isolated, n, 2))
        if a != b:
            pairs.add((min(a, b), max(a, b)))
    rows = [[] for _ in range(n)]
    for a, b in sorted(pairs, key=lambda p: (rng.random(), p)):
        w = 1 if unit else int(rng.integers(1, 100))
        rows[a].append((b, w))
        rows[b].append((a, w))
    xadj = np.cumsum([0] + [len(r) for r in rows]).astype(np.uint32)
    adj = np.array([v for r in rows for v, _ in r], np.uint32)
    ew = None if unit else np.array([w for r in rows for _, w in r], np.int32)
    vw = None if unit else rng.integers(1, 20, n).astype(np.int32)
    return H.Graph(xadj, adj, ew, vw)


@pytest.mark.parametrize("case", range(24))
def test_random_graphs_identical(case):
    rng = np.random.default_rng(1000 + case)
    n = int(rng.integers(30, 6000))
    g = _random_graph(rng, n, int(rng.integers(1, 16)), bool(case % 3 == 0), isolated=n // 10 if case % 4 == 1 else 0)
    k = [2, 3, 4, 5, 8, 16, 64, 192][case % 8]
    imb = [0.03, 0.01, 0.1, 0.0543][case % 4]
    got, want = _both(g, k, imb, int(rng.integers(0, 1 << 20)))
    np.testing.assert_array_equal(got, want)


def _coarsest(g, k):
    """The coarsest graph of the oracle's hierarchy (coarsen while n > 8k),
    rows sorted, as the solvers hand it to the initial partitioner."""
    og = O.Graph(g.xadj, g.adj, g.ew, g.vw)
    while og.n > 8 * k:
        mp, nc = O.match(og)
        if nc * 100 > og.n * 99:
            break
        og = O.contract(og, mp, nc)
    xadj, adj, ew, vw = og.arrays()
    return H.Graph(xadj, adj, ew, vw)


@pytest.mark.parametrize("name,k", [("rmat16", 64), ("rmat16_k16", 16), ("grid256", 16), ("rgg_k192", 192),
                                    ("rgg_k6", 6), ("rmat14_k512", 512)])
def test_coarsest_graphs_identical(name, k):
    if name.startswith("rmat16"):
        g = H.Graph.rmat(16, 16, 0.57, 0.19, 0.19, 1, 10, 1)
    elif name == "grid256":
        g = H.Graph.grid(256, 256)
    elif name.startswith("rgg"):
        g = H.Graph.rgg3d(131072, 14.0, 1, 100, 1, True)
    else:
        g = H.Graph.rmat(14, 16, 0.57, 0.19, 0.19, 1, 10, 2)
    c = _coarsest(g, k)
    for seed in (1, 7):
        got, want = _both(c, k, 0.03, seed)
        np.testing.assert_array_equal(got, want)


def test_im_level_imbalances_identical():
    # the IM initial mapping partitions sub-levels with adaptive imbalances
    c = _coarsest(H.Graph.rgg3d(65536, 14.0, 1, 100, 3, True), 192)
    for k, imb in ((6, 0.0099), (8, 0.0148), (4, 0.03)):
        got, want = _both(c, k, imb, 1)
        np.testing.assert_array_equal(got, want)


def test_edge_cases_identical():
    single = H.Graph(np.array([0, 0], np.uint32), np.zeros(0, np.uint32))
    for g, k in ((single, 4), (H.Graph.grid(3, 3), 16), (H.Graph.grid(10, 1), 3), (H.Graph.grid(2, 2), 2)):
        got, want = _both(g, k, 0.03, 5)
        np.testing.assert_array_equal(got, want)
    assert (H.initial_partition(H.Graph.grid(8, 8), 1) == 0).all()


def test_rejects_bad_graphs():
    with pytest.raises(H.HeiPaError):
        H.initial_partition(H.Graph(np.array([0, 1]), np.array([0])), 2)  # self loop
    with pytest.raises(H.HeiPaError):
        H.initial_partition(H.Graph(np.array([0, 1, 1]), np.array([7])), 2)  # id out of range


def test_oracle_pipeline_uses_reference_partitioner():
    # the oracle pipeline's first step is the reference's own partition of
    # the coarsest graph: partition a graph that needs no coarsening
    g = H.Graph.grid(16, 16, 1, 10, seed=2)
    og = O.Graph(g.xadj, g.adj, g.ew, g.vw)
    want = O.ref_kway(g.xadj, g.adj, np.ones(g.n, np.int32), g.ew, 64, 0.03, 3)
    np.testing.assert_array_equal(O.initial_kway(og, 64, 0.03, 3), want)
