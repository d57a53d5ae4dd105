"""CPU checks of the oracle: published test vectors, hand-derived known answers
and independent pure-Python restatements of the small building blocks
(hashes, gain buckets, distance oracle, objectives). No GPU needed."""
import math
from fractions import Fraction

import numpy as np
import pytest

import gpu_heipa as H
import oracle as O
from helpers import block_partition_grid, isolated_plus_path, k2n, perturb, star, to_oracle

M32 = 0xFFFFFFFF


# ---- hashes -------------------------------------------------------------------

def _rotl(x, r):
    return ((x << r) | (x >> (32 - r))) & M32


def _murmur3_x86_32_u32(key, seed):
    """MurmurHash3_x86_32 of the 4 little-endian bytes of `key` (Appleby's
    published algorithm), restated here independently of the oracle."""
    c1, c2 = 0xCC9E2D51, 0x1B873593
    k = (key * c1) & M32
    k = _rotl(k, 15)
    k = (k * c2) & M32
    h = seed ^ k
    h = _rotl(h, 13)
    h = (h * 5 + 0xE6546B64) & M32
    h ^= 4
    h ^= h >> 16
    h = (h * 0x85EBCA6B) & M32
    h ^= h >> 13
    h = (h * 0xC2B2AE35) & M32
    h ^= h >> 16
    return h


@pytest.mark.parametrize("key,seed,want", [
    (0x00000000, 0, 0x2362F9DE),
    (0x87654321, 0, 0xF55B516B),
    (0xFFFFFFFF, 0, 0x76293B50),
    (0x87654321, 0x5082EDEE, 0x2362F9DE),
])
def test_murmur3_published_vectors(key, seed, want):
    # Published MurmurHash3_x86_32 verification vectors for 4-byte inputs.
    assert O.murmur3_u32(key, seed) == want
    assert _murmur3_x86_32_u32(key, seed) == want


def test_murmur3_matches_restatement():
    rng = np.random.default_rng(1)
    for key, seed in zip(rng.integers(0, 1 << 32, 500), rng.integers(0, 1 << 32, 500)):
        assert O.murmur3_u32(int(key), int(seed)) == _murmur3_x86_32_u32(int(key), int(seed))


def test_xorshift32():
    def xs(x):
        x ^= (x << 13) & M32
        x ^= x >> 17
        x ^= (x << 5) & M32
        return x
    assert O.xorshift32(1) == 270369
    rng = np.random.default_rng(2)
    for x in rng.integers(1, 1 << 32, 500):
        assert O.xorshift32(int(x)) == xs(int(x))


# ---- gain buckets (jet_label_propagation.h gain_bucket) -------------------------

def _gain_bucket_exact(gx, vw):
    """Bucket of a non-positive gain: 0 for gain > 0, 1 for gain == 0, else
    25 + ceil(log_1.5(-gx/vw)) clamped to [2, 49], evaluated with exact
    rationals."""
    if gx > 0:
        return 0
    if gx == 0:
        return 1
    g = Fraction(-gx, max(vw, 1))
    k = 0
    if g >= 1:
        while k < 24 and g > Fraction(3, 2) ** k:
            k += 1
        return 25 + k
    while k < 23 and g < Fraction(2, 3) ** k:
        k += 1
    return 25 - k


def test_gain_bucket_exact_restatement():
    rng = np.random.default_rng(3)
    cases = [(1, 1), (0, 5), (-1, 1), (-3, 2), (-9, 4), (-2, 3), (-4, 9), (-1, 1 << 30), (-(1 << 30), 1)]
    cases += [(-int(a), int(b)) for a, b in zip(rng.integers(1, 1 << 20, 2000), rng.integers(1, 1 << 12, 2000))]
    cases += [(-int(a), int(b)) for a, b in zip(rng.integers(1, 50, 2000), rng.integers(1, 50, 2000))]
    for gx, vw in cases:
        assert O.gain_bucket(gx, vw) == _gain_bucket_exact(gx, vw), (gx, vw)


def test_gain_bucket_float_agrees_away_from_boundaries():
    # The reference evaluates the bucket with float log2; the integer form
    # differs from it only within ~1e-6 (relative) of a power of 1.5.
    rng = np.random.default_rng(4)
    checked = 0
    for a, b in zip(rng.integers(1, 1 << 16, 5000), rng.integers(1, 1 << 10, 5000)):
        lg = math.log(a / b, 1.5)
        if abs(lg - round(lg)) < 1e-4:
            continue
        assert O.gain_bucket(-int(a), int(b)) == O.gain_bucket_float(-int(a), int(b)), (a, b)
        checked += 1
    assert checked > 4000


# ---- distance oracle and objectives --------------------------------------------

def _distance_py(hier, dist):
    k = int(np.prod(hier))
    digits = np.zeros((k, len(hier)), np.int64)
    x = np.arange(k)
    for i, h in enumerate(hier):
        digits[:, i] = x % h
        x //= h
    D = np.zeros((k, k), np.int64)
    for a in range(k):
        diff = digits != digits[a]
        for b in range(k):
            lv = np.nonzero(diff[b])[0]
            D[a, b] = 0 if len(lv) == 0 else dist[lv[-1]]
    return D


@pytest.mark.parametrize("hier,dist", [([4, 8, 6], [1, 10, 100]), ([2, 4, 8], [1, 5, 50]), ([3, 5], [2, 7])])
def test_distance_matrix(hier, dist):
    D = O.distance_matrix(hier, dist)
    np.testing.assert_array_equal(D, _distance_py(hier, dist))
    assert D[0, 1] == dist[0] and D[0, hier[0]] == dist[1]
    assert (np.diag(D) == 0).all() and (D == D.T).all()


def _cut_py(g, part):
    rows = np.repeat(np.arange(g.n), np.diff(g.xadj.astype(np.int64)))
    w = np.ones(g.m, np.int64) if g.ew is None else g.ew.astype(np.int64)
    return int(w[part[rows] != part[g.adj]].sum()) // 2


def _J_py(g, part, D):
    rows = np.repeat(np.arange(g.n), np.diff(g.xadj.astype(np.int64)))
    w = np.ones(g.m, np.int64) if g.ew is None else g.ew.astype(np.int64)
    return int((w * D[part[rows], part[g.adj]]).sum())


def test_grid_cut_closed_form():
    # A w x h grid cut into bx x by rectangles cuts (bx-1)*h + (by-1)*w edges.
    for w, h, bx, by in [(64, 64, 8, 8), (96, 40, 4, 5), (33, 17, 3, 2)]:
        g = H.Graph.grid(w, h)
        part = block_partition_grid(w, h, bx, by)
        want = (bx - 1) * h + (by - 1) * w
        assert O.edge_cut(to_oracle(g), part) == want
        assert _cut_py(g, part) == want


def test_objectives_match_numpy():
    g = H.Graph.rmat(12, 8, seed=9)
    og = to_oracle(g)
    hier, dist = [4, 8, 2], [1, 10, 100]
    D = _distance_py(hier, dist)
    rng = np.random.default_rng(5)
    for _ in range(3):
        part = rng.integers(0, 64, g.n).astype(np.uint32)
        assert O.edge_cut(og, part) == _cut_py(g, part)
        assert O.comm_cost(og, part, hier, dist) == _J_py(g, part, D)


def test_lmax():
    assert O.lmax(65536, 16, 0.03) == math.ceil(1.03 * 4096)
    assert O.lmax(100, 3, 0.03) == math.ceil(1.03 * 100 / 3)
    assert O.lmax(7, 7, 0.0) == 1


# ---- coarsening ----------------------------------------------------------------

def _six_cycle():
    n = 6
    rows = [[] for _ in range(n)]
    for i in range(n):
        a, b, w = i, (i + 1) % n, i + 1
        rows[a].append((b, w))
        rows[b].append((a, w))
    xadj = np.cumsum([0] + [len(r) for r in rows])
    adj = np.array([v for r in rows for v, _ in r])
    ew = np.array([w for r in rows for _, w in r])
    return H.Graph(xadj, adj, ew, np.arange(1, 7))


def test_contract_kat_six_cycle():
    # Clusters {0,3},{1,4},{2,5} of the 6-cycle with edge weights 1..6 and
    # vertex weights 1..6: coarse triangle with edge weights 5 (0-1: edges 1
    # and 4), 9 (0-2: edges 6 and 3) and 7 (1-2: edges 2 and 5).
    cg = O.contract(to_oracle(_six_cycle()), np.array([0, 1, 2, 0, 1, 2]), 3)
    xadj, adj, ew, vw = cg.arrays()
    np.testing.assert_array_equal(xadj, [0, 2, 4, 6])
    np.testing.assert_array_equal(adj, [1, 2, 0, 2, 0, 1])
    np.testing.assert_array_equal(ew, [5, 9, 5, 7, 9, 7])
    np.testing.assert_array_equal(vw, [5, 7, 9])


def _check_mapping(mp, nc, n):
    assert mp.shape == (n,)
    assert (mp < nc).all()
    counts = np.bincount(mp, minlength=nc)
    assert (counts >= 1).all() and (counts <= 2).all()


@pytest.mark.parametrize("maker,args", [(star, (40,)), (k2n, (30,)), (isolated_plus_path, (50, 9))])
def test_match_special_passes_shrink(maker, args):
    g = maker(*args)
    og = to_oracle(g)
    mp, nc = O.match(og)
    _check_mapping(mp, nc, g.n)
    # Leaves of a star / twins of K_{2,n} / isolated vertices are paired by the
    # leaf, twin and relative passes, so the graph halves (within one vertex
    # per group).
    assert nc <= g.n // 2 + 2
    mp2, nc2 = O.match(og)
    np.testing.assert_array_equal(mp, mp2)
    assert nc == nc2


def test_match_and_contract_preserve_weight():
    g = H.Graph.rmat(12, 8, seed=5)
    og = to_oracle(g)
    mp, nc = O.match(og)
    _check_mapping(mp, nc, g.n)
    cg = O.contract(og, mp, nc)
    xadj, adj, ew, vw = cg.arrays()
    assert cg.n == nc
    w_in = g.n if g.vw is None else int(g.vw.sum())
    assert int(vw.sum()) == w_in
    # Contraction drops intra-cluster edges and sums parallel ones: the total
    # edge weight equals the input weight minus the weight inside clusters.
    rows = np.repeat(np.arange(g.n), np.diff(g.xadj.astype(np.int64)))
    inner = int(g.ew[mp[rows] == mp[g.adj]].astype(np.int64).sum())
    assert int(ew.astype(np.int64).sum()) == int(g.ew.astype(np.int64).sum()) - inner
    crow = np.repeat(np.arange(nc), np.diff(xadj.astype(np.int64)))
    assert (crow != adj).all()


# ---- Jet and whole pipelines (self-consistency of the oracle) -------------------

def test_jet_steps_consistent():
    w = h = 64
    g = H.Graph.grid(w, h, 1, 10, seed=2)
    og = to_oracle(g)
    k = 16
    part = perturb(block_partition_grid(w, h, 4, 4), k, 0.2, 7)
    lm = O.lmax(g.n, k, 0.03)
    jet = O.Jet(og, k, lm, part)
    obj = O.edge_cut(og, part)
    for step in ("lp", "lp", "weak", "strong", "lp"):
        moves = jet.lp(75) if step == "lp" else getattr(jet, step)()
        obj, maxw = jet.perform(moves, obj)
        st = jet.state()
        assert obj == _cut_py(g, st["map"])
        np.testing.assert_array_equal(st["bw"], np.bincount(st["map"], minlength=k))
        assert maxw == st["bw"].max()


def test_partition_pipeline_balanced():
    g = H.Graph.rmat(12, 8, seed=5)
    og = to_oracle(g)
    k = 16
    part, cut = O.partition(og, k, 0.03, False, 1)
    assert cut == _cut_py(g, part)
    bw = np.bincount(part, minlength=k)
    assert len(bw) == k and bw.max() <= O.lmax(g.n, k, 0.03)
    part2, cut2 = O.partition(og, k, 0.03, False, 1)
    np.testing.assert_array_equal(part, part2)


@pytest.mark.parametrize("mode", ["IM", "HM"])
def test_mapping_pipeline_consistent(mode):
    g = H.Graph.rgg3d(5000, 10.0, 1, 100, seed=11)
    og = to_oracle(g)
    hier, dist = [2, 4, 3], [1, 10, 100]
    part, J = (O.map_im(og, hier, dist, 0.03, 1) if mode == "IM" else O.map_hm(og, hier, dist, 0.03, False, 1))
    assert J == _J_py(g, part, _distance_py(hier, dist))
    assert part.max() < 24
