"""Checks against the committed golden vectors (tests/golden/golden.json,
written by tests/golden/make_golden.py): the oracle on the CPU, and the CUDA
path through the C ABI on the GPU."""
import hashlib
import json
import os

import numpy as np
import pytest

import gpu_heipa as H
import oracle as O
from golden.make_golden import GRAPHS, make_graph

GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")))


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()


def _og(g):
    return O.Graph(g.xadj, g.adj, g.ew, g.vw)


# ---- CPU: the oracle reproduces the golden vectors ------------------------------

def test_golden_murmur3():
    for key, seed, want in GOLDEN["murmur3"]:
        assert O.murmur3_u32(key, seed) == want


def test_golden_distance_pairs():
    d = GOLDEN["distance"]
    D = O.distance_matrix(d["hier"], d["dist"])
    for a, b, want in d["pairs"]:
        assert D[a, b] == want and D[b, a] == want


def test_golden_six_cycle():
    kat = GOLDEN["six_cycle_contraction"]
    rows = [[] for _ in range(6)]
    for i in range(6):
        rows[i].append(((i + 1) % 6, i + 1))
        rows[(i + 1) % 6].append((i, i + 1))
    xadj = np.cumsum([0] + [len(r) for r in rows])
    g = H.Graph(xadj, [v for r in rows for v, _ in r], [w for r in rows for _, w in r], np.arange(1, 7))
    cx, ca, ce, cv = O.contract(_og(g), np.array(kat["mapping"]), 3).arrays()
    assert cx.tolist() == kat["xadj"] and ca.tolist() == kat["adj"]
    assert ce.tolist() == kat["ew"] and cv.tolist() == kat["vw"]


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_golden_inputs_and_match(name):
    g = make_graph(H, name)
    want = GOLDEN["graphs"][name]
    assert (g.n, g.m, digest(g.adj)) == (want["n"], want["m"], want["adj_sha256"])
    mp, nc = O.match(_og(g))
    wm = GOLDEN["match"][name]
    assert nc == wm["n_coarse"] and digest(mp) == wm["mapping_sha256"]
    assert O.contract(_og(g), mp, nc).m == wm["coarse_m"]


@pytest.mark.parametrize("case", sorted(GOLDEN["partition"]))
def test_golden_partition_oracle(case):
    c = GOLDEN["partition"][case]
    part, cut = O.partition(_og(make_graph(H, c["graph"])), c["k"], 0.03, False, c["seed"])
    assert cut == c["cut"] and digest(part) == c["part_sha256"]


@pytest.mark.parametrize("case", sorted(GOLDEN["mapping"]))
def test_golden_mapping_oracle(case):
    c = GOLDEN["mapping"][case]
    og = _og(make_graph(H, c["graph"]))
    if c["mode"] == "IM":
        part, J = O.map_im(og, c["hier"], c["dist"], 0.03, c["seed"])
    else:
        part, J = O.map_hm(og, c["hier"], c["dist"], 0.03, c["mode"] == "HM-ultra", c["seed"])
    assert J == c["J"] and digest(part) == c["part_sha256"]


# ---- GPU: the CUDA path reproduces the golden vectors ---------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_golden_match_gpu(ctx, name):
    g = make_graph(H, name)
    dg = ctx.upload(g)
    try:
        mp, nc = ctx.match(dg)
    finally:
        dg.free()
    wm = GOLDEN["match"][name]
    assert nc == wm["n_coarse"] and digest(mp) == wm["mapping_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(GOLDEN["partition"]))
def test_golden_partition_gpu(ctx, case):
    c = GOLDEN["partition"][case]
    part, cut = ctx.partition(make_graph(H, c["graph"]), c["k"], 0.03, "default", c["seed"])
    assert cut == c["cut"] and digest(part) == c["part_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(GOLDEN["mapping"]))
def test_golden_mapping_gpu(ctx, case):
    c = GOLDEN["mapping"][case]
    part, J = ctx.process_map(make_graph(H, c["graph"]), c["hier"], c["dist"], 0.03, c["mode"], c["seed"])
    assert J == c["J"] and digest(part) == c["part_sha256"]
