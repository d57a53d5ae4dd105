"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Integer work, so every comparison is exact: mappings, coarse graphs (rows
compared after sorting; the device writes rows in hash-slot order), Jet
gains / destinations / locks / move sets, objectives and final partitions.
"""
import numpy as np
import pytest

import gpu_heipa as H
import oracle as O
from helpers import (block_partition_grid, isolated_plus_path, k2n, perturb, small_graphs, sorted_rows, star,
                     to_oracle)

pytestmark = pytest.mark.gpu

GRAPHS = small_graphs()


@pytest.mark.parametrize("name,g", GRAPHS, ids=[x[0] for x in GRAPHS])
def test_match_parity(ctx, name, g):
    dg = ctx.upload(g)
    try:
        mp, nc = ctx.match(dg)
    finally:
        dg.free()
    omp, onc = O.match(to_oracle(g))
    assert nc == onc
    np.testing.assert_array_equal(mp, omp)


@pytest.mark.parametrize("name,g", GRAPHS, ids=[x[0] for x in GRAPHS])
def test_contract_parity(ctx, name, g):
    og = to_oracle(g)
    omp, onc = O.match(og)
    oc = O.contract(og, omp, onc)
    dg = ctx.upload(g)
    try:
        dc = ctx.contract(dg, omp, onc)
        try:
            cg = dc.download()
        finally:
            dc.free()
    finally:
        dg.free()
    ox, oa, oe, ov = oc.arrays()
    assert cg.n == onc and cg.m == len(oa)
    gx, ga, ge = sorted_rows(cg.xadj, cg.adj, cg.ew)
    np.testing.assert_array_equal(gx, ox)
    np.testing.assert_array_equal(ga, oa)
    np.testing.assert_array_equal(ge, oe)
    np.testing.assert_array_equal(cg.vw, ov)


@pytest.mark.parametrize("group", [3, 4, 7, 512, 2048])
def test_contract_parity_large_clusters(ctx, group):
    # a caller-given mapping with clusters of more than two members (512 and
    # 2048 members: clusters of thousands of entries, the huge tier with its
    # rows cut into work units of many members)
    g = H.Graph.rmat(12, 8, seed=9)
    mapping = (np.arange(g.n) // group).astype(np.uint32)
    n_c = int(mapping.max()) + 1
    dg = ctx.upload(g)
    try:
        dc = ctx.contract(dg, mapping, n_c)
        cg = dc.download()
        dc.free()
    finally:
        dg.free()
    oc = O.contract(to_oracle(g), mapping, n_c)
    ox, oa, oe, ov = oc.arrays()
    gx, ga, ge = sorted_rows(cg.xadj, cg.adj, cg.ew)
    ox, oa, oe = sorted_rows(ox, oa, oe)
    np.testing.assert_array_equal(gx, ox)
    np.testing.assert_array_equal(ga, oa)
    np.testing.assert_array_equal(ge, oe)
    np.testing.assert_array_equal(cg.vw, ov)


def test_contract_kat_six_cycle(ctx):
    # 6-cycle with weights 1..6, vertex weights 1..6, clusters {0,3},{1,4},{2,5}
    n = 6
    edges = {(i, (i + 1) % n): i + 1 for i in range(n)}
    rows = [[] for _ in range(n)]
    for (a, b), w in edges.items():
        rows[a].append((b, w))
        rows[b].append((a, w))
    xadj = np.cumsum([0] + [len(r) for r in rows])
    adj = np.array([v for r in rows for v, _ in r])
    ew = np.array([w for r in rows for _, w in r])
    g = H.Graph(xadj, adj, ew, np.arange(1, 7))
    dg = ctx.upload(g)
    dc = ctx.contract(dg, np.array([0, 1, 2, 0, 1, 2]), 3)
    cg = dc.download()
    dc.free()
    dg.free()
    x, a, e = sorted_rows(cg.xadj, cg.adj, cg.ew)
    np.testing.assert_array_equal(x, [0, 2, 4, 6])
    np.testing.assert_array_equal(a, [1, 2, 0, 2, 0, 1])
    np.testing.assert_array_equal(e, [5, 9, 5, 7, 9, 7])
    np.testing.assert_array_equal(cg.vw, [5, 7, 9])


@pytest.mark.parametrize("maker,args", [(star, (40,)), (k2n, (30,)), (isolated_plus_path, (50, 9))])
def test_match_special_passes(ctx, maker, args):
    g = maker(*args)
    dg = ctx.upload(g)
    mp, nc = ctx.match(dg)
    dg.free()
    omp, onc = O.match(to_oracle(g))
    assert nc == onc
    np.testing.assert_array_equal(mp, omp)


def _jet_compare(st_gpu, st_or, keys=("map", "bw", "dest_part", "gain1", "lock", "dest_cache", "gain_cache")):
    for k in keys:
        np.testing.assert_array_equal(st_gpu[k], st_or[k], err_msg=k)


@pytest.mark.parametrize("objective", ["cut", "J"])
def test_jet_steps_grid(ctx, objective):
    g = H.Graph.grid(96, 96, 1, 10, seed=2)
    k = 16
    hier, dist = ([4, 4], [1, 10]) if objective == "J" else (None, None)
    part = perturb(block_partition_grid(96, 96, 4, 4), k, 0.08, seed=1)
    og = to_oracle(g)
    lmax = O.lmax(g.total_weight(), k, 0.03)
    obj = O.edge_cut(og, part) if objective == "cut" else O.comm_cost(og, part, hier, dist)
    dg = ctx.upload(g)
    jet = ctx.jet(dg, k, lmax, part, hier, dist)
    oj = O.Jet(og, k, lmax, part, hier, dist)
    o_gpu = o_or = obj
    try:
        for step, ratio in enumerate([25, 25, 75, 75, 25, 25]):
            mg = jet.lp(ratio)
            mo = oj.lp(ratio)
            np.testing.assert_array_equal(mg, np.sort(mo), err_msg=f"moves step {step}")
            _jet_compare(jet.state(), oj.state())
            o_gpu, w_gpu = jet.perform(o_gpu)
            o_or, w_or = oj.perform(mo, o_or)
            assert (o_gpu, w_gpu) == (o_or, w_or)
            _jet_compare(jet.state(), oj.state())
        # the tracked objective equals the recomputed one
        fin = jet.state()["map"]
        exp = O.edge_cut(og, fin) if objective == "cut" else O.comm_cost(og, fin, hier, dist)
        assert o_gpu == exp
    finally:
        jet.close()
        dg.free()


@pytest.mark.parametrize("gname", ["grid", "rmat"])
@pytest.mark.parametrize("objective", ["cut", "J"])
def test_rebalance_parity(ctx, gname, objective):
    if gname == "grid":
        g = H.Graph.grid(80, 80, 1, 10, seed=4)
        part = block_partition_grid(80, 80, 4, 4)
    else:
        g = H.Graph.rmat(13, 8, seed=9)
        part = (np.arange(g.n) % 16).astype(np.uint32)
    k = 16
    # overload blocks 0 and 5 by moving vertices into them
    rng = np.random.default_rng(3)
    idx = rng.choice(g.n, g.n // 6, replace=False)
    part = part.copy()
    part[idx[: len(idx) // 2]] = 0
    part[idx[len(idx) // 2:]] = 5
    hier, dist = ([4, 4], [1, 10]) if objective == "J" else (None, None)
    og = to_oracle(g)
    lmax = O.lmax(g.total_weight(), k, 0.03)
    obj = O.edge_cut(og, part) if objective == "cut" else O.comm_cost(og, part, hier, dist)
    dg = ctx.upload(g)
    jet = ctx.jet(dg, k, lmax, part, hier, dist)
    oj = O.Jet(og, k, lmax, part, hier, dist)
    o_gpu = o_or = obj
    try:
        for step, kind in enumerate(["weak", "weak", "strong", "strong", "weak"]):
            mg = getattr(jet, kind)()
            mo = getattr(oj, kind)()
            np.testing.assert_array_equal(mg, np.sort(mo), err_msg=f"{kind} step {step}")
            sg, so = jet.state(), oj.state()
            np.testing.assert_array_equal(sg["dest_part"][mo], so["dest_part"][mo], err_msg="dest")
            o_gpu, w_gpu = jet.perform(o_gpu)
            o_or, w_or = oj.perform(mo, o_or)
            assert (o_gpu, w_gpu) == (o_or, w_or)
            _jet_compare(jet.state(), oj.state(), ("map", "bw", "dest_cache"))
    finally:
        jet.close()
        dg.free()


# Level-loop implementations of jet_refine: one block, a cooperative grid, or
# one launch (graph) per step.
LOOP_TUNES = {"block": {"jet_fused_max_n": 65536, "jet_fused_max_m": 1 << 30, "jet_coop_max_n": 0},
              "grid": {"jet_fused_max_n": 0, "jet_coop_max_n": 65536, "jet_coop_max_m": 1 << 30,
                       "jet_coop_max_deg": 1 << 20},
              "kernels": {"jet_fused_max_n": 0, "jet_coop_max_n": 0}}


@pytest.mark.parametrize("loop", sorted(LOOP_TUNES))
@pytest.mark.parametrize("ultra", [False, True])
def test_jet_refine_parity(ctx, ultra, loop):
    g = H.Graph.rmat(13, 8, seed=21)
    k = 32
    og = to_oracle(g)
    part = (np.arange(g.n) * 7 % k).astype(np.uint32)
    lmax = O.lmax(g.total_weight(), k, 0.03)
    cut = O.edge_cut(og, part)
    maxw = int(np.bincount(part, minlength=k).max())
    c = H.Context(0, 1 << 30)
    try:
        for name, v in LOOP_TUNES[loop].items():
            c.tune(name, v)
        dg = c.upload(g)
        try:
            pg, cg, wg = c.jet_refine(dg, k, lmax, part, cut, maxw, ultra=ultra, level=1)
        finally:
            dg.free()
    finally:
        c.close()
    po, co, wo = O.jet_refine(og, k, lmax, ultra, 1, part, cut, maxw)
    assert (cg, wg) == (co, wo)
    np.testing.assert_array_equal(pg, po)
    assert cg == O.edge_cut(og, pg)


@pytest.mark.parametrize("loop", sorted(LOOP_TUNES))
def test_level_loops_pipelines(ctx, loop):
    # whole pipelines (cut and J objectives, default and ultra) with every
    # level of at most 65536 vertices on one level-loop implementation
    cases = [(H.Graph.grid(200, 150), 16, "default"), (H.Graph.rmat(15, 8, seed=5), 64, "ultra")]
    m = H.Graph.rgg3d(40000, 14.0, 1, 100, seed=8, explicit_vw=True)
    c = H.Context(0, 2 << 30)
    try:
        for name, v in LOOP_TUNES[loop].items():
            c.tune(name, v)
        for g, k, config in cases:
            part, cut = c.partition(g, k, 0.03, config, 7)
            opart, ocut = O.partition(to_oracle(g), k, 0.03, config == "ultra", 7)
            assert cut == ocut
            np.testing.assert_array_equal(part, opart)
        om = to_oracle(m)
        for mode in ("IM", "HM"):
            mp, J = c.process_map(m, [2, 4, 3], [1, 10, 100], 0.03, mode, 3)
            if mode == "IM":
                want_m, want_j = O.map_im(om, [2, 4, 3], [1, 10, 100], 0.03, 3)
            else:
                want_m, want_j = O.map_hm(om, [2, 4, 3], [1, 10, 100], 0.03, False, 3)
            assert J == want_j
            np.testing.assert_array_equal(mp, want_m)
    finally:
        c.close()


@pytest.mark.parametrize("name,g,k", [("grid256_k16", H.Graph.grid(256, 256), 16),
                                      ("rmat14_k64", H.Graph.rmat(14, 16, seed=3), 64),
                                      ("rgg_k8", H.Graph.rgg3d(30000, 14.0, 1, 100, seed=4), 8)],
                         ids=["grid256_k16", "rmat14_k64", "rgg_k8"])
def test_partition_pipeline_parity(ctx, name, g, k):
    part, cut = ctx.partition(g, k, 0.03, "default", seed=7)
    opart, ocut = O.partition(to_oracle(g), k, 0.03, False, 7)
    assert cut == ocut
    np.testing.assert_array_equal(part, opart)
    # exact checks on the output
    og = to_oracle(g)
    assert O.edge_cut(og, part) == cut
    bw = np.bincount(part, weights=(None if g.vw is None else g.vw), minlength=k)
    assert part.max() < k
    assert bw.max() <= O.lmax(g.total_weight(), k, 0.03)


@pytest.mark.parametrize("mode", ["IM", "HM", "HM-ultra"])
def test_mapping_pipeline_parity(ctx, mode):
    g = H.Graph.rgg3d(20000, 14.0, 1, 100, seed=8, explicit_vw=True)
    hier, dist = [2, 4, 3], [1, 10, 100]
    part, J = ctx.process_map(g, hier, dist, 0.03, mode, seed=3)
    og = to_oracle(g)
    if mode == "IM":
        opart, oJ = O.map_im(og, hier, dist, 0.03, 3)
    else:
        opart, oJ = O.map_hm(og, hier, dist, 0.03, mode == "HM-ultra", 3)
    assert J == oJ
    np.testing.assert_array_equal(part, opart)
    assert O.comm_cost(og, part, hier, dist) == J


def test_edge_cases(ctx):
    # empty graph, isolated vertices only, k = 1, k > n
    e = H.Graph(np.zeros(1, np.uint32), np.zeros(0, np.uint32))
    p, c = ctx.partition(e, 4)
    assert len(p) == 0 and c == 0
    iso = isolated_plus_path(300, 0)
    p, c = ctx.partition(iso, 4, seed=1)
    op, oc = O.partition(to_oracle(iso), 4, 0.03, False, 1)
    np.testing.assert_array_equal(p, op)
    assert c == 0
    g = H.Graph.grid(20, 20)
    p, c = ctx.partition(g, 1)
    assert c == 0 and (p == 0).all()
    p, c = ctx.partition(H.Graph.grid(3, 3), 16, seed=2)
    op, oc = O.partition(to_oracle(H.Graph.grid(3, 3)), 16, 0.03, False, 2)
    np.testing.assert_array_equal(p, op)


def test_invalid_inputs_rejected(ctx):
    bad = H.Graph(np.array([0, 1, 1]), np.array([5]))  # neighbour id out of range
    with pytest.raises(H.HeiPaError):
        ctx.upload(bad)
    loop = H.Graph(np.array([0, 1]), np.array([0]))  # self loop
    with pytest.raises(H.HeiPaError):
        ctx.upload(loop)
    zero_w = H.Graph(np.array([0, 1, 2]), np.array([1, 0]), np.array([0, 0]))
    with pytest.raises(H.HeiPaError):
        ctx.upload(zero_w)
    assert "invalid graph" in ctx.last_error()


def test_direct_launch_paths_equal(ctx):
    # Small test graphs take the CUDA-graph, single-block-ordering and
    # cooperative-matching paths; force the per-kernel launch paths of large
    # levels and require the same results.
    g = H.Graph.rmat(14, 16, seed=3)
    m = H.Graph.rgg3d(20000, 14.0, 1, 100, seed=8, explicit_vw=True)
    want_p, want_c = O.partition(to_oracle(g), 64, 0.03, False, 7)
    want_m, want_j = O.map_hm(to_oracle(m), [2, 4, 3], [1, 10, 100], 0.03, False, 3)
    c2 = H.Context(0, 2 << 30)
    try:
        for name in ("jet_graph_max_m", "order_small_n", "match_coop_max_n", "match_coop_max_m", "jet_fused_max_n",
                     "jet_coop_max_n"):
            c2.tune(name, 0)
        c2.tune("jet_hub_deg", 4096)
        part, cut = c2.partition(g, 64, 0.03, "default", 7)
        assert cut == want_c
        np.testing.assert_array_equal(part, want_p)
        mp, J = c2.process_map(m, [2, 4, 3], [1, 10, 100], 0.03, "HM", 3)
        assert J == want_j
        np.testing.assert_array_equal(mp, want_m)
        with pytest.raises(H.HeiPaError):
            c2.tune("no_such_threshold", 1)
    finally:
        c2.close()


@pytest.mark.parametrize("mode", [1, 2])
def test_chunk_modes_equal_oracle(mode):
    # The chunk kernels of the per-kernel Jet path with eight entries per
    # lane (1) or with bulk-copy staged row segments (2), on weighted and
    # unit-weight graphs with hub rows, and on the mapping objective.
    cases = [(H.Graph.rmat(15, 16, 0.57, 0.19, 0.19, 1, 10, 3), 64), (H.Graph.rmat(14, 16, seed=3), 32)]
    m = H.Graph.rgg3d(20000, 14.0, 1, 100, seed=8, explicit_vw=True)
    c = H.Context(0, 2 << 30)
    try:
        for name in ("jet_fused_max_n", "jet_coop_max_n"):
            c.tune(name, 0)
        c.tune("jet_chunk_mode", mode)
        for g, k in cases:
            part, cut = c.partition(g, k, 0.03, "default", 7)
            opart, ocut = O.partition(to_oracle(g), k, 0.03, False, 7)
            assert cut == ocut
            np.testing.assert_array_equal(part, opart)
        mp, J = c.process_map(m, [2, 4, 3], [1, 10, 100], 0.03, "IM", 3)
        want_m, want_j = O.map_im(to_oracle(m), [2, 4, 3], [1, 10, 100], 0.03, 3)
        assert J == want_j
        np.testing.assert_array_equal(mp, want_m)
        with pytest.raises(H.HeiPaError):
            c.tune("jet_chunk_mode", 3)
    finally:
        c.close()


def test_scalar_row_reads_equal_oracle():
    # The Jet row passes with four strided 4-byte loads per lane instead of
    # 16-byte quads (jet_vec_loads = 0): weighted and unit-weight R-MAT with
    # hub rows, a grid, and J.
    cases = [(H.Graph.rmat(15, 16, 0.57, 0.19, 0.19, 1, 10, 3), 64, "default"),
             (H.Graph.rmat(14, 16, seed=3), 32, "ultra"), (H.Graph.grid(120, 100, 1, 10, seed=4), 16, "default")]
    m = H.Graph.rgg3d(20000, 14.0, 1, 100, seed=8, explicit_vw=True)
    c = H.Context(0, 2 << 30)
    try:
        for name in ("jet_fused_max_n", "jet_coop_max_n"):
            c.tune(name, 0)
        c.tune("jet_vec_loads", 0)
        for g, k, config in cases:
            part, cut = c.partition(g, k, 0.03, config, 7)
            opart, ocut = O.partition(to_oracle(g), k, 0.03, config == "ultra", 7)
            assert cut == ocut
            np.testing.assert_array_equal(part, opart)
        mp, J = c.process_map(m, [2, 4, 3], [1, 10, 100], 0.03, "IM", 3)
        want_m, want_j = O.map_im(to_oracle(m), [2, 4, 3], [1, 10, 100], 0.03, 3)
        assert J == want_j
        np.testing.assert_array_equal(mp, want_m)
        with pytest.raises(H.HeiPaError):
            c.tune("jet_vec_loads", 2)
    finally:
        c.close()


@pytest.mark.parametrize("pct", [1, 100])
def test_cache_reset_threshold_equal_oracle(pct):
    # A perform resets every cached gain at once when its moved rows hold at
    # least pct % of the level's entries (1: nearly every perform; 100: only
    # when every row moved), else the neighbours of the moved rows one by
    # one; cut (default and ultra, whose changing filter ratio keeps the
    # scattered resets) and J.
    cases = [(H.Graph.rmat(15, 16, 0.57, 0.19, 0.19, 1, 10, 3), 64, "default"),
             (H.Graph.rmat(14, 16, seed=3), 32, "ultra"), (H.Graph.grid(120, 100, 1, 10, seed=4), 16, "default")]
    m = H.Graph.rgg3d(20000, 14.0, 1, 100, seed=8, explicit_vw=True)
    c = H.Context(0, 2 << 30)
    try:
        for name in ("jet_fused_max_n", "jet_coop_max_n"):
            c.tune(name, 0)
        c.tune("jet_inval_all_pct", pct)
        for g, k, config in cases:
            part, cut = c.partition(g, k, 0.03, config, 7)
            opart, ocut = O.partition(to_oracle(g), k, 0.03, config == "ultra", 7)
            assert cut == ocut
            np.testing.assert_array_equal(part, opart)
        mp, J = c.process_map(m, [2, 4, 3], [1, 10, 100], 0.03, "HM", 3)
        want_m, want_j = O.map_hm(to_oracle(m), [2, 4, 3], [1, 10, 100], 0.03, False, 3)
        assert J == want_j
        np.testing.assert_array_equal(mp, want_m)
        for bad in (0, 101):
            with pytest.raises(H.HeiPaError):
                c.tune("jet_inval_all_pct", bad)
    finally:
        c.close()


@pytest.mark.parametrize("hub_conn", [0, 1])
def test_hub_rows_tracked_or_rescanned_equal_oracle(hub_conn):
    # The per-kernel Jet path with every row above 64 entries a hub: the hub
    # connectivity either kept up to date by the delta pass (1) or rebuilt
    # from the rows on every pass (0); cut (default and ultra) and J.
    cases = [(H.Graph.rmat(15, 16, 0.57, 0.19, 0.19, 1, 10, 3), 64, "default"),
             (H.Graph.rmat(14, 16, seed=3), 32, "ultra"), (H.Graph.grid(120, 100, 1, 10, seed=4), 16, "default")]
    m = H.Graph.rgg3d(20000, 40.0, 1, 100, seed=8, explicit_vw=True)
    c = H.Context(0, 2 << 30)
    try:
        for name in ("jet_fused_max_n", "jet_coop_max_n"):
            c.tune(name, 0)
        c.tune("jet_hub_deg", 64)
        c.tune("jet_hub_conn", hub_conn)
        for g, k, config in cases:
            part, cut = c.partition(g, k, 0.03, config, 7)
            opart, ocut = O.partition(to_oracle(g), k, 0.03, config == "ultra", 7)
            assert cut == ocut
            np.testing.assert_array_equal(part, opart)
        mp, J = c.process_map(m, [2, 4, 3], [1, 10, 100], 0.03, "IM", 3)
        want_m, want_j = O.map_im(to_oracle(m), [2, 4, 3], [1, 10, 100], 0.03, 3)
        assert J == want_j
        np.testing.assert_array_equal(mp, want_m)
    finally:
        c.close()


def test_arena_exhaustion_is_an_error():
    small = H.Context(0, 64 << 20)
    try:
        g = H.Graph.rmat(16, 16, seed=1)
        with pytest.raises(H.HeiPaError) as e:
            small.partition(g, 8)
        assert e.value.code == 3
        # the context stays usable for a graph that fits
        p, c = small.partition(H.Graph.grid(32, 32), 4, seed=1)
        op, oc = O.partition(to_oracle(H.Graph.grid(32, 32)), 4, 0.03, False, 1)
        np.testing.assert_array_equal(p, op)
        assert c == oc
    finally:
        small.close()
