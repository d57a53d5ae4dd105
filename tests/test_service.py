"""Batched and served requests (hp_partition_batch, hp_server_*): every
result must equal the plain call's on the same input, whether the request
runs alone or concurrently with others."""
import numpy as np
import pytest

import gpu_heipa as H
import oracle as O
from conftest import has_gpu
from helpers import to_oracle


def _mix():
    return [H.Graph.grid(64, 40), H.Graph.rmat(12, 8, seed=2), H.Graph.rgg3d(15000, 10.0, 1, 10, seed=3),
            H.Graph.grid(100, 100, 1, 10, seed=4), H.Graph.rmat(13, 8, seed=5), H.Graph.rgg3d(30000, 10.0, 1, 10, seed=6),
            H.Graph.grid(20, 300), H.Graph.rmat(11, 16, seed=7)]


@pytest.mark.gpu
def test_batch_equals_plain(ctx):
    graphs = _mix()
    ks = [2, 4, 8, 16, 32, 64, 128, 256]
    out = ctx.partition_batch(graphs, ks, 0.03, "default", 1, workers=4)
    for g, k, (part, cut) in zip(graphs, ks, out):
        want, wcut = ctx.partition(g, k, 0.03, "default", 1)
        np.testing.assert_array_equal(part, want)
        assert cut == wcut
        opart, ocut = O.partition(to_oracle(g), k, 0.03, False, 1)
        np.testing.assert_array_equal(part, opart)
        assert cut == ocut


@pytest.mark.gpu
def test_server_mix_equals_alone(ctx):
    graphs = _mix()
    with H.Server(0, 2 << 30, workers=4) as srv:
        reqs = []
        for i, g in enumerate(graphs):
            if i % 3 == 2:
                reqs.append(("map", g, srv.submit_map(g, [2, 2, 2], [1, 10, 100], 0.03, "HM", 1)))
            else:
                reqs.append(("part", g, srv.submit_partition(g, 8 << (i % 3), 0.03, "default", 1)))
        mixed = [srv.wait(r) for _, _, r in reqs]
        # the same requests alone (one at a time) on the same server
        for (kind, g, _), (part, obj, lat, run) in zip(reqs, mixed):
            assert lat >= run >= 0
            i = graphs.index(g)
            if kind == "map":
                alone = srv.wait(srv.submit_map(g, [2, 2, 2], [1, 10, 100], 0.03, "HM", 1))
                want, wobj = ctx.process_map(g, [2, 2, 2], [1, 10, 100], 0.03, "HM", 1)
            else:
                alone = srv.wait(srv.submit_partition(g, 8 << (i % 3), 0.03, "default", 1))
                want, wobj = ctx.partition(g, 8 << (i % 3), 0.03, "default", 1)
            np.testing.assert_array_equal(part, alone[0])
            np.testing.assert_array_equal(part, want)
            assert obj == alone[1] == wobj


@pytest.mark.gpu
def test_server_rejects_oversized_request():
    with H.Server(0, 64 << 20, workers=2) as srv:
        g = H.Graph.rmat(16, 16, seed=1)
        rid = srv.submit_partition(g, 8)
        with pytest.raises(H.HeiPaError) as e:
            srv.wait(rid)
        assert e.value.code == 3
        # the server keeps working for requests that fit
        small = H.Graph.grid(32, 32)
        part, cut, _, _ = srv.wait(srv.submit_partition(small, 4))
        assert len(part) == small.n and cut > 0


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_server_without_device_is_an_error():
    with pytest.raises(H.HeiPaError):
        H.Server(0, 1 << 20, 2)


@pytest.mark.gpu
def test_autotune_keeps_results(ctx):
    import autotune
    graphs = [H.Graph.grid(60, 60), H.Graph.rgg3d(8000, 10.0, 1, 10, seed=2)]
    ks = [8, 16]
    before = [ctx.partition(g, k, 0.03, "default", 1) for g, k in zip(graphs, ks)]
    small = {"jet_graph_max_m": [0, 1 << 24], "order_small_n": [0, 4096], "match_coop_max_n": [0, 1 << 17],
             "match_coop_max_m": [1 << 21], "jet_fused_max_n": [0, 8192]}
    best = autotune.tune(ctx, graphs, ks, candidates=small, repeats=1)
    assert set(best) == set(autotune.DEFAULTS)
    after = [ctx.partition(g, k, 0.03, "default", 1) for g, k in zip(graphs, ks)]
    for (p0, c0), (p1, c1) in zip(before, after):
        np.testing.assert_array_equal(p0, p1)
        assert c0 == c1
    for name, v in autotune.DEFAULTS.items():  # leave the session context as it was
        ctx.tune(name, v)
