"""Bounded waits: a grid barrier whose partner block never arrives ends with
an error bit instead of hanging, and the device stays usable.

The failure is made on the device without any fault: one block of a
cooperative launch simply returns before the barrier (a flag that nothing
sets), so the others' bounded wait runs out.

Cooperative launches take a per-device slot first (one such grid at a time),
so concurrent solves whose level loops all run as full-device cooperative
grids never wait for each other's SMs.
"""
import threading
import time

import numpy as np
import pytest

import gpu_heipa as H
import oracle as O
from helpers import to_oracle


def test_selftest_rejects_bad_arguments():
    # checked before any device call
    with pytest.raises(H.HeiPaError):
        H.selftest_barrier_timeout(0, 1)


@pytest.mark.gpu
def test_grid_barrier_wait_is_bounded(ctx):
    t0 = time.perf_counter()
    err, ms = H.selftest_barrier_timeout(0, 4)
    wall = time.perf_counter() - t0
    assert err & H.DEVERR_SPIN
    assert 50.0 < ms < 30000.0 and wall < 60.0
    # the context and the device remain usable: an exact partition afterwards
    g = H.Graph.grid(64, 64)
    part, cut = ctx.partition(g, 8, 0.03, "default", 1)
    opart, ocut = O.partition(to_oracle(g), 8, 0.03, False, 1)
    assert cut == ocut
    np.testing.assert_array_equal(part, opart)


def test_coop_slot_is_exclusive():
    # host-side logic only: one holder per device; a waiter gets the slot
    # when the holder returns it; devices are independent
    dev = 7
    assert H.coop_slot_acquire(dev, 0)
    try:
        assert not H.coop_slot_acquire(dev, 50)
        assert H.coop_slot_acquire(dev + 1, 0)
        H.coop_slot_release(dev + 1)
        got = []
        t = threading.Thread(target=lambda: got.append(H.coop_slot_acquire(dev, 5000)))
        t.start()
        time.sleep(0.2)
        assert not got  # still waiting while the slot is held
        H.coop_slot_release(dev)
        t.join(10)
        assert got == [True]
    finally:
        H.coop_slot_release(dev)
    assert H.coop_slot_acquire(dev, 0)
    H.coop_slot_release(dev)


@pytest.mark.gpu
def test_concurrent_cooperative_grids(ctx):
    # Every small level runs its matching loop and Jet level loop as one
    # cooperative grid as large as the device holds (one block per vertex),
    # in concurrent HM sub-solves and concurrent batch requests. No solve may
    # fail, and every result must equal the oracle's.
    c = H.Context(0, 4 << 30)
    try:
        c.tune("jet_coop_rows", 1)
        c.tune("jet_coop_max_deg", 1 << 20)
        c.tune("match_coop_max_n", 1 << 17)
        c.tune("match_coop_max_m", 1 << 30)
        m = H.Graph.rgg3d(40000, 14.0, 1, 100, seed=8, explicit_vw=True)
        part, J = c.process_map(m, [2, 4, 3], [1, 10, 100], 0.03, "HM", 3)
        opart, oJ = O.map_hm(to_oracle(m), [2, 4, 3], [1, 10, 100], 0.03, False, 3)
        assert J == oJ
        np.testing.assert_array_equal(part, opart)
        graphs = [H.Graph.grid(80, 60), H.Graph.rmat(12, 8, seed=2), H.Graph.rgg3d(15000, 10.0, 1, 10, seed=3),
                  H.Graph.rmat(13, 8, seed=5)]
        ks = [4, 8, 16, 32]
        out = c.partition_batch(graphs, ks, 0.03, "default", 1, workers=4)
        for g, k, (p, cut) in zip(graphs, ks, out):
            op, ocut = O.partition(to_oracle(g), k, 0.03, False, 1)
            assert cut == ocut
            np.testing.assert_array_equal(p, op)
    finally:
        c.close()
