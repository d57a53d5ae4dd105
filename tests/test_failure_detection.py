"""Bounded waits: a grid barrier whose partner block never arrives ends with
an error bit instead of hanging, and the device stays usable.

The failure is made on the device without any fault: one block of a
cooperative launch simply returns before the barrier (a flag that nothing
sets), so the others' bounded wait runs out.
"""
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
