"""hp_edge_cut_noalloc: the edge cut of a caller-owned device CSR computed in
a fixed static scratch area, checked against the arena-backed hp_edge_cut and
against the CPU oracle's edge_cut on the same graph and partitions, two calls
in a row. The graph arrays live in PyTorch CUDA tensors, i.e. in memory the
library does not own.

This file is named to be collected last, so the entry point also runs after
every other GPU test has used the library on the same device."""
import numpy as np
import pytest

import gpu_heipa as H
import oracle as O

pytestmark = pytest.mark.gpu


def _device_csr(g):
    import torch
    xadj = torch.from_numpy(g.xadj.view(np.int32).copy()).cuda()
    adj = torch.from_numpy(g.adj.view(np.int32).copy()).cuda()
    ew = None if g.ew is None else torch.from_numpy(g.ew.copy()).cuda()
    torch.cuda.synchronize()
    return xadj, adj, ew


def _ptrs(xadj, adj, ew):
    return xadj.data_ptr(), adj.data_ptr(), (None if ew is None else ew.data_ptr())


@pytest.mark.parametrize("gname", ["rmat14_weighted", "grid_unit"])
def test_noalloc_matches_edge_cut_two_calls(ctx, gname):
    import torch
    if gname == "rmat14_weighted":
        g = H.Graph.rmat(14, 16, 0.57, 0.19, 0.19, 1, 10, 3)
        assert g.ew is not None
    else:
        g = H.Graph.grid(128, 96)
        assert g.ew is None
    dg = ctx.upload(g)
    try:
        xadj, adj, ew = _device_csr(g)
        px, pa, pw = _ptrs(xadj, adj, ew)
        rng = np.random.default_rng(11)
        parts = [rng.integers(0, 16, g.n, dtype=np.uint32), rng.integers(0, 64, g.n, dtype=np.uint32)]
        side = torch.cuda.Stream()
        streams = [0, side.cuda_stream]  # first call on the default stream, second on a side stream
        og = O.Graph(g.xadj, g.adj, g.ew, g.vw)
        for part, st in zip(parts, streams):
            got = H.edge_cut_noalloc(g.n, g.m, px, pa, pw, part, stream=st)
            want = O.edge_cut(og, part)
            assert got == want
            assert ctx.edge_cut(dg, part) == want
            assert got > 0
        # A partition with every vertex in one block has no cut.
        assert H.edge_cut_noalloc(g.n, g.m, px, pa, pw, np.zeros(g.n, np.uint32)) == 0
    finally:
        dg.free()


def test_noalloc_rejects_bad_input(ctx):
    g = H.Graph.grid(64, 64, 1, 9, 5)
    xadj, adj, ew = _device_csr(g)
    px, pa, pw = _ptrs(xadj, adj, ew)
    part = (np.arange(g.n) % 8).astype(np.uint32)
    want = H.edge_cut_noalloc(g.n, g.m, px, pa, pw, part)

    # Too many vertices: refused on the host before any device work.
    big = np.zeros(H.EDGE_CUT_NOALLOC_MAX_N + 1, np.uint32)
    with pytest.raises(H.HeiPaError) as e:
        H.edge_cut_noalloc(len(big), g.m, px, pa, pw, big)
    assert e.value.code == 7

    # Host memory where device memory is expected: refused on the host.
    with pytest.raises(H.HeiPaError) as e:
        H.edge_cut_noalloc(g.n, g.m, g.xadj.ctypes.data, pa, pw, part)
    assert e.value.code == 1

    # An out-of-range neighbour id: the kernel skips it and reports it.
    bad = adj.clone()
    bad[5] = g.n
    with pytest.raises(H.HeiPaError) as e:
        H.edge_cut_noalloc(g.n, g.m, px, bad.data_ptr(), pw, part)
    assert e.value.code == 5

    # A negative edge weight: rejected like hp_graph_upload rejects it.
    neg = ew.clone()
    neg[7] = -3
    with pytest.raises(H.HeiPaError) as e:
        H.edge_cut_noalloc(g.n, g.m, px, pa, neg.data_ptr(), part)
    assert e.value.code == 5

    # The partition must be host memory: a device pointer is refused (raw C
    # ABI call; the Python wrapper only takes host arrays).
    import ctypes
    import torch
    dpart = torch.from_numpy(part.view(np.int32).copy()).cuda()
    out = ctypes.c_int64(-1)
    rc = H._L.hp_edge_cut_noalloc(g.n, g.m, px, pa, pw, ctypes.c_void_p(dpart.data_ptr()), None, ctypes.byref(out))
    assert rc == 1 and out.value == -1

    # The scratch counters are cleared by every call: a good call after the
    # failures gives the same result as before.
    assert H.edge_cut_noalloc(g.n, g.m, px, pa, pw, part) == want
    assert want == O.edge_cut(O.Graph(g.xadj, g.adj, g.ew, g.vw), part)
    dg = ctx.upload(g)
    try:
        assert want == ctx.edge_cut(dg, part)
    finally:
        dg.free()
