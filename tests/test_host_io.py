"""CPU checks of the host side of the library: METIS reader/writer, the
partition writer and the synthetic workload generators. No GPU needed."""
import os

import numpy as np
import pytest

import gpu_heipa as H


def _edge_set(g):
    rows = np.repeat(np.arange(g.n), np.diff(g.xadj.astype(np.int64)))
    w = np.ones(g.m, np.int64) if g.ew is None else g.ew
    return rows, g.adj.astype(np.int64), w


def _assert_symmetric_simple(g):
    u, v, w = _edge_set(g)
    assert (u != v).all(), "self loop"
    key = u * g.n + v
    assert len(np.unique(key)) == g.m, "parallel edges"
    fwd = dict(zip(key.tolist(), np.asarray(w).tolist()))
    rev = (v * g.n + u).tolist()
    assert all(fwd.get(r) == x for r, x in zip(rev, np.asarray(w).tolist())), "asymmetric edge or weight"


def test_grid_generator():
    for w, h in [(1, 1), (1, 7), (5, 3), (64, 48)]:
        g = H.Graph.grid(w, h)
        assert g.n == w * h
        assert g.m == 2 * ((w - 1) * h + (h - 1) * w)
        assert g.ew is None and g.vw is None
        if g.m:
            _assert_symmetric_simple(g)
        assert np.diff(g.xadj.astype(np.int64)).max(initial=0) <= 4
    g = H.Graph.grid(20, 30, 1, 9, seed=3)
    assert g.ew is not None and g.ew.min() >= 1 and g.ew.max() <= 9
    _assert_symmetric_simple(g)


def test_rmat_generator():
    g = H.Graph.rmat(12, 8, 0.57, 0.19, 0.19, 1, 10, seed=5)
    assert g.n == 1 << 12
    assert g.ew.min() >= 1 and g.ew.max() <= 10
    _assert_symmetric_simple(g)
    # Deterministic per seed; another seed gives another graph.
    g2 = H.Graph.rmat(12, 8, 0.57, 0.19, 0.19, 1, 10, seed=5)
    np.testing.assert_array_equal(g.adj, g2.adj)
    np.testing.assert_array_equal(g.ew, g2.ew)
    g3 = H.Graph.rmat(12, 8, 0.57, 0.19, 0.19, 1, 10, seed=6)
    assert g3.m != g.m or not np.array_equal(g3.adj, g.adj)
    # Skewed degrees: the largest degree is far above the mean.
    deg = np.diff(g.xadj.astype(np.int64))
    assert deg.max() > 20 * deg.mean()


def test_rgg3d_generator():
    g = H.Graph.rgg3d(100000, 10.0, 1, 100, seed=11)
    assert g.n == 100000
    assert abs(g.m / g.n - 10.0) < 0.15
    assert g.vw is not None and g.vw.min() >= 1 and g.vw.max() <= 100
    assert g.ew is not None
    _assert_symmetric_simple(g)


@pytest.mark.parametrize("weights", ["none", "edges", "vertices", "both"])
def test_metis_round_trip(tmp_path, weights):
    base = H.Graph.rmat(10, 8, seed=3)
    rng = np.random.default_rng(1)
    ew = base.ew if weights in ("edges", "both") else None
    vw = rng.integers(1, 50, base.n).astype(np.int32) if weights in ("vertices", "both") else None
    g = H.Graph(base.xadj, base.adj, ew, vw)
    path = tmp_path / "g.metis"
    g.write_metis(path)
    header = open(path).readline().split()
    assert int(header[0]) == g.n and int(header[1]) == g.m // 2
    r = H.Graph.read_metis(path)
    np.testing.assert_array_equal(r.xadj, g.xadj)
    np.testing.assert_array_equal(r.adj, g.adj)
    assert (r.ew is None) == (ew is None) and (r.vw is None) == (vw is None)
    if ew is not None:
        np.testing.assert_array_equal(r.ew, ew)
    if vw is not None:
        np.testing.assert_array_equal(r.vw, vw)


def test_metis_reader_formats(tmp_path):
    # Path 0-1-2 in METIS (1-based ids), with comments, fmt 11, weights.
    text = "% comment\n3 2 11\n5 2 7\n6 1 7 3 4\n7 2 4\n"
    p = tmp_path / "p.metis"
    p.write_text(text)
    g = H.Graph.read_metis(p)
    np.testing.assert_array_equal(g.xadj, [0, 1, 3, 4])
    np.testing.assert_array_equal(g.adj, [1, 0, 2, 1])
    np.testing.assert_array_equal(g.ew, [7, 7, 4, 4])
    np.testing.assert_array_equal(g.vw, [5, 6, 7])
    # Unweighted, with an isolated vertex (empty line).
    p.write_text("3 1\n2\n1\n\n")
    g = H.Graph.read_metis(p)
    np.testing.assert_array_equal(g.xadj, [0, 1, 2, 2])
    assert g.ew is None and g.vw is None


@pytest.mark.parametrize("text", ["", "x y\n", "3 2\n2\n1 3\n", "2 1 100\n2\n1\n", "2 1\n3\n1\n"])
def test_metis_reader_errors(tmp_path, text):
    # Empty file, bad header, too few lines, vertex sizes, out-of-range id:
    # each is an error status, never an exit.
    p = tmp_path / "bad.metis"
    p.write_text(text)
    with pytest.raises(H.HeiPaError):
        H.Graph.read_metis(p)


def test_metis_reader_large_files(tmp_path):
    # Bodies above 4 MB are parsed in chunks on all host threads; the result
    # and the error behaviour must be those of the line-by-line reader.
    g = H.Graph.rmat(16, 16, seed=2)
    vw = (np.arange(g.n) % 7 + 1).astype(np.int32)
    g = H.Graph(g.xadj, g.adj, g.ew, vw)
    path = tmp_path / "big.metis"
    g.write_metis(path)
    assert os.path.getsize(path) > (8 << 20)
    lines = open(path).read().split("\n")
    # comment lines inside the body and ignored lines after the last vertex
    body = lines[1:1 + g.n]
    mid = len(body) // 2
    text = "\n".join([lines[0]] + body[:mid] + ["% a comment", "%"] + body[mid:] + ["trailing text 1 2 3", ""])
    path.write_text(text)
    r = H.Graph.read_metis(path)
    np.testing.assert_array_equal(r.xadj, g.xadj)
    np.testing.assert_array_equal(r.adj, g.adj)
    np.testing.assert_array_equal(r.ew, g.ew)
    np.testing.assert_array_equal(r.vw, vw)
    # errors deep inside a large body
    bad_id = list(body)
    bad_id[mid] = f"{vw[mid]} {g.n + 1} 3"
    bad_weight = list(body)
    bad_weight[mid + 5] = bad_weight[mid + 5].rsplit(" ", 1)[0]
    bad_char = list(body)
    bad_char[mid + 9] = bad_char[mid + 9] + " x"
    for b in (bad_id, bad_weight, bad_char, body[:-3]):
        path.write_text("\n".join([lines[0]] + b) + "\n")
        with pytest.raises(H.HeiPaError):
            H.Graph.read_metis(path)


def test_metis_writer_large_partition(tmp_path):
    part = (np.arange(700000, dtype=np.uint64) * 2654435761 % 512).astype(np.uint32)
    path = tmp_path / "part.txt"
    H.write_partition(path, part)
    got = np.loadtxt(path, dtype=np.uint32)
    np.testing.assert_array_equal(got, part)


def test_metis_reader_missing_file(tmp_path):
    with pytest.raises(H.HeiPaError):
        H.Graph.read_metis(tmp_path / "missing.metis")


def test_write_partition(tmp_path):
    part = np.array([3, 0, 2, 2, 1], np.uint32)
    path = tmp_path / "part.txt"
    H.write_partition(path, part)
    assert [int(x) for x in open(path).read().split()] == part.tolist()
    assert os.path.getsize(path) > 0
