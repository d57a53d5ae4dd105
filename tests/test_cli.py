"""The GPU-HeiPa / GPU-HeiProMap command-line tools: argument handling on the
CPU, and end-to-end runs on the GPU that must print the reference's stdout
keys and write the same partition the library call returns."""
import os
import subprocess

import numpy as np
import pytest

import gpu_heipa as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "gpu-heipa_b200", "bin")
HEIPA = os.path.join(BIN, "GPU-HeiPa")
PROMAP = os.path.join(BIN, "GPU-HeiProMap")


def _run(args, cwd=None):
    return subprocess.run(args, capture_output=True, text=True, timeout=600, cwd=cwd)


def test_cli_help_and_argument_errors(tmp_path):
    r = _run([HEIPA, "--help"])
    assert r.returncode == 0 and "--graph" in r.stdout and "--imbalance" in r.stdout
    r = _run([PROMAP, "--help"])
    assert r.returncode == 0 and "--hierarchy" in r.stdout and "--distance" in r.stdout
    # missing required options, bad values, bad config: non-zero exit, message on stderr
    for args in ([HEIPA, "-g", "x.graph"], [HEIPA, "-g", "x", "-k", "abc", "-c", "default"],
                 [HEIPA, "-g", "x", "-k", "4", "-c", "fast"], [HEIPA, "-g", "x", "-k"],
                 [PROMAP, "-g", "x", "-h", "4:8", "-d", "1:10:100", "-c", "HM"],
                 [PROMAP, "-g", "x", "-h", "4:8", "-d", "1:10", "-c", "XX"]):
        r = _run(args)
        assert r.returncode != 0 and "Error" in r.stderr, args
    # unreadable graph file
    r = _run([HEIPA, "-g", str(tmp_path / "missing.graph"), "-k", "4", "-c", "default"])
    assert r.returncode != 0 and "reading" in r.stderr
    # --deterministic is a switch (takes no value) in both tools
    for tool in (HEIPA, PROMAP):
        assert "--deterministic" in _run([tool, "--help"]).stdout
    r = _run([HEIPA, "--deterministic", "-g", str(tmp_path / "missing.graph"), "-k", "4", "-c", "default"])
    assert r.returncode != 0 and "reading" in r.stderr


def _stat(stdout, key):
    for line in stdout.splitlines():
        if line.startswith(key):
            return line.split(":", 1)[1].strip()
    raise AssertionError(f"missing key {key!r} in output:\n{stdout}")


@pytest.mark.gpu
def test_cli_partition_matches_library(tmp_path, ctx):
    g = H.Graph.rmat(14, 16, seed=7)
    path = tmp_path / "g.metis"
    g.write_metis(path)
    out = tmp_path / "part.txt"
    r = _run([HEIPA, "--graph", str(path), "--k", "16", "--imbalance", "0.03", "--config", "default", "--seed", "3",
              "--mapping", str(out)], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    for key in ("Read graph in", "#Vertices", "#Edges", "Lmax", "Init. edge-cut", "Final edge-cut",
                "Final max block w", "#empty partitions", "#oload partitions", "Coarsening", "Refinement",
                "Solved in", "Write partition in"):
        _stat(r.stdout, key)
    part = np.loadtxt(out, dtype=np.int64)
    assert len(part) == g.n
    want, cut = ctx.partition(g, 16, 0.03, "default", 3)
    np.testing.assert_array_equal(part, want)
    assert int(_stat(r.stdout, "Final edge-cut")) == cut
    assert int(_stat(r.stdout, "#oload partitions")) == 0
    # without --mapping no file is written
    r = _run([HEIPA, "-g", str(path), "-k", "16", "-c", "default"], cwd=tmp_path)
    assert r.returncode == 0 and not (tmp_path / "GPU-HeiPa_par.txt").exists()


@pytest.mark.gpu
@pytest.mark.parametrize("config", ["IM", "HM", "HM-ultra"])
def test_cli_mapping_matches_library(tmp_path, ctx, config):
    g = H.Graph.rgg3d(20000, 10.0, 1, 100, seed=11)
    path = tmp_path / "g.metis"
    g.write_metis(path)
    out = tmp_path / "map.txt"
    r = _run([PROMAP, "-g", str(path), "-h", "2:4:3", "-d", "1:10:100", "-e", "0.03", "-c", config, "--seed", "1",
              "-m", str(out)])
    assert r.returncode == 0, r.stderr
    part = np.loadtxt(out, dtype=np.int64)
    want, J = ctx.process_map(g, [2, 4, 3], [1, 10, 100], 0.03, config, 1)
    np.testing.assert_array_equal(part, want)
    assert int(_stat(r.stdout, "Final comm-cost")) == J
    assert _stat(r.stdout, "hierarchy") == "2:4:3" and int(_stat(r.stdout, "k")) == 24
