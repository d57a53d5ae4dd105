"""CPU checks of bench.py's multi-process plumbing on the gloo backend with
world size 2: max-over-ranks reduction, barriers, and the reference arm run
under torchrun (rank 0 alone prints one JSON line)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        got = bench.reduce_max([10.0 * (rank + 1), 5.0 - rank], world)
        bench.barrier(world)
        with open(f"{out_path}.{rank}", "w") as f:
            json.dump(got, f)
    finally:
        dist.destroy_process_group()


def test_reduce_max_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "r")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    for r in range(2):
        assert json.load(open(f"{out}.{r}")) == [20.0, 5.0]


def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--workload", "grid256"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port"
    # the same config object as the GPU arm prints for this workload
    assert d["config"]["n"] == 65536 and d["config"]["undirected_edges"] == 130560
    assert d["config"]["k"] == 16 and d["config"]["parallelism"] == "replicas2"
