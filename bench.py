"""Benchmark: multilevel k-way partitioning throughput (undirected edges/s).

Default workload (N=1 GPU): R-MAT scale 22, edge factor 16, (a,b,c,d) =
(0.57,0.19,0.19,0.05), self loops and duplicates removed, ids permuted from
the seed, unit vertex weights, edge weights uniform in [1,10]; k = 64,
imbalance 0.03, config default. One step = one full partition (coarsening,
contraction, initial partitioning, Jet refinement) of that graph.

value: undirected input edges / device time per step, graph resident in HBM
  (CUDA events on the library's stream, max over ranks).
e2e:   same metric through hp_partition with pinned host buffers: host->device
  copy of the CSR and device->host copy of the partition inside the timed
  region.
roofline: the dominant kernel (contraction or Jet-gain), algorithmic bytes per
  launch over its average CUDA-event duration in the timed region, against
  the measured HBM copy bandwidth.
cpu_baseline: the CPU oracle (a restatement of the reference algorithm; the
  reference itself cannot be built) on a bounded R-MAT sample, rank 0, N=1.

N > 1 GPUs: one process per GPU, each partitions its own copy of the workload
(replicas, no collective on the data path; scaling "weak").

--impl reference: the CPU oracle on a bounded sample of the same workload,
  rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-heipa_b200"))

WORKLOADS = {
    "rmat22": dict(kind="rmat", scale=22, ef=16, k=64, desc="R-MAT scale 22, edge factor 16, (0.57,0.19,0.19,0.05), "
                                                          "edge weights U[1,10], k=64, eps=0.03"),
    "rmat18": dict(kind="rmat", scale=18, ef=16, k=64, desc="R-MAT scale 18, edge factor 16, (0.57,0.19,0.19,0.05), "
                                                          "edge weights U[1,10], k=64, eps=0.03 (profiling case)"),
    "grid256": dict(kind="grid", w=256, h=256, k=16, desc="2D grid 256x256, unit weights, k=16, eps=0.03"),
}
CPU_SAMPLE_SCALE = 18
# kernel timers with algorithmic byte counts; the roofline reports the one with
# the largest device time in the timed region
ROOFLINE_KERNELS = ("contract", "jet_gain", "k_delta")
# every kernel timer of the library (printed with --kernel-timers)
KERNEL_TIMERS = ("contract", "jet_gain", "k_lp_dispatch", "k_lp_warp", "k_lp_block", "k_lp_filter", "k_afterburner",
                 "k_ab_thread", "k_ab_chunk", "k_apply", "k_delta", "k_delta_thread", "k_delta_chunk",
                 "k_weak_pick", "k_weak_dispatch", "k_weak_warp", "k_weak_block", "k_strong_pick",
                 "k_strong_dispatch", "k_strong_warp", "k_strong_block")


def make_graph(H, wl, seed):
    if wl["kind"] == "rmat":
        return H.Graph.rmat(wl["scale"], wl["ef"], 0.57, 0.19, 0.19, 1, 10, seed)
    return H.Graph.grid(wl["w"], wl["h"])


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(kernel):
    """Per-launch DRAM bytes from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_max(values, world):
    if world == 1:
        return values
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_oracle_run(H, seed, scale, k):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    g = H.Graph.rmat(scale, 16, 0.57, 0.19, 0.19, 1, 10, seed)
    og = O.Graph(g.xadj, g.adj, g.ew, g.vw)
    t0 = time.perf_counter()
    _, cut = O.partition(og, k, 0.03, False, seed)
    dt = time.perf_counter() - t0
    return g.m // 2, dt, cut


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    import gpu_heipa as H
    wl = WORKLOADS[args.workload]
    scale = CPU_SAMPLE_SCALE if wl["kind"] == "rmat" else None
    times, edges = [], 0
    for i in range(args.warmup + args.steps):
        if wl["kind"] == "rmat":
            e, dt, _ = cpu_oracle_run(H, args.seed, scale, wl["k"])
        else:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O
            g = make_graph(H, wl, args.seed)
            og = O.Graph(g.xadj, g.adj, g.ew, g.vw)
            t0 = time.perf_counter()
            O.partition(og, wl["k"], 0.03, False, args.seed)
            dt, e = time.perf_counter() - t0, g.m // 2
        if i >= args.warmup:
            times.append(dt)
            edges = e
    ms = 1000.0 * sum(times) / len(times)
    value = edges / (ms / 1000.0)
    sample = (f"R-MAT scale {scale} (same generator parameters, k={wl['k']})" if scale else wl["desc"])
    line = {
        "metric": "partition_throughput", "value": value, "unit": "edges/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": wl["desc"], "parallelism": "cpu"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": 1, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, world, rank, local):
    import gpu_heipa as H
    wl = WORKLOADS[args.workload]
    k = wl["k"]
    g = make_graph(H, wl, args.seed)
    edges = g.m // 2
    ctx = H.Context(local, H.arena_estimate(g.n, g.m, g.ew is not None, g.vw is not None))
    dg = ctx.upload(g)
    part = np.empty(g.n, np.uint32)
    for _ in range(args.warmup):
        ctx.partition_graph(dg, k, 0.03, args.config, args.seed, out=part)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier(world)
    ctx.instrument(True)
    l0 = H.kernel_launches()
    ctx.event_record(0)
    cuts = []
    for _ in range(args.steps):
        _, cut = ctx.partition_graph(dg, k, 0.03, args.config, args.seed, out=part)
        cuts.append(cut)
    ctx.event_record(1)
    ms_total = ctx.event_elapsed(0, 1)
    launches = (H.kernel_launches() - l0) / args.steps
    timing = {nm: ctx.kernel_timing(nm) for nm in ROOFLINE_KERNELS}
    if args.kernel_timers and rank == 0:
        for nm in KERNEL_TIMERS:
            t = ctx.kernel_timing(nm)
            gbs = t["bytes"] / (t["ms"] / 1e3) / 1e9 if t["ms"] and t["bytes"] else None
            print(json.dumps({"timer": nm, "ms_per_step": t["ms"] / args.steps,
                              "launches_per_step": t["launches"] / args.steps, "GB/s": gbs}), file=sys.stderr)
    ctx.instrument(False)
    barrier(world)
    clocks = sampler.stop()
    stats = ctx.last_solve_stats()
    arena_peak = ctx.arena_peak()
    dg.free()

    # e2e through the host-buffer entry point with pinned buffers
    try:
        import torch
        def pinned(a):
            if a is None:
                return None
            t = torch.from_numpy(a).pin_memory()
            return t.numpy()
        hg = H.Graph(pinned(g.xadj), pinned(g.adj), pinned(g.ew), pinned(g.vw))
        hpart = torch.empty(g.n, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    except Exception:
        hg, hpart = g, np.empty(g.n, np.uint32)
    e2e_steps = 0 if args.no_e2e else args.steps
    for _ in range(0 if args.no_e2e else max(1, args.warmup // 2)):
        ctx.partition(hg, k, 0.03, args.config, args.seed, out=hpart)
    barrier(world)
    ctx.event_record(2)
    for _ in range(e2e_steps):
        ctx.partition(hg, k, 0.03, args.config, args.seed, out=hpart)
    ctx.event_record(3)
    e2e_ms_total = ctx.event_elapsed(2, 3) if e2e_steps else 0.0
    barrier(world)
    h2d = 4 * (g.n + 1) + 4 * g.m + (4 * g.m if g.ew is not None else 0) + (4 * g.n if g.vw is not None else 0)
    d2h = 4 * g.n
    ctx.close()

    ms, e2e_ms = reduce_max([ms_total / args.steps, e2e_ms_total / max(1, e2e_steps)], world)
    if rank != 0:
        return 0
    value = world * edges / (ms / 1000.0)
    e2e_value = world * edges / (e2e_ms / 1000.0) if e2e_steps else None
    peak, peak_kind = measured_peaks()
    dom = max((x for x in timing if timing[x]["bytes"] > 0), key=lambda x: timing[x]["ms"], default="contract")
    t = timing[dom]
    roofline = None
    if t["launches"] and t["ms"] > 0:
        achieved = t["bytes"] / (t["ms"] / 1000.0) / 1e9
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                    "traffic": profile_traffic(dom),
                    "bytes_per_launch": t["bytes"] / t["launches"], "launches_per_step": t["launches"] / args.steps,
                    "avg_launch_ms": t["ms"] / t["launches"],
                    "other": {x: {"launches": timing[x]["launches"], "ms": timing[x]["ms"],
                                  "GB/s": (timing[x]["bytes"] / (timing[x]["ms"] / 1000.0) / 1e9)
                                  if timing[x]["ms"] else None} for x in timing}}
    cpu = None
    if world == 1 and not args.no_cpu_baseline and wl["kind"] == "rmat":
        e, dt, ccut = cpu_oracle_run(H, args.seed, CPU_SAMPLE_SCALE, k)
        cpu = {"value": e / dt, "unit": "edges/s", "cores": 1, "kind": "port",
               "sample": f"one partition of R-MAT scale {CPU_SAMPLE_SCALE} (same generator parameters), k={k}, "
                         f"{dt:.1f} s", "cut": ccut}
    line = {
        "metric": "partition_throughput", "value": value, "unit": "edges/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": wl["desc"], "n": g.n, "undirected_edges": edges, "k": k, "config": args.config,
                   "seed": args.seed, "parallelism": f"replicas{world}",
                   "l2": "input CSR (%.2f GB) larger than L2 (126 MB)" % (h2d / 1e9)},
        "e2e": {"value": e2e_value, "unit": "edges/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "quality": {"cut": cuts[-1], "phase_ms": stats["phase_ms"], "levels": stats["levels"],
                    "arena_peak_bytes": arena_peak},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat22", choices=sorted(WORKLOADS))
    ap.add_argument("--config", default="default", choices=["default", "ultra"])
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--kernel-timers", action="store_true", help="print every kernel timer to stderr")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            rc = run_reference(args, world, rank)
        else:
            rc = run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
