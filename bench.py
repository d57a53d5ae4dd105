"""Benchmark: multilevel k-way partitioning throughput (undirected edges/s).

Default workload (N=1 GPU): R-MAT scale 22, edge factor 16, (a,b,c,d) =
(0.57,0.19,0.19,0.05), self loops and duplicates removed, ids permuted from
the seed, unit vertex weights, edge weights uniform in [1,10]; k = 64,
imbalance 0.03, config default. One step = one full partition (coarsening,
contraction, initial partitioning, Jet refinement) of that graph.

Other workloads (--workload): grid256; the process-mapping configurations
rgg23_hm / rgg23_hm_ultra / rgg23_im (3D RGG, 8,388,608 points, mean degree
14, hierarchy 4:8:6, distance 1:10:100); rmat18 and rgg20_hm are small
profiling cases.

value: undirected input edges / device time per step, graph resident in HBM
  (CUDA events on the library's stream, max over ranks).
e2e:   same metric through hp_partition with pinned host buffers: host->device
  copy of the CSR and device->host copy of the partition inside the timed
  region.
roofline: the dominant kernel (contraction or Jet-gain), algorithmic bytes per
  launch over its average CUDA-event duration in the timed region, against
  the measured HBM copy bandwidth.
cpu_baseline: one solve of the same graph by the CPU oracle (a restatement of
  the reference algorithm; the reference itself cannot be built) on all host
  threads, rank 0, N=1.

N > 1 GPUs: one process per GPU, each partitions its own copy of the workload
(replicas, no collective on the data path; scaling "weak").

--impl reference: the CPU oracle on the same graph and task as the GPU arm
  (generated once, outside the timed region), W untimed and K timed solves on
  all host threads, rank 0 only.
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

RMAT_DESC = "R-MAT scale {s}, edge factor 16, (0.57,0.19,0.19,0.05), edge weights U[1,10], k=64, eps=0.03"
RGG_DESC = ("3D RGG {n} points, mean degree 14, edge weights U[1,100], explicit unit vertex weights, "
            "hierarchy 4:8:6, distance 1:10:100, eps=0.03, {mode}")
# task "partition": GPU-HeiPa (config from --config); task "map": GPU-HeiProMap
# with a fixed hierarchy and mode.
WORKLOADS = {
    "rmat22": dict(kind="rmat", scale=22, task="partition", k=64, desc=RMAT_DESC.format(s=22)),
    "rmat20": dict(kind="rmat", scale=20, task="partition", k=64, desc=RMAT_DESC.format(s=20) + " (profiling case)"),
    "rmat18": dict(kind="rmat", scale=18, task="partition", k=64, desc=RMAT_DESC.format(s=18) + " (profiling case)"),
    "grid256": dict(kind="grid", w=256, h=256, task="partition", k=16,
                    desc="2D grid 256x256, unit weights, k=16, eps=0.03"),
    "rgg23_hm": dict(kind="rgg", n=8388608, task="map", mode="HM", hier=[4, 8, 6], dist=[1, 10, 100],
                     desc=RGG_DESC.format(n=8388608, mode="HM")),
    "rgg23_hm_ultra": dict(kind="rgg", n=8388608, task="map", mode="HM-ultra", hier=[4, 8, 6], dist=[1, 10, 100],
                           desc=RGG_DESC.format(n=8388608, mode="HM-ultra")),
    "rgg23_im": dict(kind="rgg", n=8388608, task="map", mode="IM", hier=[4, 8, 6], dist=[1, 10, 100],
                     desc=RGG_DESC.format(n=8388608, mode="IM")),
    "batch": dict(kind="mix", task="batch", count=512, nmin=1000, nmax=200000,
                  desc="batch of 512 graphs, vertices log-uniform in [1000, 200000], generator uniform over "
                       "{grid aspect U[1,4], R-MAT ef 8, RGG mean degree 10}, edge weights U[1,10], "
                       "k power of two in 2..256, eps=0.03, default", sample=None),
    "served": dict(kind="mix", task="served", count=200, rates=(5.0, 10.0, 20.0, 50.0), emin=10000, emax=2000000,
                   desc="served: 200 Poisson requests per arrival rate (5, 10, 20, 50 /s), undirected edges "
                        "log-uniform in [1e4, 2e6], 70% partition (k power of two 2..512) / 30% mapping "
                        "(4:8:6 1:10:100, 2:4:8 1:5:50, 8:16 1:20, HM), same generators", sample=None),
    "rgg20_hm": dict(kind="rgg", n=1048576, task="map", mode="HM", hier=[4, 8, 6], dist=[1, 10, 100],
                     desc=RGG_DESC.format(n=1048576, mode="HM") + " (profiling case)"),
}
# kernel timers with algorithmic byte counts; the roofline reports the one with
# the largest device time in the timed region
ROOFLINE_KERNELS = ("contract", "jet_gain", "k_delta")
# every kernel timer of the library (printed with --kernel-timers)
KERNEL_TIMERS = ("contract", "contract_thread", "contract_warp", "contract_block", "contract_huge", "jet_gain", "k_lp_dispatch", "k_lp_warp", "k_lp_block", "k_lp_filter", "k_afterburner",
                 "k_ab_thread", "k_ab_chunk", "k_apply", "k_delta", "k_delta_thread", "k_delta_chunk", "k_hub_rebuild",
                 "k_weak_pick", "k_weak_dispatch", "k_weak_warp", "k_weak_block", "k_strong_pick",
                 "k_strong_dispatch", "k_strong_warp", "k_strong_block")


def make_graph(H, spec, seed):
    if spec["kind"] == "rmat":
        return H.Graph.rmat(spec["scale"], 16, 0.57, 0.19, 0.19, 1, 10, seed)
    if spec["kind"] == "rgg":
        return H.Graph.rgg3d(spec["n"], 14.0, 1, 100, seed, True)
    return H.Graph.grid(spec["w"], spec["h"])


def config_of(wl, args):
    return args.config if wl["task"] == "partition" else wl["mode"]


def solve_device(ctx, dg, wl, args, out):
    """One step on a graph resident in HBM; returns the objective (cut or J)."""
    if wl["task"] == "partition":
        return ctx.partition_graph(dg, wl["k"], 0.03, args.config, args.seed, out=out)[1]
    return ctx.process_map_graph(dg, wl["hier"], wl["dist"], 0.03, wl["mode"], args.seed, out=out)[1]


def solve_host(ctx, hg, wl, args, out):
    """One step through the host-buffer entry point (upload and download inside)."""
    if wl["task"] == "partition":
        return ctx.partition(hg, wl["k"], 0.03, args.config, args.seed, out=out)[1]
    return ctx.process_map(hg, wl["hier"], wl["dist"], 0.03, wl["mode"], args.seed, out=out)[1]


def oracle_solve(O, og, wl, args):
    """The CPU oracle restatement of the same task (test infrastructure)."""
    if wl["task"] == "partition":
        return O.partition(og, wl["k"], 0.03, args.config == "ultra", args.seed)[1]
    if wl["mode"] == "IM":
        return O.map_im(og, wl["hier"], wl["dist"], 0.03, args.seed)[1]
    return O.map_hm(og, wl["hier"], wl["dist"], 0.03, wl["mode"] == "HM-ultra", args.seed)[1]


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


def oracle_graph(g):
    """The CPU oracle's copy of graph g (built outside any timed region)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O, O.Graph(g.xadj, g.adj, g.ew, g.vw)


def cpu_oracle_solve(O, og, wl, args):
    """One timed solve of the oracle on all host threads: (seconds, objective)."""
    t0 = time.perf_counter()
    obj = oracle_solve(O, og, wl, args)
    return time.perf_counter() - t0, obj


L2_BYTES = 126 << 20        # B200 L2
L2_FLUSH_BYTES = 256 << 20  # written before every timed step when the input fits in L2


def input_bytes(g):
    return 4 * (g.n + 1) + 4 * g.m + (4 * g.m if g.ew is not None else 0) + (4 * g.n if g.vw is not None else 0)


def workload_config(wl, args, g, world):
    """The `config` object of both arms' lines for a plain workload on graph g."""
    h2d = input_bytes(g)
    if h2d > L2_BYTES:
        l2 = "input CSR (%.2f GB) larger than L2 (126 MB)" % (h2d / 1e9)
    else:
        l2 = ("input CSR (%.1f MB) smaller than L2 (126 MB): a 256 MB buffer is written before every timed "
              "step (L2 flush, inside the timed region)" % (h2d / 1e6))
    return {"workload": wl["desc"], "n": g.n, "undirected_edges": g.m // 2,
            "k": wl["k"] if wl["task"] == "partition" else int(np.prod(wl["hier"])), "config": config_of(wl, args),
            "seed": args.seed, "parallelism": f"replicas{world}", "l2": l2}


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    import gpu_heipa as H
    wl = WORKLOADS[args.workload]
    g = make_graph(H, wl, args.seed)  # the GPU arm's graph, generated once
    O, og = oracle_graph(g)
    edges = g.m // 2
    times, objs = [], []
    for i in range(args.warmup + args.steps):
        dt, obj = cpu_oracle_solve(O, og, wl, args)
        if i >= args.warmup:
            times.append(dt)
            objs.append(obj)
    cores = O.threads()
    ms = 1000.0 * sum(times) / len(times)
    value = edges / (ms / 1000.0)
    config = workload_config(wl, args, g, args.gpus)
    config["timing"] = "host wall clock around each oracle solve of this graph; graph generated outside"
    line = {
        "metric": "partition_throughput", "value": value, "unit": "edges/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": config,
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": cores, "kind": "port",
                         "sample": f"the full graph of config ({g.n} vertices, {edges} undirected edges), "
                                   f"{args.steps} timed solves", "objective": objs[-1]},
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


MAP_CHOICES = [([4, 8, 6], [1, 10, 100]), ([2, 4, 8], [1, 5, 50]), ([8, 16], [1, 20])]


def mixed_graph(H, rng, n_target, seed, weights=(1, 10)):
    """One graph of the batched / served mixes: grid (aspect U[1,4]), R-MAT
    (edge factor 8, vertices rounded to a power of two) or RGG (mean degree
    10), edge weights U[w_lo, w_hi]."""
    kind = int(rng.integers(0, 3))
    if kind == 0:
        aspect = float(rng.uniform(1.0, 4.0))
        w = max(2, int(round((n_target * aspect) ** 0.5)))
        h = max(2, n_target // w)
        return H.Graph.grid(w, h, weights[0], weights[1], seed)
    if kind == 1:
        scale = max(4, int(round(np.log2(n_target))))
        return H.Graph.rmat(scale, 8, 0.57, 0.19, 0.19, weights[0], weights[1], seed)
    return H.Graph.rgg3d(n_target, 10.0, weights[0], weights[1], seed, True)


def run_batch(args, world, rank, local):
    """Batched path: every graph of the mix through hp_partition_batch, against
    one plain hp_partition per graph on the same GPU (both with host buffers)."""
    import gpu_heipa as H
    wl = WORKLOADS[args.workload]
    rng = np.random.default_rng(args.seed + 1000 * rank)
    graphs, ks = [], []
    for i in range(wl["count"]):
        n_t = int(np.exp(rng.uniform(np.log(wl["nmin"]), np.log(wl["nmax"]))))
        graphs.append(mixed_graph(H, rng, n_t, args.seed + i))
        ks.append(int(2 ** rng.integers(1, 9)))
    edges = sum(g.m // 2 for g in graphs)
    big = max(graphs, key=lambda g: g.m)
    ctx = H.Context(local, 24 << 30)
    for _ in range(args.warmup):
        ctx.partition_batch(graphs[:64], ks[:64], 0.03, "default", args.seed, workers=args.workers)
    barrier(world)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        out = ctx.partition_batch(graphs, ks, 0.03, "default", args.seed, workers=args.workers)
        times.append(time.perf_counter() - t0)
    # sequential plain runs of the same graphs (one step)
    t0 = time.perf_counter()
    plain_cuts = [ctx.partition(g, k, 0.03, "default", args.seed)[1] for g, k in zip(graphs, ks)]
    plain_s = time.perf_counter() - t0
    same = all(c == pc for (_, c), pc in zip(out, plain_cuts))
    ctx.close()
    s = reduce_max([sum(times) / len(times)], world)[0]
    if rank != 0:
        return 0
    line = {
        "metric": "partition_throughput", "value": world * edges / s, "unit": "edges/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * s, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": wl["desc"], "graphs": len(graphs), "undirected_edges": edges,
                   "largest_edges": big.m // 2, "workers": args.workers, "parallelism": f"replicas{world}",
                   "timing": "host wall clock around hp_partition_batch (host buffers, uploads and downloads "
                             "inside)"},
        "e2e": {"value": world * edges / s, "unit": "edges/s", "graphs_per_s": world * len(graphs) / s,
                "h2d_bytes_per_step": int(sum(4 * (g.n + 1) + 8 * g.m for g in graphs)),
                "d2h_bytes_per_step": int(sum(4 * g.n for g in graphs))},
        "batched_vs_plain": {"batched_graphs_per_s": len(graphs) / s, "plain_graphs_per_s": len(graphs) / plain_s,
                             "speedup": plain_s / s, "same_results": same},
        "gpu_launches": None, "roofline": None, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_served(args, world, rank, local):
    """Serving loop: open-loop Poisson streams (one per arrival rate) submitted
    at their arrival times; latency = submit to result. Compared with the same
    requests run one after another through the plain calls."""
    import threading
    import gpu_heipa as H
    wl = WORKLOADS[args.workload]
    rng = np.random.default_rng(args.seed + 2000 * rank)
    reqs = []
    for i in range(wl["count"]):
        e_t = float(np.exp(rng.uniform(np.log(wl["emin"]), np.log(wl["emax"]))))
        mapping = rng.uniform() < 0.3
        n_t = max(64, int(e_t / 5.0))  # about 5 undirected edges per vertex
        g = mixed_graph(H, rng, n_t, args.seed + i, (1, 100) if mapping else (1, 10))
        if mapping:
            hier, dist = MAP_CHOICES[int(rng.integers(0, 3))]
            if g.vw is None:
                g = H.Graph(g.xadj, g.adj, g.ew, np.ones(g.n, np.int32))
            reqs.append(("map", g, (hier, dist)))
        else:
            reqs.append(("part", g, int(2 ** rng.integers(1, 10))))
    edges = sum(r[1].m // 2 for r in reqs)
    small_mask = np.array([r[1].m // 2 < 1000000 for r in reqs])
    srv = H.Server(local, 64 << 30, workers=args.workers)
    for kind, g, p in reqs[:8]:  # warm-up
        rid = srv.submit_map(g, p[0], p[1]) if kind == "map" else srv.submit_partition(g, p)
        srv.wait(rid)
    sweep = []
    results = None
    for rate in wl["rates"]:
        gaps = rng.exponential(1.0 / rate, len(reqs))
        ids, lat = [None] * len(reqs), [None] * len(reqs)

        def collector():
            for i in range(len(reqs)):
                while ids[i] is None:
                    time.sleep(0.0002)
                lat[i] = srv.wait(ids[i])

        th = threading.Thread(target=collector)
        th.start()
        t0 = time.perf_counter()
        t_next = t0
        for i, (kind, g, p) in enumerate(reqs):
            t_next += gaps[i]
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ids[i] = srv.submit_map(g, p[0], p[1]) if kind == "map" else srv.submit_partition(g, p)
        th.join()
        wall = time.perf_counter() - t0
        lats = np.array([x[2] for x in lat])
        sweep.append({"rate_per_s": rate, "wall_s": wall, "requests_per_s": len(reqs) / wall,
                      "edges_per_s": edges / wall, "p50_ms": float(np.percentile(lats, 50)),
                      "p99_ms": float(np.percentile(lats, 99)),
                      "p50_ms_under_1M_edges": float(np.percentile(lats[small_mask], 50)),
                      "p99_ms_under_1M_edges": float(np.percentile(lats[small_mask], 99))})
        results = lat
    srv.close()
    ctx = H.Context(local, H.arena_estimate(max(r[1].n for r in reqs), max(r[1].m for r in reqs), True, True))
    t1 = time.perf_counter()
    same = True
    for (kind, g, p), x in zip(reqs, results):
        if kind == "map":
            _, obj = ctx.process_map(g, p[0], p[1])
        else:
            _, obj = ctx.partition(g, p)
        same = same and obj == x[1]
    plain_s = time.perf_counter() - t1
    ctx.close()
    if rank != 0:
        return 0
    best = max(sweep, key=lambda x: x["edges_per_s"])
    line = {
        "metric": "partition_throughput", "value": best["edges_per_s"], "unit": "edges/s", "n_gpus": world,
        "steps": len(sweep), "warmup": 8, "ms_per_step": 1000 * best["wall_s"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": wl["desc"], "requests": len(reqs), "undirected_edges": edges,
                   "workers": args.workers, "timing": "host wall clock from the first arrival to the last result; "
                                                       "value = the best rate of the sweep"},
        "e2e": {"value": best["edges_per_s"], "unit": "edges/s", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": None},
        "served": {"sweep": sweep, "sequential_plain_s": plain_s,
                   "sequential_plain_requests_per_s": len(reqs) / plain_s, "same_results": same},
        "gpu_launches": None, "roofline": None, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, world, rank, local):
    import gpu_heipa as H
    wl = WORKLOADS[args.workload]
    g = make_graph(H, wl, args.seed)
    edges = g.m // 2
    # mapping (HM) runs each hierarchy level's sub-solves concurrently in the
    # arena's free space: give it twice the single-solve estimate
    scale = 2 if wl["task"] == "map" else 1
    ctx = H.Context(local, scale * H.arena_estimate(g.n, g.m, g.ew is not None, g.vw is not None))
    for t in args.tune:
        name, value = t.split("=")
        ctx.tune(name, int(value))
    dg = ctx.upload(g)
    part = np.empty(g.n, np.uint32)
    # inputs that fit in L2: write a buffer larger than L2 before every timed step
    flush = None
    if input_bytes(g) <= L2_BYTES:
        import torch
        flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")

    def l2_flush():
        if flush is not None:
            flush.zero_()
            torch.cuda.synchronize(local)

    for _ in range(args.warmup):
        l2_flush()  # (the first one also loads the fill kernel)
        solve_device(ctx, dg, wl, args, part)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier(world)
    ctx.instrument(True)
    l0 = H.kernel_launches()
    ctx.event_record(0)
    cuts = []
    for _ in range(args.steps):
        l2_flush()
        cuts.append(solve_device(ctx, dg, wl, args, part))
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
        solve_host(ctx, hg, wl, args, hpart)
    barrier(world)
    ctx.event_record(2)
    for _ in range(e2e_steps):
        l2_flush()
        solve_host(ctx, hg, wl, args, hpart)
    ctx.event_record(3)
    e2e_ms_total = ctx.event_elapsed(2, 3) if e2e_steps else 0.0
    barrier(world)
    h2d = input_bytes(g)
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
    if world == 1 and not args.no_cpu_baseline:
        O, og = oracle_graph(g)
        dt, cobj = cpu_oracle_solve(O, og, wl, args)
        cpu = {"value": edges / dt, "unit": "edges/s", "cores": O.threads(), "kind": "port",
               "sample": f"one solve of the same graph and task, {dt:.1f} s", "objective": cobj,
               "same_objective_as_gpu": cobj == cuts[-1]}
        del og
    line = {
        "metric": "partition_throughput", "value": value, "unit": "edges/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": workload_config(wl, args, g, world),
        "e2e": {"value": e2e_value, "unit": "edges/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "quality": {("cut" if wl["task"] == "partition" else "J"): cuts[-1], "phase_ms": stats["phase_ms"],
                    "levels": stats["levels"],
                    "arena_peak_bytes": arena_peak},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_quality(args, world, rank, local):
    """Quality over seeds 1..N: the objective of every seed on the GPU and,
    with --quality-oracle, of the CPU oracle restatement on the same graph
    and seed, with the geometric means."""
    if rank != 0:
        return 0
    import gpu_heipa as H
    wl = WORKLOADS[args.workload]
    g = make_graph(H, wl, args.seed)
    scale = 2 if wl["task"] == "map" else 1
    seeds = list(range(1, args.quality_seeds + 1))
    gpu, cpu, times = [], [], []
    with H.Context(local, scale * H.arena_estimate(g.n, g.m, g.ew is not None, g.vw is not None)) as ctx:
        dg = ctx.upload(g)
        part = np.empty(g.n, np.uint32)
        for sd in seeds:
            a = argparse.Namespace(**vars(args))
            a.seed = sd
            t0 = time.perf_counter()
            gpu.append(int(solve_device(ctx, dg, wl, a, part)))
            times.append(time.perf_counter() - t0)
        dg.free()
    if args.quality_oracle:
        O, og = oracle_graph(g)
        for sd in seeds:
            a = argparse.Namespace(**vars(args))
            a.seed = sd
            cpu.append(int(oracle_solve(O, og, wl, a)))

    def geomean(xs):
        return float(np.exp(np.mean(np.log(np.asarray(xs, np.float64))))) if xs and min(xs) > 0 else None

    line = {"quality_seeds": len(seeds), "workload": wl["desc"], "config": config_of(wl, args),
            "objective": "cut" if wl["task"] == "partition" else "J", "seeds": seeds, "gpu": gpu,
            "gpu_geomean": geomean(gpu), "gpu_ms_median": 1000 * statistics.median(times)}
    if cpu:
        line.update({"cpu_oracle": cpu, "cpu_oracle_geomean": geomean(cpu),
                     "gpu_over_cpu_geomean": (geomean(gpu) / geomean(cpu)) if geomean(cpu) else None,
                     "identical_every_seed": gpu == cpu})
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
    ap.add_argument("--workers", type=int, default=8, help="concurrent requests (batch / served workloads)")
    ap.add_argument("--quality-seeds", type=int, default=0,
                    help="instead of timing: objective over seeds 1..N on the GPU (geometric mean)")
    ap.add_argument("--quality-oracle", action="store_true", help="with --quality-seeds: also the CPU oracle")
    ap.add_argument("--tune", action="append", default=[], metavar="NAME=VALUE",
                    help="launch-structure threshold (hp_tune), e.g. jet_graph_max_m=0 for profiling runs")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    try:
        task = WORKLOADS[args.workload]["task"]
        if args.quality_seeds > 0 and task not in ("batch", "served"):
            rc = run_quality(args, world, rank, local)
        elif args.impl == "reference":
            if task in ("batch", "served"):
                print(json.dumps({"impl": "reference", "unavailable": "the batched and served workloads have no "
                                  "CPU restatement; their plain runs on the GPU are the comparison"}), flush=True)
                rc = 0
            else:
                rc = run_reference(args, world, rank)
        elif task == "batch":
            rc = run_batch(args, world, rank, local)
        elif task == "served":
            rc = run_served(args, world, rank, local)
        else:
            rc = run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
