"""Autotuner for the launch-structure thresholds of the partitioner
(hp_tune): which levels replay their Jet iterations as CUDA graphs, which
rebalance steps order candidates in one block, which matching loops run as
one cooperative launch, and how the Jet row passes work (hub-row tracking,
when a perform resets every cached gain at once, 16-byte or 4-byte row
reads, entries per lane). Every setting gives identical results (they only
change how the same results are computed), so tuning is a pure timing
search.

    import gpu_heipa as H, autotune
    ctx = H.Context(0, 8 << 30)
    best = autotune.tune(ctx, [H.Graph.rgg3d(200000, 10.0, 1, 10, seed=1)], [64])

The search is coordinate descent over a small candidate set per threshold,
timing hp_partition on the sample graphs (best of `repeats` runs); the best
value of each threshold is applied to ctx and returned.
"""
import time

import numpy as np

CANDIDATES = {
    "jet_graph_max_m": [0, 1 << 20, 1 << 22, 1 << 24, 1 << 26],
    "order_small_n": [0, 4096, 16384, 65536],
    "match_coop_max_n": [0, 1 << 15, 1 << 17, 1 << 19],
    "match_coop_max_m": [0, 1 << 19, 1 << 21, 1 << 23],
    "jet_fused_max_n": [0, 2048, 4096, 8192],
    "jet_fused_max_m": [1 << 16, 1 << 18, 1 << 20],
    "jet_coop_max_n": [0, 16384, 65536],
    "jet_coop_max_m": [1 << 19, 1 << 21, 1 << 23],
    "jet_coop_max_deg": [16, 32, 64],
    "jet_coop_rows": [512, 1024, 2048],
    "jet_hub_deg": [256, 1024, 4096],
    "jet_hub_conn": [0, 1],
    "jet_hub_track_pct": [25, 50, 100],
    "jet_inval_all_pct": [1, 5, 50],
    "jet_vec_loads": [0, 1],
    "jet_chunk_mode": [0, 1],
}
DEFAULTS = {"jet_graph_max_m": 1 << 24, "order_small_n": 16384, "match_coop_max_n": 1 << 17,
            "match_coop_max_m": 1 << 21, "jet_fused_max_n": 4096, "jet_fused_max_m": 1 << 18,
            "jet_coop_max_n": 65536, "jet_coop_max_m": 1 << 21, "jet_coop_max_deg": 32, "jet_coop_rows": 1024,
            "jet_hub_deg": 1024, "jet_hub_conn": 1, "jet_hub_track_pct": 50, "jet_inval_all_pct": 5,
            "jet_vec_loads": 1, "jet_chunk_mode": 0}


def _time(ctx, graphs, ks, config, seed, repeats):
    best = float("inf")
    cuts = None
    for _ in range(repeats):
        t0 = time.perf_counter()
        out = [ctx.partition(g, k, 0.03, config, seed)[1] for g, k in zip(graphs, ks)]
        best = min(best, time.perf_counter() - t0)
        cuts = out
    return best, cuts


def tune(ctx, graphs, ks, config="default", seed=1, repeats=2, candidates=None, rounds=1):
    """Returns {threshold: value} with the fastest setting found (applied to
    ctx) and checks that the objectives never change."""
    cand = candidates or CANDIDATES
    current = dict(DEFAULTS)
    for name, v in current.items():
        ctx.tune(name, v)
    base_t, ref = _time(ctx, graphs, ks, config, seed, repeats)
    for _ in range(rounds):
        for name, values in cand.items():
            best_v, best_t = current[name], base_t
            for v in values:
                if v == current[name]:
                    continue
                ctx.tune(name, v)
                t, cuts = _time(ctx, graphs, ks, config, seed, repeats)
                if cuts != ref:
                    raise RuntimeError(f"objective changed with {name}={v}: {cuts} != {ref}")
                if t < best_t:
                    best_v, best_t = v, t
            current[name] = best_v
            ctx.tune(name, best_v)
            base_t = best_t
    return current
