"""Generates tests/golden/golden.json: frozen input/output vectors for the
parity tests.

The reference cannot be built here (its Kokkos dependency is not vendored)
and ships no test fixtures, so the vectors come from two sources:
  * hand-derived known answers (published MurmurHash3_x86_32 vectors, the
    6-cycle contraction, grid cuts in closed form, distance matrices), and
  * the CPU oracle on small seeded inputs (matching, contraction, Jet
    refinement and whole pipelines), frozen so that a change in either the
    oracle or the CUDA path shows up as a diff against committed data.
Inputs are regenerated from (generator, parameters, seed); outputs are stored
as counts, objectives and SHA-256 digests of the label arrays.

Run: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "gpu-heipa_b200"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

GRAPHS = {
    "grid32": ("grid", dict(w=32, h=32)),
    "grid_w": ("grid", dict(w=40, h=24, w_lo=1, w_hi=10, seed=3)),
    "rmat11": ("rmat", dict(scale=11, edge_factor=8, seed=5)),
    "rgg": ("rgg3d", dict(n=6000, mean_degree=10.0, w_lo=1, w_hi=100, seed=11)),
}
PARTITION_CASES = [("grid32", 4), ("grid_w", 8), ("rmat11", 16), ("rgg", 8)]
MAPPING_CASES = [("rgg", "HM", [2, 2, 2], [1, 10, 100]), ("rmat11", "IM", [2, 4], [1, 10]),
                 ("grid_w", "HM-ultra", [2, 3], [1, 5])]


def make_graph(H, name):
    kind, kw = GRAPHS[name]
    if kind == "grid":
        return H.Graph.grid(kw["w"], kw["h"], kw.get("w_lo", 0), kw.get("w_hi", 0), kw.get("seed", 0))
    if kind == "rmat":
        return H.Graph.rmat(kw["scale"], kw["edge_factor"], seed=kw["seed"])
    return H.Graph.rgg3d(kw["n"], kw["mean_degree"], kw["w_lo"], kw["w_hi"], seed=kw["seed"])


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()


def main():
    import gpu_heipa as H
    import oracle as O
    O.build()
    out = {"murmur3": [[0x00000000, 0, 0x2362F9DE], [0x87654321, 0, 0xF55B516B], [0xFFFFFFFF, 0, 0x76293B50],
                       [0x87654321, 0x5082EDEE, 0x2362F9DE]],
           "six_cycle_contraction": {"mapping": [0, 1, 2, 0, 1, 2], "xadj": [0, 2, 4, 6], "adj": [1, 2, 0, 2, 0, 1],
                                     "ew": [5, 9, 5, 7, 9, 7], "vw": [5, 7, 9]},
           "distance": {"hier": [4, 8, 6], "dist": [1, 10, 100],
                        "pairs": [[0, 1, 1], [0, 4, 10], [0, 32, 100], [5, 7, 1], [3, 35, 100], [191, 160, 10]]},
           "graphs": {}, "match": {}, "partition": {}, "mapping": {}}
    for name in GRAPHS:
        g = make_graph(H, name)
        og = O.Graph(g.xadj, g.adj, g.ew, g.vw)
        out["graphs"][name] = {"n": g.n, "m": g.m, "adj_sha256": digest(g.adj)}
        mp, nc = O.match(og)
        cg = O.contract(og, mp, nc)
        out["match"][name] = {"n_coarse": nc, "mapping_sha256": digest(mp), "coarse_m": cg.m}
    for name, k in PARTITION_CASES:
        g = make_graph(H, name)
        og = O.Graph(g.xadj, g.adj, g.ew, g.vw)
        part, cut = O.partition(og, k, 0.03, False, 1)
        out["partition"][f"{name}_k{k}"] = {"graph": name, "k": k, "seed": 1, "cut": cut,
                                            "part_sha256": digest(part)}
    for name, mode, hier, dist in MAPPING_CASES:
        g = make_graph(H, name)
        og = O.Graph(g.xadj, g.adj, g.ew, g.vw)
        if mode == "IM":
            part, J = O.map_im(og, hier, dist, 0.03, 1)
        else:
            part, J = O.map_hm(og, hier, dist, 0.03, mode == "HM-ultra", 1)
        out["mapping"][f"{name}_{mode}"] = {"graph": name, "mode": mode, "hier": hier, "dist": dist, "seed": 1,
                                            "J": J, "part_sha256": digest(part)}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
