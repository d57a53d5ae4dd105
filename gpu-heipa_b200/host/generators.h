// Seeded synthetic graph generators for the benchmark workloads: 2D grid,
// R-MAT and 3D random geometric graphs. All produce symmetric CSR graphs
// without self-loops or duplicate edges and with rows sorted by neighbour id.
// Edge weights are drawn once per undirected pair, so both directions carry
// the same weight. The output depends only on the parameters and the seed.
#pragma once
#include "hp_types.h"

namespace hp {

// w x h 4-neighbour grid; vertex id = y*w + x; unit weights (empty ew/vw)
// unless w_hi > 0, in which case edge weights are uniform in [w_lo, w_hi].
HostCSR gen_grid(u32 w, u32 h, s32 w_lo, s32 w_hi, u64 seed);

// R-MAT with 2^scale vertices and edge_factor * 2^scale generated pairs,
// probabilities (a, b, c, 1-a-b-c); self-loops and duplicates dropped; vertex
// ids permuted by a seeded permutation; edge weights uniform in [w_lo, w_hi]
// (w_hi == 0 means unit weights, empty ew). Vertex weights are explicit ones
// when explicit_vw is set.
HostCSR gen_rmat(u32 scale, u32 edge_factor, double a, double b, double c, s32 w_lo, s32 w_hi, u64 seed,
                 bool explicit_vw);

// n points uniform in [0,1)^3 connected within the radius that gives the
// requested mean degree (first-order boundary correction); edge weights
// uniform in [w_lo, w_hi]; explicit unit vertex weights when explicit_vw.
HostCSR gen_rgg3d(u32 n, double mean_degree, s32 w_lo, s32 w_hi, u64 seed, bool explicit_vw);

// Radius used by gen_rgg3d for n points and the given mean degree.
double rgg3d_radius(u32 n, double mean_degree);

} // namespace hp
