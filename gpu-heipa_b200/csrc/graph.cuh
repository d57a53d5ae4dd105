// Device graph layout.
//
// A graph level lives in HBM as a padded CSR: row u occupies
// adj[rowptr[u] .. rowptr[u] + rowlen[u]) of arrays sized rowptr[n] (the
// row capacity). The input graph has rowptr = xadj and no padding; a coarse
// graph produced by contraction keeps the capacity bound of its fine rows
// (sum of member degrees), which lets contraction write every coarse row in
// one pass without a counting pre-pass. This replaces the reference's
// struct Graph (src/datastructures/graph.h:47-61: neighborhood/edges_v/
// edges_u/edges_w/weights); the COO helper edges_u is not kept.
#pragma once
#include "context.h"

namespace hp {

struct DGraph {
    u32 n = 0;
    u64 m = 0;          // directed entries actually present (sum of rowlen)
    u64 cap = 0;        // rowptr[n]
    u32 *rowptr = nullptr;  // n+1
    u32 *rowlen = nullptr;  // n
    u32 *adj = nullptr;     // cap
    s32 *ew = nullptr;      // cap, or null for unit edge weights
    s32 *vw = nullptr;      // n, or null for unit vertex weights
    s64 total_vw = 0;
};

__device__ __forceinline__ s32 g_ew(const DGraph &g, u64 j) { return g.ew ? __ldg(&g.ew[j]) : 1; }
__device__ __forceinline__ s32 g_vw(const DGraph &g, u32 u) { return g.vw ? g.vw[u] : 1; }

// Uploads a host CSR (xadj n+1, adj m, optional ew/vw) into the front of the
// arena and validates it on the device (ids in range, no self loops, weights
// >= 1). Throws HpError on invalid input.
DGraph graph_upload(Ctx &ctx, u32 n, u64 m, const u32 *xadj, const u32 *adj, const s32 *ew, const s32 *vw);

// Same, from arrays already in device memory (copied into the arena).
DGraph graph_from_device(Ctx &ctx, u32 n, u64 m, const u32 *d_xadj, const u32 *d_adj, const s32 *d_ew,
                         const s32 *d_vw, bool validate);

// Writes a compact CSR copy of g to host arrays (xadj n+1, adj m, ew m, vw n).
void graph_download(Ctx &ctx, const DGraph &g, u32 *xadj, u32 *adj, s32 *ew, s32 *vw);

// All subgraphs induced by parts 0..k-1 of `part`, in one pass over g
// (hierarchical_multisection.h:104-206 induces them one part at a time):
// subs[p] holds the vertices with part p in ascending id and, for each, its
// same-part neighbours in row order, renumbered to local ids (an empty graph
// when part p is empty); n_to_o[p] maps its vertices through n_to_o_parent
// (parent id -> root id). Arrays are allocated from the front of the arena,
// part after part.
void graph_induced_all(Ctx &ctx, const DGraph &g, const u32 *part, u32 k, const u32 *n_to_o_parent,
                       std::vector<DGraph> &subs, std::vector<u32 *> &n_to_o);

} // namespace hp
