// Coarsening: two-hop heavy-edge matching and hash contraction.
#pragma once
#include "graph.cuh"

namespace hp {

// two_hop_matcher_get_mapping (src/coarsening/two_hop_matching.h:573-650)
// with the deterministic commit rule (smallest proposer wins a receiver) and
// digest grouping by exact value for the leaf/twin/relative passes. Writes the
// fine->coarse map (device, n entries) and returns the coarse vertex count.
u32 match_graph(Ctx &ctx, const DGraph &g, u32 *mapping);

// from_Graph_Mapping (src/datastructures/graph.h:127-390): coarse vertex
// weights are summed members, coarse edges aggregate all fine edges between
// two clusters (parallel edge weights summed, self loops dropped). The
// coarse graph is allocated from the front of the arena. Rows are written in
// hash-slot order; the row contents are exact.
DGraph contract_graph(Ctx &ctx, const DGraph &g, const u32 *mapping, u32 n_c);

} // namespace hp
