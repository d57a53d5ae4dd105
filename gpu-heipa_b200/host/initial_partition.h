// Host-side initial partitioning of the coarsest graph.
//
// The reference runs a METIS-derived multilevel k-way partitioner on the host
// for the coarsest level (src/initial_partitioning/kway_partitioner/kway_core.h:
// 1527-1588) and, for process mapping with --config IM, a recursive partition
// over the hierarchy levels (src/initial_partitioning/global_multisection.h:
// 132-287). This file provides the same two services with the same algorithm
// (metis_kway.h): on the same graph, seed and imbalance the partition equals
// the reference's. It runs on graphs of a few thousand vertices, is
// sequential and deterministic, and is safe to call from concurrent threads.
#pragma once
#include "hp_types.h"

namespace hp {

// Partitions `g` into k blocks as kway_partition(HostGraph&, k, eps, seed, ...)
// does (kway_core.h:1548-1571). The result depends on the graph including its
// row order (callers pass rows sorted by neighbour id), k, eps and seed.
void initial_kway(const HostCSR &g, u32 k, double eps, u64 seed, std::vector<u32> &part);

// Imbalance for a sub-problem of a hierarchical split, as in
// src/initial_partitioning/global_multisection.h:39-48.
double adaptive_imbalance(double global_eps, s64 global_w, u32 global_k, s64 local_w, u32 local_k_rem, u64 depth);

// Recursive partition over the hierarchy levels (last level first), the IM
// initial mapping of src/initial_partitioning/global_multisection.h:259-287.
// The final block id is sum_i id_i * index_vec[l-1-i] + local id.
void global_multisection(const HostCSR &g, const std::vector<u32> &hierarchy, double eps, u64 seed,
                         std::vector<u32> &part);

// Sorts every row of `g` by neighbour id (weights follow), so that results of
// order-sensitive host code do not depend on the row order a device produced.
void sort_rows(HostCSR &g);

// Induced subgraph of the vertices with part[u] == id; vertex order and row
// order are kept. `n_to_o` receives the parent ids of the new vertices.
HostCSR induced_subgraph(const HostCSR &g, const std::vector<u32> &part, u32 id, std::vector<u32> &n_to_o);

} // namespace hp
