// ORACLE — test infrastructure only. Stand-in for the reference's
// src/datastructures/graph.h when kway_core.h is compiled on its own by
// oracle/build_ref.py (see ../utility/definitions.h): only the graph and
// partition type names that kway_core.h's unused wrapper functions
// (kway_core.h:1547-1589) mention.
#pragma once
#include "../utility/definitions.h"

namespace GPU_HeiPa {
struct HostGraph {
    vertex_t n = 0;
    vertex_t m = 0;
    weight_t g_weight = 0;
    ShimView<vertex_t> neighborhood;
    ShimView<weight_t> weights;
    ShimView<vertex_t> edges_v;
    ShimView<weight_t> edges_w;
};
struct Graph {
    vertex_t n = 0;
};
struct Partition {
    ShimView<partition_t> map;
};
inline HostGraph to_host_graph(const Graph &, DeviceExecutionSpace &) { return HostGraph{}; }
}  // namespace GPU_HeiPa
