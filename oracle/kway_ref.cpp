// ORACLE — test infrastructure only. C entry point into the reference's own
// host initial partitioner, GPU_HeiPa::ModifiedMetis::partition
// (src/initial_partitioning/kway_partitioner/kway_core.h:1527-1545), compiled
// from the reference's unmodified sources by oracle/build_ref.py into
// oracle/_ref/libkway_ref.so. Used to pin the product's restatement of that
// partitioner (gpu-heipa_b200/host/initial_partition.cpp) and, when present,
// as the oracle pipeline's initial partitioner. Never part of the product.
#include <cstdint>
#include <vector>

#include "src/initial_partitioning/kway_partitioner/kway_core.h"

extern "C" {

// Partitions the CSR graph (n vertices, xadj[n+1], adj/ew[xadj[n]], vw[n])
// into k blocks as GPU_HeiPa::kway_partition(HostGraph&, ...) does
// (kway_core.h:1548-1571): imbalance narrowed to float, seed to int.
void ref_kway_partition(uint32_t n, const uint32_t *xadj, const uint32_t *adj, const int32_t *vw, const int32_t *ew,
                        int k, double imbalance, uint64_t seed, uint32_t *part) {
    int64_t w = 0;
    for (uint32_t u = 0; u < n; ++u) w += vw[u];
    GPU_HeiPa::ModifiedMetis::Graph g((int) n, (int) xadj[n], (int) w);
    for (uint32_t u = 0; u <= n; ++u) g.rows[u] = (int) xadj[u];
    for (uint32_t u = 0; u < n; ++u) g.v_weights[u] = vw[u];
    for (uint32_t j = 0; j < xadj[n]; ++j) {
        g.edges_v[j] = (int) adj[j];
        g.edges_w[j] = ew[j];
    }
    std::vector<int> out(n);
    GPU_HeiPa::ModifiedMetis::partition(g, k, (float) imbalance, (int) seed, out);
    for (uint32_t u = 0; u < n; ++u) part[u] = (uint32_t) out[u];
}

}  // extern "C"
