// ORACLE — test infrastructure only. A CPU restatement of the reference's
// multilevel partitioning / process-mapping path, used by tests/ (and the
// CPU-baseline legs of bench.py) as the checker for the CUDA implementation.
// Nothing in the product links or calls it.
//
// Parity status: the reference (GPU-HeiPa) cannot be built here as a whole
// (Kokkos and Kokkos-Kernels are absent), ships no tests, golden vectors or
// fixtures, and its GPU phases are nondeterministic (CAS races pick matching
// partners, hash slot order and bucket offsets). This oracle therefore
// restates the reference's GPU algorithm with documented deterministic rules
// where the reference races; matching and Jet dynamics are pinned by
// hand-computed known-answer tests (contraction, distance matrix, objective
// values, hash test vectors, gain buckets) and are "parity unpinned" against
// the reference itself. The host initial partitioner is the exception: the
// reference's own plain-C++ ModifiedMetis code is compiled from its sources
// (oracle/build_ref.py) and used here directly, and the product's
// restatement of it is checked against it bit for bit.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// ---- hashes and scalar rules -------------------------------------------
int or_threads(void);  // host threads the parallel loops use (OMP_NUM_THREADS)
uint32_t or_xorshift32(uint32_t x);                 // two_hop_matching.h:93-100, graph.h:39-45
uint32_t or_murmur3_u32(uint32_t key, uint32_t seed); // Kokkos::pod_hash<u32> (MurmurHash3_x86_32, 4-byte key)
uint32_t or_gain_bucket(int32_t gx, int32_t vwgt);     // jet_label_propagation.h:147-180, exact integer rule
uint32_t or_gain_bucket_float(int32_t gx, int32_t vwgt); // same lines, literal float restatement (pin test)

// ---- graphs ------------------------------------------------------------
void *or_graph_new(uint32_t n, uint32_t m, const uint32_t *xadj, const uint32_t *adj, const int32_t *ew,
                   const int32_t *vw);
void or_graph_free(void *g);
uint32_t or_graph_n(const void *g);
uint32_t or_graph_m(const void *g);
int or_graph_has_ew(const void *g);
int or_graph_has_vw(const void *g);
void or_graph_get(const void *g, uint32_t *xadj, uint32_t *adj, int32_t *ew, int32_t *vw);

// ---- coarsening --------------------------------------------------------
uint32_t or_match(const void *g, uint32_t *mapping_out);                   // two_hop_matching.h:573-650
void *or_contract(const void *g, const uint32_t *mapping, uint32_t n_c);     // graph.h:127-390 (rows sorted)

// ---- objectives and distance oracle ------------------------------------
int64_t or_edge_cut(const void *g, const uint32_t *part);                    // edge_cut.h:71-90
int64_t or_comm_cost(const void *g, const uint32_t *part, const uint32_t *hier, const int32_t *dist, uint32_t l);
void or_distance_matrix(const uint32_t *hier, const int32_t *dist, uint32_t l, int32_t *out); // distance_oracle_matrix.h:41-90

// ---- Jet refinement on one level (state handle) -------------------------
// hier == NULL selects edge-cut Jet (jet_label_propagation.h); otherwise
// process-mapping Jet with J gains (promap_jet_label_propagation.h).
void *or_jet_new(const void *g, uint32_t k, int32_t lmax, const uint32_t *part, const uint32_t *hier,
                 const int32_t *dist, uint32_t l);
void or_jet_free(void *st);
uint32_t or_jet_lp(void *st, uint32_t ratio_pct, uint32_t *moves_out);       // jet_lp :182-354 / ProMap_jet_lp :206-330
uint32_t or_jet_weak(void *st, uint32_t *moves_out);                         // rebalance_weak :592-751
uint32_t or_jet_strong(void *st, uint32_t *moves_out);                       // rebalance_strong :356-590
void or_jet_perform(void *st, const uint32_t *moves, uint32_t count, int64_t *obj_inout, int32_t *maxw_out);
void or_jet_state(const void *st, uint32_t *map, int32_t *bw, uint32_t *dest_part, int32_t *gain1, uint32_t *lock,
                  uint32_t *dest_cache, int32_t *gain_cache);
// Whole per-level refinement (jet_refine :926-1033 / ProMap_jet_refine :1218-1311).
void or_jet_refine(const void *g, uint32_t k, int32_t lmax, int ultra, uint32_t level, uint32_t *part_inout,
                   int64_t *obj_inout, int32_t *maxw_inout, const uint32_t *hier, const int32_t *dist, uint32_t l);

// ---- whole pipelines ---------------------------------------------------
// Solver::internal_solve (solver.h:340-400); returns the final edge cut.
int64_t or_partition(const void *g, uint32_t k, double eps, int ultra, uint64_t seed, uint32_t *part_out);
// hierarchical_multisection (hierarchical_multisection.h:237-307); returns J.
int64_t or_map_hm(const void *g, const uint32_t *hier, const int32_t *dist, uint32_t l, double eps, int ultra,
                  uint64_t seed, uint32_t *part_out);
// ProMapSolver::internal_solve (promap_solver.h:244-299); returns J.
int64_t or_map_im(const void *g, const uint32_t *hier, const int32_t *dist, uint32_t l, double eps, uint64_t seed,
                  uint32_t *part_out);
// lmax = ceil((1+eps) * W / k), as solver.h:410
int32_t or_lmax(int64_t total_weight, uint32_t k, double eps);

// ---- initial partitioner -------------------------------------------------
// Installs the reference's own ModifiedMetis::partition (the C entry point of
// oracle/_ref/libkway_ref.so, built from the reference's sources by
// oracle/build_ref.py); without it the pipelines use the product's
// restatement (host/metis_kway.cpp).
void or_set_ref_kway(void *fn);
int or_uses_ref_kway(void);
// The initial partition the pipelines use (kway_core.h:1548-1571).
void or_initial_kway(const void *g, uint32_t k, double eps, uint64_t seed, uint32_t *part_out);

#ifdef __cplusplus
}
#endif
