// Level-loop drivers: Solver::internal_solve (src/datastructures/solver.h:
// 340-400, and the device constructor :144-246), ProMapSolver::internal_solve
// (src/datastructures/promap_solver.h:244-299) and the hierarchical
// multisection (src/initial_partitioning/hierarchical_multisection.h:56-307).
#pragma once
#include "coarsen.cuh"
#include "jet.cuh"

namespace hp {

struct SolveStats {
    double coarsening_ms = 0, contraction_ms = 0, initial_ms = 0, uncontraction_ms = 0, refinement_ms = 0;
    s64 initial_obj = 0;
    s32 initial_maxw = 0;
    s64 final_obj = 0;
    s32 final_maxw = 0;
    s32 lmax = 0;
    u32 levels = 0;
    std::vector<u32> level_n;
    std::vector<u64> level_m;
    void add(const SolveStats &o) {
        coarsening_ms += o.coarsening_ms;
        contraction_ms += o.contraction_ms;
        initial_ms += o.initial_ms;
        uncontraction_ms += o.uncontraction_ms;
        refinement_ms += o.refinement_ms;
    }
};

// lmax = ceil((1 + eps) * W / k)  (solver.h:410)
s32 lmax_of(s64 total_weight, u32 k, double eps);

// k-way edge-cut partition of g into `part` (device, g.n entries); returns the
// final edge cut.
s64 solve_partition(Ctx &ctx, const DGraph &g, u32 k, double eps, bool ultra, u64 seed, u32 *part,
                    SolveStats *stats);

// Process mapping. mode 0: IM (J-gain Jet over the multilevel hierarchy with
// a global-multisection initial mapping); 1: HM; 2: HM-ultra (recursive
// multisection with edge-cut sub-solves). Returns J (int64).
s64 solve_mapping(Ctx &ctx, const DGraph &g, const std::vector<u32> &hier, const std::vector<s32> &dist, double eps,
                  int mode, u64 seed, u32 *part, SolveStats *stats);

// Bytes of device arena a solve of a graph with n vertices and m directed
// entries needs (hierarchy plus scratch), with a safety margin.
size_t arena_estimate(u32 n, u64 m, bool has_ew, bool has_vw);
// Device bytes one request of a batch or a served stream reserves.
size_t request_estimate(u32 n, u64 m, bool has_ew, bool has_vw);

} // namespace hp
