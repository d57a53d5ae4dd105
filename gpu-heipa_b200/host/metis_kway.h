// The reference's host initial partitioner, restated: the METIS-derived
// multilevel k-way partitioner GPU_HeiPa::ModifiedMetis::partition
// (src/initial_partitioning/kway_partitioner/kway_core.h:1527-1545) that the
// reference runs on the coarsest graph of every solve (solver.h:483 through
// kway_core.h:1548-1588) and, level by level, for the IM initial mapping
// (global_multisection.h:132-287).
//
// Same steps, constants, float expressions and tie rules as the reference, so
// that on the same graph (same vertex and row order) the partition is
// identical; the test suite checks this against the reference's own code
// compiled from its sources. Differences in form, not in results:
//  * the pseudo-random numbers come from a per-call generator that produces
//    the same sequence as the C library's srand()/rand() (the reference calls
//    the process-wide rand(), which would make concurrent calls interfere);
//  * an empty graph returns an empty partition (the reference divides by
//    zero there).
#pragma once
#include "hp_types.h"

namespace hp {

// The C library's default rand() sequence (the additive feedback generator
// r[i] = r[i-3] + r[i-31] over 32-bit words, seeded by a Lehmer generator
// and with the first 310 outputs discarded), as a value type.
class LibcRand {
public:
    explicit LibcRand(u32 seed = 1) { seed_with(seed); }
    void seed_with(u32 seed);
    int next();  // the value rand() would return

private:
    s32 r_[31];
    int f_ = 3, b_ = 0;  // front and rear taps into r_
};

// Partitions the CSR graph (rows in the order given) into k blocks exactly as
// ModifiedMetis::partition(g, k, imbalance, seed, part) does.
void metis_kway(u32 n, const u32 *xadj, const u32 *adj, const s32 *vw, const s32 *ew, int k, float imbalance,
                int seed, u32 *part);

} // namespace hp
