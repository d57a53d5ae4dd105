// Jet label-propagation refinement on the device for the edge cut
// (src/refinement/jet_label_propagation.h) and for the process-mapping
// objective J(C,D,Pi) (src/refinement/promap_jet_label_propagation.h).
//
// Connectivity rows are not stored for ordinary vertices: every pass that
// needs conn(u, b) aggregates it on the fly from the CSR row and the current
// labels (registers for degree <= 16, a per-warp shared-memory table up to
// the hub threshold, hub rows in chunks). Hub rows of the per-kernel level
// loop (k <= 256) keep their k block sums instead, updated by the delta pass
// or rebuilt per hub when stale (JetLevel::prepare_kernel_loop). The
// dest/gain cache of the reference (dest_cache/gain_cache, invalidated when
// the vertex or one of its neighbours moves) is kept, so a pass only reaches
// vertices whose neighbourhood changed.
#pragma once
#include "graph.cuh"

namespace hp {

// Hierarchy distance oracle computed from label digits instead of a k x k
// matrix (src/distance_oracles/distance_oracle_matrix.h:64-99): every block id
// gets a code with its mixed-radix digits packed low digit first; the
// distance of two different blocks is distance[level of the highest
// differing digit].
struct DistOracle {
    u32 k = 0;
    std::vector<u32> hier;
    std::vector<s32> dist;
    u32 *code = nullptr;     // device, k entries
    s32 *bitdist = nullptr;  // device, 32 entries: distance by highest differing bit
};

DistOracle make_dist_oracle(Ctx &ctx, const std::vector<u32> &hier, const std::vector<s32> &dist);

__device__ __forceinline__ s32 dist_of(const u32 *code, const s32 *bitdist, u32 a, u32 b) {
    if (a == b) return 0;
    const u32 x = __ldg(&code[a]) ^ __ldg(&code[b]);
    return __ldg(&bitdist[31 - __clz(x)]);
}

// Objectives (int64): edge_cut.h:71-90 (halved) and comm_cost.h:36-56 (not).
s64 edge_cut_dev(Ctx &ctx, const DGraph &g, const u32 *part);
s64 comm_cost_dev(Ctx &ctx, const DGraph &g, const u32 *part, const DistOracle &D);

// Block weights of a labelling (partition.h:107-123) and their maximum.
void block_weights(Ctx &ctx, const DGraph &g, const u32 *part, u32 k, s32 *bw);
s32 max_block_weight(Ctx &ctx, const s32 *bw, u32 k);

// Per-level Jet state (device arrays from the arena's back end).
struct JetLevel {
    Ctx *ctx = nullptr;
    DGraph g;
    u32 k = 0;
    s32 lmax = 0;
    s32 g_weight = 0;
    const DistOracle *D = nullptr;  // null: edge cut
    u32 *map = nullptr;
    s32 *bw = nullptr;
    u32 *dest_cache = nullptr;
    s32 *gain_cache = nullptr;
    u32 *lock = nullptr;
    u32 *dest_part = nullptr;
    s32 *gain1 = nullptr;
    u32 *cand = nullptr;
    u32 *moves = nullptr;
    u32 *heavy = nullptr;
    u32 *heavy2 = nullptr;
    unsigned long long *items = nullptr;  // chunk work items (afterburner, delta)
    u32 items_cap = 0;
    s32 *hubacc = nullptr;  // hub-row connectivity accumulators (direct tables, small k), or null
    u32 *hubcnt = nullptr;  // hub-row finished-chunk counters
    u32 hub_cap = 0;        // hub-row slots
    unsigned long long *dlab = nullptr;   // per-kernel loop: packed label / moved / old label / hub slot
    unsigned long long *abrec = nullptr;  // per-kernel loop: packed gain / target / label (afterburner)
    u32 *hub_cur = nullptr;                           // tracked hubs: current generation of the sums (device word)
    u32 *hub_gen = nullptr;                           // tracked hubs: generation each hub's sums were built for
    const u32 *hub_vertex = nullptr;                  // tracked hubs: row of each hub slot
    unsigned long long hub_track_max = 0;             // tracked hubs: update while moved entries <= this
    u32 hub_deg = 0;        // hub threshold and chunk length (entries)
    s32 *abacc = nullptr;  // afterburner partial sums of multi-chunk rows
    u32 *abcnt = nullptr;  // afterburner finished-chunk counts of multi-chunk rows
    u32 blk_slots = 0;  // block-tier table size
    bool warp_direct = false;  // warp tier: direct-indexed (else hashed) tables
    u32 warp_slots = 0;        // warp tier: table slots per warp
    u32 warp_smem = 0;         // warp tier: dynamic shared memory per block
    size_t gain_rec = SIZE_MAX;   // instrumentation record of the last gain pass
    size_t delta_rec = SIZE_MAX;  // instrumentation record of the last delta pass
    // true when every cached gain would be recomputed identically from an
    // unchanged neighbourhood (then perform may reset all caches at once)
    bool cache_pure = false;

    void setup(Ctx &c, const DGraph &gr, u32 kk, s32 lm, const DistOracle *d, const u32 *part);
    // Each of these fills `moves` and leaves the move count in the status
    // word's MOVES counter (no host synchronisation for lp()).
    void lp(u32 ratio_pct);
    void weak();
    void strong();
    // Applies the moves; leaves the objective delta and the new maximum block
    // weight in the status word.
    void perform();
    // Single pass helpers used by tests: recompute gains for all vertices
    // whose cache is invalid (the "Jet-gain" kernel).
    // Before the per-kernel level loop: packed per-vertex words for the delta
    // pass and the afterburner, and, with direct tables and k <= 256, tracked
    // connectivity of the hub rows (Tunables::jet_hub_conn): the gain and
    // rebalance passes read a hub's k sums instead of rescanning its row, the
    // delta pass keeps the sums up to date (or, after many moves, advances
    // their generation), and a pass rebuilds the stale sums of the hubs it
    // needs (rebuild_hubs, after its dispatch).
    void prepare_kernel_loop();
    void rebuild_hubs();
    void gain_pass(u32 ratio_pct);

    // One Jet iteration: the step (0 = lp with ratio_pct, 1 = weak, 2 =
    // strong), perform, and the status word copied to the host; returns after
    // the stream is idle. With `graphs`, the sequence is captured into a CUDA
    // graph on first use (per step kind and ratio) and replayed afterwards,
    // so an iteration costs one graph launch and one host synchronisation.
    bool graphs = false;
    void run_step(int kind, u32 ratio_pct);
    void release_graphs();
    JetLevel() = default;
    JetLevel(const JetLevel &) = delete;
    JetLevel &operator=(const JetLevel &) = delete;
    ~JetLevel() { release_graphs(); }

private:
    struct StepGraph {
        int kind;
        u32 ratio;
        cudaGraphExec_t exec;
        unsigned long long kernels;  // kernel launches in the captured sequence
    };
    std::vector<StepGraph> step_graphs;
};

// Levels up to Tunables::jet_graph_max_m CSR entries replay their Jet
// iterations as CUDA graphs (launch and synchronisation cost dominates there).

// Status word slots used by Jet.
constexpr int ST_MOVES = 3;
constexpr int ST_HEAVY = 4;
constexpr int ST_CAND = 5;
constexpr int ST_HEAVY2 = 6;
constexpr int ST_AUX = 7;
constexpr int SUM_DELTA = 2;
constexpr int SUM_PERF_ENTRIES = 5;  // row entries of the moved vertices (perform)
constexpr int MAX_BW = 0;

// jet_refine (jet_label_propagation.h:926-1033) / ProMap_jet_refine
// (promap_jet_label_propagation.h:1218-1311). `part` (device, g.n) holds the
// input labelling and receives the best labelling found; obj / maxw are the
// running objective (edge cut or J) and maximum block weight.
void jet_refine(Ctx &ctx, const DGraph &g, u32 *part, u32 k, s32 lmax, bool ultra, u32 level, s64 &obj, s32 &maxw,
                const DistOracle *D);

} // namespace hp
