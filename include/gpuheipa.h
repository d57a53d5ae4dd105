/*
 * C ABI of the B200 multilevel graph partitioner / process mapper.
 *
 * Every entry point returns an int status (HP_OK == 0) and never exits or
 * aborts; hp_last_error() returns the message of the last failure on a
 * context. Host buffers are owned by the caller. Device memory is owned by the
 * context's arena, which allocates LIFO like the reference's
 * KokkosMemoryStack (src/datastructures/kokkos_memory_stack.h:36-206): graph
 * handles must be freed in reverse order of creation.
 *
 * The reference exposes this path only as header-only C++ templates; the
 * comment above each function names the reference interface it replaces.
 * Conventions: n = vertices, m = directed CSR entries (2x undirected edges,
 * src/datastructures/host_graph.h:195), ids uint32, weights int32 (>= 1),
 * objectives int64. A NULL weight array means unit weights ("uniform").
 */
#ifndef GPUHEIPA_H
#define GPUHEIPA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    HP_OK = 0,
    HP_ERR_ARG = 1,
    HP_ERR_CUDA = 2,
    HP_ERR_OOM = 3,
    HP_ERR_IO = 4,
    HP_ERR_GRAPH = 5,
    HP_ERR_DEVICE = 6,
    HP_ERR_TOO_LARGE = 7, /* input larger than a fixed-size entry point accepts */
    HP_ERR_BUSY = 8       /* a bounded wait for a shared resource timed out */
};

/* Mapping modes for hp_map / hp_map_graph (GPU-HeiProMap --config). */
enum { HP_MAP_IM = 0, HP_MAP_HM = 1, HP_MAP_HM_ULTRA = 2 };

typedef struct hp_ctx hp_ctx;
typedef struct hp_graph hp_graph;
typedef struct hp_jet hp_jet;
typedef struct hp_host_graph hp_host_graph;

/* ---- context ------------------------------------------------------------------ */

/* Replaces Kokkos::initialize + initialize_kokkos_memory_stack
 * (app/GPU-HeiPa.cpp:44, src/datastructures/kokkos_memory_stack.h:57). */
int hp_ctx_create(int device, size_t arena_bytes, hp_ctx **out);
/* Replaces destroy(mem_stack) + Kokkos::finalize (kokkos_memory_stack.h:195-206). */
int hp_ctx_destroy(hp_ctx *ctx);
/* Message of the last failed call on ctx ("" if none). */
const char *hp_last_error(const hp_ctx *ctx);
/* Arena bytes a solve of an (n, m) graph needs; replaces the sizing rules of
 * configuration.h:79 and promap_solver.h:307-311. */
size_t hp_arena_estimate(uint32_t n, uint64_t m, int has_edge_weights, int has_vertex_weights);
/* Peak arena bytes used so far. */
size_t hp_arena_peak(const hp_ctx *ctx);

/* ---- device graphs -------------------------------------------------------- */

/* Replaces from_HostGraph (src/datastructures/graph.h:63-125). Validates ids,
 * self loops and weights on the device. */
int hp_graph_upload(hp_ctx *ctx, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj,
                    const int32_t *ew, const int32_t *vw, hp_graph **out);
/* Replaces free_graph (graph.h:438-443); LIFO order. */
int hp_graph_free(hp_ctx *ctx, hp_graph *g);
/* n, m (directed entries present) and total vertex weight of a device graph. */
int hp_graph_info(const hp_graph *g, uint32_t *n, uint64_t *m, int64_t *total_vw);
/* Replaces to_host_graph (graph.h:413-436): compact CSR copy to host arrays
 * (xadj n+1, adj m, ew m, vw n; any may be NULL). Row order is the device's. */
int hp_graph_download(hp_ctx *ctx, const hp_graph *g, uint32_t *xadj, uint32_t *adj, int32_t *ew, int32_t *vw);

/* ---- phase kernels -------------------------------------------------------- */

/* Replaces two_hop_matcher_get_mapping (src/coarsening/two_hop_matching.h:573)
 * with deterministic tie rules; writes mapping (n entries, host). */
int hp_match(hp_ctx *ctx, const hp_graph *g, uint32_t *mapping, uint32_t *n_coarse);
/* Replaces from_Graph_Mapping (src/datastructures/graph.h:127-390): contracts
 * g with a host mapping (values < n_coarse) into a new device graph. */
int hp_contract(hp_ctx *ctx, const hp_graph *g, const uint32_t *mapping, uint32_t n_coarse, hp_graph **out);
/* Replaces jet_refine (src/refinement/jet_label_propagation.h:926) when
 * hier == NULL, and ProMap_jet_refine (promap_jet_label_propagation.h:1218)
 * otherwise; part (host, n) is refined in place; obj and maxw are the running
 * objective and maximum block weight (in/out). */
int hp_jet_refine(hp_ctx *ctx, const hp_graph *g, uint32_t k, int32_t lmax, int ultra, uint32_t level,
                  uint32_t *part, int64_t *obj, int32_t *maxw, const uint32_t *hier, const int32_t *dist,
                  uint32_t levels);

/* One Jet iteration at a time, for stepping and inspection (the phases of
 * jet_refine: jet_lp :182, rebalance_weak :592, rebalance_strong :356,
 * perform_moves :753; ProMap variants likewise). */
int hp_jet_begin(hp_ctx *ctx, const hp_graph *g, uint32_t k, int32_t lmax, const uint32_t *part,
                 const uint32_t *hier, const int32_t *dist, uint32_t levels, hp_jet **out);
int hp_jet_lp(hp_jet *jet, uint32_t ratio_pct, uint32_t *moves, uint32_t *count);
int hp_jet_weak(hp_jet *jet, uint32_t *moves, uint32_t *count);
int hp_jet_strong(hp_jet *jet, uint32_t *moves, uint32_t *count);
/* Applies the moves selected by the last lp/weak/strong call. */
int hp_jet_perform(hp_jet *jet, int64_t *obj, int32_t *maxw);
/* Copies the per-vertex Jet state (any pointer may be NULL). */
int hp_jet_state(hp_jet *jet, uint32_t *map, int32_t *bw, uint32_t *dest_part, int32_t *gain1, uint32_t *lock,
                 uint32_t *dest_cache, int32_t *gain_cache);
int hp_jet_end(hp_jet *jet);

/* Replaces edge_cut (src/utility/edge_cut.h:71-90) and comm_cost
 * (src/utility/comm_cost.h:36-56) with int64 sums. part is a host array. */
int hp_edge_cut(hp_ctx *ctx, const hp_graph *g, const uint32_t *part, int64_t *cut);
int hp_comm_cost(hp_ctx *ctx, const hp_graph *g, const uint32_t *part, const uint32_t *hier, const int32_t *dist,
                 uint32_t levels, int64_t *J);

/* Edge cut without any memory allocation. No counterpart in the reference:
 * it computes the same objective as hp_edge_cut (edge_cut, src/utility/
 * edge_cut.h:71-90) for callers that cannot allocate device memory at call
 * time -- a graph held in another framework's memory pool (a PyTorch tensor, a
 * serving engine that reserved HBM up front), where cudaMalloc would stall all
 * streams of the device or fail, and where no hp_ctx (whose arena is sized for
 * whole solves) exists.
 *
 * Inputs: a compact CSR on the current device (d_xadj: n+1 offsets with
 * d_xadj[n] == m; d_adj: m neighbour ids; d_ew: m weights or NULL for unit
 * weights), a HOST partition `part` of n labels, and a cudaStream_t (NULL =
 * the legacy default stream). The call stages `part` in a fixed static device
 * scratch area of this library (16 MiB + 256 B per device, reserved by the
 * driver when the library's module is loaded), runs one kernel on `stream`
 * and waits for that stream before it returns *cut.
 *
 * Limits and behaviour:
 *  - n > HP_EDGE_CUT_NOALLOC_MAX_N returns HP_ERR_TOO_LARGE before any device
 *    work; use hp_edge_cut for larger graphs.
 *  - Graph pointers that are not device memory of the current device, or a
 *    `part` in device memory, return HP_ERR_ARG; rows with d_xadj[u+1] <
 *    d_xadj[u] or > m, ids >= n and edge weights <= 0 (the graphs that
 *    hp_graph_upload rejects) are skipped by the kernel and reported as
 *    HP_ERR_GRAPH.
 *  - A failing CUDA call returns HP_ERR_CUDA with the runtime's error state
 *    cleared, so it is not reported again against the caller's later work.
 *  - The first call on a device resolves the scratch address on that device
 *    (and loads the module there); make that first call before any stream
 *    capture begins. Later calls only read a table.
 *  - The scratch counters are cleared by every call before its kernel; the
 *    staging area needs no initial value.
 *  - All calls on one device share the one scratch area: calls that overlap
 *    (from several host threads, or on streams the caller does not order) race
 *    and can return wrong results. Serialise them.
 * No cudaMalloc, cudaFree or allocating library routine is called. */
#define HP_EDGE_CUT_NOALLOC_MAX_N 4194304u
int hp_edge_cut_noalloc(uint32_t n, uint32_t m, const uint32_t *d_xadj, const uint32_t *d_adj, const int32_t *d_ew,
                        const uint32_t *part, void *stream, int64_t *cut);

/* ---- whole solves ---------------------------------------------------------- */

/* Replaces Solver(config).solve(HostGraph&) (src/datastructures/solver.h:248)
 * for GPU-HeiPa --config default|ultra. Host CSR in, host partition out. */
int hp_partition(hp_ctx *ctx, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj, const int32_t *ew,
                 const int32_t *vw, uint32_t k, double imbalance, int ultra, uint64_t seed, uint32_t *part,
                 int64_t *cut);
/* Same on an uploaded graph (the device-resident path). */
int hp_partition_graph(hp_ctx *ctx, const hp_graph *g, uint32_t k, double imbalance, int ultra, uint64_t seed,
                       uint32_t *part, int64_t *cut);
/* Replaces ProMapSolver<DistanceOracleMatrix>(config).solve / solve_multisection
 * (src/datastructures/promap_solver.h:146,238) for GPU-HeiProMap --config
 * IM|HM|HM-ultra. Returns J over directed entries in *J. */
int hp_map(hp_ctx *ctx, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj, const int32_t *ew,
           const int32_t *vw, const uint32_t *hier, const int32_t *dist, uint32_t levels, double imbalance, int mode,
           uint64_t seed, uint32_t *part, int64_t *J);
int hp_map_graph(hp_ctx *ctx, const hp_graph *g, const uint32_t *hier, const int32_t *dist, uint32_t levels,
                 double imbalance, int mode, uint64_t seed, uint32_t *part, int64_t *J);

/* Phase timings (ms) of the last solve on ctx: coarsening, contraction,
 * initial partitioning, uncontraction, refinement (solver.h:319-328 keys). */
int hp_last_solve_stats(const hp_ctx *ctx, double *phase_ms5, int64_t *initial_obj, int32_t *lmax,
                        uint32_t *levels);
/* Maximum block weight after initial partitioning and at the end of the last
 * solve (the "Init./Final max block w" lines of solver.h:301-329). */
int hp_last_solve_maxw(const hp_ctx *ctx, int32_t *initial_maxw, int32_t *final_maxw);
/* Size of hierarchy level `index` of the last solve (level 0 = input), the
 * per-level "n m" lines of solver.h:358; HP_ERR_ARG past the last level. */
int hp_last_solve_level(const hp_ctx *ctx, uint32_t index, uint32_t *n, uint64_t *m);

/* Diagnostics of the bounded waits: launches `blocks` (>= 2, all resident at
 * once) cooperative blocks of which one never reaches a grid barrier; the
 * others give up after the barrier's bounded wait (about a second), set
 * HP_DEVERR_SPIN in the kernel's error word and end. *err_bits receives that
 * word, *ms (if non-NULL) the kernel's duration. Returns HP_OK when the call
 * ran (whatever the bits), HP_ERR_ARG for a bad device or block count. The
 * cooperative Jet level loop and matching loop use the same barrier. No
 * counterpart in the reference. */
#define HP_DEVERR_SPIN 8u
int hp_selftest_barrier_timeout(int device, uint32_t blocks, uint32_t *err_bits, double *ms);

/* Diagnostics of the cooperative-launch budget (host only, no device work).
 * Grids whose blocks wait for one another at grid barriers (the cooperative
 * Jet level loop and matching loop, and the self-test above) share a budget
 * of as many blocks as the device has SMs: a grid of b blocks holds min(b,
 * budget) of it until its kernel has completed, and a larger grid holds all
 * of it. The grids running together then have at most one block per SM in
 * all, so they always become resident together and never wait for each
 * other. hp_coop_slot_acquire takes the whole budget of `device` (waiting at
 * most timeout_ms for every running cooperative grid to finish; HP_ERR_BUSY
 * when that did not happen) and hp_coop_slot_release returns it; a caller
 * that holds it delays every cooperative launch of this library on that
 * device. No counterpart in the reference (it runs one solve on one
 * stream). */
int hp_coop_slot_acquire(int device, int timeout_ms);
int hp_coop_slot_release(int device);

/* Sets a size threshold that chooses between equivalent implementations
 * (results are identical; only the launch structure changes): "jet_graph_max_m"
 * (levels up to this many CSR entries replay Jet iterations as CUDA graphs;
 * 0 = never), "order_small_n" (single-block rebalance ordering up to this many
 * vertices, at most 65536; 0 = never), "match_coop_max_n" / "match_coop_max_m"
 * (one cooperative launch for the matching loop of levels up to these sizes;
 * 0 = never), "jet_fused_max_n" / "jet_fused_max_m" (the whole refinement loop
 * of a level in one single-block launch up to these sizes, vertices capped at
 * 65536, when k <= 1024, or k <= 256 for the mapping objective; 0 = never),
 * "jet_coop_max_n" / "jet_coop_max_m" / "jet_coop_max_deg" (likewise as one
 * cooperative grid of 1024-thread blocks for larger sparse levels, up to this
 * many vertices, entries and entries per vertex; 0 = never), "jet_coop_rows"
 * (vertices per block of that grid),
 * "jet_hub_deg" (Jet connectivity passes with k <= 256: rows longer than this
 * are split into chunks of this many entries, one warp each; 64..4096),
 * "jet_chunk_mode" (the Jet chunk kernels read row entries 4 (0) or 8 (1) per
 * lane from global memory, or (2) stage row segments in shared memory with
 * bulk copies, 8 per lane; values above 2 are rejected), "jet_hub_conn" (1:
 * the per-kernel Jet loop keeps the block connectivity of hub rows up to date
 * from the moved vertices instead of rescanning the rows every pass; 0: rescan),
 * "jet_hub_track_pct" (with jet_hub_conn = 1: a perform whose moved rows hold
 * more entries than this percentage of all hub-row entries lets the next pass
 * rebuild the hub sums from the rows instead of updating them),
 * "jet_inval_all_pct" (1..100: where a recomputed gain equals a still-valid
 * cached one, a perform whose moved rows hold at least this percentage of the
 * level's entries resets every cached gain with one sequential fill instead of
 * one scattered reset per entry of the moved rows), "jet_vec_loads" (1: the
 * Jet row passes read CSR entries as 16-byte quads of four, one vector load
 * of adj and one of ew per lane; 0: four strided 4-byte loads; values above
 * 1 are rejected).
 * Unknown names return HP_ERR_ARG. No counterpart in the reference. */
int hp_tune(hp_ctx *ctx, const char *name, int64_t value);

/* Enables CUDA-event timing of the contraction and Jet-gain kernels on ctx;
 * hp_kernel_timing reports launches, total ms and algorithmic bytes. */
int hp_instrument(hp_ctx *ctx, int enable);
int hp_kernel_timing(hp_ctx *ctx, const char *name, uint64_t *launches, double *ms, double *bytes);
/* Per-launch records of the kernel timers in launch order (at most 2^20 per
 * enable): name, device milliseconds and algorithmic bytes of record `index`;
 * index 0 first waits for the stream. Returns HP_ERR_ARG past the last record.
 * A profiling aid without a counterpart in the reference. */
int hp_kernel_log(hp_ctx *ctx, uint64_t index, char *name, size_t name_len, double *ms, double *bytes);

/* Records event `slot` (0..7) on the context's stream; hp_event_elapsed
 * returns the milliseconds between two recorded slots (synchronises). */
int hp_event_record(hp_ctx *ctx, int slot);
int hp_event_elapsed(hp_ctx *ctx, int slot_a, int slot_b, float *ms);
/* Kernels launched by this process so far. */
uint64_t hp_kernel_launches(void);
/* Diagnostic phase timers (synchronising; off by default). hp_profile resets
 * them; hp_profile_entry enumerates (name, total ms, count) by index and
 * returns HP_ERR_ARG past the last entry. */
int hp_profile(hp_ctx *ctx, int enable);
int hp_profile_entry(const hp_ctx *ctx, uint32_t index, char *name, size_t name_len, double *ms, uint64_t *count);

/* ---- batched and served requests --------------------------------------------- */

/* One graph of a batch (host buffers, caller-owned). The results part (n
 * labels), cut and status are written by hp_partition_batch. */
typedef struct hp_batch_item {
    uint32_t n;
    uint64_t m;
    const uint32_t *xadj;
    const uint32_t *adj;
    const int32_t *ew; /* NULL: unit edge weights */
    const int32_t *vw; /* NULL: unit vertex weights */
    uint32_t k;
    double imbalance;
    int ultra;
    uint64_t seed;
    uint32_t *part; /* out */
    int64_t cut;    /* out */
    int status;     /* out: HP_OK or this item's error */
} hp_batch_item;

/* Partitions `count` independent graphs (GPU-HeiPa each, the same result as
 * hp_partition on that graph alone). Up to `workers` graphs (0: 8) run at
 * once on their own streams, each admitted by a device-memory estimate of its
 * solve (input + 96 B per entry + 256 B per vertex + 16 MiB) into the
 * context's free arena. Returns HP_OK, or the first failing item's status
 * (hp_last_error names the item). No counterpart in the reference, which
 * solves one graph per process. */
int hp_partition_batch(hp_ctx *ctx, hp_batch_item *items, uint32_t count, uint32_t workers);

/* Serving loop: requests are queued on submit and run as soon as a worker
 * (0: 8) and enough of the server's device buffer (buffer_bytes, allocated at
 * create) are free, oldest first, with smaller requests allowed past a
 * blocked one a bounded number of times. Each request's result equals the
 * plain call's (hp_partition / hp_map) on the same input. Host buffers passed
 * to a submit must stay valid until its hp_server_wait returns. Safe to call
 * from several host threads. No counterpart in the reference. */
typedef struct hp_server hp_server;
int hp_server_create(int device, size_t buffer_bytes, uint32_t workers, hp_server **out);
int hp_server_submit_partition(hp_server *s, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj,
                               const int32_t *ew, const int32_t *vw, uint32_t k, double imbalance, int ultra,
                               uint64_t seed, uint32_t *part, uint64_t *request);
int hp_server_submit_map(hp_server *s, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj,
                         const int32_t *ew, const int32_t *vw, const uint32_t *hier, const int32_t *dist,
                         uint32_t levels, double imbalance, int mode, uint64_t seed, uint32_t *part,
                         uint64_t *request);
/* done = 1 when the request has finished (or is unknown). */
int hp_server_poll(hp_server *s, uint64_t request, int *done);
/* Blocks until the request finishes; returns its status and writes its
 * objective (cut or J), latency (submit to finish) and run time in ms. */
int hp_server_wait(hp_server *s, uint64_t request, int64_t *objective, double *latency_ms, double *run_ms);
/* Message of the last failed request returned by hp_server_wait. */
const char *hp_server_last_error(hp_server *s);
/* Finishes every queued request, then frees the server. */
int hp_server_destroy(hp_server *s);

/* ---- host utilities (no device work) --------------------------------------- */

/* Replaces from_file (src/datastructures/host_graph.h:154-247). */
int hp_read_metis(const char *path, hp_host_graph **out);
/* Synthetic generators for the benchmark workloads. */
int hp_gen_grid(uint32_t w, uint32_t h, int32_t w_lo, int32_t w_hi, uint64_t seed, hp_host_graph **out);
int hp_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, int32_t w_lo, int32_t w_hi,
                uint64_t seed, int explicit_vw, hp_host_graph **out);
int hp_gen_rgg3d(uint32_t n, double mean_degree, int32_t w_lo, int32_t w_hi, uint64_t seed, int explicit_vw,
                 hp_host_graph **out);
/* Sizes (has_ew/has_vw: 0 when weights are unit) and contents of a host graph. */
int hp_host_graph_info(const hp_host_graph *g, uint32_t *n, uint64_t *m, int *has_ew, int *has_vw);
int hp_host_graph_copy(const hp_host_graph *g, uint32_t *xadj, uint32_t *adj, int32_t *ew, int32_t *vw);
int hp_host_graph_free(hp_host_graph *g);
/* Writes a METIS file (fmt 0/1/10/11 from the flags). */
int hp_write_metis(const char *path, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj,
                   const int32_t *ew, const int32_t *vw);
/* Replaces write_partition (src/utility/util.h:288-329): one id per line. */
int hp_write_partition(const char *path, const uint32_t *part, uint32_t n);

/* Replaces kway_partition(HostGraph&, k, imbalance, seed, HostPartition&)
 * (src/initial_partitioning/kway_partitioner/kway_core.h:1548-1571): the
 * reference's METIS-derived host partitioner, which every solve runs on its
 * coarsest graph. Host CSR in (rows in the order given; vw / ew NULL for unit
 * weights), n labels < k out. The imbalance is narrowed to float and the seed
 * to int as in the reference; on the same graph, k, imbalance and seed the
 * partition equals the reference's. HP_ERR_GRAPH for ids out of range or self
 * loops; safe to call from concurrent threads. */
int hp_initial_partition(uint32_t n, const uint32_t *xadj, const uint32_t *adj, const int32_t *vw, const int32_t *ew,
                         uint32_t k, double imbalance, uint64_t seed, uint32_t *part);

#ifdef __cplusplus
}
#endif

#endif /* GPUHEIPA_H */
