// Execution context: one device, one stream, one device-memory arena and a
// small pinned status block through which kernels report counts, sums and
// error bits to the host (one synchronisation per read).
//
// The arena replaces the reference's KokkosMemoryStack
// (src/datastructures/kokkos_memory_stack.h:36-206): one up-front device
// allocation, LIFO allocation from the front (long-lived: graph hierarchy,
// mappings, partitions) and from the back (per-phase scratch), 256-byte
// alignment, and an error return instead of abort() on exhaustion.
#pragma once
#include <cuda_runtime.h>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace hp {

struct HpError {
    int code;
    std::string msg;
};

#define HP_CUDA(x)                                                                                   \
    do {                                                                                             \
        cudaError_t e_ = (x);                                                                        \
        if (e_ != cudaSuccess)                                                                       \
            throw ::hp::HpError{::hp::HP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define HP_LAUNCH_CHECK() HP_CUDA(cudaGetLastError())

class Arena {
public:
    void init(size_t bytes);
    // Uses [p, p + bytes) of memory owned by someone else (never freed here).
    void attach(void *p, size_t bytes);
    void destroy();
    void *front(size_t bytes);
    void *back(size_t bytes);
    size_t front_mark() const { return front_; }
    size_t back_mark() const { return back_; }
    void front_release(size_t mark) { front_ = mark; }
    void back_release(size_t mark) { back_ = mark; }
    size_t capacity() const { return size_; }
    size_t used() const { return front_ + (size_ - back_); }
    size_t peak() const { return peak_; }
    char *base() const { return base_; }

private:
    char *base_ = nullptr;
    size_t size_ = 0, front_ = 0, back_ = 0, peak_ = 0;
    bool owns_ = true;
};

// Restores the back (scratch) end of the arena when leaving a scope.
struct ScratchScope {
    Arena &a;
    size_t mark;
    explicit ScratchScope(Arena &ar) : a(ar), mark(ar.back_mark()) {}
    ~ScratchScope() { a.back_release(mark); }
};

// Values kernels report to the host; lives in device memory and is copied to
// a pinned mirror when the host needs it.
struct DevStatus {
    u32 err;          // DevErr bits
    u32 cnt[15];      // list lengths and other counters
    long long sum[8]; // 64-bit sums (objective deltas, ...)
    int imax[8];      // maxima (block weights, ...)
};

// Optional per-kernel timing with CUDA events on the context's stream. When
// enabled, instrumented launch sites record an event pair and the
// algorithmic bytes of the launch; resolve() (after a stream sync) turns the
// pairs into per-name totals.
struct Instr {
    struct Rec {
        std::string name;
        cudaEvent_t a, b;
        double bytes;
    };
    struct Total {
        std::string name;
        u64 launches = 0;
        double ms = 0.0;
        double bytes = 0.0;
    };
    struct Logged {
        std::string name;
        double ms;
        double bytes;
    };
    static constexpr size_t LOG_MAX = 1u << 20;  // resolved records kept in launch order
    bool enabled = false;
    bool capturing = false;  // stream capture in progress: records are skipped
    std::vector<Rec> pending;
    std::vector<Total> totals;
    std::vector<Logged> log;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t get_event();
    // begin() returns a record index (or SIZE_MAX when disabled) for end().
    size_t begin(cudaStream_t s, const char *name, double bytes);
    void end(cudaStream_t s, size_t idx);
    void resolve();  // requires the stream to be idle
    void clear();
    void destroy();
};

// Diagnostic phase timers: when enabled, a scope synchronises the stream on
// entry and exit and accumulates wall-clock milliseconds per name. Off by
// default (no synchronisation is added to the normal path).
struct PhaseProf {
    bool enabled = false;
    bool capturing = false;  // stream capture in progress: scopes are skipped
    std::vector<std::pair<std::string, double> > totals;
    std::vector<std::pair<std::string, u64> > counts;
    void add(const char *name, double ms);
    void clear() {
        totals.clear();
        counts.clear();
    }
};

// Size thresholds that choose between equivalent implementations (results
// are identical either way; only the launch structure differs).
struct Tunables {
    u64 jet_graph_max_m = 1ull << 24;  // Jet iterations replayed as CUDA graphs up to this many entries
    u32 order_small_n = 16384;         // single-block rebalance ordering up to this many vertices
    u32 match_coop_max_n = 1u << 17;   // cooperative matching loop up to this many vertices ...
    u64 match_coop_max_m = 1ull << 21; // ... and entries
    u32 jet_fused_max_n = 4096;        // whole Jet level loop in one block up to this many vertices ...
    u64 jet_fused_max_m = 1ull << 18;  // ... and entries
    u32 jet_coop_max_n = 65536;        // ... else as a cooperative grid up to this many vertices ...
    u64 jet_coop_max_m = 1ull << 21;   // ... and entries ...
    u32 jet_coop_max_deg = 32;         // ... and average degree (dense levels keep the whole GPU)
    u32 jet_coop_rows = 1024;          // vertices per block of that grid
    u32 jet_hub_deg = 1024;            // Jet table passes: rows above this length are cut into chunks of it (64..4096)
    u32 jet_chunk_mode = 0;            // chunk kernels: 0 = 4 entries per lane, 1 = 8, 2 = bulk-copy staged rows
    u32 jet_hub_conn = 1;              // per-kernel Jet loop: keep hub-row connectivity up to date (1) or rescan (0)
    u32 jet_hub_track_pct = 50;        // ... updated while the moved rows hold <= this % of the hub-row entries
    u32 jet_vec_loads = 1;             // Jet row passes read row entries as 16-byte quads (1) or 4-byte strided loads (0)
    u32 jet_inval_all_pct = 5;         // a perform whose moved rows hold >= this % of all entries resets every cache at once
};

struct Ctx {
    int device = 0;
    Tunables tune;
    int sm_count = NUM_SMS_HINT;
    cudaStream_t stream = nullptr;
    Arena arena;
    DevStatus *d_status = nullptr;
    DevStatus *h_status = nullptr;
    std::string last_error;
    bool owns_arena = true;
    Instr instr;
    PhaseProf prof;
    cudaEvent_t events[8] = {};
    cudaEvent_t event(int slot);  // created on first use
    // Worker contexts (own stream and status word, no arena of their own)
    // for running independent sub-solves concurrently; created on first use
    // and kept until destroy().
    std::vector<std::unique_ptr<Ctx> > workers;
    Ctx &worker(size_t i);

    void init(int dev, size_t arena_bytes);
    void destroy();
    template<typename T>
    T *falloc(size_t n) {
        return (T *) arena.front(sizeof(T) * (n == 0 ? 1 : n));
    }
    template<typename T>
    T *balloc(size_t n) {
        return (T *) arena.back(sizeof(T) * (n == 0 ? 1 : n));
    }
    void zero_status();                 // async, clears everything including err
    void zero_counters();               // async, keeps err
    const DevStatus &read_status();     // syncs the stream
    void sync();
    void check_device_error();          // reads status; throws on error bits
    u32 grid(u64 items, u32 per_block) const {
        u64 b = (items + per_block - 1) / per_block;
        if (b == 0) b = 1;
        u64 cap = (u64) sm_count * 16;
        return (u32) (b > cap ? cap : b);
    }
};

// Cooperative launches (grids whose blocks wait for one another at grid
// barriers) share a per-device budget of S blocks, S = the SM count.
// Concurrent solves (HM sub-solves, batch and server requests) may each want
// such a grid. A grid of b blocks takes min(b, S) of the budget and gives it
// back after its kernel has completed; a grid of more than S blocks takes all
// of it and runs alone (the cooperative launch itself checks that it fits).
// Why this is enough: the grids holding budget have at most S blocks in all,
// and every block fits on an SM that holds none of them (it launched at all).
// While any of those blocks is still waiting to start, fewer than S SMs hold
// blocks of these grids, so some SM holds none; the waiting block starts
// there once the ordinary kernels on that SM end, and those never wait for
// anything. So all blocks of all running grids become resident together, and
// no grid waits at a barrier for SMs that another waiting grid holds.
class CoopSlots {
public:
    // Takes min(blocks, budget) blocks of `device`'s budget (waiting while
    // they are not free); budget = the device's SM count.
    static void acquire(int device, u32 blocks, u32 budget);
    static void release(int device, u32 blocks, u32 budget);
    // The whole budget (no other cooperative grid runs); waits at most
    // timeout_ms, false when it did not become free.
    static bool try_acquire_all_for(int device, int timeout_ms);
    static void release_all(int device);
};

// Holds `blocks` of the device's cooperative budget for the lifetime of the
// scope. The destructor first waits for `stream` (errors ignored), so the
// budget is never returned while the grid may still run, even when the scope
// is left by an exception between the launch and the status read.
struct CoopGuard {
    int device;
    cudaStream_t stream;
    u32 blocks, budget;
    CoopGuard(int dev, cudaStream_t s, u32 b, u32 sms) : device(dev), stream(s), blocks(b), budget(sms) {
        CoopSlots::acquire(dev, blocks, budget);
    }
    ~CoopGuard() {
        cudaStreamSynchronize(stream);
        CoopSlots::release(device, blocks, budget);
    }
    CoopGuard(const CoopGuard &) = delete;
    CoopGuard &operator=(const CoopGuard &) = delete;
};

// Thrown when a cooperative grid's bounded barrier wait gave up
// (DEV_ERR_SPIN): the caller redoes that work on its per-kernel launch path.
struct CoopSpin {};

// Records a CUDA-event pair around the launches in a C++ scope when
// instrumentation is enabled (no synchronisation).
struct KernTimer {
    Ctx &c;
    size_t idx;
    KernTimer(Ctx &ctx, const char *name, double bytes = 0.0);
    ~KernTimer();
};

// RAII scope for PhaseProf.
struct ProfScope {
    Ctx &c;
    const char *name;
    double t0 = 0;
    ProfScope(Ctx &ctx, const char *nm);
    ~ProfScope();
};

} // namespace hp
