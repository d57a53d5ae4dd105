// Jet refinement kernels. Semantics: src/refinement/jet_label_propagation.h
// and src/refinement/promap_jet_label_propagation.h with the deterministic
// tie rules documented in jet.cuh (lowest block id on best-block ties,
// mini-bucket order by vertex id, fallback slots in ascending vertex id).
#include "jet.cuh"
#include "stage.cuh"

#include <mutex>
#include <optional>
#include <vector>
#include "prims.cuh"

#include <algorithm>

namespace hp {
namespace {

constexpr u32 JT = 16;             // thread-level rows up to this degree
constexpr u32 JW_DEG = 4096;       // warp-level rows up to this degree ...
constexpr u32 JW_SLOTS = 1024;     // ... whose block table fits this per-warp capacity
constexpr int JW_BLOCK = 128;      // 4 warps per block
constexpr u32 JB_SLOTS = 16384;    // largest per-block table (128 KB)
constexpr int JB_BLOCK = 512;
constexpr u32 EMPTY = NO_BLOCK_ID;
// Hub rows of the table-based passes are cut into chunks of hub_deg entries
// (Tunables::jet_hub_deg), one warp each, when tables are direct-indexed and
// k <= HUB_K; the chunks' partial connectivity is summed per row in global
// memory and the last chunk to finish completes the row. With chunking
// available, rows of more than hub_deg entries count as hubs, so that no warp
// scans a long row alone.
constexpr u32 HUB_K = 256;
constexpr int ST_CHUNKS = 8;  // status slot: hub chunk items of the current pass
constexpr u32 NOKEY = 0xFFFFFFFFu;
// During perform, map[] holds the new label of every vertex and the MOVED
// bit marks the vertices that changed block in this iteration; their old
// label is in dest_part[] (the reference's swap, perform_moves :794-795).
constexpr u32 MOVED = 0x80000000u;
// dlab (per-kernel level loop): label, moved bit, old label and hub slot of
// a vertex in one word, so that the delta pass needs one gather per
// neighbour.
constexpr unsigned long long DL_LABEL = 0xFFFFull;           // label (k <= MAX_K)
constexpr unsigned long long DL_MOVED = 1ull << 16;          // changed block in this perform
constexpr int DL_OLD_SHIFT = 17;                              // old label (valid with DL_MOVED)
constexpr unsigned long long DL_OLD = 0xFFFFull << DL_OLD_SHIFT;
constexpr int DL_SLOT_SHIFT = 33;                             // tracked hub slot + 1 (0: not a tracked hub)
constexpr u32 DL_MAX_HUBS = 0x7FFFFFFEu;

// Block-tier table size: a row never has more distinct blocks than k.
inline u32 block_slots_for(u32 k) {
    u32 t = 64;
    while (t < 2 * k && t < JB_SLOTS) t <<= 1;
    return t;
}

struct JArgs {
    DGraph g;
    u32 k;
    u32 blk_slots;  // block-tier table size (power of two)
    s32 lmax;
    s32 g_weight;
    const u32 *code;     // non-null: process-mapping objective
    const s32 *bitdist;
    u32 *map;
    s32 *bw;
    u32 *dest_cache;
    s32 *gain_cache;
    u32 *lock;
    u32 *dest_part;
    s32 *gain1;
    u32 *cand;
    u32 *moves;
    u32 *heavy;
    u32 *heavy2;
    unsigned long long *items;  // chunk work items (afterburner, delta): (vertex << 32) | chunk
    u32 items_cap;
    unsigned long long inval_all_min;  // moved-row entries from which perform resets every cache
    s32 *hubacc;  // hub rows: k partial-connectivity sums per row slot (zero between uses), or null
    u32 *hubcnt;  // hub rows: finished chunks per row slot (zero between uses)
    u32 hub_cap;  // row slots of hubacc / hubcnt
    u32 hub_deg;  // hub threshold and chunk length (entries) when hubacc is set
    // Per-kernel level loop: dlab[v] packs v's label (DL_LABEL bits), its
    // moved bit (DL_MOVED), its old label while moved (DL_OLD) and, with
    // tracked hubs, its hub slot + 1 (above DL_SLOT_SHIFT). Null in the
    // single-launch level loop.
    unsigned long long *dlab;
    // Afterburner records (per-kernel level loop): gain1 (low 32 bits),
    // dest_part (next 16) and label (top 16) of a vertex, written by the
    // filter, so that a neighbour costs one gather. Null: separate arrays.
    unsigned long long *abrec;
    // Row entries read as 16-byte quads (Tunables::jet_vec_loads) in the
    // kernels that support it; else four strided 4-byte loads.
    u32 vec;
    // Tracked hub connectivity (k <= HUB_K, hub_cur set): hubacc then
    // holds, for every hub row h and block b, the row's connection to b at
    // hubacc[h * k + b] (the two counters one moved neighbour changes share a
    // cache line; a block-major layout measured slower), kept up to date by
    // the delta pass. Without tracking, hub rows are rescanned in chunks on
    // every pass.
    // A perform whose moved rows hold more than hub_track_max entries does
    // not update the hub sums but advances the generation *hub_cur; a pass
    // that needs the sums of a hub whose generation (hub_gen) is older
    // rebuilds that hub's sums from its row first (hub_vertex: the row of
    // each hub slot). hub_cur is null without tracking.
    unsigned long long hub_track_max;
    u32 *hub_cur;
    u32 *hub_gen;
    const u32 *hub_vertex;
    s32 *abacc;  // afterburner partial sums of multi-chunk rows (zero between uses)
    u32 *abcnt;  // afterburner finished chunks of multi-chunk rows (zero between uses)
    DevStatus *st;
};

__device__ __forceinline__ s32 D(const JArgs &a, u32 x, u32 y) { return dist_of(a.code, a.bitdist, x, y); }

// ---- group abstraction: warp (BLK=false) or block (BLK=true) ---------------------
template<bool BLK>
struct Grp {
    static __device__ __forceinline__ u32 tid() { return BLK ? threadIdx.x : (u32) lane_id(); }
    static __device__ __forceinline__ u32 size() { return BLK ? blockDim.x : 32u; }
    static __device__ __forceinline__ void sync() {
        if (BLK) __syncthreads();
        else __syncwarp();
    }
    static __device__ __forceinline__ unsigned long long max_u64(unsigned long long v, unsigned long long *sm) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long y = __shfl_xor_sync(FULL, v, o);
            v = y > v ? y : v;
        }
        if (!BLK) return v;
        if (lane_id() == 0) sm[warp_in_block()] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long r = 0;
            for (u32 w = 0; w < (blockDim.x >> 5); ++w) r = sm[w] > r ? sm[w] : r;
            sm[32] = r;
        }
        __syncthreads();
        v = sm[32];
        __syncthreads();
        return v;
    }
    static __device__ __forceinline__ long long sum_s64(long long v, long long *sm) {
        v = warp_sum<long long>(v);
        if (!BLK) return v;
        if (lane_id() == 0) sm[warp_in_block()] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            long long r = 0;
            for (u32 w = 0; w < (blockDim.x >> 5); ++w) r += sm[w];
            sm[32] = r;
        }
        __syncthreads();
        v = sm[32];
        __syncthreads();
        return v;
    }
};

// Loads of Jet state (labels, targets, gains) that the calling kernel does not
// write go through the non-coherent path (NC); the fused small-level kernel,
// which writes them between its phases, uses plain loads.
template<bool NC, typename T>
__device__ __forceinline__ T ldj(const T *p) {
    return NC ? __ldg(p) : *p;
}

// Loads B row entries (ids and weights) strided by nthreads from t0.
template<int B>
__device__ __forceinline__ void load_entries(const JArgs &a, u64 beg, u32 t0, u32 to, u32 nthreads, u32 (&v)[B],
                                             s32 (&w)[B]) {
#pragma unroll
    for (int j = 0; j < B; ++j) {
        const u32 t = t0 + j * nthreads;
        v[j] = t < to ? __ldg(&a.g.adj[beg + t]) : SENTINEL;  // SENTINEL == EMPTY
        w[j] = t < to ? g_ew(a.g, beg + t) : 0;
    }
}

// 128-bit row reads: the four CSR entries of quad qi (positions [4 qi,
// 4 qi + 4)) with one 16-byte load of adj and one of ew; entries outside
// [lo, hi) come back as SENTINEL with weight 0. Whole quads are read: CSR
// arrays come from the arena, whose allocations are 256-byte aligned and
// padded to 256 bytes, so a quad holding an entry lies inside its array's
// allocation.
__device__ __forceinline__ void load_quad(const JArgs &a, u64 qi, u64 lo, u64 hi, u32 (&v)[4], s32 (&w)[4]) {
    const uint4 q = __ldg(reinterpret_cast<const uint4 *>(a.g.adj) + qi);
    int4 r = make_int4(1, 1, 1, 1);
    if (a.g.ew) r = __ldg(reinterpret_cast<const int4 *>(a.g.ew) + qi);
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
    w[0] = r.x;
    w[1] = r.y;
    w[2] = r.z;
    w[3] = r.w;
    const u64 p = qi * 4;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (p + j < lo || p + j >= hi) {
            v[j] = SENTINEL;
            w[j] = 0;
        }
}

// Quad qi of the entries [lo, hi) if it holds any of them (returns true),
// else SENTINEL / 0 in v and w (returns false).
__device__ __forceinline__ bool next_quad(const JArgs &a, u64 qi, u64 lo, u64 hi, u32 (&v)[4], s32 (&w)[4]) {
    if (qi * 4 >= hi) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            v[j] = SENTINEL;
            w[j] = 0;
        }
        return false;
    }
    load_quad(a, qi, lo, hi, v, w);
    return true;
}

__device__ __forceinline__ u32 thash(u32 key, u32 mask) { return (key * 2654435761u >> 7) & mask; }

__device__ __forceinline__ u32 table_mask_for(u32 len, u32 k, u32 cap) {
    u32 want = 2 * (len < k ? len : k);
    u32 t = 64;
    while (t < want && t < cap) t <<= 1;
    return t - 1;
}

// Aggregates conn(u, .) into the group's hashed table (cleared on entry).
// Four entries per thread are loaded before they are inserted.
template<bool BLK, bool NC = true>
__device__ __forceinline__ void table_build(const JArgs &a, u32 u, u32 *tk, s32 *tv, u32 mask) {
    const u64 beg = __ldg(&a.g.rowptr[u]);
    const u32 len = __ldg(&a.g.rowlen[u]);
    const u32 gs = Grp<BLK>::size();
    for (u32 t0 = Grp<BLK>::tid(); t0 < len; t0 += 4 * gs) {
        u32 bb[4];
        s32 ww[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const u32 t = t0 + j * gs;
            bb[j] = t < len ? __ldg(&a.g.adj[beg + t]) : EMPTY;
            ww[j] = t < len ? g_ew(a.g, beg + t) : 0;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (bb[j] != EMPTY) bb[j] = ldj<NC>(&a.map[bb[j]]);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const u32 b = bb[j];
            if (b == EMPTY) continue;
            u32 h = thash(b, mask);
            bool ok = false;
            for (u32 p = 0; p <= mask; ++p) {
                const u32 prev = atomicCAS(&tk[h], EMPTY, b);
                if (prev == EMPTY || prev == b) {
                    atomicAdd(&tv[h], ww[j]);
                    ok = true;
                    break;
                }
                h = (h + 1) & mask;
            }
            if (!ok) set_error(&a.st->err, DEV_ERR_HASH_FULL);
        }
    }
    Grp<BLK>::sync();
}

template<bool BLK>
__device__ __forceinline__ void table_clear(u32 *tk, s32 *tv, u32 mask) {
    Grp<BLK>::sync();
    for (u32 s = Grp<BLK>::tid(); s <= mask; s += Grp<BLK>::size()) {
        tk[s] = EMPTY;
        tv[s] = 0;
    }
    Grp<BLK>::sync();
}

// Direct-indexed variant for small k: tv[b] = conn(u, b) for b < k (0 = no
// connection; weights are positive), so an entry costs one shared-memory add
// and no compare-and-swap. Four entries per thread are loaded (ids, then
// labels) before any table update, which keeps four gathers in flight.
template<bool BLK, bool NC = true>
__device__ __forceinline__ void dtable_build_range(const JArgs &a, u32 u, s32 *tv, u32 from, u32 len) {
    const u64 beg = __ldg(&a.g.rowptr[u]);
    const u32 gs = Grp<BLK>::size(), tid = Grp<BLK>::tid();
    if (NC && a.vec) {
        // the same with the entries read as 16-byte quads
        const u64 lo = beg + from, hi = beg + len;
        u64 qi = (lo >> 2) + tid;
        u32 b[4];
        s32 w[4];
        if (next_quad(a, qi, lo, hi, b, w)) {
            for (;;) {
                const u64 qn = qi + gs;
                u32 bn[4];
                s32 wn[4];
                const bool more = next_quad(a, qn, lo, hi, bn, wn);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (b[j] != EMPTY) b[j] = ldj<NC>(&a.map[b[j]]);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (b[j] != EMPTY) atomicAdd(&tv[b[j]], w[j]);
                if (!more) break;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    b[j] = bn[j];
                    w[j] = wn[j];
                }
                qi = qn;
            }
        }
        Grp<BLK>::sync();
        return;
    }
    if (NC) {
        // kernels that do not write labels: the next four entries are loaded
        // while the current four labels are gathered
        u32 t0 = from + tid;
        if (t0 < len) {
            u32 b[4];
            s32 w[4];
            load_entries<4>(a, beg, t0, len, gs, b, w);
            for (;;) {
                const u32 t1 = t0 + 4 * gs;
                u32 bn[4];
                s32 wn[4];
                load_entries<4>(a, beg, t1, len, gs, bn, wn);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (b[j] != EMPTY) b[j] = ldj<NC>(&a.map[b[j]]);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (b[j] != EMPTY) atomicAdd(&tv[b[j]], w[j]);
                if (t1 >= len) break;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    b[j] = bn[j];
                    w[j] = wn[j];
                }
                t0 = t1;
            }
        }
        Grp<BLK>::sync();
        return;
    }
    for (u32 t0 = from + tid; t0 < len; t0 += 4 * gs) {
        u32 b[4];
        s32 w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const u32 t = t0 + j * gs;
            b[j] = t < len ? __ldg(&a.g.adj[beg + t]) : EMPTY;
            w[j] = t < len ? g_ew(a.g, beg + t) : 0;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (b[j] != EMPTY) b[j] = ldj<NC>(&a.map[b[j]]);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (b[j] != EMPTY) atomicAdd(&tv[b[j]], w[j]);
    }
    Grp<BLK>::sync();
}

template<bool BLK, bool NC = true>
__device__ __forceinline__ void dtable_build(const JArgs &a, u32 u, s32 *tv) {
    dtable_build_range<BLK, NC>(a, u, tv, 0, __ldg(&a.g.rowlen[u]));
}

template<bool BLK>
__device__ __forceinline__ void dtable_clear(s32 *tv, u32 k) {
    Grp<BLK>::sync();
    for (u32 s = Grp<BLK>::tid(); s < k; s += Grp<BLK>::size()) tv[s] = 0;
    Grp<BLK>::sync();
}

// Connectivity table of one row: direct-indexed (DIRECT) or hashed.
template<bool BLK, bool DIRECT, bool NC = true>
struct ConnTable {
    u32 *tk;
    s32 *tv;
    u32 mask;  // hashed: slots - 1
    u32 k;
    __device__ __forceinline__ void build(const JArgs &a, u32 u) {
        if (DIRECT) dtable_build<BLK, NC>(a, u, tv);
        else table_build<BLK, NC>(a, u, tk, tv, mask);
    }
    __device__ __forceinline__ u32 slots() const { return DIRECT ? k : mask + 1; }
    __device__ __forceinline__ u32 key(u32 s) const { return DIRECT ? (tv[s] != 0 ? s : EMPTY) : tk[s]; }
    __device__ __forceinline__ s32 val(u32 s) const { return tv[s]; }
    __device__ __forceinline__ void clear() {
        if (DIRECT) dtable_clear<BLK>(tv, k);
        else table_clear<BLK>(tk, tv, mask);
    }
};

// Thread-level connectivity row in registers (degree <= JT).
struct TRow {
    u32 b[JT];
    s32 c[JT];
};

// Connectivity row of a vertex of at most JT entries, in registers. All
// entries are loaded first and their labels gathered together (JT independent
// loads in flight instead of a chain of JT), then equal blocks are merged into
// their first occurrence. Labels are not written by the kernels that call
// this, so they are read through the non-coherent path.
template<bool NC = true>
__device__ __forceinline__ void trow_build(const JArgs &a, u32 u, TRow &r) {
    const u64 beg = __ldg(&a.g.rowptr[u]);
    const u32 len = __ldg(&a.g.rowlen[u]);
#pragma unroll
    for (int s = 0; s < (int) JT; ++s) {
        r.b[s] = (u32) s < len ? __ldg(&a.g.adj[beg + s]) : EMPTY;
        r.c[s] = (u32) s < len ? g_ew(a.g, beg + s) : 0;
    }
#pragma unroll
    for (int s = 0; s < (int) JT; ++s)
        if (r.b[s] != EMPTY) r.b[s] = ldj<NC>(&a.map[r.b[s]]);
#pragma unroll
    for (int s = 1; s < (int) JT; ++s) {
#pragma unroll
        for (int t = 0; t < s; ++t)
            if (r.b[s] != EMPTY && r.b[t] == r.b[s]) {
                r.c[t] = wadd(r.c[t], r.c[s]);
                r.b[s] = EMPTY;
                r.c[s] = 0;
            }
    }
}

__device__ __forceinline__ unsigned long long cut_key(s32 c, u32 b) {
    return ((unsigned long long) (u32) c << 32) | (u32) ~b;
}
__device__ __forceinline__ unsigned long long delta_key(s32 d, u32 b) {
    return ((unsigned long long) ((u32) d ^ 0x80000000u) << 32) | (u32) ~b;
}

// ---- Jet LP best block (jet_lp :193-238 / ProMap_jet_lp :219-263) ------------------

__device__ __forceinline__ void lp_store(const JArgs &a, u32 u, u32 best, s32 gain) {
    a.gain_cache[u] = gain;
    a.dest_cache[u] = best;
    a.dest_part[u] = best;
}

__device__ __forceinline__ void lp_finish_cut(const JArgs &a, u32 u, s32 own, unsigned long long bk, u32 ratio) {
    u32 best = NO_MOVE;
    s32 gain = 0;
    if (bk) {
        const s32 bc = (s32) (u32) (bk >> 32);
        if (bc >= own || (s64) own - (s64) bc < ((s64) ratio * (s64) own) / 100) {
            best = ~(u32) bk;
            gain = wsub(bc, own);
        }
    }
    lp_store(a, u, best, gain);
}

__device__ __forceinline__ void lp_finish_map(const JArgs &a, u32 u, unsigned long long bk) {
    u32 best = NO_MOVE;
    s32 gain = 0;
    if (bk) {
        const s32 d = (s32) ((u32) (bk >> 32) ^ 0x80000000u);
        if (d >= 0) {
            best = ~(u32) bk;
            gain = d;
        }
    }
    lp_store(a, u, best, gain);
}

template<bool NC = true>
__device__ __forceinline__ void lp_thread(const JArgs &a, u32 u, u32 ratio) {
    TRow r;
    trow_build<NC>(a, u, r);
    const u32 o = a.map[u];
    unsigned long long bk = 0;
    if (!a.code) {
        s32 own = 0;
#pragma unroll
        for (int s = 0; s < (int) JT; ++s) {
            if (r.b[s] == EMPTY) continue;
            if (r.b[s] == o) own = r.c[s];
            else {
                unsigned long long k = cut_key(r.c[s], r.b[s]);
                bk = k > bk ? k : bk;
            }
        }
        lp_finish_cut(a, u, own, bk, ratio);
    } else {
#pragma unroll
        for (int s = 0; s < (int) JT; ++s) {
            if (r.b[s] == EMPTY || r.b[s] == o) continue;
            s32 d = 0;
#pragma unroll
            for (int t = 0; t < (int) JT; ++t)
                if (r.b[t] != EMPTY) d = wadd(d, wmul(r.c[t], wsub(D(a, o, r.b[t]), D(a, r.b[s], r.b[t]))));
            unsigned long long k = delta_key(d, r.b[s]);
            bk = k > bk ? k : bk;
        }
        lp_finish_map(a, u, bk);
    }
}

// Best block of u from its built connectivity table T (clears T).
template<bool BLK, bool DIRECT, bool NC = true>
__device__ __forceinline__ void lp_finish_group(const JArgs &a, u32 u, u32 ratio, ConnTable<BLK, DIRECT, NC> T,
                                                unsigned long long *smu, long long *sms) {
    const u32 o = a.map[u];
    unsigned long long bk = 0;
    long long own = 0;
    const u32 ns = T.slots();
    for (u32 s = Grp<BLK>::tid(); s < ns; s += Grp<BLK>::size()) {
        const u32 b = T.key(s);
        if (b == EMPTY) continue;
        if (b == o) {
            own = T.val(s);
            continue;
        }
        unsigned long long k;
        if (!a.code) {
            k = cut_key(T.val(s), b);
        } else {
            s32 d = 0;
            for (u32 t = 0; t < ns; ++t) {
                const u32 id = T.key(t);
                if (id != EMPTY) d = wadd(d, wmul(T.val(t), wsub(D(a, o, id), D(a, b, id))));
            }
            k = delta_key(d, b);
        }
        bk = k > bk ? k : bk;
    }
    bk = Grp<BLK>::max_u64(bk, smu);
    own = Grp<BLK>::sum_s64(own, sms);
    if (Grp<BLK>::tid() == 0) {
        if (!a.code) lp_finish_cut(a, u, (s32) own, bk, ratio);
        else lp_finish_map(a, u, bk);
    }
    T.clear();
}

template<bool BLK, bool DIRECT, bool NC = true>
__device__ __forceinline__ void lp_group(const JArgs &a, u32 u, u32 ratio, ConnTable<BLK, DIRECT, NC> T,
                                         unsigned long long *smu, long long *sms) {
    T.build(a, u);
    lp_finish_group<BLK, DIRECT, NC>(a, u, ratio, T, smu, sms);
}

// Direct-indexed tables are used when k fits the table and, for the mapping
// objective (whose candidate scoring loops over the whole table), k is small.
__device__ __forceinline__ bool use_direct(const JArgs &a, u32 cap) {
    return a.k <= cap && (!a.code || a.k <= 256);
}

// Tier of a row for the table-based kernels: 0 thread, 1 warp, 2 block.
__device__ __forceinline__ int table_tier(u32 len, u32 k, u32 warp_max = JW_DEG) {
    if (len <= JT) return 0;
    const u32 d = len < k ? len : k;
    return (len <= warp_max && 2 * d <= JW_SLOTS) ? 1 : 2;
}

// Adds per-thread counts to the status word with one atomic per block.
__device__ __forceinline__ void block_count(u32 *cnt, unsigned long long *sum, u32 c, unsigned long long e) {
    __shared__ u32 sc[32];
    __shared__ unsigned long long se[32];
    c = warp_sum<u32>(c);
    e = warp_sum<unsigned long long>(e);
    if (lane_id() == 0) {
        sc[warp_in_block()] = c;
        se[warp_in_block()] = e;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 tc = 0;
        unsigned long long te = 0;
        for (u32 w = 0; w < (blockDim.x >> 5); ++w) {
            tc += sc[w];
            te += se[w];
        }
        if (tc && cnt) atomicAdd(cnt, tc);
        if (te && sum) atomicAdd(sum, te);
    }
}

// Neighbour-loop kernels (afterburner, delta): rows up to CHUNK_THREAD_MAX
// entries are handled by one thread; longer rows are cut into chunks of
// CHUNK entries, one warp each, so that hub rows spread over the whole GPU.
constexpr u32 CHUNK_THREAD_MAX = 32;
constexpr u32 CHUNK = 1024;

__device__ __forceinline__ u32 chunks_of(u32 len) { return (len + CHUNK - 1) / CHUNK; }

// Appends nch chunk items of row u (all lanes of the warp call this; lanes
// with nch == 0 append nothing). One atomic per warp reserves the slots.
__device__ __forceinline__ void warp_emit_chunks(const JArgs &a, u32 u, u32 nch, u32 *counter) {
    u32 incl = nch;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(FULL, incl, o);
        if (lane_id() >= o) incl += y;
    }
    const u32 wtot = __shfl_sync(FULL, incl, 31);
    u32 wbase = 0;
    if (lane_id() == 31 && wtot) wbase = atomicAdd(counter, wtot);
    wbase = __shfl_sync(FULL, wbase, 31);
    const u32 first = wbase + incl - nch;
    for (u32 c = 0; c < nch; ++c) {
        if (first + c < a.items_cap) a.items[first + c] = ((unsigned long long) u << 32) | c;
        else set_error(&a.st->err, DEV_ERR_RANGE);
    }
}

// Entries [from, to) of chunk item `it`.
__device__ __forceinline__ void chunk_range(const JArgs &a, unsigned long long it, u32 &u, u32 &from, u32 &to,
                                            u32 &nch) {
    u = (u32) (it >> 32);
    from = (u32) it * CHUNK;
    const u32 len = __ldg(&a.g.rowlen[u]);
    to = len - from < CHUNK ? len : from + CHUNK;
    nch = chunks_of(len);
}

// Chunk items of a hub row in row slot h (warp-collective; lanes with len 0
// emit nothing). Slots beyond the accumulator capacity are reported as an
// error and skipped.
__device__ __forceinline__ void emit_hub_chunks(const JArgs &a, u32 h, u32 len) {
    u32 nch = len ? (len + a.hub_deg - 1) / a.hub_deg : 0u;
    if (nch && h >= a.hub_cap) {
        set_error(&a.st->err, DEV_ERR_RANGE);
        nch = 0;
    }
    warp_emit_chunks(a, h, nch, &a.st->cnt[ST_CHUNKS]);
}

// Hub rows met by a table pass's dispatch (warp-collective; `hub` marks hub
// row u, list slot s2). Without tracking, every hub row is cut into chunk
// items for k_hub. With tracking, a hub whose sums are older than the current
// generation gets its sums zeroed, its generation advanced and its chunk items
// emitted for k_hub_rebuild, which runs before the pass reads the sums; hubs
// the pass does not need are left as they are.
__device__ __forceinline__ void hub_dispatch(const JArgs &a, u32 s2, bool hub, u32 u) {
    if (!a.hubacc) return;
    if (!a.hub_cur) {
        emit_hub_chunks(a, s2, hub ? a.g.rowlen[u] : 0u);
        return;
    }
    u32 h = 0, len = 0;
    if (hub) {
        h = (u32) (a.dlab[u] >> DL_SLOT_SHIFT) - 1u;  // k_hub_tracked reports a row without a slot
        const u32 cur = *a.hub_cur;
        if (h < a.hub_cap && a.hub_gen[h] != cur) {
            a.hub_gen[h] = cur;
            for (u32 b = 0; b < a.k; ++b) a.hubacc[(u64) h * a.k + b] = 0;
            len = a.g.rowlen[u];
        }
    }
    emit_hub_chunks(a, h, len);
}

__global__ void __launch_bounds__(BLOCK) k_lp_dispatch(JArgs a, u32 ratio) {
    const u64 stride = (u64) gridDim.x * blockDim.x;
    u32 nrec = 0;
    unsigned long long erec = 0;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < a.g.n; base += stride) {
        const u32 u = (u32) (base + threadIdx.x);
        int cls = 0;
        if (u < a.g.n) {
            const u32 dc = a.dest_cache[u];
            if (dc != NULL_PART) {
                a.dest_part[u] = dc;
            } else {
                const u32 len = a.g.rowlen[u];
                ++nrec;
                cls = table_tier(len, a.k, a.hubacc ? a.hub_deg : JW_DEG);
                // a tracked hub row is not scanned: it reads its k sums
                // (counted as k / 3 entries of 12 bytes)
                erec += (cls == 2 && a.hub_cur) ? (a.k + 2) / 3 : len;
                if (cls == 0) lp_thread(a, u, ratio);
            }
        }
        u32 s1 = warp_append(&a.st->cnt[ST_HEAVY], cls == 1);
        if (cls == 1) a.heavy[s1] = u;
        u32 s2 = warp_append(&a.st->cnt[ST_HEAVY2], cls == 2);
        if (cls == 2) a.heavy2[s2] = u;
        hub_dispatch(a, s2, cls == 2, u);
    }
    block_count(&a.st->cnt[ST_AUX], (unsigned long long *) &a.st->sum[4], nrec, erec);
}

// Per-warp shared memory of the warp-tier kernels (dynamic, sized by the
// host): a direct-indexed table of wslots >= k values, or a hashed table of
// wslots keys followed by wslots values.
template<bool DIRECT>
__device__ __forceinline__ u32 *warp_table(u32 wslots) {
    extern __shared__ u32 dsm[];
    u32 *w = dsm + warp_in_block() * (DIRECT ? wslots : 2 * wslots);
    for (u32 s = lane_id(); s < (DIRECT ? wslots : 2 * wslots); s += 32) w[s] = (!DIRECT && s < wslots) ? EMPTY : 0u;
    __syncwarp();
    return w;
}

template<bool DIRECT>
__global__ void __launch_bounds__(JW_BLOCK) k_lp_warp(JArgs a, u32 ratio, u32 wslots) {
    u32 *w = warp_table<DIRECT>(wslots);
    u32 *tk = w;
    s32 *tv = (s32 *) (DIRECT ? w : w + wslots);
    const u32 total = a.st->cnt[ST_HEAVY];
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        const u32 u = a.heavy[i];
        const u32 mask = DIRECT ? 0u : table_mask_for(a.g.rowlen[u], a.k, wslots);
        lp_group<false, DIRECT>(a, u, ratio, ConnTable<false, DIRECT>{tk, tv, mask, a.k}, nullptr, nullptr);
    }
}

__global__ void __launch_bounds__(JB_BLOCK) k_lp_block(JArgs a, u32 ratio) {
    const u32 total = a.st->cnt[ST_HEAVY2];
    if (blockIdx.x >= total) return;
    extern __shared__ u32 dsm[];
    u32 *tk = dsm;
    s32 *tv = (s32 *) (dsm + a.blk_slots);
    __shared__ unsigned long long smu[33];
    __shared__ long long sms[33];
    for (u32 s = threadIdx.x; s < a.blk_slots; s += blockDim.x) {
        tk[s] = EMPTY;
        tv[s] = 0;
    }
    __syncthreads();
    const bool direct = use_direct(a, a.blk_slots);
    for (u32 i = blockIdx.x; i < total; i += gridDim.x) {
        const u32 u = a.heavy2[i];
        const u32 mask = table_mask_for(a.g.rowlen[u], a.k, a.blk_slots);
        if (direct) lp_group<true, true>(a, u, ratio, ConnTable<true, true>{tk, tv, mask, a.k}, smu, sms);
        else lp_group<true, false>(a, u, ratio, ConnTable<true, false>{tk, tv, mask, a.k}, smu, sms);
    }
}

// filter potentially viable moves (:247-258); also resets the list counters
// of the gain pass for the afterburner that follows (the gain kernels are done)
__global__ void __launch_bounds__(BLOCK) k_lp_filter(JArgs a) {
    __shared__ u32 sm[33];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.st->cnt[ST_HEAVY] = 0;
        a.st->cnt[ST_HEAVY2] = 0;
    }
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < a.g.n; base += stride) {
        const u32 u = (u32) (base + threadIdx.x);
        bool c = false;
        if (u < a.g.n) {
            const u32 dp = a.dest_part[u];
            c = dp != NO_MOVE && a.lock[u] == 0;
            const s32 g1 = c ? a.gain_cache[u] : GAIN_MIN;
            a.gain1[u] = g1;
            if (!c) a.lock[u] = 0;
            if (a.abrec)
                a.abrec[u] = (unsigned long long) (u32) g1 | ((unsigned long long) (dp & 0xFFFFu) << 32) |
                             ((unsigned long long) (a.map[u] & 0xFFFFu) << 48);
        }
        const u32 s = block_append(&a.st->cnt[ST_CAND], c, sm);
        if (c) a.cand[s] = u;
    }
}

// afterburner (:269-331 / ProMap :273-320): the terms of four loaded row
// entries of u (v = SENTINEL marks an empty slot).
template<bool NC>
__device__ __forceinline__ s32 ab_batch(const JArgs &a, u32 u, s32 ug, u32 ou, u32 nu, const u32 (&v)[4],
                                        const s32 (&w)[4]) {
    u32 nv[4], ov[4];
    s32 vg[4];
    // only neighbours that move first (higher gain, or equal gain and a
    // lower id) contribute: their target and label come with the gain in
    // one record (abrec) or are gathered after the gains
    bool first[4];
    if (a.abrec) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const unsigned long long r = v[j] != SENTINEL ? ldj<NC>(&a.abrec[v[j]]) : 0ull;
            vg[j] = (s32) (u32) r;
            nv[j] = (u32) (r >> 32) & 0xFFFFu;
            ov[j] = (u32) (r >> 48);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) first[j] = v[j] != SENTINEL && (vg[j] > ug || (vg[j] == ug && v[j] < u));
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) vg[j] = v[j] != SENTINEL ? ldj<NC>(&a.gain1[v[j]]) : 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            first[j] = v[j] != SENTINEL && (vg[j] > ug || (vg[j] == ug && v[j] < u));
            if (first[j]) {
                nv[j] = ldj<NC>(&a.dest_part[v[j]]);
                ov[j] = ldj<NC>(&a.map[v[j]]);
            }
        }
    }
    s32 change = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!first[j]) continue;
        s32 t;
        if (!a.code) {
            t = wmul(w[j], (s32) (nv[j] == nu) - (s32) (nv[j] == ou) + (s32) (ov[j] == ou) - (s32) (ov[j] == nu));
        } else {
            const s32 before_u = wsub(D(a, ou, ov[j]), D(a, nu, ov[j]));
            const s32 after_u = wsub(D(a, ou, nv[j]), D(a, nu, nv[j]));
            t = wmul(w[j], wsub(after_u, before_u));
        }
        change = wadd(change, t);
    }
    return change;
}

// Sum of the afterburner terms over entries [from, to) of u's row, strided
// over a group of threads (wrap-around s32 arithmetic). The gains, targets
// and labels read here are not written by the afterburner kernels, so they
// are gathered through the non-coherent path, four entries at a time; with
// PF the next four row entries are loaded while those are gathered.
template<bool NC = true, bool PF = false>
__device__ __forceinline__ s32 ab_range(const JArgs &a, u32 u, s32 ug, u32 ou, u32 nu, u32 from, u32 to, u32 tid,
                                        u32 nthreads) {
    const u64 beg = __ldg(&a.g.rowptr[u]);
    s32 change = 0;
    if (PF) {
        u32 t0 = from + tid;
        if (t0 >= to) return 0;
        u32 v[4];
        s32 w[4];
        load_entries<4>(a, beg, t0, to, nthreads, v, w);
        for (;;) {
            const u32 t1 = t0 + 4 * nthreads;
            u32 vn[4];
            s32 wn[4];
            load_entries<4>(a, beg, t1, to, nthreads, vn, wn);
            change = wadd(change, ab_batch<NC>(a, u, ug, ou, nu, v, w));
            if (t1 >= to) break;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                v[j] = vn[j];
                w[j] = wn[j];
            }
            t0 = t1;
        }
        return change;
    }
    for (u32 t0 = from + tid; t0 < to; t0 += 4 * nthreads) {
        u32 v[4];
        s32 w[4];
        load_entries<4>(a, beg, t0, to, nthreads, v, w);
        change = wadd(change, ab_batch<NC>(a, u, ug, ou, nu, v, w));
    }
    return change;
}

// The same with 128-bit row reads (quads tid, tid + gs, ... of the segment).
template<bool NC = true>
__device__ __forceinline__ s32 ab_range_quads(const JArgs &a, u32 u, s32 ug, u32 ou, u32 nu, u32 from, u32 to,
                                              u32 tid, u32 gs) {
    const u64 beg = __ldg(&a.g.rowptr[u]);
    const u64 lo = beg + from, hi = beg + to;
    u64 qi = (lo >> 2) + tid;
    u32 v[4];
    s32 w[4];
    if (!next_quad(a, qi, lo, hi, v, w)) return 0;
    s32 change = 0;
    for (;;) {
        const u64 qn = qi + gs;
        u32 vn[4];
        s32 wn[4];
        const bool more = next_quad(a, qn, lo, hi, vn, wn);
        change = wadd(change, ab_batch<NC>(a, u, ug, ou, nu, v, w));
        if (!more) break;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            v[j] = vn[j];
            w[j] = wn[j];
        }
        qi = qn;
    }
    return change;
}

template<bool VEC>
__global__ void __launch_bounds__(BLOCK) k_ab_thread(JArgs a) {
    __shared__ u32 sm[33];
    const u32 total = a.st->cnt[ST_CAND];
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < total; base += stride) {
        const u64 i = base + threadIdx.x;
        bool lock = false;
        u32 u = 0, nch = 0;
        if (i < total) {
            u = a.cand[i];
            const u32 len = __ldg(&a.g.rowlen[u]);
            if (len <= CHUNK_THREAD_MAX) {
                const s32 ug = __ldg(&a.gain1[u]);
                const u32 ou = __ldg(&a.map[u]), nu = __ldg(&a.dest_part[u]);
                const s32 ch = VEC ? ab_range_quads(a, u, ug, ou, nu, 0, len, 0, 1)
                                   : ab_range(a, u, ug, ou, nu, 0, len, 0, 1);
                if (wadd(ug, ch) >= 0) {
                    a.lock[u] = 1;
                    lock = true;
                }
            } else {
                nch = chunks_of(len);
            }
        }
        warp_emit_chunks(a, u, nch, &a.st->cnt[ST_HEAVY]);
        const u32 s3 = block_append(&a.st->cnt[ST_MOVES], lock, sm);
        if (lock) a.moves[s3] = u;
    }
}

// One warp per chunk item. A row of one chunk is decided by its warp; for a
// row of several chunks each warp adds its partial sum to abacc[u] and the
// last warp to finish (counted in abcnt[u], after a fence) decides and resets
// both words, so nothing waits for another warp.
template<bool VEC>
__global__ void __launch_bounds__(BLOCK, 4) k_ab_chunk(JArgs a) {
    u32 total = a.st->cnt[ST_HEAVY];
    if (total > a.items_cap) total = a.items_cap;
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        u32 u, from, to, nch;
        chunk_range(a, __ldg(&a.items[i]), u, from, to, nch);
        const s32 ug = __ldg(&a.gain1[u]);
        const u32 ou = __ldg(&a.map[u]), nu = __ldg(&a.dest_part[u]);
        const s32 part = VEC ? ab_range_quads(a, u, ug, ou, nu, from, to, lane_id(), 32)
                             : ab_range<true, true>(a, u, ug, ou, nu, from, to, lane_id(), 32);
        const s32 change = (s32) warp_sum<u32>((u32) part);
        if (lane_id() == 0) {
            bool decide = nch == 1;
            s32 tot = change;
            if (!decide) {
                atomicAdd(&a.abacc[u], change);
                __threadfence();
                if (atomicAdd(&a.abcnt[u], 1u) == nch - 1) {
                    tot = atomicExch(&a.abacc[u], 0);
                    a.abcnt[u] = 0;
                    decide = true;
                }
            }
            if (decide && wadd(ug, tot) >= 0) {
                a.lock[u] = 1;
                a.moves[atomicAdd(&a.st->cnt[ST_MOVES], 1u)] = u;
            }
        }
    }
}

// ---- perform_moves (:753-924 / ProMap :1103-1216) -----------------------------------



// Invalidates the caches of the neighbours in entries [from, to) of u's row
// and returns their objective contribution (strided over a group of threads).
// Labels and old labels are not written while the delta kernels run, so they
// are read through the non-coherent path; four entries per thread are loaded
// (ids, then labels, then old labels of moved neighbours) before the cache
// resets are stored, which keeps four dependent gathers in flight.
// Objective contribution and cache resets of B loaded entries (v = SENTINEL
// marks an empty slot) of a row whose vertex has new label nu and old label
// ou (um: it changed block). All B labels are gathered, then the old labels
// of moved neighbours, so B dependent gathers are in flight at a time.
// Whether this perform updates the tracked hub sums (else it advances their
// generation, so that every hub's sums count as stale): read by every delta
// kernel after k_apply has counted the entries.
__device__ __forceinline__ bool hub_update_now(const JArgs &a) {
    return a.hub_cur && (unsigned long long) a.st->sum[SUM_PERF_ENTRIES] <= a.hub_track_max;
}

template<int B, bool NC>
__device__ __forceinline__ long long delta_batch(const JArgs &a, u32 nu, u32 ou, bool um, const u32 (&v)[B],
                                                 const s32 (&w)[B], bool inval, bool hub_upd) {
    long long acc = 0;
    if (um && a.dlab) {
        // one gather of dlab gives the neighbour's label, moved bit, old
        // label and hub slot; tracked hub neighbours move w from ou to nu in
        // their connectivity (integer atomics: the sums do not depend on
        // their order)
        unsigned long long xv[B];
#pragma unroll
        for (int j = 0; j < B; ++j) xv[j] = v[j] != SENTINEL ? ldj<NC>(&a.dlab[v[j]]) : 0ull;
#pragma unroll
        for (int j = 0; j < B; ++j) {
            if (v[j] == SENTINEL) continue;
            const u32 nv = (u32) (xv[j] & DL_LABEL);
            const u32 ov = (xv[j] & DL_MOVED) ? (u32) ((xv[j] & DL_OLD) >> DL_OLD_SHIFT) : nv;
            long long c;
            if (!a.code) c = (long long) w[j] * ((long long) (nu != nv) - (long long) (ou != ov));
            else c = (long long) w[j] * ((long long) D(a, nu, nv) - (long long) D(a, ou, ov));
            acc += (xv[j] & DL_MOVED) ? c : 2 * c;
            const u32 hs = (u32) (xv[j] >> DL_SLOT_SHIFT);
            if (hs && hub_upd) {
                atomicSub(&a.hubacc[(u64) (hs - 1) * a.k + ou], w[j]);
                atomicAdd(&a.hubacc[(u64) (hs - 1) * a.k + nu], w[j]);
            }
        }
    } else if (um) {
        u32 xv[B], ov[B];
#pragma unroll
        for (int j = 0; j < B; ++j) xv[j] = v[j] != SENTINEL ? ldj<NC>(&a.map[v[j]]) : 0;
#pragma unroll
        for (int j = 0; j < B; ++j) ov[j] = (xv[j] & MOVED) ? ldj<NC>(&a.dest_part[v[j]]) : (xv[j] & ~MOVED);
#pragma unroll
        for (int j = 0; j < B; ++j) {
            if (v[j] == SENTINEL) continue;
            const u32 nv = xv[j] & ~MOVED;
            long long c;
            if (!a.code) c = (long long) w[j] * ((long long) (nu != nv) - (long long) (ou != ov[j]));
            else c = (long long) w[j] * ((long long) D(a, nu, nv) - (long long) D(a, ou, ov[j]));
            acc += (xv[j] & MOVED) ? c : 2 * c;
        }
    }
    if (inval) {
#pragma unroll
        for (int j = 0; j < B; ++j)
            if (v[j] != SENTINEL) a.dest_cache[v[j]] = NULL_PART;
    }
    return acc;
}

// With PF, the next batch's row entries are loaded before the current
// batch's label gathers, so the row read and the gathers overlap.
template<bool NC = true, int B = 4, bool PF = false>
__device__ __forceinline__ long long delta_range(const JArgs &a, u32 u, u32 from, u32 to, u32 tid, u32 nthreads,
                                                 bool inval, bool hub_upd = false) {
    const u64 beg = __ldg(&a.g.rowptr[u]);
    const u32 x = ldj<NC>(&a.map[u]);
    const bool um = (x & MOVED) != 0;
    const u32 nu = x & ~MOVED;
    const u32 ou = um ? ldj<NC>(&a.dest_part[u]) : nu;
    long long acc = 0;
    if (PF) {
        u32 t0 = from + tid;
        if (t0 >= to) return 0;
        u32 v[B];
        s32 w[B];
        load_entries<B>(a, beg, t0, to, nthreads, v, w);
        for (;;) {
            const u32 t1 = t0 + B * nthreads;
            u32 vn[B];
            s32 wn[B];
            load_entries<B>(a, beg, t1, to, nthreads, vn, wn);
            acc += delta_batch<B, NC>(a, nu, ou, um, v, w, inval, hub_upd);
            if (t1 >= to) break;
#pragma unroll
            for (int j = 0; j < B; ++j) {
                v[j] = vn[j];
                w[j] = wn[j];
            }
            t0 = t1;
        }
        return acc;
    }
    for (u32 t0 = from + tid; t0 < to; t0 += B * nthreads) {
        u32 v[B];
        s32 w[B];
        load_entries<B>(a, beg, t0, to, nthreads, v, w);
        acc += delta_batch<B, NC>(a, nu, ou, um, v, w, inval, hub_upd);
    }
    return acc;
}

// The same with 128-bit row reads: thread tid of a group of gs takes quads
// tid, tid + gs, ... of the row segment, the next quad loaded while the
// current one's labels are gathered.
template<bool NC = true>
__device__ __forceinline__ long long delta_range_quads(const JArgs &a, u32 u, u32 from, u32 to, u32 tid, u32 gs,
                                                       bool inval, bool hub_upd) {
    const u64 beg = __ldg(&a.g.rowptr[u]);
    const u32 x = ldj<NC>(&a.map[u]);
    const bool um = (x & MOVED) != 0;
    const u32 nu = x & ~MOVED;
    const u32 ou = um ? ldj<NC>(&a.dest_part[u]) : nu;
    const u64 lo = beg + from, hi = beg + to;
    u64 qi = (lo >> 2) + tid;
    u32 v[4];
    s32 w[4];
    if (!next_quad(a, qi, lo, hi, v, w)) return 0;
    long long acc = 0;
    for (;;) {
        const u64 qn = qi + gs;
        u32 vn[4];
        s32 wn[4];
        const bool more = next_quad(a, qn, lo, hi, vn, wn);
        acc += delta_batch<4, NC>(a, nu, ou, um, v, w, inval, hub_upd);
        if (!more) break;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            v[j] = vn[j];
            w[j] = wn[j];
        }
        qi = qn;
    }
    return acc;
}

// The same over len entries staged in shared memory (one warp, B per lane).
template<int B>
__device__ __forceinline__ long long delta_staged(const JArgs &a, u32 u, const u32 *sadj, const s32 *sew, u32 len,
                                                  bool inval, bool hub_upd) {
    const u32 x = __ldg(&a.map[u]);
    const bool um = (x & MOVED) != 0;
    const u32 nu = x & ~MOVED;
    const u32 ou = um ? __ldg(&a.dest_part[u]) : nu;
    long long acc = 0;
    for (u32 t0 = (u32) lane_id(); t0 < len; t0 += 32u * B) {
        u32 v[B];
        s32 w[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const u32 t = t0 + 32u * j;
            v[j] = t < len ? sadj[t] : SENTINEL;
            w[j] = t < len ? (sew ? sew[t] : 1) : 0;
        }
        acc += delta_batch<B, true>(a, nu, ou, um, v, w, inval, hub_upd);
    }
    return acc;
}

// When the moved rows hold at least inval_all_min entries (a percentage of the
// level's entries, Tunables::jet_inval_all_pct), most caches are invalidated
// anyway (on an R-MAT level, moved rows with 5% of the entries reach nearly
// every vertex): the delta kernels then skip the scattered resets, one 4-byte
// store per entry, and k_inval_unmark resets all caches with one sequential
// fill. Only enabled where a recomputed gain equals the cached one for every
// vertex whose neighbourhood did not change (a fixed filter ratio per level,
// or the mapping objective).
__device__ __forceinline__ bool scattered_inval(const JArgs &a) {
    return (unsigned long long) a.st->sum[SUM_PERF_ENTRIES] < a.inval_all_min;
}

// Last perform kernel: resets every cache when the delta pass skipped the
// scattered resets, and clears the moved bits.
__global__ void k_inval_unmark(JArgs a) {
    if (!scattered_inval(a))
        for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < a.g.n; u += gridDim.x * blockDim.x)
            a.dest_cache[u] = NULL_PART;
    const u32 total = a.st->cnt[ST_MOVES];
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const u32 u = a.moves[i];
        a.map[u] &= ~MOVED;
        if (a.dlab) a.dlab[u] &= ~DL_MOVED;
    }
}

// First perform kernel: clears the counters and sums perform accumulates.
__global__ void k_perform_reset(DevStatus *st) {
    if (threadIdx.x == 0) {
        st->cnt[ST_HEAVY] = 0;
        st->cnt[ST_HEAVY2] = 0;
        st->sum[SUM_DELTA] = 0;
        st->sum[SUM_PERF_ENTRIES] = 0;
    }
}

// Adds a per-thread s64 to the status word with one atomic per block.
__device__ __forceinline__ void block_add_s64(long long v, long long *dst) {
    __shared__ long long sl[32];
    v = warp_sum<long long>(v);
    if (lane_id() == 0) sl[warp_in_block()] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long r = 0;
        for (u32 w = 0; w < (blockDim.x >> 5); ++w) r += sl[w];
        if (r) atomicAdd((unsigned long long *) dst, (unsigned long long) r);
    }
}

template<bool VEC>
__global__ void __launch_bounds__(BLOCK) k_delta_thread(JArgs a) {
    const u32 total = a.st->cnt[ST_MOVES];
    const bool inval = scattered_inval(a);
    const bool hub_upd = hub_update_now(a);
    if (a.hub_cur && !hub_upd && blockIdx.x == 0 && threadIdx.x == 0) *a.hub_cur += 1u;
    const u64 stride = (u64) gridDim.x * blockDim.x;
    long long acc = 0;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < total; base += stride) {
        const u64 i = base + threadIdx.x;
        u32 u = 0, nch = 0;
        if (i < total) {
            u = a.moves[i];
            const u32 len = __ldg(&a.g.rowlen[u]);
            if (len <= CHUNK_THREAD_MAX)
                acc += VEC ? delta_range_quads(a, u, 0, len, 0, 1, inval, hub_upd)
                           : delta_range(a, u, 0, len, 0, 1, inval, hub_upd);
            else nch = chunks_of(len);
        }
        warp_emit_chunks(a, u, nch, &a.st->cnt[ST_HEAVY]);
    }
    block_add_s64(acc, &a.st->sum[SUM_DELTA]);
    if (blockIdx.x == 0) {
        // maximum block weight after the moves (k_apply has finished)
        __shared__ s32 mx[32];
        s32 m = 0;
        for (u32 b = threadIdx.x; b < a.k; b += blockDim.x) m = a.bw[b] > m ? a.bw[b] : m;
        m = __reduce_max_sync(FULL, m);
        if (lane_id() == 0) mx[warp_in_block()] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            s32 r = 0;
            for (u32 w = 0; w < (blockDim.x >> 5); ++w) r = mx[w] > r ? mx[w] : r;
            a.st->imax[MAX_BW] = r;
        }
    }
}

// Six blocks per SM (at most 40 registers): the pass is bound by dependent
// gathers, so resident warps matter more than registers. The objective delta
// is added with one atomic per warp, so no warp waits for the others of its
// block at the end.
template<int B, bool VEC = false>
__global__ void __launch_bounds__(BLOCK, (B > 4 || VEC) ? 4 : 5) k_delta_chunk(JArgs a) {
    u32 total = a.st->cnt[ST_HEAVY];
    if (total > a.items_cap) total = a.items_cap;
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    const bool inval = scattered_inval(a);
    const bool hub_upd = hub_update_now(a);
    long long acc = 0;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        u32 u, from, to, nch;
        chunk_range(a, __ldg(&a.items[i]), u, from, to, nch);
        if (VEC) acc += delta_range_quads(a, u, from, to, lane_id(), 32, inval, hub_upd);
        else acc += delta_range<true, B, B <= 4>(a, u, from, to, lane_id(), 32, inval, hub_upd);
    }
    acc = warp_sum<long long>(acc);
    if (lane_id() == 0 && acc) atomicAdd((unsigned long long *) &a.st->sum[SUM_DELTA], (unsigned long long) acc);
}

// Chunk items of the delta pass with their row segments staged in shared
// memory by bulk copies (stage.cuh), eight entries per lane in flight.
constexpr int STAGE_BLOCK = 128;
constexpr int STAGE_BLOCKS_PER_SM = 6;
constexpr size_t stage_smem() { return (STAGE_BLOCK / 32) * sizeof(WarpStage); }

__global__ void __launch_bounds__(STAGE_BLOCK, STAGE_BLOCKS_PER_SM) k_delta_staged(JArgs a) {
    extern __shared__ __align__(16) unsigned char stage_sm[];
    WarpStage &S = reinterpret_cast<WarpStage *>(stage_sm)[warp_in_block()];
    u32 total = a.st->cnt[ST_HEAVY];
    if (total > a.items_cap) total = a.items_cap;
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    const bool inval = scattered_inval(a);
    const bool hub_upd = hub_update_now(a);
    long long acc = 0;
    staged_items(
        a.g, S, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps, total, &a.st->err,
        [&](u32 i, u32 &u, u32 &from, u32 &to) {
            u32 nch;
            chunk_range(a, __ldg(&a.items[i]), u, from, to, nch);
        },
        [&](u32 u, const u32 *sadj, const s32 *sew, u32 len, u32) { acc += delta_staged<8>(a, u, sadj, sew, len, inval, hub_upd); },
        [&](u32, u32) {});
    acc = warp_sum<long long>(acc);
    if (lane_id() == 0 && acc) atomicAdd((unsigned long long *) &a.st->sum[SUM_DELTA], (unsigned long long) acc);
}

constexpr u32 APPLY_SMEM_K = 4096;  // block weights accumulated in shared memory up to this k

__global__ void __launch_bounds__(BLOCK) k_apply(JArgs a) {
    extern __shared__ s32 sbw[];
    const u32 total = a.st->cnt[ST_MOVES];
    const bool local = a.k <= APPLY_SMEM_K;
    if (blockIdx.x * blockDim.x >= total) return;
    if (local) {
        for (u32 b = threadIdx.x; b < a.k; b += blockDim.x) sbw[b] = 0;
        __syncthreads();
    }
    long long entries = 0;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const u32 u = a.moves[i];
        const u32 ou = a.map[u], nu = a.dest_part[u];
        const s32 w = g_vw(a.g, u);
        if (ou != nu) {
            if (local) {
                atomicSub(&sbw[ou], w);
                atomicAdd(&sbw[nu], w);
            } else {
                atomicSub(&a.bw[ou], w);
                atomicAdd(&a.bw[nu], w);
            }
        }
        a.map[u] = ou != nu ? (nu | MOVED) : nu;
        if (a.dlab)
            a.dlab[u] = (a.dlab[u] & ~(DL_LABEL | DL_MOVED | DL_OLD)) | nu |
                        (ou != nu ? DL_MOVED | ((unsigned long long) ou << DL_OLD_SHIFT) : 0ull);
        a.dest_part[u] = ou;
        a.dest_cache[u] = NULL_PART;
        entries += a.g.rowlen[u];
    }
    if (local) {
        __syncthreads();
        for (u32 b = threadIdx.x; b < a.k; b += blockDim.x)
            if (sbw[b]) atomicAdd(&a.bw[b], sbw[b]);
    }
    // row entries the delta pass will read (byte accounting of the timers)
    block_add_s64(entries, &a.st->sum[SUM_PERF_ENTRIES]);
}

__global__ void k_max_bw(const s32 *bw, u32 k, int *out) {
    s32 m = 0;
    for (u32 b = threadIdx.x; b < k; b += blockDim.x) m = bw[b] > m ? bw[b] : m;
    m = __reduce_max_sync(FULL, m);
    __shared__ s32 sm[32];
    if (lane_id() == 0) sm[warp_in_block()] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        s32 r = 0;
        for (u32 w = 0; w < (blockDim.x >> 5); ++w) r = sm[w] > r ? sm[w] : r;
        *out = r;
    }
}

// ---- rebalancing (rebalance_weak :592-751, rebalance_strong :356-590) ----------------

struct RbArgs {
    s32 opt;
    s32 max_b_w;
    u32 sections;
    const u32 *under;
    u32 *keys;  // per vertex: mini-bucket key or NOKEY
};

// weak: best non-overloaded block by connection (:645-687)
__device__ __forceinline__ void weak_finish(const JArgs &a, const RbArgs &r, u32 u, u32 o, s32 own,
                                            unsigned long long bk) {
    const u32 n_under = a.st->cnt[ST_AUX];
    u32 best = o;
    s32 gain = 0;
    const s32 best_w = bk ? (s32) (u32) (bk >> 32) : 0;
    if (best_w <= 0) {
        if (n_under > 0) best = r.under[u % n_under];
        gain = -own;
    } else {
        best = ~(u32) bk;
        gain = wsub(best_w, own);
    }
    a.dest_part[u] = best;
    const s32 vw = g_vw(a.g, u);
    r.keys[u] = (o != best) ? (MAX_BUCKETS * o + gain_bucket(gain, vw)) * r.sections + (u % r.sections) : NOKEY;
}

// strong: average connection to non-full blocks minus own (:404-442)
__device__ __forceinline__ void strong_finish(const JArgs &a, const RbArgs &r, u32 u, u32 o, s32 own, s32 sum,
                                              s32 count) {
    if (count == 0) count = 1;
    const s32 gain = wsub(sum / count, own);
    const s32 vw = g_vw(a.g, u);
    const s32 excess = a.bw[o] - a.lmax;
    r.keys[u] = (MAX_BUCKETS * o + gain_bucket(gain, vw < excess ? vw : excess)) * r.sections + (u % r.sections) + 1;
}

template<bool STRONG>
__device__ __forceinline__ bool rb_qualifies(const JArgs &a, const RbArgs &r, u32 o, s32 vw, s32 maxv) {
    const s64 ow = a.bw[o];
    if (ow <= a.lmax) return false;
    if (!STRONG) return 2 * (s64) vw < 3 * (ow - r.opt);
    return (s64) vw <= 2 * (s64) maxv && (s64) vw < 2 * (ow - r.opt);
}

template<bool STRONG, bool NC = true>
__device__ __forceinline__ void rb_thread(const JArgs &a, const RbArgs &r, u32 u, u32 o) {
    TRow row;
    trow_build<NC>(a, u, row);
    s32 own = 0, sum = 0, count = 0;
    unsigned long long bk = 0;
#pragma unroll
    for (int s = 0; s < (int) JT; ++s) {
        const u32 b = row.b[s];
        if (b == EMPTY) continue;
        if (b == o) {
            own = row.c[s];
            continue;
        }
        if (a.bw[b] < r.max_b_w) {
            if (STRONG) {
                sum = wadd(sum, row.c[s]);
                ++count;
            } else {
                unsigned long long k = cut_key(row.c[s], b);
                bk = k > bk ? k : bk;
            }
        }
    }
    if (STRONG) strong_finish(a, r, u, o, own, sum, count);
    else weak_finish(a, r, u, o, own, bk);
}

template<bool STRONG, bool BLK, bool DIRECT, bool NC = true>
__device__ __forceinline__ void rb_finish_group(const JArgs &a, const RbArgs &r, u32 u,
                                                ConnTable<BLK, DIRECT, NC> T, unsigned long long *smu,
                                                long long *sms) {
    const u32 o = a.map[u];
    long long own = 0, sum = 0, count = 0;
    unsigned long long bk = 0;
    const u32 ns = T.slots();
    for (u32 s = Grp<BLK>::tid(); s < ns; s += Grp<BLK>::size()) {
        const u32 b = T.key(s);
        if (b == EMPTY) continue;
        if (b == o) {
            own = T.val(s);
            continue;
        }
        if (a.bw[b] < r.max_b_w) {
            if (STRONG) {
                sum = (long long) wadd((s32) sum, T.val(s));
                ++count;
            } else {
                unsigned long long k = cut_key(T.val(s), b);
                bk = k > bk ? k : bk;
            }
        }
    }
    own = Grp<BLK>::sum_s64(own, sms);
    if (STRONG) {
        // s32 wrap-around sum: reduce the low 32 bits
        sum = (long long) (s32) (u32) (unsigned long long) Grp<BLK>::sum_s64((long long) (u32) (s32) sum, sms);
        count = Grp<BLK>::sum_s64(count, sms);
    } else {
        bk = Grp<BLK>::max_u64(bk, smu);
    }
    if (Grp<BLK>::tid() == 0) {
        if (STRONG) strong_finish(a, r, u, o, (s32) own, (s32) sum, (s32) count);
        else weak_finish(a, r, u, o, (s32) own, bk);
    }
    T.clear();
}

template<bool STRONG, bool BLK, bool DIRECT, bool NC = true>
__device__ __forceinline__ void rb_group(const JArgs &a, const RbArgs &r, u32 u, ConnTable<BLK, DIRECT, NC> T,
                                         unsigned long long *smu, long long *sms) {
    T.build(a, u);
    rb_finish_group<STRONG, BLK, DIRECT, NC>(a, r, u, T, smu, sms);
}

template<bool STRONG>
__global__ void __launch_bounds__(BLOCK) k_rb_dispatch(JArgs a, RbArgs r) {
    const s32 maxv = a.st->imax[1];
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < a.g.n; base += stride) {
        const u32 u = (u32) (base + threadIdx.x);
        int cls = 0;
        if (u < a.g.n) {
            const u32 o = a.map[u];
            if (!rb_qualifies<STRONG>(a, r, o, g_vw(a.g, u), maxv)) {
                if (!STRONG) a.dest_part[u] = o;
                r.keys[u] = NOKEY;
            } else {
                cls = table_tier(a.g.rowlen[u], a.k, a.hubacc ? a.hub_deg : JW_DEG);
                if (cls == 0) rb_thread<STRONG>(a, r, u, o);
            }
        }
        u32 s1 = warp_append(&a.st->cnt[ST_HEAVY], cls == 1);
        if (cls == 1) a.heavy[s1] = u;
        u32 s2 = warp_append(&a.st->cnt[ST_HEAVY2], cls == 2);
        if (cls == 2) a.heavy2[s2] = u;
        hub_dispatch(a, s2, cls == 2, u);
    }
}

template<bool STRONG, bool DIRECT>
__global__ void __launch_bounds__(JW_BLOCK) k_rb_warp(JArgs a, RbArgs r, u32 wslots) {
    u32 *w = warp_table<DIRECT>(wslots);
    u32 *tk = w;
    s32 *tv = (s32 *) (DIRECT ? w : w + wslots);
    const u32 total = a.st->cnt[ST_HEAVY];
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        const u32 u = a.heavy[i];
        const u32 mask = DIRECT ? 0u : table_mask_for(a.g.rowlen[u], a.k, wslots);
        rb_group<STRONG, false, DIRECT>(a, r, u, ConnTable<false, DIRECT>{tk, tv, mask, a.k}, nullptr, nullptr);
    }
}

template<bool STRONG>
__global__ void __launch_bounds__(JB_BLOCK) k_rb_block(JArgs a, RbArgs r) {
    const u32 total = a.st->cnt[ST_HEAVY2];
    if (blockIdx.x >= total) return;
    extern __shared__ u32 dsm[];
    u32 *tk = dsm;
    s32 *tv = (s32 *) (dsm + a.blk_slots);
    __shared__ unsigned long long smu[33];
    __shared__ long long sms[33];
    for (u32 s = threadIdx.x; s < a.blk_slots; s += blockDim.x) {
        tk[s] = EMPTY;
        tv[s] = 0;
    }
    __syncthreads();
    const bool direct = use_direct(a, a.blk_slots);
    for (u32 i = blockIdx.x; i < total; i += gridDim.x) {
        const u32 u = a.heavy2[i];
        const u32 mask = table_mask_for(a.g.rowlen[u], a.k, a.blk_slots);
        if (direct) rb_group<STRONG, true, true>(a, r, u, ConnTable<true, true>{tk, tv, mask, a.k}, smu, sms);
        else rb_group<STRONG, true, false>(a, r, u, ConnTable<true, false>{tk, tv, mask, a.k}, smu, sms);
    }
}

// Hub rows in chunks (KIND 0: Jet gain, 1: weak pick, 2: strong pick). A
// warp aggregates its chunk in a direct-indexed table, adds the non-zero sums
// to the row's accumulator in global memory, and counts itself finished after
// a fence; the warp that finishes last reads the full row back (bypassing L1),
// resets the accumulator and completes the row with the ordinary finishing
// code. No warp waits for another.
template<int KIND>
__global__ void __launch_bounds__(JW_BLOCK) k_hub(JArgs a, u32 ratio, RbArgs r) {
    u32 *w = warp_table<true>(a.k);
    s32 *tv = (s32 *) w;
    const ConnTable<false, true> T{w, tv, 0, a.k};
    u32 total = a.st->cnt[ST_CHUNKS];
    if (total > a.items_cap) total = a.items_cap;
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    const u32 lane = lane_id();
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        const unsigned long long it = a.items[i];
        const u32 h = (u32) (it >> 32);
        const u32 u = a.heavy2[h];
        const u32 len = __ldg(&a.g.rowlen[u]);
        const u32 from = (u32) it * a.hub_deg;
        const u32 to = len - from < a.hub_deg ? len : from + a.hub_deg;
        const u32 nch = (len + a.hub_deg - 1) / a.hub_deg;
        dtable_build_range<false>(a, u, tv, from, to);
        s32 *acc = a.hubacc + (u64) h * a.k;
        for (u32 b = lane; b < a.k; b += 32) {
            const s32 v = tv[b];
            if (v) {
                atomicAdd(&acc[b], v);
                tv[b] = 0;
            }
        }
        __threadfence();
        __syncwarp();
        u32 last = 0;
        if (lane == 0) last = atomicAdd(&a.hubcnt[h], 1u) == nch - 1 ? 1u : 0u;
        last = __shfl_sync(FULL, last, 0);
        if (!last) continue;
        __threadfence();
        for (u32 b = lane; b < a.k; b += 32) {
            tv[b] = __ldcg(&acc[b]);
            acc[b] = 0;
        }
        if (lane == 0) a.hubcnt[h] = 0;
        __syncwarp();
        if (KIND == 0) lp_finish_group<false, true>(a, u, ratio, T, nullptr, nullptr);
        else rb_finish_group<KIND == 2, false, true>(a, r, u, T, nullptr, nullptr);
    }
}

// Tracked hubs: one warp per hub row of the pass's hub list (heavy2) loads
// the row's connectivity from hubacc into its direct table and completes the
// row with the ordinary finishing code (gain: KIND 0, weak: 1, strong: 2).
template<int KIND>
__global__ void __launch_bounds__(JW_BLOCK) k_hub_tracked(JArgs a, u32 ratio, RbArgs r) {
    u32 *w = warp_table<true>(a.k);
    s32 *tv = (s32 *) w;
    const ConnTable<false, true> T{w, tv, 0, a.k};
    const u32 total = a.st->cnt[ST_HEAVY2];
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        const u32 u = a.heavy2[i];
        const u32 hs = (u32) (a.dlab[u] >> DL_SLOT_SHIFT);
        if (hs == 0 || hs > a.hub_cap) {  // not a tracked hub: cannot happen for rows above hub_deg
            if (lane_id() == 0) set_error(&a.st->err, DEV_ERR_RANGE);
            continue;
        }
        for (u32 b = lane_id(); b < a.k; b += 32) tv[b] = a.hubacc[(u64) (hs - 1) * a.k + b];
        __syncwarp();
        if (KIND == 0) lp_finish_group<false, true>(a, u, ratio, T, nullptr, nullptr);
        else rb_finish_group<KIND == 2, false, true>(a, r, u, T, nullptr, nullptr);
    }
}

// Level set-up of tracked hubs: numbers the hub rows (rows of more than
// hub_deg entries), writes dlab for every vertex and sums the hub rows'
// lengths into the status word's sum[0].
__global__ void __launch_bounds__(BLOCK) k_hub_number(JArgs a) {
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < a.g.n; base += stride) {
        const u32 u = (u32) (base + threadIdx.x);
        const bool hub = u < a.g.n && a.g.rowlen[u] > a.hub_deg;
        const u32 slot = warp_append(&a.st->cnt[ST_HEAVY2], hub);
        const bool ok = hub && slot < a.hub_cap && slot < DL_MAX_HUBS;
        if (hub && !ok) set_error(&a.st->err, DEV_ERR_RANGE);
        if (ok) a.heavy2[slot] = u;
        if (ok) const_cast<u32 *>(a.hub_vertex)[slot] = u;
        if (u < a.g.n) a.dlab[u] = a.map[u] | (ok ? (unsigned long long) (slot + 1) << DL_SLOT_SHIFT : 0ull);
        if (ok) atomicAdd((unsigned long long *) &a.st->sum[0], (unsigned long long) a.g.rowlen[u]);
    }
}

// Rebuilds the tracked connectivity of the hubs the dispatch found stale
// (their sums zeroed there) from their chunk items; each warp adds its
// chunk's block sums to the row's hubacc entries.
__global__ void __launch_bounds__(JW_BLOCK) k_hub_rebuild(JArgs a) {
    u32 *w = warp_table<true>(a.k);
    s32 *tv = (s32 *) w;
    u32 total = a.st->cnt[ST_CHUNKS];
    if (total > a.items_cap) total = a.items_cap;
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    const u32 lane = lane_id();
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        const unsigned long long it = a.items[i];
        const u32 h = (u32) (it >> 32);
        const u32 u = a.hub_vertex[h];
        const u32 len = __ldg(&a.g.rowlen[u]);
        const u32 from = (u32) it * a.hub_deg;
        const u32 to = len - from < a.hub_deg ? len : from + a.hub_deg;
        dtable_build_range<false>(a, u, tv, from, to);
        for (u32 b = lane; b < a.k; b += 32) {
            const s32 v = tv[b];
            if (v) {
                atomicAdd(&a.hubacc[(u64) h * a.k + b], v);
                tv[b] = 0;
            }
        }
        __syncwarp();
    }
}

// dlab of every vertex without tracked hubs: the label alone.
__global__ void k_dlab_init(JArgs a) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < a.g.n; u += gridDim.x * blockDim.x) a.dlab[u] = a.map[u];
}

// underloaded_blocks (:614-627): ordered list of blocks below max_b_w.
__device__ __forceinline__ void under_block(const s32 *bw, u32 k, s32 max_b_w, u32 *under, u32 *n_under) {
    __shared__ u32 sm[32];
    u32 carry = 0;
    for (u32 base = 0; base < k; base += blockDim.x) {
        const u32 b = base + threadIdx.x;
        const u32 f = (b < k && bw[b] < max_b_w) ? 1u : 0u;
        u32 tot;
        const u32 p = block_exclusive_scan<u32>(f, tot, sm);
        if (f) under[carry + p] = b;
        carry += tot;
    }
    if (threadIdx.x == 0) *n_under = carry;
}

__global__ void k_under(const s32 *bw, u32 k, s32 max_b_w, u32 *under, u32 *n_under) {
    under_block(bw, k, max_b_w, under, n_under);
}

// find max size (:377-385): largest free capacity below max_b_w (INT32_MIN if none)
__device__ __forceinline__ void maxv_block(const s32 *bw, u32 k, s32 max_b_w, int *out) {
    s32 m = INT32_MIN;
    for (u32 b = threadIdx.x; b < k; b += blockDim.x)
        if (bw[b] < max_b_w && max_b_w - bw[b] > m) m = max_b_w - bw[b];
    m = __reduce_max_sync(FULL, m);
    __shared__ s32 sm[32];
    if (lane_id() == 0) sm[warp_in_block()] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        s32 r = INT32_MIN;
        for (u32 w = 0; w < (blockDim.x >> 5); ++w) r = sm[w] > r ? sm[w] : r;
        *out = r;
    }
}

__global__ void k_maxv(const s32 *bw, u32 k, s32 max_b_w, int *out) { maxv_block(bw, k, max_b_w, out); }

// B(x) for x = p * width, p in [0, k]: weight of candidates with key < x.
__global__ void k_bounds(const u32 *skeys, const long long *prefix, const u32 *d_c, u32 k, u32 width, long long *B) {
    const u32 c = *d_c;
    for (u32 p = blockIdx.x * blockDim.x + threadIdx.x; p <= k; p += gridDim.x * blockDim.x) {
        const u64 x = (u64) p * width;
        u32 lo = 0, hi = c;
        while (lo < hi) {
            const u32 mid = (lo + hi) >> 1;
            if ((u64) skeys[mid] < x) lo = mid + 1;
            else hi = mid;
        }
        B[p] = prefix[lo];
    }
}

__global__ void k_weak_filter(JArgs a, const u32 *svals, const long long *prefix, const long long *B,
                              const u32 *d_c) {
    const u32 c = *d_c;
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < c; base += stride) {
        const u64 i = base + threadIdx.x;
        bool take = false;
        u32 u = 0;
        if (i < c) {
            u = svals[i];
            const u32 o = a.map[u];
            const long long score = prefix[i] - B[o];
            take = score < (long long) a.bw[o] - a.lmax;
        }
        const u32 s = warp_append(&a.st->cnt[ST_MOVES], take);
        if (take) a.moves[s] = u;
    }
}

__global__ void k_strong_filter(JArgs a, const u32 *svals, const long long *prefix, const long long *B,
                                const u32 *d_c, long long *evict_adjust, long long *mpre) {
    const u32 c = *d_c;
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < c; base += stride) {
        const u64 i = base + threadIdx.x;
        bool take = false;
        u32 u = 0;
        if (i < c) {
            u = svals[i];
            const u32 o = a.map[u];
            const long long score = prefix[i] - B[o];
            const long long limit = (long long) a.bw[o] - a.lmax;
            if (score < limit) {
                take = true;
                const long long vw = g_vw(a.g, u);
                if (score + vw >= limit) evict_adjust[o] = score + vw;
            }
        }
        const u32 s = warp_append(&a.st->cnt[ST_MOVES], take);
        if (take) {
            a.moves[s] = u;
            mpre[s] = prefix[i];
        }
    }
}

// cookie cutter (:524-551), one block
__device__ __forceinline__ void cookie_block(const s32 *bw, u32 k, s32 max_b_w, const long long *B, long long *ea,
                                             long long *es, long long *max_v, long long *sm) {
    long long carry = 0, carry2 = 0;
    for (u32 base = 0; base < k; base += blockDim.x) {
        const u32 p = base + threadIdx.x;
        long long add = 0, cap = 0;
        if (p < k) {
            add = ea[p];
            if (add == 0) add = B[p + 1] - B[p];
            cap = max_b_w > bw[p] ? (long long) max_b_w - bw[p] : 0;
        }
        long long tot, tot2;
        const long long pa = block_exclusive_scan<long long>(add, tot, sm);
        const long long pc = block_exclusive_scan<long long>(cap, tot2, sm);
        if (p < k) {
            ea[p] = B[p] - (carry + pa);
            es[p + 1] = carry2 + pc + cap;
        }
        carry += tot;
        carry2 += tot2;
    }
    if (threadIdx.x == 0) {
        es[0] = 0;
        *max_v = carry;
    }
}

__global__ void k_cookie(const s32 *bw, u32 k, s32 max_b_w, const long long *B, long long *ea, long long *es,
                         long long *max_v) {
    __shared__ long long sm[32];
    cookie_block(bw, k, max_b_w, B, ea, es, max_v, sm);
}

__device__ __forceinline__ s32 chunk_of(const long long *es, u32 k, long long tg) {
    // largest id in [0, k] with es[id] <= tg (es non-decreasing, es[0] = 0)
    u32 lo = 0, hi = k + 1;
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (es[mid] <= tg) lo = mid + 1;
        else hi = mid;
    }
    return (s32) lo - 1;
}

// First attempt of one evicted vertex; returns true when it needs a fallback
// slot.
__device__ __forceinline__ bool strong_assign_one(const JArgs &a, u32 u, long long mpre_j, const long long *ea,
                                                  const long long *es) {
    const u32 o = a.map[u];
    const long long vw = g_vw(a.g, u);
    const long long tg = mpre_j - ea[o];
    const s32 id = chunk_of(es, a.k, tg);
    if (id < (s32) a.k && vw / 2 <= es[id + 1] - tg) {
        a.dest_part[u] = (u32) id;
        return false;
    }
    a.dest_part[u] = o;
    return id < (s32) a.k;
}

// adjust_scores (:560-584): first attempt for every evicted vertex; those
// that need a fallback slot are collected.
__global__ void k_strong_assign(JArgs a, const long long *mpre, const long long *ea, const long long *es, u32 *fail,
                                u32 *n_fail) {
    const u32 total = a.st->cnt[ST_MOVES];
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < total; base += stride) {
        const u64 j = base + threadIdx.x;
        bool f = false;
        u32 u = 0;
        if (j < total) {
            u = a.moves[j];
            f = strong_assign_one(a, u, mpre[j], ea, es);
        }
        const u32 s = warp_append(n_fail, f);
        if (f) fail[s] = u;
    }
}

// dst[i] = src[i] for i < *d_count.
__global__ void k_copy_count(u32 *dst, const u32 *src, const u32 *d_count) {
    const u32 c = *d_count;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

// Fallback slots in ascending vertex order (one thread; at most one
// straddling vertex per chunk boundary reaches this).
__device__ __forceinline__ void strong_fallback_seq(const JArgs &a, const u32 *fail, u32 nf, const long long *es,
                                                    long long *max_v) {
    long long mv = *max_v;
    for (u32 i = 0; i < nf; ++i) {
        const u32 u = fail[i];
        const u32 o = a.map[u];
        const long long vw = g_vw(a.g, u);
        u32 dest = o;
        for (u32 guard = 0; guard < 2 * a.k + 4; ++guard) {
            const long long tg = mv;
            mv += vw;
            const s32 id = chunk_of(es, a.k, tg);
            if (id >= (s32) a.k) break;
            if (vw / 2 <= es[id + 1] - tg) {
                dest = (u32) id;
                break;
            }
        }
        a.dest_part[u] = dest;
    }
    *max_v = mv;
}

__global__ void k_strong_fallback(JArgs a, const u32 *fail, const u32 *d_nf, const long long *es, long long *max_v) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const u32 nf = *d_nf;
    if (nf) strong_fallback_seq(a, fail, nf, es, max_v);
}

__device__ __forceinline__ int bits_for_u32(u32 x) { return x ? 32 - __clz(x) : 0; }

// ---- rebalance ordering of small levels in one block -------------------------------

// Levels of at most Tunables::order_small_n vertices run the whole ordering of a
// rebalance step (candidate compaction, stable sort by mini-bucket key,
// weight prefix, bucket bounds, move selection and, for strong rebalancing,
// the cookie cutter and slot assignment) in one 1024-thread block instead of
// ~25 small launches. The block reads and writes its own arrays only, with a
// __syncthreads() between phases.
constexpr u32 ORDER_SMALL_N = 1u << 16;  // upper bound of Tunables::order_small_n
constexpr int OB = 1024;

struct OrderScratch {
    u32 *cands, *ck, *cands2, *ck2;
    long long *prefix, *B;
    long long *ea, *es, *mpre;  // strong only
    u32 *fail, *fail2;          // strong only
};

// Stable LSD radix sort (8-bit digits) of (k0[i], v0[i]), i < cnt, by key bits
// [0, bits), ping-ponging with (k1, v1); returns true when the result is in
// (k1, v1). All OB threads call it.
__device__ bool block_sort_pairs(u32 *k0, u32 *v0, u32 *k1, u32 *v1, u32 cnt, int bits, u32 *offs,
                                 u32 (*wc)[256], u32 *scan_sm) {
    const u32 tid = threadIdx.x, w = warp_in_block(), lane = lane_id();
    const unsigned lt = (1u << lane) - 1u;
    bool flipped = false;
    for (int shift = 0; shift < bits; shift += 8) {
        if (tid < 256) offs[tid] = 0;
        __syncthreads();
        for (u32 i = tid; i < cnt; i += OB) atomicAdd(&offs[(k0[i] >> shift) & 255u], 1u);
        __syncthreads();
        u32 tot;
        const u32 v = tid < 256 ? offs[tid] : 0u;
        const u32 p = block_exclusive_scan<u32>(v, tot, scan_sm);
        if (tid < 256) offs[tid] = p;
        __syncthreads();
        for (u32 base = 0; base < cnt; base += OB) {
            for (u32 j = tid; j < 32 * 256; j += OB) wc[j >> 8][j & 255] = 0;
            __syncthreads();
            const u32 i = base + tid;
            const bool valid = i < cnt;
            const u32 key = valid ? k0[i] : 0u;
            const u32 d = valid ? ((key >> shift) & 255u) : 256u;
            const unsigned mask = __match_any_sync(FULL, d);
            if (valid && (u32) (__ffs(mask) - 1) == lane) wc[w][d] = (u32) __popc(mask);
            __syncthreads();
            if (valid) {
                u32 off = offs[d] + (u32) __popc(mask & lt);
                for (u32 x = 0; x < w; ++x) off += wc[x][d];
                k1[off] = key;
                v1[off] = v0[i];
            }
            __syncthreads();
            if (tid < 256) {
                u32 add = 0;
                for (u32 x = 0; x < OB / 32; ++x) add += wc[x][tid];
                offs[tid] += add;
            }
            __syncthreads();
        }
        u32 *t = k0;
        k0 = k1;
        k1 = t;
        t = v0;
        v0 = v1;
        v1 = t;
        flipped = !flipped;
    }
    return flipped;
}

// Whole-block body (OB threads); leaves the move count in cnt[ST_MOVES].
struct OrderSmem {
    u32 offs[256];
    u32 wc[OB / 32][256];
    u32 scan_sm[32];
    long long lsm[32];
    u32 cnt_sm[3];  // candidates, moves, fallbacks
};

template<bool STRONG>
__device__ void order_small_body(const JArgs &a, const RbArgs &r, u32 width, int key_bits, const OrderScratch &S,
                                 s32 max_b_w, OrderSmem &sm) {
    u32 *offs = sm.offs, *scan_sm = sm.scan_sm, *cnt_sm = sm.cnt_sm;
    u32 (*wc)[256] = sm.wc;
    long long *lsm = sm.lsm;
    const u32 tid = threadIdx.x, n = a.g.n;
    if (tid < 3) cnt_sm[tid] = 0;
    if (STRONG)
        for (u32 b = tid; b < a.k; b += OB) S.ea[b] = 0;
    __syncthreads();
    // 1. candidates in ascending vertex id with their keys
    for (u32 base = 0; base < n; base += OB) {
        const u32 u = base + tid;
        const bool c = u < n && r.keys[u] != NOKEY;
        u32 tot;
        const u32 p = block_exclusive_scan<u32>(c ? 1u : 0u, tot, scan_sm) + cnt_sm[0];
        if (c) {
            S.cands[p] = u;
            S.ck[p] = r.keys[u];
        }
        __syncthreads();
        if (tid == 0) cnt_sm[0] += tot;
        __syncthreads();
    }
    const u32 cc = cnt_sm[0];
    // 2. stable sort by key
    u32 *sk = S.ck, *sv = S.cands;
    if (block_sort_pairs(S.ck, S.cands, S.ck2, S.cands2, cc, key_bits, offs, wc, scan_sm)) {
        sk = S.ck2;
        sv = S.cands2;
    }
    // 3. weight prefix over the sorted candidates (prefix[cc] = total)
    long long carry = 0;
    for (u32 base = 0; base <= cc; base += OB) {
        const u32 i = base + tid;
        const long long v = i < cc ? (long long) g_vw(a.g, sv[i]) : 0;
        long long tot;
        const long long p = block_exclusive_scan<long long>(v, tot, lsm) + carry;
        if (i <= cc) S.prefix[i] = p;
        carry += tot;
        __syncthreads();
    }
    // 4. B(x) for x = p * width, p in [0, k]
    for (u32 pb = tid; pb <= a.k; pb += OB) {
        const u64 x = (u64) pb * width;
        u32 lo = 0, hi = cc;
        while (lo < hi) {
            const u32 mid = (lo + hi) >> 1;
            if ((u64) sk[mid] < x) lo = mid + 1;
            else hi = mid;
        }
        S.B[pb] = S.prefix[lo];
    }
    __syncthreads();
    // 5. moves
    for (u32 i = tid; i < cc; i += OB) {
        const u32 u = sv[i];
        const u32 o = a.map[u];
        const long long score = S.prefix[i] - S.B[o];
        const long long limit = (long long) a.bw[o] - a.lmax;
        if (score < limit) {
            const u32 s = atomicAdd(&cnt_sm[1], 1u);
            a.moves[s] = u;
            if (STRONG) {
                S.mpre[s] = S.prefix[i];
                const long long vw = g_vw(a.g, u);
                if (score + vw >= limit) S.ea[o] = score + vw;
            }
        }
    }
    __syncthreads();
    const u32 nm = cnt_sm[1];
    if (!STRONG) {
        if (tid == 0) a.st->cnt[ST_MOVES] = nm;
        return;
    }
    // 6. cookie cutter
    long long *max_v = (long long *) &a.st->sum[3];
    cookie_block(a.bw, a.k, max_b_w, S.B, S.ea, S.es, max_v, lsm);
    __syncthreads();
    // 7. first slot attempt
    for (u32 j = tid; j < nm; j += OB) {
        const u32 u = a.moves[j];
        if (strong_assign_one(a, u, S.mpre[j], S.ea, S.es)) S.fail[atomicAdd(&cnt_sm[2], 1u)] = u;
    }
    __syncthreads();
    // 8. fallback slots in ascending vertex id
    const u32 nf = cnt_sm[2];
    if (nf) {
        u32 *fk = S.fail, *fv = S.fail2;
        // sort ids (keys) carrying themselves as values: (fail, fail2) -> sorted
        for (u32 i = tid; i < nf; i += OB) S.fail2[i] = S.fail[i];
        __syncthreads();
        u32 *k1 = S.cands, *v1 = S.cands2;  // free after step 5
        if (block_sort_pairs(S.fail, S.fail2, k1, v1, nf, bits_for_u32(n), offs, wc, scan_sm)) fk = k1;
        __syncthreads();
        (void) fv;
        if (tid == 0) strong_fallback_seq(a, fk, nf, S.es, max_v);
    }
    if (tid == 0) a.st->cnt[ST_MOVES] = nm;
}

template<bool STRONG>
__global__ void __launch_bounds__(OB, 1) k_order_small(JArgs a, RbArgs r, u32 width, int key_bits, OrderScratch S,
                                                        s32 max_b_w) {
    __shared__ OrderSmem sm;
    order_small_body<STRONG>(a, r, width, key_bits, S, max_b_w, sm);
}

// ---- fused refinement of small and mid-size levels --------------------------------------

// The whole level loop of jet_refine in one launch of 1024-thread blocks: the
// iteration control (ratios, weak/strong switching, best-labelling tracking)
// and per iteration the same steps as the per-kernel path (gain pass, filter,
// afterburner, weak or strong rebalancing with the one-block ordering,
// perform). Levels of at most Tunables::jet_fused_max_n vertices run it in a
// single block (phases separated by __syncthreads()); levels of at most
// Tunables::jet_coop_max_n vertices run it as a cooperative grid (phases
// separated by grid barriers; block 0 alone does the ordering). State written
// in one phase is read in a later phase with plain loads after the barrier
// (never through the non-coherent path). Every branch of the control flow
// depends only on values all threads read after the same barrier, so every
// thread reaches every barrier. The result equals the per-kernel path's (a
// parity test forces both).
constexpr int FB = OB;                  // threads per block (= the ordering block)
constexpr u32 FUSED_MAX_N = 1u << 16;   // upper bound of both vertex thresholds (one-block ordering)
constexpr u32 FUSED_AB_THREAD = 32;     // afterburner / delta rows handled by one thread
constexpr int FC_N = 4;  // counters per set: warp rows, block rows, candidates, moves
constexpr int FS_N = 2;  // sums per set: moved-row entries, objective delta

struct FusedCtl {
    u32 n_ratios;
    u32 ratios[17];
    s32 lmax;
    u32 promap;
    long long obj;  // in: objective of the input labelling; out: best objective
    s32 maxw;       // in / out: maximum block weight
    u32 iterations; // out: Jet iterations run
};

struct FusedArgs {
    RbArgs weak, strong;
    u32 width;
    int bits_weak, bits_strong;
    OrderScratch S;
    u32 *under;       // writable alias of weak.under
    u32 *part;        // receives the best labelling
    u32 *gcnt;        // cooperative grid: 2 sets of FC_N counters (zero on entry)
    long long *gsum;  // cooperative grid: 2 sets of FS_N sums (zero on entry)
    u32 *bar;         // cooperative grid: barrier words (zero on entry)
};

// Barrier of the team: the block, or the cooperative grid (bounded wait;
// false once a wait gave up).
template<bool COOP>
__device__ __forceinline__ bool team_sync(u32 *bar, u32 *err) {
    if (COOP) return grid_barrier(bar, err);
    __syncthreads();
    return true;
}

// Loads a value that decides the control flow (counts, sums, block weights)
// after a barrier: from L2 on a grid (global memory), a volatile load within
// one block (shared or global memory), so every thread sees the same value.
template<bool COOP, typename T>
__device__ __forceinline__ T ld_team(const T *p) {
    return COOP ? __ldcg(p) : *(const volatile T *) p;
}

__device__ __forceinline__ long long block_sum_ll(long long v, long long *sm) {
    v = warp_sum<long long>(v);
    if (lane_id() == 0) sm[warp_in_block()] = v;
    __syncthreads();
    long long r = 0;
    if (threadIdx.x == 0) {
        for (u32 w = 0; w < (blockDim.x >> 5); ++w) r += sm[w];
        sm[32] = r;
    }
    __syncthreads();
    r = sm[32];
    __syncthreads();
    return r;
}

// Adds v over all threads into *slot (zero beforehand), synchronises the team
// and reads the total into out; false once a barrier wait gave up.
template<bool COOP>
__device__ __forceinline__ bool team_sum(long long v, long long *slot, long long *sm, u32 *bar, u32 *err,
                                         long long &out) {
    v = block_sum_ll(v, sm);
    if (threadIdx.x == 0 && v) atomicAdd((unsigned long long *) slot, (unsigned long long) v);
    if (!team_sync<COOP>(bar, err)) return false;
    out = ld_team<COOP>(slot);
    return true;
}

#define TEAM_SYNC()                                          \
    do {                                                     \
        if (!team_sync<COOP>(F.bar, &a.st->err)) goto finish; \
    } while (0)

template<bool COOP>
__global__ void __launch_bounds__(FB, 1) k_jet_loop(JArgs a, FusedArgs F, FusedCtl *ctl) {
    extern __shared__ s32 fsm[];
    const u32 tid = threadIdx.x, lane = lane_id(), warp = warp_in_block(), n = a.g.n, k = a.k;
    s32 *wtab = fsm + warp * k;  // per-warp direct table
    s32 *btab = fsm + 32u * k;   // block table
    s32 *sbd = fsm + 33u * k;    // block-weight changes of this block's moves
    __shared__ u32 scnt[2 * FC_N];
    __shared__ long long ssum[2 * FS_N];
    __shared__ long long sl[33];
    __shared__ unsigned long long smu[33];
    __shared__ long long sms[33];
    __shared__ s32 smx[32];
    __shared__ OrderSmem osm;
    for (u32 i = tid; i < 34u * k; i += FB) fsm[i] = 0;
    if (!COOP && tid < 2 * FC_N) scnt[tid] = 0;
    if (!COOP && tid < 2 * FS_N) ssum[tid] = 0;
    __syncthreads();
    u32 *const cnt_base = COOP ? F.gcnt : scnt;
    long long *const sum_base = COOP ? F.gsum : ssum;
    const u32 nthreads = gridDim.x * FB;
    const u32 wbase0 = blockIdx.x * FB + warp * 32u;  // first row of this warp in grid-stride loops
    const u32 gwarps = gridDim.x * (FB / 32), gw = blockIdx.x * (FB / 32) + warp;
    const ConnTable<false, true, false> WT{nullptr, wtab, 0, k};
    const ConnTable<true, true, false> BT{nullptr, btab, 0, k};
    const bool promap = ctl->promap != 0;
    const s32 lmax = ctl->lmax;
    const u32 n_ratios = ctl->n_ratios;
    long long obj = ctl->obj, best_obj = obj;
    s32 maxw = ctl->maxw, best_max = maxw;
    u32 iterations = 0, it = 0;
    for (u32 ri = 0; ri < n_ratios; ++ri) {
        const u32 ratio = ctl->ratios[ri];
        u32 balance_iteration = 0, iteration = 0;
        while (iteration < JET_MAX_ITERATIONS) {
            iteration += 1;
            ++iterations;
            // counter set of this iteration (zero); the other set is cleared
            // after the first barrier, when every thread is done reading it
            const u32 set = it & 1u;
            ++it;
            u32 *const cnt = cnt_base + set * FC_N;
            long long *const sum = sum_base + set * FS_N;
            const bool clears = blockIdx.x == 0 && tid < (u32) FC_N;
            bool lp_iter = false;
            int step;
            if (maxw <= lmax) {
                step = 0;
                lp_iter = true;
                balance_iteration = 0;
            } else if (!promap) {
                step = balance_iteration < JET_MAX_WEAK_ITERATIONS ? 1 : 2;
            } else {
                balance_iteration++;
                step = balance_iteration < JET_MAX_WEAK_ITERATIONS ? 1 : 2;
            }
            u32 nm;
            if (step == 0) {
                // gain pass (jet_lp :193-238): cached targets, else recompute
                for (u32 wb = wbase0; wb < n; wb += nthreads) {
                    const u32 u = wb + lane;
                    int cls = -1;
                    if (u < n) {
                        const u32 dc = a.dest_cache[u];
                        if (dc != NULL_PART) {
                            a.dest_part[u] = dc;
                        } else {
                            cls = table_tier(a.g.rowlen[u], k);
                            if (cls == 0) lp_thread<false>(a, u, ratio);
                        }
                    }
                    const u32 s1 = warp_append(&cnt[0], cls == 1);
                    if (cls == 1) a.heavy[s1] = u;
                    const u32 s2 = warp_append(&cnt[1], cls == 2);
                    if (cls == 2) a.heavy2[s2] = u;
                }
                TEAM_SYNC();
                if (clears) cnt_base[(set ^ 1u) * FC_N + tid] = 0;
                if (clears && tid < (u32) FS_N) sum_base[(set ^ 1u) * FS_N + tid] = 0;
                const u32 n1 = ld_team<COOP>(&cnt[0]), n2 = ld_team<COOP>(&cnt[1]);
                for (u32 i = gw; i < n1; i += gwarps) lp_group<false, true, false>(a, a.heavy[i], ratio, WT, nullptr, nullptr);
                for (u32 i = blockIdx.x; i < n2; i += gridDim.x) lp_group<true, true, false>(a, a.heavy2[i], ratio, BT, smu, sms);
                TEAM_SYNC();
                // filter (:247-258)
                for (u32 wb = wbase0; wb < n; wb += nthreads) {
                    const u32 u = wb + lane;
                    bool c = false;
                    if (u < n) {
                        c = a.dest_part[u] != NO_MOVE && a.lock[u] == 0;
                        if (c) {
                            a.gain1[u] = a.gain_cache[u];
                        } else {
                            a.gain1[u] = GAIN_MIN;
                            a.lock[u] = 0;
                        }
                    }
                    const u32 s3 = warp_append(&cnt[2], c);
                    if (c) a.cand[s3] = u;
                }
                TEAM_SYNC();
                // afterburner: short rows by a thread, longer ones by the whole warp
                const u32 nc = ld_team<COOP>(&cnt[2]);
                for (u32 wb = wbase0; wb < nc; wb += nthreads) {
                    const u32 i = wb + lane;
                    u32 u = 0, len = 0;
                    bool lock = false;
                    if (i < nc) {
                        u = a.cand[i];
                        len = a.g.rowlen[u];
                        if (len <= FUSED_AB_THREAD) {
                            const s32 ug = a.gain1[u];
                            lock = wadd(ug, ab_range<false>(a, u, ug, a.map[u], a.dest_part[u], 0, len, 0, 1)) >= 0;
                        }
                    }
                    unsigned longer = __ballot_sync(FULL, i < nc && len > FUSED_AB_THREAD);
                    while (longer) {
                        const int src = __ffs(longer) - 1;
                        longer &= longer - 1;
                        const u32 v = __shfl_sync(FULL, u, src), lv = __shfl_sync(FULL, len, src);
                        const s32 vg = a.gain1[v];
                        const s32 change = (s32) warp_sum<u32>(
                            (u32) ab_range<false>(a, v, vg, a.map[v], a.dest_part[v], 0, lv, lane, 32));
                        if (lane == (u32) src) lock = wadd(vg, change) >= 0;
                    }
                    if (lock) a.lock[u] = 1;
                    const u32 s4 = warp_append(&cnt[3], lock);
                    if (lock) a.moves[s4] = u;
                }
                TEAM_SYNC();
                nm = ld_team<COOP>(&cnt[3]);
            } else {
                // rebalancing picks (rebalance_weak :592-751 / rebalance_strong :356-590)
                const bool strong = step == 2;
                const RbArgs &r = strong ? F.strong : F.weak;
                if (blockIdx.x == 0) {
                    if (strong) maxv_block(a.bw, k, r.max_b_w, &a.st->imax[1]);
                    else under_block(a.bw, k, r.max_b_w, F.under, &a.st->cnt[ST_AUX]);
                }
                TEAM_SYNC();
                if (clears) cnt_base[(set ^ 1u) * FC_N + tid] = 0;
                if (clears && tid < (u32) FS_N) sum_base[(set ^ 1u) * FS_N + tid] = 0;
                const s32 maxv = ld_team<COOP>(&a.st->imax[1]);
                for (u32 wb = wbase0; wb < n; wb += nthreads) {
                    const u32 u = wb + lane;
                    int cls = -1;
                    if (u < n) {
                        const u32 o = a.map[u];
                        const bool q = strong ? rb_qualifies<true>(a, r, o, g_vw(a.g, u), maxv)
                                              : rb_qualifies<false>(a, r, o, g_vw(a.g, u), maxv);
                        if (!q) {
                            if (!strong) a.dest_part[u] = o;
                            r.keys[u] = NOKEY;
                        } else {
                            cls = table_tier(a.g.rowlen[u], k);
                            if (cls == 0) {
                                if (strong) rb_thread<true, false>(a, r, u, o);
                                else rb_thread<false, false>(a, r, u, o);
                            }
                        }
                    }
                    const u32 s1 = warp_append(&cnt[0], cls == 1);
                    if (cls == 1) a.heavy[s1] = u;
                    const u32 s2 = warp_append(&cnt[1], cls == 2);
                    if (cls == 2) a.heavy2[s2] = u;
                }
                TEAM_SYNC();
                const u32 n1 = ld_team<COOP>(&cnt[0]), n2 = ld_team<COOP>(&cnt[1]);
                for (u32 i = gw; i < n1; i += gwarps) {
                    if (strong) rb_group<true, false, true, false>(a, r, a.heavy[i], WT, nullptr, nullptr);
                    else rb_group<false, false, true, false>(a, r, a.heavy[i], WT, nullptr, nullptr);
                }
                for (u32 i = blockIdx.x; i < n2; i += gridDim.x) {
                    if (strong) rb_group<true, true, true, false>(a, r, a.heavy2[i], BT, smu, sms);
                    else rb_group<false, true, true, false>(a, r, a.heavy2[i], BT, smu, sms);
                }
                TEAM_SYNC();
                if (blockIdx.x == 0) {
                    if (strong) order_small_body<true>(a, r, F.width, F.bits_strong, F.S, r.max_b_w, osm);
                    else order_small_body<false>(a, r, F.width, F.bits_weak, F.S, r.max_b_w, osm);
                }
                TEAM_SYNC();
                nm = ld_team<COOP>(&a.st->cnt[ST_MOVES]);
            }
            // perform_moves (:753-924): labels with the moved bit, block weights
            long long entries = 0;
            for (u32 i = blockIdx.x * FB + tid; i < nm; i += nthreads) {
                const u32 u = a.moves[i];
                const u32 ou = a.map[u], nu = a.dest_part[u];
                const s32 w = g_vw(a.g, u);
                if (ou != nu) {
                    atomicSub(&sbd[ou], w);
                    atomicAdd(&sbd[nu], w);
                }
                a.map[u] = ou != nu ? (nu | MOVED) : nu;
                a.dest_part[u] = ou;
                a.dest_cache[u] = NULL_PART;
                entries += a.g.rowlen[u];
            }
            __syncthreads();
            for (u32 b = tid; b < k; b += FB)
                if (sbd[b]) {
                    atomicAdd(&a.bw[b], sbd[b]);
                    sbd[b] = 0;
                }
            long long ent = 0;
            if (!team_sum<COOP>(entries, &sum[0], sl, F.bar, &a.st->err, ent)) goto finish;
            const bool inval = (unsigned long long) ent < a.inval_all_min;
            s32 m = 0;
            for (u32 b = tid; b < k; b += FB) {
                const s32 x = ld_team<COOP>(&a.bw[b]);
                m = x > m ? x : m;
            }
            m = __reduce_max_sync(FULL, m);
            if (lane == 0) smx[warp] = m;
            __syncthreads();
            s32 new_maxw = 0;
            for (u32 w = 0; w < FB / 32; ++w) new_maxw = smx[w] > new_maxw ? smx[w] : new_maxw;
            // exact objective change and the neighbours' cache resets
            long long acc = 0;
            for (u32 wb = wbase0; wb < nm; wb += nthreads) {
                const u32 i = wb + lane;
                u32 u = 0, len = 0;
                if (i < nm) {
                    u = a.moves[i];
                    len = a.g.rowlen[u];
                    if (len <= FUSED_AB_THREAD) acc += delta_range<false>(a, u, 0, len, 0, 1, inval);
                }
                unsigned longer = __ballot_sync(FULL, i < nm && len > FUSED_AB_THREAD);
                while (longer) {
                    const int src = __ffs(longer) - 1;
                    longer &= longer - 1;
                    const u32 v = __shfl_sync(FULL, u, src), lv = __shfl_sync(FULL, len, src);
                    acc += delta_range<false>(a, v, 0, lv, lane, 32, inval);
                }
            }
            long long d = 0;
            if (!team_sum<COOP>(acc, &sum[1], sl, F.bar, &a.st->err, d)) goto finish;
            if (!inval)
                for (u32 u = blockIdx.x * FB + tid; u < n; u += nthreads) a.dest_cache[u] = NULL_PART;
            for (u32 i = blockIdx.x * FB + tid; i < nm; i += nthreads) a.map[a.moves[i]] &= ~MOVED;
            // control (jet_label_propagation.h:966-1030, promap :1250-1305):
            // 1 = next iteration, 2 = next ratio
            int action = 0;
            if (!promap) {
                if (nm == 0) {
                    if (lp_iter) {
                        action = 2;
                    } else if (balance_iteration < JET_MAX_WEAK_ITERATIONS) {
                        balance_iteration = JET_MAX_WEAK_ITERATIONS;
                        action = 1;
                    } else {
                        action = 2;
                    }
                } else if (!lp_iter) {
                    balance_iteration++;
                }
            } else if (nm == 0) {
                action = 1;
            }
            bool copy = false;
            if (action == 0) {
                obj += promap ? d : d / 2;
                maxw = new_maxw;
                const bool leq = promap ? (maxw < best_max) : (maxw <= best_max);
                if (best_max > lmax && maxw < best_max) {
                    copy = true;
                    iteration = 0;
                } else if (obj < best_obj && (maxw <= lmax || leq)) {
                    if (1000 * obj < 999 * best_obj) iteration = 0;  // PHI = 0.999
                    copy = true;
                }
                if (copy) {
                    best_obj = obj;
                    best_max = maxw;
                }
            }
            if (copy)  // the moved bits may still be set here: mask them
                for (u32 u = blockIdx.x * FB + tid; u < n; u += nthreads) F.part[u] = a.map[u] & ~MOVED;
            TEAM_SYNC();
            if (action == 2) break;
        }
    }
    if (blockIdx.x == 0 && tid == 0) {
        ctl->obj = best_obj;
        ctl->maxw = best_max;
        ctl->iterations = iterations;
    }
finish:;
}

#undef TEAM_SYNC

// ---- objectives ------------------------------------------------------------------

__global__ void k_objective(DGraph g, const u32 *part, const u32 *code, const s32 *bitdist, unsigned long long *out) {
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    long long acc = 0;
    for (u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < g.n; u += warps) {
        const u64 beg = g.rowptr[u];
        const u32 len = g.rowlen[u];
        const u32 pu = part[u];
        for (u32 t = lane_id(); t < len; t += 32) {
            const u32 pv = part[g.adj[beg + t]];
            const long long w = g_ew(g, beg + t);
            if (code) acc += w * dist_of(code, bitdist, pu, pv);
            else acc += pu != pv ? w : 0;
        }
    }
    acc = warp_sum<long long>(acc);
    if (lane_id() == 0 && acc) atomicAdd(out, (unsigned long long) acc);
}

__global__ void k_block_weights(DGraph g, const u32 *part, s32 *bw) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < g.n; u += gridDim.x * blockDim.x)
        atomicAdd(&bw[part[u]], g_vw(g, u));
}

JArgs make_args(JetLevel &L) {
    JArgs a;
    a.g = L.g;
    a.k = L.k;
    a.lmax = L.lmax;
    a.g_weight = L.g_weight;
    a.code = L.D ? L.D->code : nullptr;
    a.bitdist = L.D ? L.D->bitdist : nullptr;
    a.map = L.map;
    a.bw = L.bw;
    a.dest_cache = L.dest_cache;
    a.gain_cache = L.gain_cache;
    a.lock = L.lock;
    a.dest_part = L.dest_part;
    a.gain1 = L.gain1;
    a.cand = L.cand;
    a.moves = L.moves;
    a.heavy = L.heavy;
    a.heavy2 = L.heavy2;
    a.items = L.items;
    a.items_cap = L.items_cap;
    a.abacc = L.abacc;
    a.inval_all_min = L.cache_pure ? (L.g.m * L.ctx->tune.jet_inval_all_pct + 99) / 100 : ~0ull;
    a.hubacc = L.hubacc;
    a.hubcnt = L.hubcnt;
    a.hub_cap = L.hub_cap;
    a.hub_deg = L.hub_deg;
    a.dlab = L.dlab;
    a.abrec = L.abrec;
    a.vec = L.ctx->tune.jet_vec_loads;
    a.hub_track_max = L.hub_track_max;
    a.hub_cur = L.hub_cur;
    a.hub_gen = L.hub_gen;
    a.hub_vertex = L.hub_vertex;
    a.abcnt = L.abcnt;
    a.st = L.ctx->d_status;
    a.blk_slots = L.blk_slots;
    return a;
}

void sections_of(u32 n, u32 k, u32 &sections, u32 &width) {
    sections = MAX_SECTIONS;
    u32 section_size = (n + sections * k) / (sections * k);
    if (section_size < 4096) {
        section_size = 4096;
        sections = (n + section_size * k) / (section_size * k);
    }
    width = MAX_BUCKETS * sections;
}

// Raises the dynamic shared-memory limit of the block-tier kernels, once per
// device (function attributes are per device; several host threads may get
// here at once).
void set_big_smem() {
    static std::mutex mu;
    static std::vector<int> done;
    int dev = 0;
    HP_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    for (int d: done)
        if (d == dev) return;
    const int smem = (int) (JB_SLOTS * 8);
    HP_CUDA(cudaFuncSetAttribute(k_lp_block, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    HP_CUDA(cudaFuncSetAttribute(k_rb_block<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    HP_CUDA(cudaFuncSetAttribute(k_rb_block<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    HP_CUDA(cudaFuncSetAttribute(k_jet_loop<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int) (34 * JW_SLOTS * sizeof(s32))));
    HP_CUDA(cudaFuncSetAttribute(k_jet_loop<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int) (34 * JW_SLOTS * sizeof(s32))));
    // staged chunk kernels: the full shared-memory carveout, so that
    // STAGE_BLOCKS_PER_SM blocks of stage_smem() bytes fit on an SM
    HP_CUDA(cudaFuncSetAttribute(k_delta_staged, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    done.push_back(dev);
}

} // namespace

// ---- distance oracle -----------------------------------------------------------------

DistOracle make_dist_oracle(Ctx &ctx, const std::vector<u32> &hier, const std::vector<s32> &dist) {
    DistOracle D;
    D.hier = hier;
    D.dist = dist;
    const u32 l = (u32) hier.size();
    if (l == 0 || dist.size() != l) throw HpError{HP_ERR_ARG, "hierarchy and distance must have the same length"};
    u64 k = 1;
    std::vector<u32> bits(l), off(l);
    u32 total = 0;
    for (u32 t = 0; t < l; ++t) {
        if (hier[t] == 0) throw HpError{HP_ERR_ARG, "hierarchy entries must be positive"};
        k *= hier[t];
        u32 b = 0;
        while ((1ull << b) < hier[t]) ++b;
        bits[t] = b;
        off[t] = total;
        total += b;
    }
    if (k > MAX_K || total > 32) throw HpError{HP_ERR_ARG, "hierarchy too large"};
    D.k = (u32) k;
    std::vector<u32> code(k);
    for (u32 i = 0; i < k; ++i) {
        u32 x = i, c = 0;
        for (u32 t = 0; t < l; ++t) {
            c |= (x % hier[t]) << off[t];
            x /= hier[t];
        }
        code[i] = c;
    }
    std::vector<s32> bd(32, 0);
    for (u32 t = 0; t < l; ++t)
        for (u32 b = 0; b < bits[t]; ++b) bd[off[t] + b] = dist[t];
    D.code = ctx.falloc<u32>(k);
    D.bitdist = ctx.falloc<s32>(32);
    HP_CUDA(cudaMemcpyAsync(D.code, code.data(), sizeof(u32) * k, cudaMemcpyHostToDevice, ctx.stream));
    HP_CUDA(cudaMemcpyAsync(D.bitdist, bd.data(), sizeof(s32) * 32, cudaMemcpyHostToDevice, ctx.stream));
    ctx.sync();  // host vectors go out of scope
    return D;
}

s64 edge_cut_dev(Ctx &ctx, const DGraph &g, const u32 *part) {
    ctx.zero_counters();
    k_objective<<<ctx.grid((u64) g.n * 32, BLOCK), BLOCK, 0, ctx.stream>>>(
        g, part, nullptr, nullptr, (unsigned long long *) &ctx.d_status->sum[0]); note_launch();
    HP_LAUNCH_CHECK();
    return ctx.read_status().sum[0] / 2;
}

s64 comm_cost_dev(Ctx &ctx, const DGraph &g, const u32 *part, const DistOracle &D) {
    ctx.zero_counters();
    k_objective<<<ctx.grid((u64) g.n * 32, BLOCK), BLOCK, 0, ctx.stream>>>(
        g, part, D.code, D.bitdist, (unsigned long long *) &ctx.d_status->sum[0]); note_launch();
    HP_LAUNCH_CHECK();
    return ctx.read_status().sum[0];
}

void block_weights(Ctx &ctx, const DGraph &g, const u32 *part, u32 k, s32 *bw) {
    HP_CUDA(cudaMemsetAsync(bw, 0, sizeof(s32) * k, ctx.stream));
    k_block_weights<<<ctx.grid(g.n, BLOCK), BLOCK, 0, ctx.stream>>>(g, part, bw); note_launch();
    HP_LAUNCH_CHECK();
}

s32 max_block_weight(Ctx &ctx, const s32 *bw, u32 k) {
    ctx.zero_counters();
    k_max_bw<<<1, 1024, 0, ctx.stream>>>(bw, k, &ctx.d_status->imax[MAX_BW]); note_launch();
    HP_LAUNCH_CHECK();
    return ctx.read_status().imax[MAX_BW];
}

// ---- JetLevel -----------------------------------------------------------------------

void JetLevel::setup(Ctx &c, const DGraph &gr, u32 kk, s32 lm, const DistOracle *d, const u32 *part) {
    ProfScope prof(c, "jet.setup");
    ctx = &c;
    g = gr;
    k = kk;
    lmax = lm;
    D = d;
    g_weight = (s32) gr.total_vw;
    const u32 n = g.n;
    map = c.balloc<u32>(n);
    bw = c.balloc<s32>(k);
    dest_cache = c.balloc<u32>(n);
    gain_cache = c.balloc<s32>(n);
    lock = c.balloc<u32>(n);
    dest_part = c.balloc<u32>(n);
    gain1 = c.balloc<s32>(n);
    cand = c.balloc<u32>(n);
    moves = c.balloc<u32>(n);
    heavy = c.balloc<u32>(n);
    heavy2 = c.balloc<u32>(n);
    blk_slots = block_slots_for(k);
    // warp tier: direct-indexed table of k values when k is small enough
    // (for the mapping objective the candidate scoring loops over the table,
    // so only up to 256 blocks), else a hashed table of JW_SLOTS slots
    warp_direct = k <= JW_SLOTS && (d == nullptr || k <= 256);
    warp_slots = warp_direct ? k : JW_SLOTS;
    warp_smem = (JW_BLOCK / 32) * (warp_direct ? 1u : 2u) * warp_slots * (u32) sizeof(u32);
    // chunk items (afterburner candidates, delta moves, hub chunks; each
    // vertex at most once): one per row of <= CHUNK (hub_deg) entries, so at
    // most n + m / min(CHUNK, hub_deg) + 1
    hub_deg = std::min<u32>(JW_DEG, std::max<u32>(64, c.tune.jet_hub_deg));
    items_cap = (u32) std::min<u64>(0xFFFFFFFFull, (u64) n + g.m / std::min<u32>(CHUNK, hub_deg) + 1);
    items = c.balloc<unsigned long long>(items_cap);
    // hub-row accumulators (rows of more than hub_deg entries: fewer than
    // m / hub_deg + 1 of them) when the tables are direct-indexed and k small
    hubacc = nullptr;
    hubcnt = nullptr;
    hub_cap = 0;
    dlab = nullptr;
    abrec = nullptr;
    hub_cur = nullptr;
    hub_gen = nullptr;
    hub_vertex = nullptr;
    hub_track_max = 0;
    if (warp_direct && k <= HUB_K) {
        hub_cap = (u32) std::min<u64>(n, g.m / hub_deg + 1);
        hubacc = c.balloc<s32>((u64) hub_cap * k);
        hubcnt = c.balloc<u32>(hub_cap);
        HP_CUDA(cudaMemsetAsync(hubacc, 0, sizeof(s32) * (u64) hub_cap * k, c.stream));
        HP_CUDA(cudaMemsetAsync(hubcnt, 0, sizeof(u32) * hub_cap, c.stream));
    }
    abacc = c.balloc<s32>(n);
    abcnt = c.balloc<u32>(n);
    HP_CUDA(cudaMemsetAsync(abacc, 0, sizeof(s32) * n, c.stream));
    HP_CUDA(cudaMemsetAsync(abcnt, 0, sizeof(u32) * n, c.stream));
    HP_CUDA(cudaMemcpyAsync(map, part, sizeof(u32) * n, cudaMemcpyDeviceToDevice, c.stream));
    device_fill<u32>(c, dest_cache, n, NULL_PART);
    HP_CUDA(cudaMemsetAsync(gain_cache, 0, sizeof(s32) * n, c.stream));
    HP_CUDA(cudaMemsetAsync(lock, 0, sizeof(u32) * n, c.stream));
    device_fill<u32>(c, dest_part, n, NO_MOVE);
    HP_CUDA(cudaMemsetAsync(gain1, 0, sizeof(s32) * n, c.stream));
    block_weights(c, g, map, k, bw);
    set_big_smem();
}

void JetLevel::prepare_kernel_loop() {
    Ctx &c = *ctx;
    ProfScope prof(c, "jet.prepare");
    dlab = c.balloc<unsigned long long>(g.n);
    abrec = c.balloc<unsigned long long>(g.n);
    if (!hubacc || !c.tune.jet_hub_conn || hub_cap > DL_MAX_HUBS) {
        JArgs a = make_args(*this);
        k_dlab_init<<<c.grid(g.n, BLOCK), BLOCK, 0, c.stream>>>(a); note_launch();
        HP_LAUNCH_CHECK();
        return;
    }
    hub_cur = c.balloc<u32>(1);
    hub_gen = c.balloc<u32>(hub_cap);
    u32 *vertex = c.balloc<u32>(hub_cap);
    hub_vertex = vertex;
    // every hub starts stale: generation 0x01010101 against 0; the passes
    // build the sums of the hubs they need
    HP_CUDA(cudaMemsetAsync(hub_gen, 0, sizeof(u32) * hub_cap, c.stream));
    HP_CUDA(cudaMemsetAsync(hub_cur, 1, sizeof(u32), c.stream));
    c.zero_counters();
    JArgs a = make_args(*this);
    k_hub_number<<<c.grid(g.n, BLOCK), BLOCK, 0, c.stream>>>(a); note_launch();
    HP_LAUNCH_CHECK();
    const DevStatus &st = c.read_status();
    if (st.err) throw HpError{HP_ERR_DEVICE, "hub numbering reported error bits " + std::to_string(st.err)};
    // updates pay while the moved rows hold at most jet_hub_track_pct percent
    // of the hub rows' entries
    const unsigned long long hub_entries = (unsigned long long) st.sum[0];
    hub_track_max = hub_entries / 100 * c.tune.jet_hub_track_pct;
    c.zero_counters();
}

// Rebuilds the sums of the stale hubs the pass's dispatch found (no host
// synchronisation: the item count stays on the device).
void JetLevel::rebuild_hubs() {
    if (!hub_cur) return;
    Ctx &c = *ctx;
    JArgs a = make_args(*this);
    KernTimer kt(c, "k_hub_rebuild");
    k_hub_rebuild<<<c.grid((u64) items_cap * 32, JW_BLOCK), JW_BLOCK, (JW_BLOCK / 32) * k * sizeof(u32), c.stream>>>(a);
    note_launch();
}

void JetLevel::gain_pass(u32 ratio_pct) {
    Ctx &c = *ctx;
    ProfScope prof(c, "jet.gain");
    JArgs a = make_args(*this);
    const u32 n = g.n;
    gain_rec = c.instr.begin(c.stream, "jet_gain", 0.0);
    {
        KernTimer kt(c, "k_lp_dispatch");
        k_lp_dispatch<<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a, ratio_pct); note_launch();
    }
    // the hub sums the pass needs are rebuilt under their own timer (the
    // gain pass's algorithmic bytes count a tracked hub as its k sums)
    c.instr.end(c.stream, gain_rec);
    rebuild_hubs();
    const size_t gain_rec2 = c.instr.begin(c.stream, "jet_gain", 0.0);
    {
        KernTimer kt(c, "k_lp_warp");
        if (warp_direct) {
            k_lp_warp<true><<<c.grid((u64) n * 32, JW_BLOCK), JW_BLOCK, warp_smem, c.stream>>>(a, ratio_pct, warp_slots);
        } else {
            k_lp_warp<false><<<c.grid((u64) n * 32, JW_BLOCK), JW_BLOCK, warp_smem, c.stream>>>(a, ratio_pct, warp_slots);
        }
        note_launch();
    }
    {
        KernTimer kt(c, "k_lp_block");
        if (hub_cur) {
            k_hub_tracked<0><<<c.grid((u64) hub_cap * 32, JW_BLOCK), JW_BLOCK, (JW_BLOCK / 32) * k * sizeof(u32),
                               c.stream>>>(a, ratio_pct, RbArgs{});
        } else if (hubacc) {
            k_hub<0><<<c.grid((u64) items_cap * 32, JW_BLOCK), JW_BLOCK, (JW_BLOCK / 32) * k * sizeof(u32), c.stream>>>(
                a, ratio_pct, RbArgs{});
        } else {
            k_lp_block<<<c.sm_count * 4, JB_BLOCK, blk_slots * 8, c.stream>>>(a, ratio_pct);
        }
        note_launch();
    }
    HP_LAUNCH_CHECK();
    c.instr.end(c.stream, gain_rec2);
}

void JetLevel::lp(u32 ratio_pct) {
    Ctx &c = *ctx;
    c.zero_counters();
    gain_pass(ratio_pct);
    ProfScope prof(c, "jet.filter_afterburner");
    JArgs a = make_args(*this);
    const u32 n = g.n;
    {
        KernTimer kt(c, "k_lp_filter");
        k_lp_filter<<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a); note_launch();
    }
    KernTimer kt(c, "k_afterburner");
    {
        KernTimer kt1(c, "k_ab_thread");
        if (a.vec) k_ab_thread<true><<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a);
        else k_ab_thread<false><<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a);
        note_launch();
    }
    {
        KernTimer kt1(c, "k_ab_chunk");
        if (a.vec) k_ab_chunk<true><<<c.grid((u64) items_cap * 32, BLOCK), BLOCK, 0, c.stream>>>(a);
        else k_ab_chunk<false><<<c.grid((u64) items_cap * 32, BLOCK), BLOCK, 0, c.stream>>>(a);
        note_launch();
    }
    HP_LAUNCH_CHECK();
}

void JetLevel::weak() {
    Ctx &c = *ctx;
    ProfScope prof(c, "jet.weak");
    const u32 n = g.n;
    const s32 opt = (g_weight + (s32) (k - 1)) / (s32) k;
    s32 max_b_w = (s32) ((99 * (s64) lmax) / 100);
    if (max_b_w < lmax - 100) max_b_w = lmax - 100;
    u32 sections, width;
    sections_of(n, k, sections, width);
    ScratchScope ss(c.arena);
    u32 *under = c.balloc<u32>(k);
    u32 *keys = c.balloc<u32>(n);
    c.zero_counters();
    k_under<<<1, 1024, 0, c.stream>>>(bw, k, max_b_w, under, &c.d_status->cnt[ST_AUX]); note_launch();
    JArgs a = make_args(*this);
    RbArgs r{opt, max_b_w, sections, under, keys};
    {
        ProfScope p2(c, "weak.pick");
        KernTimer kt(c, "k_weak_pick");
        {
            KernTimer kt1(c, "k_weak_dispatch");
            k_rb_dispatch<false><<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a, r); note_launch();
        }
        rebuild_hubs();
        {
            KernTimer kt1(c, "k_weak_warp");
            if (warp_direct) {
                k_rb_warp<false, true><<<c.grid((u64) n * 32, JW_BLOCK), JW_BLOCK, warp_smem, c.stream>>>(a, r, warp_slots);
            } else {
                k_rb_warp<false, false><<<c.grid((u64) n * 32, JW_BLOCK), JW_BLOCK, warp_smem, c.stream>>>(a, r, warp_slots);
            }
            note_launch();
        }
        {
            KernTimer kt1(c, "k_weak_block");
            if (hub_cur) {
                k_hub_tracked<1><<<c.grid((u64) hub_cap * 32, JW_BLOCK), JW_BLOCK, (JW_BLOCK / 32) * k * sizeof(u32),
                                   c.stream>>>(a, 0u, r);
            } else if (hubacc) {
                k_hub<1><<<c.grid((u64) items_cap * 32, JW_BLOCK), JW_BLOCK, (JW_BLOCK / 32) * k * sizeof(u32),
                               c.stream>>>(a, 0u, r);
            } else {
                k_rb_block<false><<<c.sm_count * 4, JB_BLOCK, blk_slots * 8, c.stream>>>(a, r);
            }
            note_launch();
        }
    }
    ProfScope p3(c, "weak.order");
    HP_LAUNCH_CHECK();
    if (n <= std::min<u32>(c.tune.order_small_n, ORDER_SMALL_N)) {
        OrderScratch S{};
        S.cands = c.balloc<u32>(n);
        S.ck = c.balloc<u32>(n);
        S.cands2 = c.balloc<u32>(n);
        S.ck2 = c.balloc<u32>(n);
        S.prefix = c.balloc<long long>((u64) n + 1);
        S.B = c.balloc<long long>((u64) k + 1);
        k_order_small<false><<<1, OB, 0, c.stream>>>(a, r, width, bits_for((u64) MAX_BUCKETS * k * sections + 1), S,
                                                     max_b_w); note_launch();
        HP_LAUNCH_CHECK();
        return;
    }
    // ordered candidates (ascending id), then a stable sort by mini-bucket key
    u32 *cands = c.balloc<u32>(n);
    u32 *ck = c.balloc<u32>(n);
    device_scan<u32>(
        c, n, [=] __device__(u64 i) -> u32 { return keys[i] != NOKEY ? 1u : 0u; },
        [=] __device__(u64 i, u32 p, u32 v) {
            if (v) {
                cands[p] = (u32) i;
                ck[p] = keys[i];
            }
        },
        &c.d_status->cnt[ST_CAND]);
    // the candidate count stays on the device: the sort, the scan and the
    // filter read it there (no host synchronisation inside the step)
    const u32 *d_cc = &c.d_status->cnt[ST_CAND];
    radix_sort_pairs<u32>(c, ck, cands, n, 0, bits_for((u64) MAX_BUCKETS * k * sections + 1), d_cc);
    long long *prefix = c.balloc<long long>((u64) n + 1);
    const DGraph gg = g;
    device_scan<long long>(
        c, (u64) n + 1,
        [=] __device__(u64 i) -> long long { return i < *d_cc ? (long long) g_vw(gg, cands[i]) : 0; },
        [=] __device__(u64 i, long long p, long long) { prefix[i] = p; }, (long long *) nullptr, d_cc, 1);
    long long *B = c.balloc<long long>((u64) k + 1);
    k_bounds<<<c.grid(k + 1, BLOCK), BLOCK, 0, c.stream>>>(ck, prefix, d_cc, k, width, B); note_launch();
    HP_CUDA(cudaMemsetAsync(&c.d_status->cnt[ST_MOVES], 0, sizeof(u32), c.stream));
    k_weak_filter<<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a, cands, prefix, B, d_cc); note_launch();
    HP_LAUNCH_CHECK();
}

void JetLevel::strong() {
    Ctx &c = *ctx;
    ProfScope prof(c, "jet.strong");
    const u32 n = g.n;
    const s32 opt = (g_weight + (s32) (k - 1)) / (s32) k;
    const s32 max_b_w = std::max<s32>(opt + 1, (s32) ((99 * (s64) lmax) / 100));
    u32 sections, width;
    sections_of(n, k, sections, width);
    ScratchScope ss(c.arena);
    u32 *keys = c.balloc<u32>(n);
    c.zero_counters();
    k_maxv<<<1, 1024, 0, c.stream>>>(bw, k, max_b_w, &c.d_status->imax[1]); note_launch();
    JArgs a = make_args(*this);
    RbArgs r{opt, max_b_w, sections, nullptr, keys};
    {
        ProfScope p2(c, "strong.pick");
        KernTimer kt(c, "k_strong_pick");
        {
            KernTimer kt1(c, "k_strong_dispatch");
            k_rb_dispatch<true><<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a, r); note_launch();
        }
        rebuild_hubs();
        {
            KernTimer kt1(c, "k_strong_warp");
            if (warp_direct) {
                k_rb_warp<true, true><<<c.grid((u64) n * 32, JW_BLOCK), JW_BLOCK, warp_smem, c.stream>>>(a, r, warp_slots);
            } else {
                k_rb_warp<true, false><<<c.grid((u64) n * 32, JW_BLOCK), JW_BLOCK, warp_smem, c.stream>>>(a, r, warp_slots);
            }
            note_launch();
        }
        {
            KernTimer kt1(c, "k_strong_block");
            if (hub_cur) {
                k_hub_tracked<2><<<c.grid((u64) hub_cap * 32, JW_BLOCK), JW_BLOCK, (JW_BLOCK / 32) * k * sizeof(u32),
                                   c.stream>>>(a, 0u, r);
            } else if (hubacc) {
                k_hub<2><<<c.grid((u64) items_cap * 32, JW_BLOCK), JW_BLOCK, (JW_BLOCK / 32) * k * sizeof(u32),
                               c.stream>>>(a, 0u, r);
            } else {
                k_rb_block<true><<<c.sm_count * 4, JB_BLOCK, blk_slots * 8, c.stream>>>(a, r);
            }
            note_launch();
        }
    }
    ProfScope p3(c, "strong.order");
    HP_LAUNCH_CHECK();
    if (n <= std::min<u32>(c.tune.order_small_n, ORDER_SMALL_N)) {
        OrderScratch S{};
        S.cands = c.balloc<u32>(n);
        S.ck = c.balloc<u32>(n);
        S.cands2 = c.balloc<u32>(n);
        S.ck2 = c.balloc<u32>(n);
        S.prefix = c.balloc<long long>((u64) n + 1);
        S.B = c.balloc<long long>((u64) k + 1);
        S.ea = c.balloc<long long>(k);
        S.es = c.balloc<long long>((u64) k + 1);
        S.mpre = c.balloc<long long>((u64) n + 1);
        S.fail = c.balloc<u32>(n);
        S.fail2 = c.balloc<u32>(n);
        k_order_small<true><<<1, OB, 0, c.stream>>>(a, r, width, bits_for((u64) MAX_BUCKETS * k * sections + 2), S,
                                                    max_b_w); note_launch();
        HP_LAUNCH_CHECK();
        return;
    }
    u32 *cands = c.balloc<u32>(n);
    u32 *ck = c.balloc<u32>(n);
    device_scan<u32>(
        c, n, [=] __device__(u64 i) -> u32 { return keys[i] != NOKEY ? 1u : 0u; },
        [=] __device__(u64 i, u32 p, u32 v) {
            if (v) {
                cands[p] = (u32) i;
                ck[p] = keys[i];
            }
        },
        &c.d_status->cnt[ST_CAND]);
    const u32 *d_cc = &c.d_status->cnt[ST_CAND];
    radix_sort_pairs<u32>(c, ck, cands, n, 0, bits_for((u64) MAX_BUCKETS * k * sections + 2), d_cc);
    long long *prefix = c.balloc<long long>((u64) n + 1);
    const DGraph gg = g;
    device_scan<long long>(
        c, (u64) n + 1,
        [=] __device__(u64 i) -> long long { return i < *d_cc ? (long long) g_vw(gg, cands[i]) : 0; },
        [=] __device__(u64 i, long long p, long long) { prefix[i] = p; }, (long long *) nullptr, d_cc, 1);
    long long *B = c.balloc<long long>((u64) k + 1);
    k_bounds<<<c.grid(k + 1, BLOCK), BLOCK, 0, c.stream>>>(ck, prefix, d_cc, k, width, B); note_launch();
    long long *ea = c.balloc<long long>(k);
    long long *es = c.balloc<long long>((u64) k + 1);
    long long *mpre = c.balloc<long long>((u64) n + 1);
    HP_CUDA(cudaMemsetAsync(ea, 0, sizeof(long long) * k, c.stream));
    HP_CUDA(cudaMemsetAsync(&c.d_status->cnt[ST_MOVES], 0, sizeof(u32), c.stream));
    k_strong_filter<<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a, cands, prefix, B, d_cc, ea, mpre); note_launch();
    long long *max_v = (long long *) &c.d_status->sum[3];
    k_cookie<<<1, 1024, 0, c.stream>>>(bw, k, max_b_w, B, ea, es, max_v); note_launch();
    u32 *fail = c.balloc<u32>(n);
    u32 *n_fail = &c.d_status->cnt[ST_HEAVY];
    HP_CUDA(cudaMemsetAsync(n_fail, 0, sizeof(u32), c.stream));
    k_strong_assign<<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a, mpre, ea, es, fail, n_fail); note_launch();
    HP_LAUNCH_CHECK();
    {
        // fallback slots in ascending vertex id; the failure count stays on
        // the device (usually zero: every kernel then returns at once)
        u32 *fk = c.balloc<u32>(n);
        k_copy_count<<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(fk, fail, n_fail); note_launch();
        radix_sort_pairs<u32>(c, fk, fail, n, 0, bits_for(n), n_fail);
        k_strong_fallback<<<1, 32, 0, c.stream>>>(a, fail, n_fail, es, max_v); note_launch();
        HP_LAUNCH_CHECK();
    }
}

void JetLevel::perform() {
    Ctx &c = *ctx;
    ProfScope prof(c, "jet.perform");
    JArgs a = make_args(*this);
    const u32 n = g.n;
    k_perform_reset<<<1, 32, 0, c.stream>>>(c.d_status); note_launch();
    {
        // labels first (new label + MOVED bit, old label in dest_part) ...
        ProfScope p2(c, "perform.apply");
        KernTimer kt(c, "k_apply");
        k_apply<<<c.grid(n, BLOCK), BLOCK, k <= APPLY_SMEM_K ? k * sizeof(s32) : 0, c.stream>>>(a); note_launch();
    }
    {
        // ... then the exact objective change and the neighbours' cache resets
        ProfScope p3(c, "perform.delta");
        KernTimer kt(c, "k_delta");
        delta_rec = kt.idx;
        {
            KernTimer kt1(c, "k_delta_thread");
            if (a.vec) k_delta_thread<true><<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a);
            else k_delta_thread<false><<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a);
            note_launch();
        }
        {
            KernTimer kt1(c, "k_delta_chunk");
            if (c.tune.jet_chunk_mode == 2 && stage_ok(g)) {
                const u32 blocks = (u32) std::min<u64>(((u64) items_cap * 32 + STAGE_BLOCK - 1) / STAGE_BLOCK,
                                                       (u64) c.sm_count * STAGE_BLOCKS_PER_SM);
                k_delta_staged<<<std::max<u32>(blocks, 1), STAGE_BLOCK, stage_smem(), c.stream>>>(a);
            } else if (c.tune.jet_chunk_mode == 1) {
                k_delta_chunk<8><<<c.grid((u64) items_cap * 32, BLOCK), BLOCK, 0, c.stream>>>(a);
            } else {
                if (a.vec) k_delta_chunk<4, true><<<c.grid((u64) items_cap * 32, BLOCK), BLOCK, 0, c.stream>>>(a);
                else k_delta_chunk<4><<<c.grid((u64) items_cap * 32, BLOCK), BLOCK, 0, c.stream>>>(a);
            }
            note_launch();
        }
        k_inval_unmark<<<c.grid(n, BLOCK), BLOCK, 0, c.stream>>>(a); note_launch();
    }
    HP_LAUNCH_CHECK();
}

void JetLevel::release_graphs() {
    for (StepGraph &sg: step_graphs) cudaGraphExecDestroy(sg.exec);
    step_graphs.clear();
}

void JetLevel::run_step(int kind, u32 ratio_pct) {
    Ctx &c = *ctx;
    auto body = [&] {
        if (kind == 0) lp(ratio_pct);
        else if (kind == 1) weak();
        else strong();
        perform();
        HP_CUDA(cudaMemcpyAsync(c.h_status, c.d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, c.stream));
    };
    if (!graphs) {
        body();
        c.sync();
        return;
    }
    cudaGraphExec_t exec = nullptr;
    unsigned long long kernels = 0;
    for (const StepGraph &sg: step_graphs)
        if (sg.kind == kind && sg.ratio == ratio_pct) {
            exec = sg.exec;
            kernels = sg.kernels;
        }
    if (!exec) {
        // Scratch allocated inside the step is released when it returns and
        // nothing else allocates while the level's iterations run, so the
        // addresses baked into the graph stay valid for every replay.
        cudaGraph_t graph = nullptr;
        const unsigned long long before = t_kernel_launches;
        HP_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        c.instr.capturing = c.prof.capturing = true;
        try {
            body();
        } catch (...) {
            c.instr.capturing = c.prof.capturing = false;
            cudaStreamEndCapture(c.stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        c.instr.capturing = c.prof.capturing = false;
        HP_CUDA(cudaStreamEndCapture(c.stream, &graph));
        // the capture records launches without running them: count them
        // on every replay instead
        kernels = t_kernel_launches - before;
        g_kernel_launches -= kernels;
        const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        HP_CUDA(e);
        step_graphs.push_back(StepGraph{kind, ratio_pct, exec, kernels});
    }
    HP_CUDA(cudaGraphLaunch(exec, c.stream));
    g_kernel_launches += kernels;
    c.sync();
}

// The whole level loop in one k_jet_loop launch (warp_direct levels of at
// most FUSED_MAX_N vertices): one block, or a cooperative grid of `blocks`
// blocks; writes the best labelling to part.
static void jet_refine_fused(Ctx &ctx, JetLevel &L, const std::vector<u32> &ratios, bool promap, u32 *part,
                             s64 &obj, s32 &maxw, u32 blocks) {
    const u32 n = L.g.n, k = L.k;
    const s32 opt = (L.g_weight + (s32) (k - 1)) / (s32) k;
    u32 sections, width;
    sections_of(n, k, sections, width);
    FusedArgs F{};
    F.weak.opt = F.strong.opt = opt;
    F.weak.max_b_w = std::max<s32>(L.lmax - 100, (s32) ((99 * (s64) L.lmax) / 100));
    F.strong.max_b_w = std::max<s32>(opt + 1, (s32) ((99 * (s64) L.lmax) / 100));
    F.weak.sections = F.strong.sections = sections;
    F.under = ctx.balloc<u32>(k);
    F.weak.under = F.under;
    F.weak.keys = F.strong.keys = ctx.balloc<u32>(n);
    F.width = width;
    F.bits_weak = bits_for((u64) MAX_BUCKETS * k * sections + 1);
    F.bits_strong = bits_for((u64) MAX_BUCKETS * k * sections + 2);
    OrderScratch &S = F.S;
    S.cands = ctx.balloc<u32>(n);
    S.ck = ctx.balloc<u32>(n);
    S.cands2 = ctx.balloc<u32>(n);
    S.ck2 = ctx.balloc<u32>(n);
    S.prefix = ctx.balloc<long long>((u64) n + 1);
    S.B = ctx.balloc<long long>((u64) k + 1);
    S.ea = ctx.balloc<long long>(k);
    S.es = ctx.balloc<long long>((u64) k + 1);
    S.mpre = ctx.balloc<long long>((u64) n + 1);
    S.fail = ctx.balloc<u32>(n);
    S.fail2 = ctx.balloc<u32>(n);
    F.part = part;
    F.gcnt = ctx.balloc<u32>(2 * FC_N);
    F.gsum = ctx.balloc<long long>(2 * FS_N);
    F.bar = ctx.balloc<u32>(2);
    HP_CUDA(cudaMemsetAsync(F.bar, 0, 2 * sizeof(u32), ctx.stream));
    HP_CUDA(cudaMemsetAsync(F.gcnt, 0, 2 * FC_N * sizeof(u32), ctx.stream));
    HP_CUDA(cudaMemsetAsync(F.gsum, 0, 2 * FS_N * sizeof(long long), ctx.stream));
    FusedCtl h{};
    h.n_ratios = (u32) ratios.size();
    for (size_t i = 0; i < ratios.size() && i < 17; ++i) h.ratios[i] = ratios[i];
    h.lmax = L.lmax;
    h.promap = promap ? 1u : 0u;
    h.obj = obj;
    h.maxw = maxw;
    FusedCtl *d = ctx.balloc<FusedCtl>(1);
    HP_CUDA(cudaMemcpyAsync(d, &h, sizeof(FusedCtl), cudaMemcpyHostToDevice, ctx.stream));
    ctx.zero_counters();
    const size_t smem = 34 * (size_t) k * sizeof(s32);
    JArgs a = make_args(L);
    std::optional<CoopGuard> coop;  // cooperative budget (grid blocks), until the kernel has completed
    if (blocks <= 1) {
        KernTimer kt(ctx, "k_jet_fused");
        k_jet_loop<false><<<1, FB, smem, ctx.stream>>>(a, F, d); note_launch();
    } else {
        coop.emplace(ctx.device, ctx.stream, blocks, (u32) ctx.sm_count);
        KernTimer kt(ctx, "k_jet_coop");
        void *args[] = {&a, &F, &d};
        HP_CUDA(cudaLaunchCooperativeKernel((const void *) k_jet_loop<true>, dim3(blocks), dim3(FB), args, smem,
                                            ctx.stream));
        note_launch();
    }
    HP_LAUNCH_CHECK();
    HP_CUDA(cudaMemcpyAsync(&h, d, sizeof(FusedCtl), cudaMemcpyDeviceToHost, ctx.stream));
    const DevStatus &st = ctx.read_status();
    if (st.err & DEV_ERR_SPIN) throw CoopSpin{};
    if (st.err) throw HpError{HP_ERR_DEVICE, "Jet kernel reported error bits " + std::to_string(st.err)};
    obj = h.obj;
    maxw = h.maxw;
}

// Blocks of the cooperative level loop for a level of n vertices (0 when it
// does not apply): one per Tunables::jet_coop_rows vertices, at least two, at
// most as many as fit on the GPU at once.
static u32 coop_blocks(Ctx &ctx, u32 n, u32 k) {
    int per_sm = 0;
    HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jet_loop<true>, FB,
                                                          34 * (size_t) k * sizeof(s32)));
    if (per_sm <= 0) return 0;
    const u64 rows = std::max<u32>(1, ctx.tune.jet_coop_rows);
    const u64 want = ((u64) n + rows - 1) / rows;
    return (u32) std::max<u64>(2, std::min<u64>(want, (u64) per_sm * ctx.sm_count));
}

void jet_refine(Ctx &ctx, const DGraph &g, u32 *part, u32 k, s32 lmax, bool ultra, u32 level, s64 &obj, s32 &maxw,
                const DistOracle *D) {
    if (g.n == 0 || k <= 1) return;
    ScratchScope ss(ctx.arena);
    JetLevel L;
    L.setup(ctx, g, k, lmax, D, part);
    const bool promap = D != nullptr;
    // one filter ratio per level (or none for the mapping objective): a
    // recomputed gain then equals a still-valid cached one
    L.cache_pure = promap || !ultra;
    L.graphs = g.m <= ctx.tune.jet_graph_max_m && !ctx.prof.enabled;
    s64 best_obj = obj;
    s32 best_max = maxw;
    std::vector<u32> ratios;
    if (ultra && !promap) ratios = {85, 80, 75, 70, 65, 60, 55, 50, 45, 40, 35, 30, 25, 20, 15, 10, 5};
    else ratios = {level == 0 ? 25u : 75u};
    if (L.warp_direct && !ctx.prof.enabled) {
        if (g.n <= std::min<u32>(ctx.tune.jet_fused_max_n, FUSED_MAX_N) && g.m <= ctx.tune.jet_fused_max_m) {
            jet_refine_fused(ctx, L, ratios, promap, part, obj, maxw, 1);
            return;
        }
        if (g.n <= std::min<u32>(ctx.tune.jet_coop_max_n, FUSED_MAX_N) && g.m <= ctx.tune.jet_coop_max_m &&
            g.m <= (u64) ctx.tune.jet_coop_max_deg * g.n) {
            set_big_smem();
            const u32 blocks = coop_blocks(ctx, g.n, k);
            if (blocks) {
                // the level's input labelling, kept for the per-kernel path
                // should the cooperative loop give up at a grid barrier
                u32 *saved = ctx.balloc<u32>(g.n);
                HP_CUDA(cudaMemcpyAsync(saved, part, sizeof(u32) * g.n, cudaMemcpyDeviceToDevice, ctx.stream));
                const s64 obj0 = obj;
                const s32 maxw0 = maxw;
                try {
                    jet_refine_fused(ctx, L, ratios, promap, part, obj, maxw, blocks);
                    return;
                } catch (const CoopSpin &) {
                    HP_CUDA(cudaMemcpyAsync(part, saved, sizeof(u32) * g.n, cudaMemcpyDeviceToDevice, ctx.stream));
                    ctx.zero_status();
                    obj = obj0;
                    maxw = maxw0;
                    L.setup(ctx, g, k, lmax, D, part);
                }
            }
        }
    }
    L.prepare_kernel_loop();
    for (u32 ratio: ratios) {
        u32 balance_iteration = 0, iteration = 0;
        while (iteration < JET_MAX_ITERATIONS) {
            iteration += 1;
            bool lp_iter = false;
            int step = 0;
            if (!promap) {
                if (maxw <= lmax) {
                    step = 0;
                    lp_iter = true;
                    balance_iteration = 0;
                } else if (balance_iteration < JET_MAX_WEAK_ITERATIONS) {
                    step = 1;
                } else {
                    step = 2;
                }
            } else {
                if (maxw <= lmax) {
                    step = 0;
                    lp_iter = true;
                    balance_iteration = 0;
                } else {
                    balance_iteration++;
                    step = balance_iteration < JET_MAX_WEAK_ITERATIONS ? 1 : 2;
                }
            }
            L.run_step(step, ratio);
            const DevStatus &st = *ctx.h_status;
            if (st.err) throw HpError{HP_ERR_DEVICE, "Jet kernel reported error bits " + std::to_string(st.err)};
            const u32 nm = st.cnt[ST_MOVES];
            if (lp_iter && L.gain_rec < ctx.instr.pending.size()) {
                // algorithmic bytes of the gain pass: every vertex reads its
                // cache entry and writes dest_part (8 B); a recomputed vertex
                // instead reads its offset, length and own label and writes
                // dest_part and both caches (16 B in all), and each entry of
                // its row costs adj + ew + the label gather (12 B)
                const double nrec = st.cnt[ST_AUX], erec = (double) st.sum[4];
                ctx.instr.pending[L.gain_rec].bytes = 8.0 * (g.n - nrec) + 16.0 * nrec + 12.0 * erec;
            }
            if (L.delta_rec < ctx.instr.pending.size()) {
                // algorithmic bytes of the delta pass (all tiers and the
                // unmark pass): per move its list entry, offset, length, label
                // and old label and the unmark read-modify-write (36 B); per
                // entry of a moved row adj (+ ew), the neighbour's label and
                // its cache reset
                const double ent = (double) st.sum[SUM_PERF_ENTRIES];
                const bool all = L.cache_pure &&
                                 (u64) st.sum[SUM_PERF_ENTRIES] >= (g.m * ctx.tune.jet_inval_all_pct + 99) / 100;
                ctx.instr.pending[L.delta_rec].bytes =
                    36.0 * nm + (g.ew ? 16.0 : 12.0) * ent - (all ? 4.0 * ent - 4.0 * g.n : 0.0);
            }
            if (!promap) {
                if (nm == 0) {
                    if (lp_iter) break;
                    if (balance_iteration < JET_MAX_WEAK_ITERATIONS) {
                        balance_iteration = JET_MAX_WEAK_ITERATIONS;
                        continue;
                    }
                    break;
                }
                if (!lp_iter) balance_iteration++;
            } else if (nm == 0) {
                continue;
            }
            const s64 d = st.sum[SUM_DELTA];
            obj += promap ? d : d / 2;
            maxw = st.imax[MAX_BW];
            const bool leq = promap ? (maxw < best_max) : (maxw <= best_max);
            if (best_max > lmax && maxw < best_max) {
                HP_CUDA(cudaMemcpyAsync(part, L.map, sizeof(u32) * g.n, cudaMemcpyDeviceToDevice, ctx.stream));
                best_obj = obj;
                best_max = maxw;
                iteration = 0;
            } else if (obj < best_obj && (maxw <= lmax || leq)) {
                if (1000 * obj < 999 * best_obj) iteration = 0;  // PHI = 0.999
                HP_CUDA(cudaMemcpyAsync(part, L.map, sizeof(u32) * g.n, cudaMemcpyDeviceToDevice, ctx.stream));
                best_obj = obj;
                best_max = maxw;
            }
        }
    }
    obj = best_obj;
    maxw = best_max;
    ctx.sync();
}

} // namespace hp
