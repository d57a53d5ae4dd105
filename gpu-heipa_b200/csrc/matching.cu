// Two-hop heavy-edge matching on the device; the semantics follow
// src/coarsening/two_hop_matching.h:93-650 with the deterministic commit and
// grouping rules documented in coarsen.cuh.
#include "coarsen.cuh"
#include "prims.cuh"



namespace hp {
namespace {

// Reads of vcmap: plain in kernels that do not write it, L2-coherent (no L1)
// in the fused matching loop, where other blocks write it between phases.
template<bool COH>
__device__ __forceinline__ u32 ld_vc(const u32 *p) {
    return COH ? __ldcg(p) : *p;
}

// Argmax over the eligible neighbours of u of (edge weight, xorshift(v + r)),
// r = xorshift(u ^ seed): pick_neighbor_flat two_hop_matching.h:102-141.
template<bool INITIAL, bool COH = false>
__device__ __forceinline__ u32 pick_thread(const DGraph &g, const u32 *vcmap, u32 u, u32 seed) {
    const u32 r = xorshift32(u ^ seed);
    const u64 beg = g.rowptr[u];
    const u32 len = g.rowlen[u];
    if (len > THREAD_DEG_MAX) return SENTINEL;  // callers use this for short rows only
    // rows of at most THREAD_DEG_MAX entries: load the entries, gather their
    // match state together, then take the argmax in entry order
    u32 vs[THREAD_DEG_MAX];
    s32 ws[THREAD_DEG_MAX];
    bool ok[THREAD_DEG_MAX];
#pragma unroll
    for (int t = 0; t < (int) THREAD_DEG_MAX; ++t) {
        vs[t] = (u32) t < len ? g.adj[beg + t] : SENTINEL;
        ws[t] = ((u32) t < len && g.ew) ? g.ew[beg + t] : 0;
    }
#pragma unroll
    for (int t = 0; t < (int) THREAD_DEG_MAX; ++t)
        ok[t] = vs[t] != SENTINEL && (INITIAL || ld_vc<COH>(&vcmap[vs[t]]) == SENTINEL);
    u32 h = SENTINEL, tbb = 0;
    s32 maxw = 0;
#pragma unroll
    for (int t = 0; t < (int) THREAD_DEG_MAX; ++t) {
        if (!ok[t]) continue;
        const u32 v = vs[t];
        if (g.ew) {
            const s32 w = ws[t];
            if (maxw < w) {
                maxw = w;
                h = v;
                tbb = xorshift32(v + r);
                continue;
            }
            if (maxw != w) continue;
        }
        const u32 tb = xorshift32(v + r);
        if (tb >= tbb) {
            h = v;
            tbb = tb;
        }
    }
    return h;
}

// Group version of pick_thread (pick_neighbor_team :143-188 selects the same
// vertex): every thread of a warp or block keeps the argmax of its strided
// share of the row, then the group reduces.
struct PickLocal {
    bool found;
    s32 w;
    u32 tb;
    u32 h;
};

template<bool INITIAL, bool COH = false>
__device__ __forceinline__ PickLocal pick_local(const DGraph &g, const u32 *vcmap, u32 u, u32 seed, u32 tid,
                                                u32 nthreads) {
    const u32 r = xorshift32(u ^ seed);
    const u64 beg = g.rowptr[u];
    const u32 len = g.rowlen[u];
    PickLocal p{false, 0, 0, SENTINEL};
    // four entries per thread are loaded and their match state gathered
    // before they are compared (entries are visited in the same order)
    for (u32 t0 = tid; t0 < len; t0 += 4 * nthreads) {
        u32 vs[4];
        s32 ws[4];
        bool ok[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const u32 t = t0 + j * nthreads;
            vs[j] = t < len ? g.adj[beg + t] : SENTINEL;
            ws[j] = (t < len && g.ew) ? g.ew[beg + t] : 0;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            ok[j] = vs[j] != SENTINEL && (INITIAL || ld_vc<COH>(&vcmap[vs[j]]) == SENTINEL);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (!ok[j]) continue;
            const u32 tb = xorshift32(vs[j] + r);
            if (!p.found || ws[j] > p.w || (ws[j] == p.w && tb >= p.tb)) p = PickLocal{true, ws[j], tb, vs[j]};
        }
    }
    return p;
}

// Warp argmax of (w, tb); all lanes receive the winner (or an empty pick).
__device__ __forceinline__ PickLocal pick_reduce_warp(PickLocal p) {
    const s32 wbest = __reduce_max_sync(FULL, p.found ? p.w : INT32_MIN);
    if (wbest == INT32_MIN) return PickLocal{false, 0, 0, SENTINEL};
    const bool elig = p.found && p.w == wbest;
    const u32 tbest = __reduce_max_sync(FULL, elig ? p.tb : 0u);
    const unsigned win = __ballot_sync(FULL, elig && p.tb == tbest);
    return PickLocal{true, wbest, tbest, __shfl_sync(FULL, p.h, __ffs(win) - 1)};
}

template<bool INITIAL, bool COH = false>
__device__ __forceinline__ u32 pick_warp(const DGraph &g, const u32 *vcmap, u32 u, u32 seed) {
    return pick_reduce_warp(pick_local<INITIAL, COH>(g, vcmap, u, seed, lane_id(), 32)).h;
}

// Block argmax: warp winners go through shared memory to thread 0.
template<bool INITIAL, bool COH = false>
__device__ __forceinline__ u32 pick_block(const DGraph &g, const u32 *vcmap, u32 u, u32 seed, PickLocal *sm) {
    PickLocal p = pick_reduce_warp(pick_local<INITIAL, COH>(g, vcmap, u, seed, threadIdx.x, blockDim.x));
    if (lane_id() == 0) sm[warp_in_block()] = p;
    __syncthreads();
    u32 h = SENTINEL;
    if (threadIdx.x == 0) {
        PickLocal best{false, 0, 0, SENTINEL};
        for (u32 w = 0; w < (blockDim.x >> 5); ++w) {
            const PickLocal q = sm[w];
            if (q.found && (!best.found || q.w > best.w || (q.w == best.w && q.tb > best.tb))) best = q;
        }
        h = best.h;
    }
    __syncthreads();
    return h;
}

constexpr u32 PICK_WARP_MAX = 4096;  // longer rows are picked by a whole block
constexpr int PICK_BLOCK = 512;

// Appends u to the warp list (tier 1) or block list (tier 2).
__device__ __forceinline__ void append_tier(int tier, u32 u, u32 *heavy, u32 *heavy_cnt, u32 *huge, u32 *huge_cnt) {
    const u32 s1 = warp_append(heavy_cnt, tier == 1);
    if (tier == 1) heavy[s1] = u;
    const u32 s2 = warp_append(huge_cnt, tier == 2);
    if (tier == 2) huge[s2] = u;
}

__device__ __forceinline__ int pick_tier(u32 len) {
    return len <= THREAD_DEG_MAX ? 0 : (len <= PICK_WARP_MAX ? 1 : 2);
}

__global__ void k_match_init(DGraph g, u32 *vcmap, u32 *hn, u32 seed, u32 *heavy, u32 *heavy_cnt, u32 *huge,
                             u32 *huge_cnt) {
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < g.n; base += stride) {
        const u32 u = (u32) (base + threadIdx.x);
        int tier = 0;
        if (u < g.n) {
            vcmap[u] = SENTINEL;
            const u32 len = g.rowlen[u];
            if (!g.ew) {
                // initial_pick_uniform two_hop_matching.h:279-284
                hn[u] = len ? g.adj[g.rowptr[u] + (xorshift32(u ^ seed) % len)] : SENTINEL;
            } else {
                tier = pick_tier(len);
                hn[u] = tier == 0 ? pick_thread<true>(g, vcmap, u, seed) : SENTINEL;
            }
        }
        append_tier(tier, u, heavy, heavy_cnt, huge, huge_cnt);
    }
}

template<bool INITIAL>
__global__ void k_pick_heavy(DGraph g, const u32 *vcmap, u32 *hn, u32 seed, const u32 *list, const u32 *cnt) {
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    const u32 c = *cnt;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < c; i += warps) {
        const u32 u = list[i];
        const u32 h = pick_warp<INITIAL>(g, vcmap, u, seed);
        if (lane_id() == 0) hn[u] = h;
    }
}

template<bool INITIAL>
__global__ void __launch_bounds__(PICK_BLOCK) k_pick_huge(DGraph g, const u32 *vcmap, u32 *hn, u32 seed,
                                                          const u32 *list, const u32 *cnt) {
    __shared__ PickLocal sm[32];
    const u32 c = *cnt;
    for (u32 i = blockIdx.x; i < c; i += gridDim.x) {
        const u32 u = list[i];
        const u32 h = pick_block<INITIAL>(g, vcmap, u, seed, sm);
        if (threadIdx.x == 0) hn[u] = h;
    }
}

__device__ __forceinline__ bool commit_cond(u32 u, u32 v, u32 r) {
    return r > 0 ? (murmur3_u32(u + r) < murmur3_u32(v + r)) : (u < v);
}

// commit_p1 two_hop_matching.h:313-319: mark receivers.
__global__ void k_mark(const u32 *list, u32 cnt, const u32 *hn, u32 *vcmap, u32 r) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const u32 u = list[i];
        const u32 v = hn[u];
        if (v == SENTINEL || vcmap[u] != SENTINEL) continue;
        if (!commit_cond(u, v, r)) vcmap[u] = SENTINEL - 1;
    }
}

// commit_p2 two_hop_matching.h:320-327, deterministic: every proposer whose
// target is a receiver offers itself; the smallest offer of the current epoch
// wins (tags decrease with the epoch so stale offers lose).
__global__ void k_claim(const u32 *list, u32 cnt, const u32 *hn, const u32 *vcmap, unsigned long long *claim,
                        u32 tag) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const u32 u = list[i];
        const u32 v = hn[u];
        if (v == SENTINEL || vcmap[u] != SENTINEL) continue;
        if (vcmap[v] == SENTINEL - 1) atomicMin(&claim[v], ((unsigned long long) tag << 32) | u);
    }
}

// Resolves one sub-round (each thread writes only its own vcmap entry: the
// CAS winner pair of p2 and the reset of p3, :320-332) and marks the
// receivers of the next sub-round when next_r >= 0.
__global__ void k_resolve(const u32 *list, u32 cnt, const u32 *hn, u32 *vcmap, const unsigned long long *claim,
                          u32 tag, int next_r) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const u32 u = list[i];
        u32 s = vcmap[u];
        const u32 v = hn[u];
        if (s == SENTINEL - 1) {
            const unsigned long long c = claim[u];
            if ((u32) (c >> 32) == tag) {
                const u32 p = (u32) c;
                s = u < p ? u : p;
            } else {
                s = SENTINEL;
            }
        } else if (s == SENTINEL && v != SENTINEL) {
            const unsigned long long c = claim[v];
            if ((u32) (c >> 32) == tag && (u32) c == u) s = u < v ? u : v;
        }
        if (next_r >= 0 && s == SENTINEL && v != SENTINEL && !commit_cond(u, v, (u32) next_r)) s = SENTINEL - 1;
        vcmap[u] = s;
    }
}

// Re-pick for list vertices whose target got matched (:336-374).
__global__ void k_repick(DGraph g, const u32 *list, u32 cnt, const u32 *vcmap, u32 *hn, u32 seed, u32 *heavy,
                         u32 *heavy_cnt, u32 *huge, u32 *huge_cnt) {
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < cnt; base += stride) {
        const u64 i = base + threadIdx.x;
        int tier = 0;
        u32 u = 0;
        if (i < cnt) {
            u = list[i];
            const u32 h = hn[u];
            if (vcmap[u] == SENTINEL && h != SENTINEL && vcmap[h] != SENTINEL) {
                tier = pick_tier(g.rowlen[u]);
                if (tier == 0) hn[u] = pick_thread<false>(g, vcmap, u, seed);
            }
        }
        append_tier(tier, u, heavy, heavy_cnt, huge, huge_cnt);
    }
}

// The whole matching loop of one level in one cooperative launch (grid-wide
// barriers between the phases the per-phase kernels above run separately):
// per round the receiver marks, four commit sub-rounds of claim and resolve,
// the re-pick (thread, warp and block tiers) and the compaction of the
// still-unmatched list. Data written by other blocks is read through L2
// (__ldcg), never from L1. The list order does not affect the result (claims
// keep the smallest proposer, picks are per vertex), so the compaction
// appends atomically. ctr: [0] next list length, [1] warp-tier picks, [2]
// block-tier picks, [3] rounds run, [4] error.
constexpr u32 MATCH_MAX_ROUNDS = 100000;
// upper bound of Tunables::match_coop_max_n (the grid of the fused loop holds
// every list entry in a few grid-stride passes)
constexpr u32 MATCH_COOP_MAX_N = 1u << 20;

__global__ void __launch_bounds__(PICK_BLOCK) k_match_loop(DGraph g, u32 *vcmap, u32 *hn, u32 *list, u32 *list2,
                                                           u32 cnt, unsigned long long *claim, u32 *heavy, u32 *huge,
                                                           u32 *ctr, u32 seed, u32 *bar, u32 *err) {
    __shared__ PickLocal sm[32];
    const u64 gtid = (u64) blockIdx.x * blockDim.x + threadIdx.x;
    const u64 gsize = (u64) gridDim.x * blockDim.x;
    const u32 warps = (u32) (gsize >> 5);
    const u32 gwarp = (u32) (gtid >> 5);
    u32 epoch = 0;
    for (u32 round = 0; cnt > 0; ++round) {
        if (round >= MATCH_MAX_ROUNDS) {
            if (gtid == 0) ctr[4] = 1;
            break;
        }
        const u32 round_seed = seed ^ (round * 0x9e3779b1u);
        if (gtid == 0) {
            ctr[0] = 0;
            ctr[1] = 0;
            ctr[2] = 0;
        }
        // commit_p1: receivers of sub-round 0
        for (u64 i = gtid; i < cnt; i += gsize) {
            const u32 u = list[i];
            const u32 v = __ldcg(&hn[u]);
            if (v == SENTINEL || __ldcg(&vcmap[u]) != SENTINEL) continue;
            if (!commit_cond(u, v, 0)) vcmap[u] = SENTINEL - 1;
        }
        if (!grid_barrier(bar, err)) return;
        for (u32 r = 0; r < 4; ++r) {
            ++epoch;
            const u32 tag = 0xFFFFFFFFu - epoch;
            for (u64 i = gtid; i < cnt; i += gsize) {
                const u32 u = list[i];
                const u32 v = __ldcg(&hn[u]);
                if (v == SENTINEL || __ldcg(&vcmap[u]) != SENTINEL) continue;
                if (__ldcg(&vcmap[v]) == SENTINEL - 1) atomicMin(&claim[v], ((unsigned long long) tag << 32) | u);
            }
            if (!grid_barrier(bar, err)) return;
            const int next_r = r < 3 ? (int) r + 1 : -1;
            for (u64 i = gtid; i < cnt; i += gsize) {
                const u32 u = list[i];
                u32 st = __ldcg(&vcmap[u]);
                const u32 v = __ldcg(&hn[u]);
                if (st == SENTINEL - 1) {
                    const unsigned long long c = __ldcg(&claim[u]);
                    st = (u32) (c >> 32) == tag ? (u < (u32) c ? u : (u32) c) : SENTINEL;
                } else if (st == SENTINEL && v != SENTINEL) {
                    const unsigned long long c = __ldcg(&claim[v]);
                    if ((u32) (c >> 32) == tag && (u32) c == u) st = u < v ? u : v;
                }
                if (next_r >= 0 && st == SENTINEL && v != SENTINEL && !commit_cond(u, v, (u32) next_r))
                    st = SENTINEL - 1;
                vcmap[u] = st;
            }
            if (!grid_barrier(bar, err)) return;
        }
        // re-pick for vertices whose target got matched
        for (u64 base = (u64) blockIdx.x * blockDim.x; base < cnt; base += gsize) {
            const u64 i = base + threadIdx.x;
            int tier = 0;
            u32 u = 0;
            if (i < cnt) {
                u = list[i];
                const u32 h = __ldcg(&hn[u]);
                if (__ldcg(&vcmap[u]) == SENTINEL && h != SENTINEL && __ldcg(&vcmap[h]) != SENTINEL) {
                    tier = pick_tier(g.rowlen[u]);
                    if (tier == 0) hn[u] = pick_thread<false, true>(g, vcmap, u, round_seed);
                }
            }
            append_tier(tier, u, heavy, &ctr[1], huge, &ctr[2]);
        }
        if (!grid_barrier(bar, err)) return;
        const u32 nh = __ldcg(&ctr[1]), ng = __ldcg(&ctr[2]);
        for (u32 i = gwarp; i < nh; i += warps) {
            const u32 u = heavy[i];
            const u32 h = pick_warp<false, true>(g, vcmap, u, round_seed);
            if (lane_id() == 0) hn[u] = h;
        }
        for (u32 i = blockIdx.x; i < ng; i += gridDim.x) {
            const u32 u = huge[i];
            const u32 h = pick_block<false, true>(g, vcmap, u, round_seed, sm);
            if (threadIdx.x == 0) hn[u] = h;
        }
        if (!grid_barrier(bar, err)) return;
        // still unmatched with a target: next round's list
        for (u64 i = gtid; i < cnt; i += gsize) {
            const u32 u = list[i];
            if (__ldcg(&vcmap[u]) == SENTINEL && __ldcg(&hn[u]) != SENTINEL) list2[atomicAdd(&ctr[0], 1u)] = u;
        }
        if (!grid_barrier(bar, err)) return;
        cnt = __ldcg(&ctr[0]);
        u32 *t = list;
        list = list2;
        list2 = t;
        if (gtid == 0) ctr[3] = round + 1;
        if (!grid_barrier(bar, err)) return;  // every thread has read ctr[0] before the next round clears it
    }
}

__global__ void k_count_unmapped(const u32 *vcmap, u32 n, u32 *out) {
    u32 c = 0;
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) c += vcmap[u] == SENTINEL;
    c = warp_sum<u32>(c);
    if (lane_id() == 0 && c) atomicAdd(out, c);
}

// Twin digest: sum over neighbours of (h + h^2), h = pod_hash(v) in u64
// (:454-466). One warp per candidate.
__global__ void k_twin_digest(DGraph g, const u32 *cands, const u32 *cnt, unsigned long long *dig) {
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    const u32 c = *cnt;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < c; i += warps) {
        const u32 u = cands[i];
        const u64 beg = g.rowptr[u];
        const u32 len = g.rowlen[u];
        unsigned long long s = 0;
        for (u32 t = lane_id(); t < len; t += 32) {
            unsigned long long y = murmur3_u32(g.adj[beg + t]);
            s += y * y + y;
        }
        s = warp_sum<unsigned long long>(s);
        if (lane_id() == 0) dig[i] = s;
    }
}

// Relative digest: neighbour of minimum degree, then maximum edge weight,
// then lowest id (:545-565 with the id tie rule). One warp per candidate.
__global__ void k_rel_digest(DGraph g, const u32 *cands, const u32 *cnt, u32 *dig) {
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    const u32 c = *cnt;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < c; i += warps) {
        const u32 u = cands[i];
        const u64 beg = g.rowptr[u];
        const u32 len = g.rowlen[u];
        unsigned long long best = ~0ull;
        u32 bv = SENTINEL;
        for (u32 t = lane_id(); t < len; t += 32) {
            const u32 v = g.adj[beg + t];
            const u32 d = g.rowlen[v];
            const s32 w = g_ew(g, beg + t);
            const unsigned long long key = ((unsigned long long) d << 32) | (u32) (INT32_MAX - w);
            if (key < best || (key == best && v < bv)) {
                best = key;
                bv = v;
            }
        }
        unsigned long long kmin = best;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long y = __shfl_xor_sync(FULL, kmin, o);
            kmin = y < kmin ? y : kmin;
        }
        const u32 vmin = __reduce_min_sync(FULL, best == kmin ? bv : SENTINEL);
        if (lane_id() == 0) dig[i] = vmin;
    }
}

// Pairs sorted candidates: ranks 2j and 2j+1 within a digest group match.
__global__ void k_pair(const u32 *cands, const u32 *gid, const u32 *gstart, u32 cnt, u32 *vcmap) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const u32 rank = i - gstart[gid[i]];
        if (rank & 1u) {
            const u32 a = cands[i - 1], b = cands[i];
            const u32 cv = a < b ? a : b;
            vcmap[a] = cv;
            vcmap[b] = cv;
        }
    }
}

__global__ void k_singletons(u32 *vcmap, u32 n) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
        if (vcmap[u] == SENTINEL) vcmap[u] = u;
}

__global__ void k_final_map(const u32 *vcmap, const u32 *rank, u32 *mapping, u32 n) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
        mapping[u] = rank[vcmap[u]];
}

// matchHash (:205-253) under the grouping rule: stable sort by digest, then
// pair neighbours in each group.
template<typename K>
void pair_by_digest(Ctx &ctx, u32 *cands, K *keys, u32 cnt, u32 *vcmap) {
    if (cnt < 2) return;
    ScratchScope ss(ctx.arena);
    radix_sort_pairs<K>(ctx, keys, cands, cnt, 0, 8 * (int) sizeof(K));
    u32 *gid = ctx.balloc<u32>(cnt);
    u32 *gstart = ctx.balloc<u32>(cnt);
    device_scan<u32>(
        ctx, cnt, [=] __device__(u64 i) -> u32 { return (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u; },
        [=] __device__(u64 i, u32 p, u32 v) {
            gid[i] = p + v - 1;
            if (v) gstart[p] = (u32) i;
        },
        (u32 *) nullptr);
    k_pair<<<ctx.grid(cnt, BLOCK), BLOCK, 0, ctx.stream>>>(cands, gid, gstart, cnt, vcmap); note_launch();
    HP_LAUNCH_CHECK();
}

u32 count_unmapped(Ctx &ctx, const u32 *vcmap, u32 n) {
    ctx.zero_counters();
    k_count_unmapped<<<ctx.grid(n, BLOCK), BLOCK, 0, ctx.stream>>>(vcmap, n, &ctx.d_status->cnt[1]); note_launch();
    HP_LAUNCH_CHECK();
    return ctx.read_status().cnt[1];
}

} // namespace

// One matching of g into mapping; allow_coop selects the single cooperative
// launch for the round loop of small levels.
static u32 match_graph_impl(Ctx &ctx, const DGraph &g, u32 *mapping, bool allow_coop) {
    const u32 n = g.n;
    ScratchScope ss(ctx.arena);
    u32 *vcmap = ctx.balloc<u32>(n);
    u32 *hn = ctx.balloc<u32>(n);
    u32 *list = ctx.balloc<u32>(n);
    u32 *list2 = ctx.balloc<u32>(n);
    u32 *heavy = ctx.balloc<u32>(n);
    u32 *huge = ctx.balloc<u32>(n);
    unsigned long long *claim = ctx.balloc<unsigned long long>(n);
    HP_CUDA(cudaMemsetAsync(claim, 0xFF, sizeof(unsigned long long) * n, ctx.stream));
    u32 *heavy_cnt = &ctx.d_status->cnt[2];
    u32 *huge_cnt = &ctx.d_status->cnt[3];
    const u32 hgrid = (u32) ctx.sm_count * 4;
    const u32 seed = MATCH_SEED;
    const u32 wgrid = ctx.grid((u64) n * 32, BLOCK);

    ctx.zero_counters();
    k_match_init<<<ctx.grid(n, BLOCK), BLOCK, 0, ctx.stream>>>(g, vcmap, hn, seed, heavy, heavy_cnt, huge, huge_cnt); note_launch();
    k_pick_heavy<true><<<wgrid, BLOCK, 0, ctx.stream>>>(g, vcmap, hn, seed, heavy, heavy_cnt); note_launch();
    k_pick_huge<true><<<hgrid, PICK_BLOCK, 0, ctx.stream>>>(g, vcmap, hn, seed, huge, huge_cnt); note_launch();
    device_iota(ctx, list, n);
    HP_LAUNCH_CHECK();

    // the round loop: on small levels (launch and synchronisation cost
    // dominates) one cooperative launch, else one launch per phase with a
    // host read per round (large levels need more threads than fit at once)
    int per_sm = 0;
    if (allow_coop && n <= std::min<u32>(ctx.tune.match_coop_max_n, MATCH_COOP_MAX_N) &&
        g.m <= ctx.tune.match_coop_max_m)
        HP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_match_loop, PICK_BLOCK, 0));
    if (per_sm > 0) {
        u32 *ctr = &ctx.d_status->cnt[8];  // 5 words, then the barrier's 2 words; cleared below
        u32 *bar = &ctx.d_status->cnt[13];
        u32 *err = &ctx.d_status->err;
        HP_CUDA(cudaMemsetAsync(ctr, 0, 7 * sizeof(u32), ctx.stream));
        const u32 want = (u32) std::max<u64>(1, ((u64) n + PICK_BLOCK - 1) / PICK_BLOCK);
        const u32 grid = std::min<u32>(want, (u32) (per_sm * ctx.sm_count));
        DGraph gg = g;
        u32 *pl = list, *pl2 = list2;
        u32 cnt0 = n;
        u32 sd = seed;
        void *args[] = {&gg, &vcmap, &hn, &pl, &pl2, &cnt0, &claim, &heavy, &huge, &ctr, &sd, &bar, &err};
        // cooperative budget (grid blocks), held until the kernel has completed
        CoopGuard coop(ctx.device, ctx.stream, grid, (u32) ctx.sm_count);
        HP_CUDA(cudaLaunchCooperativeKernel((const void *) k_match_loop, dim3(grid), dim3(PICK_BLOCK), args, 0,
                                            ctx.stream));
        note_launch();
        const DevStatus &st = ctx.read_status();
        if (st.err & DEV_ERR_SPIN) throw CoopSpin{};
        if (st.cnt[12]) throw HpError{HP_ERR_DEVICE, "matching did not converge"};
    } else {
        u32 cnt = n;
        u32 round = 0, epoch = 0;
        while (cnt > 0) {
            const u32 round_seed = seed ^ (round * 0x9e3779b1u);
            const u32 grid = ctx.grid(cnt, BLOCK);
            k_mark<<<grid, BLOCK, 0, ctx.stream>>>(list, cnt, hn, vcmap, 0); note_launch();
            for (u32 r = 0; r < 4; ++r) {
                ++epoch;
                const u32 tag = 0xFFFFFFFFu - epoch;
                k_claim<<<grid, BLOCK, 0, ctx.stream>>>(list, cnt, hn, vcmap, claim, tag); note_launch();
                k_resolve<<<grid, BLOCK, 0, ctx.stream>>>(list, cnt, hn, vcmap, claim, tag, r < 3 ? (int) r + 1 : -1);
                note_launch();
            }
            ctx.zero_counters();
            k_repick<<<grid, BLOCK, 0, ctx.stream>>>(g, list, cnt, vcmap, hn, round_seed, heavy, heavy_cnt, huge,
                                                     huge_cnt); note_launch();
            k_pick_heavy<false><<<wgrid, BLOCK, 0, ctx.stream>>>(g, vcmap, hn, round_seed, heavy, heavy_cnt);
            note_launch();
            k_pick_huge<false><<<hgrid, PICK_BLOCK, 0, ctx.stream>>>(g, vcmap, hn, round_seed, huge, huge_cnt);
            note_launch();
            HP_LAUNCH_CHECK();
            const u32 *l = list;
            device_select(
                ctx, cnt, [=] __device__(u64 i) -> bool {
                    const u32 u = l[i];
                    return vcmap[u] == SENTINEL && hn[u] != SENTINEL;
                },
                [=] __device__(u64 i) -> u32 { return l[i]; }, list2, &ctx.d_status->cnt[0]);
            cnt = ctx.read_status().cnt[0];
            std::swap(list, list2);
            ++round;
            if (round > 100000) throw HpError{HP_ERR_DEVICE, "matching did not converge"};
        }
    }

    u32 unmapped = count_unmapped(ctx, vcmap, n);
    // leaf matching (:395-425)
    if ((u64) unmapped * 4 > (u64) n) {
        ScratchScope s2(ctx.arena);
        u32 *cands = ctx.balloc<u32>(n);
        u32 *dig = ctx.balloc<u32>(n);
        ctx.zero_counters();
        const DGraph gg = g;
        device_scan<u32>(
            ctx, n, [=] __device__(u64 i) -> u32 { return (vcmap[i] == SENTINEL && gg.rowlen[i] == 1) ? 1u : 0u; },
            [=] __device__(u64 i, u32 p, u32 v) {
                if (v) {
                    cands[p] = (u32) i;
                    dig[p] = gg.adj[gg.rowptr[i]];
                }
            },
            &ctx.d_status->cnt[0]);
        u32 c = ctx.read_status().cnt[0];
        pair_by_digest<u32>(ctx, cands, dig, c, vcmap);
        unmapped = count_unmapped(ctx, vcmap, n);
    }
    // twin matching (:427-524)
    if ((u64) unmapped * 4 > (u64) n) {
        ScratchScope s2(ctx.arena);
        u32 *cands = ctx.balloc<u32>(n);
        unsigned long long *dig = ctx.balloc<unsigned long long>(n);
        ctx.zero_counters();
        device_select(
            ctx, n, [=] __device__(u64 i) -> bool { return vcmap[i] == SENTINEL; },
            [=] __device__(u64 i) -> u32 { return (u32) i; }, cands, &ctx.d_status->cnt[0]);
        k_twin_digest<<<wgrid, BLOCK, 0, ctx.stream>>>(g, cands, &ctx.d_status->cnt[0], dig); note_launch();
        HP_LAUNCH_CHECK();
        u32 c = ctx.read_status().cnt[0];
        pair_by_digest<unsigned long long>(ctx, cands, dig, c, vcmap);
        unmapped = count_unmapped(ctx, vcmap, n);
    }
    // relative matching (:526-571)
    if ((u64) unmapped * 4 > (u64) n) {
        ScratchScope s2(ctx.arena);
        u32 *cands = ctx.balloc<u32>(n);
        u32 *dig = ctx.balloc<u32>(n);
        ctx.zero_counters();
        device_select(
            ctx, n, [=] __device__(u64 i) -> bool { return vcmap[i] == SENTINEL; },
            [=] __device__(u64 i) -> u32 { return (u32) i; }, cands, &ctx.d_status->cnt[0]);
        k_rel_digest<<<wgrid, BLOCK, 0, ctx.stream>>>(g, cands, &ctx.d_status->cnt[0], dig); note_launch();
        HP_LAUNCH_CHECK();
        u32 c = ctx.read_status().cnt[0];
        pair_by_digest<u32>(ctx, cands, dig, c, vcmap);
    }
    // coarse ids (:611-641)
    k_singletons<<<ctx.grid(n, BLOCK), BLOCK, 0, ctx.stream>>>(vcmap, n); note_launch();
    HP_LAUNCH_CHECK();
    u32 *rank = list2;
    ctx.zero_counters();
    device_scan<u32>(
        ctx, n, [=] __device__(u64 i) -> u32 { return vcmap[i] == (u32) i ? 1u : 0u; },
        [=] __device__(u64 i, u32 p, u32 v) {
            if (v) rank[i] = p;
        },
        &ctx.d_status->cnt[0]);
    k_final_map<<<ctx.grid(n, BLOCK), BLOCK, 0, ctx.stream>>>(vcmap, rank, mapping, n); note_launch();
    HP_LAUNCH_CHECK();
    return ctx.read_status().cnt[0];
}

u32 match_graph(Ctx &ctx, const DGraph &g, u32 *mapping) {
    if (g.n == 0) return 0;
    ProfScope prof_all(ctx, "match");
    try {
        return match_graph_impl(ctx, g, mapping, true);
    } catch (const CoopSpin &) {
        // the cooperative round loop gave up at a grid barrier: matching is
        // a deterministic function of the graph, so redoing it from the
        // start on the per-phase path gives the same mapping
        ctx.zero_status();
        return match_graph_impl(ctx, g, mapping, false);
    }
}

} // namespace hp
