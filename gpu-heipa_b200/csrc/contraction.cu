// Graph contraction (src/datastructures/graph.h:127-390) as one aggregation
// pass over the member rows of every coarse vertex. Coarse rows are
// aggregated in registers (row capacity <= 16), a per-warp shared-memory hash
// table (<= 256), a per-block shared-memory table (<= 4096) or a global hash
// table (larger), and written straight into the padded coarse CSR at the
// capacity offsets.
#include <algorithm>
#include <vector>

#include "coarsen.cuh"
#include "prims.cuh"

namespace hp {
namespace {

constexpr u32 EMPTY = 0xFFFFFFFFu;
constexpr u32 C_THREAD_MAX = 16;
constexpr u32 C_WARP_MAX = 256;
constexpr u32 C_WARP_BITS = 9;  // 512 slots per warp
constexpr u32 C_WARP_SLOTS = 1u << C_WARP_BITS;
constexpr u32 C_BLOCK_MAX = 4096;
constexpr u32 C_BLOCK_BITS = 13;  // 8192 slots per block
constexpr u32 C_BLOCK_SLOTS = 1u << C_BLOCK_BITS;
constexpr u32 C_BLOCK_SMALL_MAX = 1024;  // block tier with a 2048-slot table (16 KB) up to this capacity
constexpr u32 C_BLOCK_SMALL_BITS = 11;
constexpr int C_WARP_BLOCK = 128;  // 4 warps per block for the warp kernel
constexpr int C_HUGE_BLOCK = 1024;
constexpr int C_ST_BLOCK_LARGE = 3;  // status slot: clusters of the large block tier
constexpr int C_ST_HUGE_TICKET = 4;  // status slot: next huge cluster to be taken by a block

__device__ __forceinline__ u32 hslot(u32 key, u32 bits) { return (key * 2654435761u) >> (32 - bits); }

__global__ void k_cluster_stats(DGraph g, const u32 *map, u32 *cnt, u32 *capsum, s32 *cw) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < g.n; u += gridDim.x * blockDim.x) {
        const u32 c = map[u];
        atomicAdd(&cnt[c], 1u);
        atomicAdd(&capsum[c], g.rowlen[u]);
        atomicAdd(&cw[c], g_vw(g, u));
    }
}

__global__ void k_fill_members(const u32 *map, u32 n, u32 *cursor, u32 *mlist) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        const u32 pos = atomicAdd(&cursor[map[u]], 1u);
        mlist[pos] = u;
    }
}

struct CArgs {
    DGraph g;         // fine graph
    const u32 *map;   // fine -> coarse
    const u32 *moff;  // member offsets (n_c + 1)
    const u32 *mlist; // members
    DGraph c;         // coarse graph (rowptr, rowlen, adj, ew written here)
    u32 *err;
    unsigned long long *m_out;
};

// Thread-per-coarse-vertex aggregation in registers for capacities <= 16;
// larger coarse vertices are appended to the warp / block / huge lists.
struct TierLists {
    u32 *wl, *wcnt;    // warp tier
    u32 *bl, *bcnt;    // block tier, 2048-slot tables
    u32 *bl2, *b2cnt;  // block tier, 8192-slot tables
    u32 *hl, *hcnt;    // huge clusters
    u32 *hcap;         // huge clusters: row capacity (entries of the member rows)
    u32 *hoffc;        // per coarse vertex: offset of its global table (huge clusters)
    unsigned long long *hbump;  // global table slots handed out
};

__global__ void k_contract_small(CArgs a, TierLists L) {
    const u64 stride = (u64) gridDim.x * blockDim.x;
    unsigned long long msum = 0;
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < a.c.n; base += stride) {
        const u32 c = (u32) (base + threadIdx.x);
        u32 cls = 0;  // 0 none, 1 warp, 2 block, 3 huge
        u32 cap = 0;
        if (c < a.c.n) {
            cap = a.c.rowptr[c + 1] - a.c.rowptr[c];
            const u32 m0 = a.moff[c], mc = a.moff[c + 1] - m0;
            if (cap <= C_THREAD_MAX && mc <= 2) {
                // matched clusters have one or two members: the (at most 16)
                // entries of their rows are loaded first, then all coarse ids
                // are gathered at once, then aggregated in registers (larger
                // clusters of a caller-given mapping go to the warp tier)
                const u32 u0 = a.mlist[m0];
                const u32 u1 = mc > 1 ? a.mlist[m0 + 1] : u0;
                const u64 b0 = a.g.rowptr[u0], b1 = a.g.rowptr[u1];
                const u32 l0 = a.g.rowlen[u0], l1 = mc > 1 ? a.g.rowlen[u1] : 0u;
                u32 keys[C_THREAD_MAX];
                s32 ws[C_THREAD_MAX];
#pragma unroll
                for (int s = 0; s < (int) C_THREAD_MAX; ++s) {
                    const u32 t = (u32) s;
                    keys[s] = EMPTY;
                    ws[s] = 0;
                    if (t < l0 + l1) {
                        const u64 e = t < l0 ? b0 + t : b1 + (t - l0);
                        keys[s] = __ldg(&a.g.adj[e]);
                        ws[s] = g_ew(a.g, e);
                    }
                }
#pragma unroll
                for (int s = 0; s < (int) C_THREAD_MAX; ++s)
                    if (keys[s] != EMPTY) {
                        keys[s] = __ldg(&a.map[keys[s]]);
                        if (keys[s] == c) keys[s] = EMPTY;  // self loop
                    }
                // merge equal coarse ids into their first occurrence
#pragma unroll
                for (int s = 1; s < (int) C_THREAD_MAX; ++s) {
#pragma unroll
                    for (int t = 0; t < s; ++t)
                        if (keys[s] != EMPTY && keys[t] == keys[s]) {
                            ws[t] = wadd(ws[t], ws[s]);
                            keys[s] = EMPTY;
                        }
                }
                u64 pos = a.c.rowptr[c];
                u32 cntu = 0;
#pragma unroll
                for (int s = 0; s < (int) C_THREAD_MAX; ++s)
                    if (keys[s] != EMPTY) {
                        a.c.adj[pos + cntu] = keys[s];
                        a.c.ew[pos + cntu] = ws[s];
                        ++cntu;
                    }
                a.c.rowlen[c] = cntu;
                msum += cntu;
            } else if (cap <= C_WARP_MAX) {
                cls = 1;  // includes small clusters of more than two members
            } else if (cap <= C_BLOCK_SMALL_MAX) {
                cls = 2;
            } else if (cap <= C_BLOCK_MAX) {
                cls = 4;
            } else {
                cls = 3;
                L.hoffc[c] = (u32) atomicAdd(L.hbump, (unsigned long long) (2 * cap));
            }
        }
        u32 s1 = warp_append(L.wcnt, cls == 1);
        if (cls == 1) L.wl[s1] = c;
        u32 s2 = warp_append(L.bcnt, cls == 2);
        if (cls == 2) L.bl[s2] = c;
        u32 s4 = warp_append(L.b2cnt, cls == 4);
        if (cls == 4) L.bl2[s4] = c;
        u32 s3 = warp_append(L.hcnt, cls == 3);
        if (cls == 3) {
            L.hl[s3] = c;
            L.hcap[s3] = cap;
        }
    }
    msum = warp_sum<unsigned long long>(msum);
    if (lane_id() == 0 && msum) atomicAdd(a.m_out, msum);
}

// Calls insert(cv, w) for every entry of the member rows of cluster c whose
// coarse neighbour cv differs from c; entries are strided over a group of
// `nt` threads starting at `tid` across the concatenated member rows (one or
// two members), four entries per thread loaded before they are inserted.
// Loads four entries t0, t0 + nt, ... of the concatenated rows [b0, b0 + l0)
// and [b1, b1 + l1) (total = l0 + l1); empty slots get EMPTY.
__device__ __forceinline__ void load_pair_entries(const CArgs &a, u64 b0, u32 l0, u64 b1, u32 total, u32 t0, u32 nt,
                                                  u32 (&cv)[4], s32 (&w)[4]) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const u32 t = t0 + j * nt;
        cv[j] = EMPTY;
        w[j] = 0;
        if (t < total) {
            const u64 e = t < l0 ? b0 + t : b1 + (t - l0);
            cv[j] = __ldg(&a.g.adj[e]);
            w[j] = g_ew(a.g, e);
        }
    }
}

// Calls insert(cv, w) for every entry of the member rows of cluster c whose
// coarse neighbour cv differs from c; entries are strided over a group of
// `nt` threads starting at `tid` across the concatenated member rows (one or
// two members at a time), four entries per thread loaded before their coarse
// ids are gathered, and the next four loaded while those are gathered and
// inserted.
template<typename Insert>
__device__ __forceinline__ void for_cluster_entries(const CArgs &a, u32 c, u32 tid, u32 nt, Insert insert) {
    const u32 m0 = a.moff[c], mc = a.moff[c + 1] - m0;
    for (u32 mi = 0; mi < mc; mi += 2) {
        const u32 u0 = a.mlist[m0 + mi];
        const u32 u1 = mi + 1 < mc ? a.mlist[m0 + mi + 1] : u0;
        const u64 b0 = a.g.rowptr[u0], b1 = a.g.rowptr[u1];
        const u32 l0 = a.g.rowlen[u0], l1 = mi + 1 < mc ? a.g.rowlen[u1] : 0u;
        const u32 total = l0 + l1;
        u32 t0 = tid;
        if (t0 >= total) continue;
        u32 cv[4];
        s32 w[4];
        load_pair_entries(a, b0, l0, b1, total, t0, nt, cv, w);
        for (;;) {
            const u32 t1 = t0 + 4 * nt;
            u32 cvn[4];
            s32 wn[4];
            load_pair_entries(a, b0, l0, b1, total, t1, nt, cvn, wn);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (cv[j] != EMPTY) cv[j] = __ldg(&a.map[cv[j]]);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (cv[j] != EMPTY && cv[j] != c) insert(cv[j], w[j]);
            if (t1 >= total) break;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                cv[j] = cvn[j];
                w[j] = wn[j];
            }
            t0 = t1;
        }
    }
}

// Inserts (cv, w) into an open-addressing table with linear probing.
__device__ __forceinline__ bool table_insert(u32 *tk, s32 *tw, u32 mask, u32 h, u32 cv, s32 w) {
    for (u32 probe = 0; probe <= mask; ++probe) {
        const u32 prev = atomicCAS(&tk[h], EMPTY, cv);
        if (prev == EMPTY || prev == cv) {
            atomicAdd(&tw[h], w);
            return true;
        }
        h = (h + 1) & mask;
    }
    return false;
}

__global__ void __launch_bounds__(C_WARP_BLOCK) k_contract_warp(CArgs a, const u32 *wl, const u32 *wcnt) {
    __shared__ u32 tk_all[C_WARP_BLOCK / 32][C_WARP_SLOTS];
    __shared__ s32 tw_all[C_WARP_BLOCK / 32][C_WARP_SLOTS];
    u32 *tk = tk_all[warp_in_block()];
    s32 *tw = tw_all[warp_in_block()];
    const int lane = lane_id();
    for (u32 s = lane; s < C_WARP_SLOTS; s += 32) {
        tk[s] = EMPTY;
        tw[s] = 0;
    }
    __syncwarp();
    const u32 total = *wcnt;
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long msum = 0;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        const u32 c = wl[i];
        const u32 cap = a.c.rowptr[c + 1] - a.c.rowptr[c];
        u32 bits = 6;
        while ((1u << bits) < 2 * cap && bits < C_WARP_BITS) ++bits;
        const u32 tsz = 1u << bits;
        for_cluster_entries(a, c, (u32) lane, 32u, [&](u32 cv, s32 w) {
            if (!table_insert(tk, tw, tsz - 1, hslot(cv, bits), cv, w)) set_error(a.err, DEV_ERR_HASH_FULL);
        });
        __syncwarp();
        const u64 out = a.c.rowptr[c];
        u32 cntu = 0;
        for (u32 s0 = 0; s0 < tsz; s0 += 32) {
            const u32 s = s0 + lane;
            const u32 key = tk[s];
            const bool has = key != EMPTY;
            const unsigned mask = __ballot_sync(FULL, has);
            if (has) {
                const u32 p = cntu + __popc(mask & ((1u << lane) - 1u));
                a.c.adj[out + p] = key;
                a.c.ew[out + p] = tw[s];
                tk[s] = EMPTY;
                tw[s] = 0;
            }
            cntu += __popc(mask);
        }
        if (lane == 0) a.c.rowlen[c] = cntu;
        msum += cntu;
        __syncwarp();
    }
    if (lane == 0 && msum) atomicAdd(a.m_out, msum);
}

// Emits the non-empty slots of a block-wide table into the coarse row and
// resets them (thread t owns slots t, t + NT, ...).
__device__ __forceinline__ u32 block_emit(u32 *tk, s32 *tw, u32 slots, u64 out, u32 *adj, s32 *ew,
                                          u32 *smem_scan) {
    u32 cnt = 0;
    for (u32 s = threadIdx.x; s < slots; s += blockDim.x) cnt += tk[s] != EMPTY;
    u32 tot;
    u32 p = block_exclusive_scan<u32>(cnt, tot, smem_scan);
    for (u32 s = threadIdx.x; s < slots; s += blockDim.x) {
        const u32 key = tk[s];
        if (key != EMPTY) {
            adj[out + p] = key;
            ew[out + p] = tw[s];
            ++p;
            tk[s] = EMPTY;
            tw[s] = 0;
        }
    }
    return tot;
}

__global__ void __launch_bounds__(BLOCK) k_contract_block(CArgs a, const u32 *bl, const u32 *bcnt, u32 max_bits) {
    extern __shared__ u32 dsm[];
    const u32 slots = 1u << max_bits;
    u32 *tk = dsm;
    s32 *tw = (s32 *) (dsm + slots);
    __shared__ u32 scan_sm[32];
    for (u32 s = threadIdx.x; s < slots; s += blockDim.x) {
        tk[s] = EMPTY;
        tw[s] = 0;
    }
    __syncthreads();
    const u32 total = *bcnt;
    unsigned long long msum = 0;
    for (u32 i = blockIdx.x; i < total; i += gridDim.x) {
        const u32 c = bl[i];
        // table of the next power of two >= 2 * capacity (<= C_BLOCK_SLOTS)
        const u32 cap = a.c.rowptr[c + 1] - a.c.rowptr[c];
        u32 bits = 9;
        while ((1u << bits) < 2 * cap && bits < max_bits) ++bits;
        const u32 tsz = 1u << bits;
        for_cluster_entries(a, c, threadIdx.x, blockDim.x, [&](u32 cv, s32 w) {
            if (!table_insert(tk, tw, tsz - 1, hslot(cv, bits), cv, w)) set_error(a.err, DEV_ERR_HASH_FULL);
        });
        __syncthreads();
        const u32 cntu = block_emit(tk, tw, tsz, a.c.rowptr[c], a.c.adj, a.c.ew, scan_sm);
        if (threadIdx.x == 0) a.c.rowlen[c] = cntu;
        msum += cntu;
        __syncthreads();
    }
    if (threadIdx.x == 0 && msum) atomicAdd(a.m_out, msum);
}

__device__ __forceinline__ u32 range_hash(u32 key, u32 size) {
    return (u32) (((u64) (key * 2654435761u) * (u64) size) >> 32);
}

// One global hash table per huge cluster; a slot is (key, weight) in one
// 8-byte word pair, so an insert touches one cache line (the tables of the
// hub clusters of a large level do not fit in L2).
struct HugeSlot {
    u32 key;
    s32 w;
};

// Blocks take clusters from hl (largest first) through a ticket, so that no
// block is left with several large clusters while others are idle.
__global__ void __launch_bounds__(C_HUGE_BLOCK) k_contract_huge(CArgs a, const u32 *hl, const u32 *hcnt,
                                                               const u32 *hoff, HugeSlot *slots, u32 *ticket) {
    __shared__ u32 scan_sm[32];
    __shared__ u32 s_next;
    const u32 total = *hcnt;
    unsigned long long msum = 0;
    for (;;) {
        if (threadIdx.x == 0) s_next = atomicAdd(ticket, 1u);
        __syncthreads();
        const u32 i = s_next;
        if (i >= total) break;
        const u32 c = hl[i];
        const u32 cap = a.c.rowptr[c + 1] - a.c.rowptr[c];
        const u32 tsz = 2 * cap;
        HugeSlot *tb = slots + hoff[c];
        for (u32 s = threadIdx.x; s < tsz; s += blockDim.x) tb[s] = HugeSlot{EMPTY, 0};
        __syncthreads();
        // one entry per thread at a time: batching four entries here (as the
        // other tiers do) measured slower, the table atomics then dominate
        for (u32 mi = a.moff[c]; mi < a.moff[c + 1]; ++mi) {
            const u32 u = a.mlist[mi];
            const u64 beg = a.g.rowptr[u];
            const u32 len = a.g.rowlen[u];
            for (u32 t = threadIdx.x; t < len; t += blockDim.x) {
                const u32 cv = a.map[a.g.adj[beg + t]];
                if (cv == c) continue;
                const s32 w = g_ew(a.g, beg + t);
                u32 h = range_hash(cv, tsz);
                bool ok = false;
                for (u32 probe = 0; probe < tsz; ++probe) {
                    const u32 prev = atomicCAS(&tb[h].key, EMPTY, cv);
                    if (prev == EMPTY || prev == cv) {
                        atomicAdd(&tb[h].w, w);
                        ok = true;
                        break;
                    }
                    h = (h + 1 == tsz) ? 0 : h + 1;
                }
                if (!ok) set_error(a.err, DEV_ERR_HASH_FULL);
            }
        }
        __syncthreads();
        // emit in chunks of blockDim.x slots
        const u64 out = a.c.rowptr[c];
        u32 cntu = 0;
        for (u32 s0 = 0; s0 < tsz; s0 += blockDim.x) {
            const u32 s = s0 + threadIdx.x;
            const HugeSlot sl = s < tsz ? tb[s] : HugeSlot{EMPTY, 0};
            const bool has = sl.key != EMPTY;
            u32 tot;
            const u32 p = block_exclusive_scan<u32>(has ? 1u : 0u, tot, scan_sm);
            if (has) {
                a.c.adj[out + cntu + p] = sl.key;
                a.c.ew[out + cntu + p] = sl.w;
            }
            cntu += tot;
        }
        if (threadIdx.x == 0) a.c.rowlen[c] = cntu;
        msum += cntu;
        __syncthreads();
    }
    if (threadIdx.x == 0 && msum) atomicAdd(a.m_out, msum);
}

} // namespace

DGraph contract_graph(Ctx &ctx, const DGraph &g, const u32 *mapping, u32 n_c) {
    ProfScope prof(ctx, "contract");
    DGraph c;
    c.n = n_c;
    c.cap = g.m;
    c.total_vw = g.total_vw;
    c.rowptr = ctx.falloc<u32>((u64) n_c + 1);
    c.rowlen = ctx.falloc<u32>(n_c);
    c.vw = ctx.falloc<s32>(n_c);
    c.adj = ctx.falloc<u32>(c.cap);
    c.ew = ctx.falloc<s32>(c.cap);

    ScratchScope ss(ctx.arena);
    u32 *cnt = ctx.balloc<u32>(n_c);
    u32 *capsum = ctx.balloc<u32>(n_c);
    u32 *moff = ctx.balloc<u32>((u64) n_c + 1);
    u32 *cursor = ctx.balloc<u32>(n_c);
    u32 *mlist = ctx.balloc<u32>(g.n);
    u32 *wl = ctx.balloc<u32>(n_c);
    u32 *bl = ctx.balloc<u32>(n_c);
    u32 *bl2 = ctx.balloc<u32>(n_c);
    u32 *hl = ctx.balloc<u32>(n_c);
    u32 *hcap = ctx.balloc<u32>(n_c);
    u32 *hoffc = ctx.balloc<u32>(n_c);
    HP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(u32) * n_c, ctx.stream));
    HP_CUDA(cudaMemsetAsync(capsum, 0, sizeof(u32) * n_c, ctx.stream));
    HP_CUDA(cudaMemsetAsync(c.vw, 0, sizeof(s32) * n_c, ctx.stream));
    k_cluster_stats<<<ctx.grid(g.n, BLOCK), BLOCK, 0, ctx.stream>>>(g, mapping, cnt, capsum, c.vw); note_launch();
    HP_LAUNCH_CHECK();
    u32 *rowptr = c.rowptr;
    device_scan<u32>(
        ctx, (u64) n_c + 1, [=] __device__(u64 i) -> u32 { return i < n_c ? cnt[i] : 0u; },
        [=] __device__(u64 i, u32 p, u32) {
            moff[i] = p;
            if (i < n_c) cursor[i] = p;
        },
        (u32 *) nullptr);
    device_scan<u32>(
        ctx, (u64) n_c + 1, [=] __device__(u64 i) -> u32 { return i < n_c ? capsum[i] : 0u; },
        [=] __device__(u64 i, u32 p, u32) { rowptr[i] = p; }, (u32 *) nullptr);
    k_fill_members<<<ctx.grid(g.n, BLOCK), BLOCK, 0, ctx.stream>>>(mapping, g.n, cursor, mlist); note_launch();
    HP_LAUNCH_CHECK();

    ctx.zero_counters();
    DevStatus *st = ctx.d_status;
    CArgs a{g, mapping, moff, mlist, c, &st->err, (unsigned long long *) &st->sum[1]};
    const size_t rec0 = ctx.instr.begin(ctx.stream, "contract", 0.0);
    const size_t rec_t = ctx.instr.begin(ctx.stream, "contract_thread", 0.0);
    TierLists TL{wl, &st->cnt[0], bl, &st->cnt[1], bl2, &st->cnt[C_ST_BLOCK_LARGE], hl, &st->cnt[2], hcap, hoffc,
                 (unsigned long long *) &st->sum[0]};
    k_contract_small<<<ctx.grid(n_c, BLOCK), BLOCK, 0, ctx.stream>>>(a, TL); note_launch();
    HP_LAUNCH_CHECK();
    ctx.instr.end(ctx.stream, rec_t);
    ctx.instr.end(ctx.stream, rec0);
    const DevStatus &s1 = ctx.read_status();
    const u32 nw = s1.cnt[0], nb = s1.cnt[1], nh = s1.cnt[2], nb2 = s1.cnt[C_ST_BLOCK_LARGE];
    const u64 hslots = (u64) s1.sum[0];
    if (nw) {
        KernTimer kt(ctx, "contract");
        KernTimer kt1(ctx, "contract_warp");
        k_contract_warp<<<ctx.grid((u64) nw * 32, C_WARP_BLOCK), C_WARP_BLOCK, 0, ctx.stream>>>(a, wl, &st->cnt[0]); note_launch();
        HP_LAUNCH_CHECK();
    }
    if (nb) {
        // clusters of up to C_BLOCK_SMALL_MAX entries: 16 KB tables, so
        // eight 256-thread blocks fit on an SM
        const size_t smem = ((size_t) 1 << C_BLOCK_SMALL_BITS) * 8;
        KernTimer kt(ctx, "contract");
        KernTimer kt1(ctx, "contract_block");
        k_contract_block<<<(u32) std::min<u64>(nb, (u64) ctx.sm_count * 8), BLOCK, smem, ctx.stream>>>(
            a, bl, &st->cnt[1], C_BLOCK_SMALL_BITS); note_launch();
        HP_LAUNCH_CHECK();
    }
    if (nb2) {
        const size_t smem = (size_t) C_BLOCK_SLOTS * 8;
        HP_CUDA(cudaFuncSetAttribute(k_contract_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        KernTimer kt(ctx, "contract");
        KernTimer kt1(ctx, "contract_block");
        k_contract_block<<<(u32) std::min<u64>(nb2, (u64) ctx.sm_count * 3), BLOCK, smem, ctx.stream>>>(
            a, bl2, &st->cnt[C_ST_BLOCK_LARGE], C_BLOCK_BITS); note_launch();
        HP_LAUNCH_CHECK();
    }
    if (nh) {
        // largest clusters first (their rows differ by two orders of
        // magnitude; a block that took a large one late would finish alone)
        std::vector<u32> hv(nh), hc(nh), order(nh);
        HP_CUDA(cudaMemcpyAsync(hv.data(), hl, sizeof(u32) * nh, cudaMemcpyDeviceToHost, ctx.stream));
        HP_CUDA(cudaMemcpyAsync(hc.data(), hcap, sizeof(u32) * nh, cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        for (u32 i = 0; i < nh; ++i) order[i] = i;
        std::sort(order.begin(), order.end(), [&](u32 x, u32 y) { return hc[x] != hc[y] ? hc[x] > hc[y] : hv[x] < hv[y]; });
        for (u32 i = 0; i < nh; ++i) hc[i] = hv[order[i]];
        HP_CUDA(cudaMemcpyAsync(hl, hc.data(), sizeof(u32) * nh, cudaMemcpyHostToDevice, ctx.stream));
        ctx.sync();
        HugeSlot *slots = ctx.balloc<HugeSlot>(hslots);
        KernTimer kt(ctx, "contract");
        KernTimer kt1(ctx, "contract_huge");
        k_contract_huge<<<(u32) std::min<u64>(nh, (u64) ctx.sm_count * 2), C_HUGE_BLOCK, 0, ctx.stream>>>(
            a, hl, &st->cnt[2], hoffc, slots, &st->cnt[C_ST_HUGE_TICKET]); note_launch();
        HP_LAUNCH_CHECK();
    }
    const DevStatus &s2 = ctx.read_status();
    if (s2.err & DEV_ERR_HASH_FULL) throw HpError{HP_ERR_DEVICE, "contraction hash table overflow"};
    c.m = (u64) s2.sum[1];
    // algorithmic bytes of the aggregation pass (roofline accounting): member
    // lists, fine offsets/lengths/weights, fine rows and weights, map gather,
    // coarse rows, weights and lengths
    if (rec0 < ctx.instr.pending.size()) {
        const double fine_e = g.ew ? 12.0 : 8.0;
        ctx.instr.pending[rec0].bytes = 12.0 * g.n + fine_e * (double) g.m + 8.0 * n_c + 8.0 * (double) c.m;
    }
    return c;
}

} // namespace hp
