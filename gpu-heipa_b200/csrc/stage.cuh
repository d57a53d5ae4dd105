// Per-warp staging of CSR row segments into shared memory with the Blackwell
// bulk-copy engine: cp.async.bulk (global -> this CTA's shared memory, no
// multicast) whose completion is counted in bytes on an mbarrier. Each warp
// owns two stages; while it gathers the labels of one segment's neighbours,
// the copy of its next segment is already in flight, so the row reads of a
// long row leave the critical path of the dependent label gathers.
//
// Alignment: a bulk copy needs a 16-byte aligned source, destination and
// size. A segment [e0, e1) of a row is copied as the 4-entry groups that
// cover it, [e0 & ~3, (e1 + 3) & ~3), and indexed from e0 & 3. Reading up to
// the next multiple of 4 entries stays inside the array: every CSR array of a
// DGraph lives in a context arena (or an arena slice starting on a 4096-byte
// boundary), whose allocations start on 256-byte boundaries and are rounded
// up to a multiple of 256 bytes. Launch sites check stage_ok() on the host
// and take the unstaged kernels otherwise.
//
// Waits are bounded: a wait that runs out sets DEV_ERR_SPIN, waits (again
// bounded) for the warp's other copy in flight and ends the warp's loop, so
// the kernel returns and the host reports the error.
#pragma once
#include "common.cuh"
#include "graph.cuh"

namespace hp {

constexpr u32 SEG = 512;          // entries per staged segment
constexpr u32 SEG_PAD = SEG + 8;  // room for rounding both ends to 4-entry groups
constexpr u32 STAGE_SPINS = 1u << 22;

// Shared memory of one warp: two stages of row ids and edge weights, and one
// mbarrier per stage.
struct WarpStage {
    u32 adj[2][SEG_PAD];
    s32 ew[2][SEG_PAD];
    unsigned long long bar[2];
};

// Host check: the graph's row arrays are 16-byte aligned.
inline bool stage_ok(const DGraph &g) {
    return ((uintptr_t) g.adj & 15u) == 0 && ((uintptr_t) g.ew & 15u) == 0;
}

__device__ __forceinline__ u32 smem_addr(const void *p) { return (u32) __cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes initialised mbarriers visible to the bulk-copy (async) proxy.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this thread's earlier shared-memory accesses before later async-proxy
// writes to the same buffer.
__device__ __forceinline__ void proxy_fence_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, u32 bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, u32 parity) {
    u32 done;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the phase with the given parity. Every lane of the warp
// waits (so that each sees the copied data) and the result is warp-uniform.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, u32 parity) {
    bool ok = false;
    for (u32 i = 0; i < STAGE_SPINS && !ok; ++i) ok = mbar_try_wait(bar, parity);
    return __all_sync(FULL, ok);
}

// Lane 0: starts the copy of entries [e0, e1) of g's rows into stage s.
__device__ __forceinline__ void stage_issue(const DGraph &g, WarpStage &S, int s, u64 e0, u64 e1) {
    const u64 a0 = e0 & ~3ull, a1 = (e1 + 3) & ~3ull;
    const u32 bytes = (u32) (a1 - a0) * 4u;
    proxy_fence_smem();
    mbar_arrive_expect_tx(&S.bar[s], g.ew ? 2u * bytes : bytes);
    bulk_copy_g2s(S.adj[s], g.adj + a0, bytes, &S.bar[s]);
    if (g.ew) bulk_copy_g2s(S.ew[s], g.ew + a0, bytes, &S.bar[s]);
}

// Runs one warp over the work items first, first + stride, ... < total. Item
// i covers entries [from, to) of row u (range(i, u, from, to)); the entries
// are staged SEG at a time and passed to body(u, adj, ew, len, item) as
// shared-memory arrays (ew is null for unit edge weights); done(u, item) runs
// after the item's last segment. Every lane of the warp calls this. Returns
// false when a wait ran out (DEV_ERR_SPIN is set in *err).
template<typename Range, typename Body, typename Done>
__device__ __forceinline__ bool staged_items(const DGraph &g, WarpStage &S, u32 first, u32 stride, u32 total,
                                             u32 *err, Range range, Body body, Done done) {
    const u32 lane = (u32) lane_id();
    if (lane == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        mbar_init_fence();
    }
    __syncwarp();
    if (first >= total) return true;
    u32 parity = 0u;  // bit s: phase parity of stage s
    u32 i = first, u, from, to;
    range(i, u, from, to);
    u64 beg = __ldg(&g.rowptr[u]);
    u32 seg = from;
    int s = 0;
    if (lane == 0) stage_issue(g, S, 0, beg + seg, beg + (to - seg < SEG ? to : seg + SEG));
    for (;;) {
        // the next segment: the rest of this row, else the next item
        u32 ni = i, nu = u, nfrom = from, nto = to, nseg = seg + SEG;
        u64 nbeg = beg;
        bool more = nseg < to;
        if (!more) {
            ni = i + stride;
            more = ni < total;
            if (more) {
                range(ni, nu, nfrom, nto);
                nbeg = __ldg(&g.rowptr[nu]);
                nseg = nfrom;
            }
        }
        if (more && lane == 0)
            stage_issue(g, S, s ^ 1, nbeg + nseg, nbeg + (nto - nseg < SEG ? nto : nseg + SEG));
        if (!mbar_wait_bounded(&S.bar[s], (parity >> s) & 1u)) {
            set_error(err, DEV_ERR_SPIN);
            if (more) mbar_wait_bounded(&S.bar[s ^ 1], (parity >> (s ^ 1)) & 1u);
            __syncwarp();
            return false;
        }
        parity ^= 1u << s;
        const u32 len = (to - seg < SEG ? to : seg + SEG) - seg;
        const u32 off = (u32) ((beg + seg) & 3ull);
        body(u, S.adj[s] + off, g.ew ? S.ew[s] + off : (const s32 *) nullptr, len, i);
        __syncwarp();
        if (seg + SEG >= to) done(u, i);
        if (!more) return true;
        i = ni;
        u = nu;
        from = nfrom;
        to = nto;
        seg = nseg;
        beg = nbeg;
        s ^= 1;
    }
}

} // namespace hp
