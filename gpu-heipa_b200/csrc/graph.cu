#include "graph.cuh"
#include "prims.cuh"

namespace hp {

__global__ void k_iota(u32 *p, u64 n) {
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64) gridDim.x * blockDim.x) p[i] = (u32) i;
}

void device_iota(Ctx &ctx, u32 *p, u64 n) {
    if (n == 0) return;
    k_iota<<<ctx.grid(n, BLOCK), BLOCK, 0, ctx.stream>>>(p, n); note_launch();
    HP_LAUNCH_CHECK();
}

// rowlen from offsets; sums vertex weights; checks vertex weights.
__global__ void k_rows(DGraph g, u32 *err, long long *vw_sum) {
    s64 local = 0;
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < g.n; u += gridDim.x * blockDim.x) {
        u32 a = g.rowptr[u], b = g.rowptr[u + 1];
        if (b < a) {
            set_error(err, DEV_ERR_RANGE);
            b = a;
        }
        g.rowlen[u] = b - a;
        s32 w = g_vw(g, u);
        if (w < 1) set_error(err, DEV_ERR_BAD_WEIGHT);
        local += w;
    }
    local = warp_sum<long long>(local);
    if (lane_id() == 0) atomicAdd((unsigned long long *) vw_sum, (unsigned long long) local);
}

// Checks neighbour ids and edge weights; one warp per row.
__global__ void k_validate_edges(DGraph g, u32 *err) {
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < g.n; u += warps) {
        const u64 beg = g.rowptr[u];
        const u32 len = g.rowlen[u];
        for (u32 t = lane_id(); t < len; t += 32) {
            u32 v = g.adj[beg + t];
            if (v >= g.n || v == u) set_error(err, DEV_ERR_BAD_ID);
            if (g.ew && g.ew[beg + t] < 1) set_error(err, DEV_ERR_BAD_WEIGHT);
        }
    }
}

static void finish_graph(Ctx &ctx, DGraph &g, bool validate) {
    ctx.zero_status();
    k_rows<<<ctx.grid(g.n, BLOCK), BLOCK, 0, ctx.stream>>>(g, &ctx.d_status->err, &ctx.d_status->sum[0]); note_launch();
    HP_LAUNCH_CHECK();
    if (validate && g.cap > 0) {
        k_validate_edges<<<ctx.grid((u64) g.n * 32, BLOCK), BLOCK, 0, ctx.stream>>>(g, &ctx.d_status->err); note_launch();
        HP_LAUNCH_CHECK();
    }
    const DevStatus &s = ctx.read_status();
    if (s.err & (DEV_ERR_BAD_ID | DEV_ERR_RANGE))
        throw HpError{HP_ERR_GRAPH, "invalid graph: neighbour id out of range, self loop or bad offsets"};
    if (s.err & DEV_ERR_BAD_WEIGHT) throw HpError{HP_ERR_GRAPH, "invalid graph: weights must be >= 1"};
    g.total_vw = s.sum[0];
    if (g.total_vw > INT32_MAX) throw HpError{HP_ERR_GRAPH, "total vertex weight exceeds the 32-bit range"};
    g.m = g.cap;
}

DGraph graph_upload(Ctx &ctx, u32 n, u64 m, const u32 *xadj, const u32 *adj, const s32 *ew, const s32 *vw) {
    if (m >= 0xFFFFFFFFull) throw HpError{HP_ERR_ARG, "graph has too many edges for 32-bit offsets"};
    if (xadj == nullptr || (m > 0 && adj == nullptr)) throw HpError{HP_ERR_ARG, "null CSR array"};
    if ((u64) xadj[n] != m || xadj[0] != 0) throw HpError{HP_ERR_GRAPH, "xadj[0] must be 0 and xadj[n] must equal m"};
    DGraph g;
    g.n = n;
    g.cap = m;
    g.rowptr = ctx.falloc<u32>((u64) n + 1);
    g.rowlen = ctx.falloc<u32>(n);
    g.adj = ctx.falloc<u32>(m);
    if (ew) g.ew = ctx.falloc<s32>(m);
    if (vw) g.vw = ctx.falloc<s32>(n);
    HP_CUDA(cudaMemcpyAsync(g.rowptr, xadj, sizeof(u32) * ((u64) n + 1), cudaMemcpyHostToDevice, ctx.stream));
    if (m) HP_CUDA(cudaMemcpyAsync(g.adj, adj, sizeof(u32) * m, cudaMemcpyHostToDevice, ctx.stream));
    if (ew && m) HP_CUDA(cudaMemcpyAsync(g.ew, ew, sizeof(s32) * m, cudaMemcpyHostToDevice, ctx.stream));
    if (vw && n) HP_CUDA(cudaMemcpyAsync(g.vw, vw, sizeof(s32) * n, cudaMemcpyHostToDevice, ctx.stream));
    finish_graph(ctx, g, true);
    return g;
}

DGraph graph_from_device(Ctx &ctx, u32 n, u64 m, const u32 *d_xadj, const u32 *d_adj, const s32 *d_ew,
                         const s32 *d_vw, bool validate) {
    DGraph g;
    g.n = n;
    g.cap = m;
    g.rowptr = ctx.falloc<u32>((u64) n + 1);
    g.rowlen = ctx.falloc<u32>(n);
    g.adj = ctx.falloc<u32>(m);
    if (d_ew) g.ew = ctx.falloc<s32>(m);
    if (d_vw) g.vw = ctx.falloc<s32>(n);
    HP_CUDA(cudaMemcpyAsync(g.rowptr, d_xadj, sizeof(u32) * ((u64) n + 1), cudaMemcpyDeviceToDevice, ctx.stream));
    if (m) HP_CUDA(cudaMemcpyAsync(g.adj, d_adj, sizeof(u32) * m, cudaMemcpyDeviceToDevice, ctx.stream));
    if (d_ew && m) HP_CUDA(cudaMemcpyAsync(g.ew, d_ew, sizeof(s32) * m, cudaMemcpyDeviceToDevice, ctx.stream));
    if (d_vw && n) HP_CUDA(cudaMemcpyAsync(g.vw, d_vw, sizeof(s32) * n, cudaMemcpyDeviceToDevice, ctx.stream));
    finish_graph(ctx, g, validate);
    return g;
}

// Copies padded rows into a compact CSR (one warp per row).
__global__ void k_compact_rows(DGraph g, const u32 *off, u32 *adj, s32 *ew) {
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < g.n; u += warps) {
        const u64 src = g.rowptr[u], dst = off[u];
        const u32 len = g.rowlen[u];
        for (u32 t = lane_id(); t < len; t += 32) {
            adj[dst + t] = g.adj[src + t];
            ew[dst + t] = g_ew(g, src + t);
        }
    }
}

void graph_download(Ctx &ctx, const DGraph &g, u32 *xadj, u32 *adj, s32 *ew, s32 *vw) {
    ScratchScope ss(ctx.arena);
    u32 *off = ctx.balloc<u32>((u64) g.n + 1);
    const u32 *rowlen = g.rowlen;
    device_scan<u32>(
        ctx, g.n + 1, [=] __device__(u64 i) -> u32 { return i < g.n ? rowlen[i] : 0u; },
        [=] __device__(u64 i, u32 p, u32) { off[i] = p; }, (u32 *) nullptr);
    u32 *dadj = ctx.balloc<u32>(g.m);
    s32 *dew = ctx.balloc<s32>(g.m);
    k_compact_rows<<<ctx.grid((u64) g.n * 32, BLOCK), BLOCK, 0, ctx.stream>>>(g, off, dadj, dew); note_launch();
    HP_LAUNCH_CHECK();
    if (xadj) HP_CUDA(cudaMemcpyAsync(xadj, off, sizeof(u32) * ((u64) g.n + 1), cudaMemcpyDeviceToHost, ctx.stream));
    if (adj && g.m) HP_CUDA(cudaMemcpyAsync(adj, dadj, sizeof(u32) * g.m, cudaMemcpyDeviceToHost, ctx.stream));
    if (ew && g.m) HP_CUDA(cudaMemcpyAsync(ew, dew, sizeof(s32) * g.m, cudaMemcpyDeviceToHost, ctx.stream));
    if (vw) {
        if (g.vw) HP_CUDA(cudaMemcpyAsync(vw, g.vw, sizeof(s32) * g.n, cudaMemcpyDeviceToHost, ctx.stream));
        else
            for (u32 u = 0; u < g.n; ++u) vw[u] = 1;
    }
    ctx.sync();
}

// ---- induced subgraph (hierarchical multisection) ------------------------------

// Per-vertex count of neighbours inside the block (one warp per vertex).
__global__ void k_sub_degrees(DGraph g, const u32 *part, u32 id, u32 *deg) {
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < g.n; u += warps) {
        u32 c = 0;
        if (part[u] == id) {
            const u64 beg = g.rowptr[u];
            const u32 len = g.rowlen[u];
            for (u32 t = lane_id(); t < len; t += 32) c += part[g.adj[beg + t]] == id;
            c = warp_sum<u32>(c);
        }
        if (lane_id() == 0) deg[u] = c;
    }
}

// Writes the rows of the block's vertices; row order is kept with a warp
// ballot compaction.
__global__ void k_sub_fill(DGraph g, const u32 *part, u32 id, const u32 *local, const u32 *eoff, DGraph s) {
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < g.n; u += warps) {
        if (part[u] != id) continue;
        const u32 lu = local[u];
        const u64 beg = g.rowptr[u];
        const u32 len = g.rowlen[u];
        u64 out = eoff[u];
        if (lane_id() == 0) {
            s.rowptr[lu] = (u32) out;
            s.vw[lu] = g_vw(g, u);
        }
        for (u32 t0 = 0; t0 < len; t0 += 32) {
            u32 t = t0 + lane_id();
            bool keep = false;
            u32 v = 0;
            if (t < len) {
                v = g.adj[beg + t];
                keep = part[v] == id;
            }
            unsigned mask = __ballot_sync(FULL, keep);
            if (keep) {
                u64 pos = out + __popc(mask & ((1u << lane_id()) - 1u));
                s.adj[pos] = local[v];
                s.ew[pos] = g_ew(g, beg + t);
            }
            out += __popc(mask);
        }
    }
}

__global__ void k_sub_rowlen(DGraph s, u32 m) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < s.n; u += gridDim.x * blockDim.x) {
        u32 end = (u + 1 < s.n) ? s.rowptr[u + 1] : m;
        s.rowlen[u] = end - s.rowptr[u];
        if (u + 1 == s.n) s.rowptr[s.n] = m;
    }
}

DGraph graph_induced(Ctx &ctx, const DGraph &g, const u32 *part, u32 id, u32 *n_to_o_out, u32 &sub_n) {
    ScratchScope ss(ctx.arena);
    u32 *counts = &ctx.d_status->cnt[0];
    ctx.zero_counters();
    u32 *local = ctx.balloc<u32>(g.n);
    u32 *eoff = ctx.balloc<u32>((u64) g.n + 1);
    u32 *deg = ctx.balloc<u32>(g.n);
    device_scan<u32>(
        ctx, g.n, [=] __device__(u64 i) -> u32 { return part[i] == id ? 1u : 0u; },
        [=] __device__(u64 i, u32 p, u32 v) {
            if (v) {
                local[i] = p;
                n_to_o_out[p] = (u32) i;
            }
        },
        counts + 0);
    k_sub_degrees<<<ctx.grid((u64) g.n * 32, BLOCK), BLOCK, 0, ctx.stream>>>(g, part, id, deg); note_launch();
    HP_LAUNCH_CHECK();
    device_scan<u32>(
        ctx, g.n, [=] __device__(u64 i) -> u32 { return deg[i]; }, [=] __device__(u64 i, u32 p, u32) { eoff[i] = p; },
        counts + 1);
    const DevStatus &st = ctx.read_status();
    sub_n = st.cnt[0];
    const u32 sub_m = st.cnt[1];
    DGraph s;
    s.n = sub_n;
    s.cap = sub_m;
    s.m = sub_m;
    s.rowptr = ctx.falloc<u32>((u64) sub_n + 1);
    s.rowlen = ctx.falloc<u32>(sub_n);
    s.adj = ctx.falloc<u32>(sub_m);
    s.ew = ctx.falloc<s32>(sub_m);
    s.vw = ctx.falloc<s32>(sub_n);
    if (sub_n == 0) return s;
    k_sub_fill<<<ctx.grid((u64) g.n * 32, BLOCK), BLOCK, 0, ctx.stream>>>(g, part, id, local, eoff, s); note_launch();
    k_sub_rowlen<<<ctx.grid(sub_n, BLOCK), BLOCK, 0, ctx.stream>>>(s, sub_m); note_launch();
    HP_LAUNCH_CHECK();
    // total vertex weight of the subgraph
    ctx.zero_counters();
    const s32 *svw = s.vw;
    long long *sum = &ctx.d_status->sum[0];
    device_scan<long long>(
        ctx, sub_n, [=] __device__(u64 i) -> long long { return svw[i]; }, [=] __device__(u64, long long, long long) {},
        sum);
    s.total_vw = ctx.read_status().sum[0];
    return s;
}

} // namespace hp
