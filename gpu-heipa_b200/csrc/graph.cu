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

// ---- induced subgraphs (hierarchical multisection): all parts in one pass --------------

struct IndPart {
    u32 *rowptr, *rowlen, *adj;
    s32 *ew, *vw;
    u32 *n_to_o;
    u32 n, vstart;
    u64 m, ebase;
};

constexpr u32 IND_SMEM_K = 1024;  // per-block part histograms in shared memory up to this k

// Same-part degree of every vertex, and per part: vertices, entries, vertex
// weight (block histograms in shared memory for small k).
__global__ void k_ind_count(DGraph g, const u32 *part, u32 k, u32 *deg, u32 *cnt_v, unsigned long long *cnt_e,
                            unsigned long long *sum_vw, u32 *err) {
    __shared__ u32 sv[IND_SMEM_K];
    __shared__ unsigned long long se[IND_SMEM_K], sw[IND_SMEM_K];
    const bool local = k <= IND_SMEM_K;
    if (local) {
        for (u32 p = threadIdx.x; p < k; p += blockDim.x) {
            sv[p] = 0;
            se[p] = 0;
            sw[p] = 0;
        }
        __syncthreads();
    }
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < g.n; u += warps) {
        const u32 p = part[u];
        if (p >= k) {
            if (lane_id() == 0) {
                set_error(err, DEV_ERR_RANGE);
                deg[u] = 0;
            }
            continue;
        }
        const u64 beg = g.rowptr[u];
        const u32 len = g.rowlen[u];
        u32 c = 0;
        for (u32 t = lane_id(); t < len; t += 32) c += part[g.adj[beg + t]] == p;
        c = warp_sum<u32>(c);
        if (lane_id() == 0) {
            deg[u] = c;
            const s32 w = g_vw(g, u);
            if (local) {
                atomicAdd(&sv[p], 1u);
                atomicAdd(&se[p], (unsigned long long) c);
                atomicAdd(&sw[p], (unsigned long long) (long long) w);
            } else {
                atomicAdd(&cnt_v[p], 1u);
                atomicAdd(&cnt_e[p], (unsigned long long) c);
                atomicAdd(&sum_vw[p], (unsigned long long) (long long) w);
            }
        }
    }
    if (local) {
        __syncthreads();
        for (u32 p = threadIdx.x; p < k; p += blockDim.x)
            if (sv[p]) {
                atomicAdd(&cnt_v[p], sv[p]);
                atomicAdd(&cnt_e[p], se[p]);
                atomicAdd(&sum_vw[p], sw[p]);
            }
    }
}

// Local ids (rank within the part in ascending vertex id, from the sorted
// order), composed root ids, row offsets, row lengths and vertex weights.
__global__ void k_ind_local(DGraph g, const u32 *skey, const u32 *sval, const u32 *pre, const u32 *deg,
                            const IndPart *T, const u32 *n_to_o_parent, u32 *local_of) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
        const u32 p = skey[i], u = sval[i];
        const IndPart P = T[p];
        const u32 lu = i - P.vstart;
        local_of[u] = lu;
        P.n_to_o[lu] = n_to_o_parent[u];
        P.rowptr[lu] = (u32) (pre[i] - P.ebase);
        P.rowlen[lu] = deg[u];
        P.vw[lu] = g_vw(g, u);
        if (lu + 1 == P.n) P.rowptr[P.n] = (u32) P.m;
    }
}

// Rows of every subgraph, in parent row order (warp ballot compaction).
__global__ void k_ind_fill(DGraph g, const u32 *part, const u32 *local_of, const IndPart *T, u32 k) {
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < g.n; u += warps) {
        const u32 p = part[u];
        if (p >= k) continue;
        const IndPart P = T[p];
        const u64 beg = g.rowptr[u];
        const u32 len = g.rowlen[u];
        u64 out = P.rowptr[local_of[u]];
        for (u32 t0 = 0; t0 < len; t0 += 32) {
            const u32 t = t0 + lane_id();
            bool keep = false;
            u32 v = 0;
            if (t < len) {
                v = g.adj[beg + t];
                keep = part[v] == p;
            }
            const unsigned mask = __ballot_sync(FULL, keep);
            if (keep) {
                const u64 pos = out + __popc(mask & ((1u << lane_id()) - 1u));
                P.adj[pos] = local_of[v];
                P.ew[pos] = g_ew(g, beg + t);
            }
            out += __popc(mask);
        }
    }
}

void graph_induced_all(Ctx &ctx, const DGraph &g, const u32 *part, u32 k, const u32 *n_to_o_parent,
                       std::vector<DGraph> &subs, std::vector<u32 *> &n_to_o) {
    subs.assign(k, DGraph{});
    n_to_o.assign(k, nullptr);
    if (g.n == 0 || k == 0) return;
    // per-part sizes (front allocations below must not sit under scratch:
    // the scratch of this function is taken from the back)
    ScratchScope ss(ctx.arena);
    u32 *deg = ctx.balloc<u32>(g.n);
    u32 *cnt_v = ctx.balloc<u32>(k);
    unsigned long long *cnt_e = ctx.balloc<unsigned long long>(k);
    unsigned long long *sum_vw = ctx.balloc<unsigned long long>(k);
    HP_CUDA(cudaMemsetAsync(cnt_v, 0, sizeof(u32) * k, ctx.stream));
    HP_CUDA(cudaMemsetAsync(cnt_e, 0, sizeof(unsigned long long) * k, ctx.stream));
    HP_CUDA(cudaMemsetAsync(sum_vw, 0, sizeof(unsigned long long) * k, ctx.stream));
    ctx.zero_status();
    k_ind_count<<<ctx.grid((u64) g.n * 32, BLOCK), BLOCK, 0, ctx.stream>>>(g, part, k, deg, cnt_v, cnt_e, sum_vw,
                                                                          &ctx.d_status->err); note_launch();
    HP_LAUNCH_CHECK();
    std::vector<u32> hv(k);
    std::vector<unsigned long long> he(k), hw(k);
    HP_CUDA(cudaMemcpyAsync(hv.data(), cnt_v, sizeof(u32) * k, cudaMemcpyDeviceToHost, ctx.stream));
    HP_CUDA(cudaMemcpyAsync(he.data(), cnt_e, sizeof(unsigned long long) * k, cudaMemcpyDeviceToHost, ctx.stream));
    HP_CUDA(cudaMemcpyAsync(hw.data(), sum_vw, sizeof(unsigned long long) * k, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.check_device_error();
    // per-part arrays (front of the arena, part after part)
    std::vector<IndPart> T(k);
    u64 vstart = 0, ebase = 0;
    for (u32 p = 0; p < k; ++p) {
        IndPart &P = T[p];
        P.n = hv[p];
        P.m = he[p];
        P.vstart = (u32) vstart;
        P.ebase = ebase;
        vstart += P.n;
        ebase += P.m;
        if (P.n == 0) continue;
        DGraph &s = subs[p];
        s.n = P.n;
        s.m = s.cap = P.m;
        s.rowptr = P.rowptr = ctx.falloc<u32>((u64) P.n + 1);
        s.rowlen = P.rowlen = ctx.falloc<u32>(P.n);
        s.adj = P.adj = ctx.falloc<u32>(P.m);
        s.ew = P.ew = ctx.falloc<s32>(P.m);
        s.vw = P.vw = ctx.falloc<s32>(P.n);
        s.total_vw = (s64) hw[p];
        n_to_o[p] = P.n_to_o = ctx.falloc<u32>(P.n);
    }
    if (ebase > 0xFFFFFFFFull) throw HpError{HP_ERR_ARG, "induced subgraphs exceed 32-bit offsets"};
    IndPart *dT = ctx.balloc<IndPart>(k);
    HP_CUDA(cudaMemcpyAsync(dT, T.data(), sizeof(IndPart) * k, cudaMemcpyHostToDevice, ctx.stream));
    // vertices grouped by part, ascending id within each part (stable sort)
    u32 *skey = ctx.balloc<u32>(g.n);
    u32 *sval = ctx.balloc<u32>(g.n);
    HP_CUDA(cudaMemcpyAsync(skey, part, sizeof(u32) * g.n, cudaMemcpyDeviceToDevice, ctx.stream));
    device_iota(ctx, sval, g.n);
    radix_sort_pairs<u32>(ctx, skey, sval, g.n, 0, bits_for(k));
    // entry offsets in that order: parts are contiguous, so part p's rows
    // start at its ebase
    u32 *pre = ctx.balloc<u32>(g.n);
    device_scan<u32>(
        ctx, g.n, [=] __device__(u64 i) -> u32 { return deg[sval[i]]; },
        [=] __device__(u64 i, u32 q, u32) { pre[i] = q; }, (u32 *) nullptr);
    u32 *local_of = ctx.balloc<u32>(g.n);
    k_ind_local<<<ctx.grid(g.n, BLOCK), BLOCK, 0, ctx.stream>>>(g, skey, sval, pre, deg, dT, n_to_o_parent,
                                                                local_of); note_launch();
    k_ind_fill<<<ctx.grid((u64) g.n * 32, BLOCK), BLOCK, 0, ctx.stream>>>(g, part, local_of, dT, k); note_launch();
    HP_LAUNCH_CHECK();
    ctx.sync();  // the scratch (table, order, local ids) is released on return
}


} // namespace hp
