#include "solver.cuh"
#include "prims.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <exception>
#include <mutex>
#include <thread>

#include "../host/initial_partition.h"

namespace hp {
namespace {

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

__global__ void k_project(const u32 *coarse_part, const u32 *map, u32 *fine_part, u32 n) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
        fine_part[u] = coarse_part[map[u]];
}

__global__ void k_scatter_leaf(const u32 *tmp, const u32 *n_to_o, u32 n, u32 offset, u32 *global_part) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
        global_part[n_to_o[u]] = offset + tmp[u];
}

// Downloads the coarsest graph with rows in canonical (sorted) order.
HostCSR download_sorted(Ctx &ctx, const DGraph &g) {
    HostCSR h;
    h.n = g.n;
    h.m = (u32) g.m;
    h.xadj.resize((size_t) g.n + 1);
    h.adj.resize(g.m);
    h.ew.resize(g.m);
    h.vw.resize(g.n);
    graph_download(ctx, g, h.xadj.data(), h.adj.data(), h.ew.data(), h.vw.data());
    sort_rows(h);
    return h;
}

struct Hierarchy {
    std::vector<DGraph> graphs;
    std::vector<u32 *> maps;
};

// Coarsen while n > 8k (solver.h:343-347); stops early when a matching
// shrinks its level by less than 1% (the reference has no such check and
// loops on graphs that stop coarsening; every level here costs arena space).
void coarsen(Ctx &ctx, const DGraph &g, u32 k, Hierarchy &H, SolveStats *stats) {
    H.graphs.push_back(g);
    while (H.graphs.back().n > 8 * k) {
        const DGraph cur = H.graphs.back();
        auto t0 = Clock::now();
        u32 *mp = ctx.falloc<u32>(cur.n);
        const u32 nc = match_graph(ctx, cur, mp);
        if (stats) stats->coarsening_ms += ms_since(t0);
        if ((u64) nc * 100 > (u64) cur.n * 99) break;
        auto t1 = Clock::now();
        DGraph c = contract_graph(ctx, cur, mp, nc);
        if (stats) stats->contraction_ms += ms_since(t1);
        H.graphs.push_back(c);
        H.maps.push_back(mp);
    }
    if (stats) {
        stats->levels = (u32) H.graphs.size();
        for (const DGraph &x: H.graphs) {
            stats->level_n.push_back(x.n);
            stats->level_m.push_back(x.m);
        }
    }
}

// Uncoarsen + refine every level (solver.h:381-398).
void uncoarsen(Ctx &ctx, Hierarchy &H, u32 *coarse_part, u32 *part_out, u32 k, s32 lmax, bool ultra, s64 &obj,
               s32 &maxw, const DistOracle *D, SolveStats *stats) {
    u32 *cpart = coarse_part;
    for (size_t l = H.maps.size(); l > 0; --l) {
        const DGraph &fine = H.graphs[l - 1];
        auto t0 = Clock::now();
        u32 *fpart = (l == 1) ? part_out : ctx.falloc<u32>(fine.n);
        k_project<<<ctx.grid(fine.n, BLOCK), BLOCK, 0, ctx.stream>>>(cpart, H.maps[l - 1], fpart, fine.n); note_launch();
        HP_LAUNCH_CHECK();
        if (stats) {
            ctx.sync();
            stats->uncontraction_ms += ms_since(t0);
        }
        auto t1 = Clock::now();
        jet_refine(ctx, fine, fpart, k, lmax, ultra, (u32) (l - 1), obj, maxw, D);
        if (stats) stats->refinement_ms += ms_since(t1);
        cpart = fpart;
    }
    if (H.maps.empty())
        HP_CUDA(cudaMemcpyAsync(part_out, cpart, sizeof(u32) * H.graphs[0].n, cudaMemcpyDeviceToDevice, ctx.stream));
}

} // namespace

s32 lmax_of(s64 total_weight, u32 k, double eps) {
    return (s32) std::ceil((1.0 + eps) * ((double) total_weight / (double) k));
}

size_t request_estimate(u32 n, u64 m, bool has_ew, bool has_vw) {
    // the terms of arena_estimate with the per-vertex and scratch shares of
    // the hierarchy rounded up and a small fixed reserve instead of 512 MiB,
    // so that small requests of a served stream reserve little memory
    const double in = 4.0 * ((double) n + 1) * 2 + 4.0 * (double) m * (has_ew ? 2 : 1) + (has_vw ? 4.0 * n : 0.0);
    return (size_t) (in + 96.0 * (double) m + 256.0 * (double) n + 16.0 * 1024 * 1024);
}

size_t arena_estimate(u32 n, u64 m, bool has_ew, bool has_vw) {
    // input graph + hierarchy (every padded level holds up to the fine level's
    // m entries of 8 bytes; power-law graphs keep ~90% of their edges for the
    // first ~8 levels, so 10 levels' worth are budgeted) + per-level mappings
    // and Jet state (~60 n words) + matching / contraction scratch (global
    // hash tables for hub rows).
    const double in = 4.0 * ((double) n + 1) * 2 + 4.0 * (double) m * (has_ew ? 2 : 1) + (has_vw ? 4.0 * n : 0.0);
    const double hier = 80.0 * (double) m;
    const double per_vertex = 240.0 * (double) n;
    const double scratch = 16.0 * (double) m;
    return (size_t) (in + hier + per_vertex + scratch + (512.0 * 1024 * 1024));
}

s64 solve_partition(Ctx &ctx, const DGraph &g, u32 k, double eps, bool ultra, u64 seed, u32 *part,
                    SolveStats *stats) {
    if (k == 0) throw HpError{HP_ERR_ARG, "k must be positive"};
    if (k > MAX_K) throw HpError{HP_ERR_ARG, "k too large"};
    if (g.n == 0) return 0;
    if (k == 1) {
        HP_CUDA(cudaMemsetAsync(part, 0, sizeof(u32) * g.n, ctx.stream));
        ctx.sync();
        return 0;
    }
    const size_t front_mark = ctx.arena.front_mark();
    const s32 lmax = lmax_of(g.total_vw, k, eps);
    Hierarchy H;
    coarsen(ctx, g, k, H, stats);
    const DGraph &coarsest = H.graphs.back();
    // initial partitioning on the host (kway_core.h:1573-1588)
    auto t0 = Clock::now();
    ProfScope prof_ip(ctx, "initial_partitioning");
    HostCSR hc = download_sorted(ctx, coarsest);
    std::vector<u32> hpart;
    initial_kway(hc, k, eps, seed, hpart);
    u32 *cpart = ctx.falloc<u32>(coarsest.n);
    HP_CUDA(cudaMemcpyAsync(cpart, hpart.data(), sizeof(u32) * coarsest.n, cudaMemcpyHostToDevice, ctx.stream));
    s64 obj = edge_cut_dev(ctx, coarsest, cpart);
    s32 *bw = ctx.falloc<s32>(k);
    block_weights(ctx, coarsest, cpart, k, bw);
    s32 maxw = max_block_weight(ctx, bw, k);
    if (stats) {
        stats->initial_ms += ms_since(t0);
        stats->initial_obj = obj;
        stats->initial_maxw = maxw;
        stats->lmax = lmax;
    }
    uncoarsen(ctx, H, cpart, part, k, lmax, ultra, obj, maxw, nullptr, stats);
    ctx.sync();
    ctx.arena.front_release(front_mark);
    if (stats) {
        stats->final_obj = obj;
        stats->final_maxw = maxw;
    }
    return obj;
}

namespace {

// One sub-solve of the hierarchical multisection: a subgraph (in the main
// arena), its map to input vertex ids, the path of block ids that leads to it,
// and its partition.
struct HmTask {
    DGraph g;
    const u32 *n_to_o = nullptr;
    std::vector<u32> identifier;
    u32 *part = nullptr;
};

// Arena bytes a worker needs for one sub-solve of g (hierarchy, Jet scratch
// and sorting buffers; the subgraph itself lives in the main arena).
size_t worker_bytes(const DGraph &g) { return 96 * (size_t) g.m + 256 * (size_t) g.n + (64ull << 20); }

constexpr size_t HM_MAX_WORKERS = 32;

// Runs fn(ctx_w, task) for every task. The sub-solves are independent and
// deterministic, so they run concurrently on worker contexts (one host
// thread, stream and status word each, arena slices carved from the main
// arena's free space); with room for one slice only, they run in order on the
// main context. Results do not depend on the number of workers.
template<typename Fn>
void run_hm_tasks(Ctx &ctx, std::vector<HmTask> &tasks, Fn fn) {
    size_t slice = 0;
    for (const HmTask &t: tasks) slice = std::max(slice, worker_bytes(t.g));
    slice = (slice + 4095) & ~(size_t) 4095;
    const size_t free_bytes = ctx.arena.back_mark() - ctx.arena.front_mark();
    size_t W = std::min<size_t>(tasks.size(), HM_MAX_WORKERS);
    if (slice) W = std::min<size_t>(W, free_bytes / slice);
    if (W <= 1) {
        for (HmTask &t: tasks) fn(ctx, t);
        return;
    }
    ScratchScope ss(ctx.arena);
    char *slab = ctx.balloc<char>(W * slice);
    ctx.sync();  // subgraphs and partition arrays are ready before workers start
    std::vector<Ctx *> wc(W);
    for (size_t w = 0; w < W; ++w) {
        wc[w] = &ctx.worker(w);
        wc[w]->arena.attach(slab + w * slice, slice);
    }
    std::atomic<size_t> next{0};
    std::vector<std::exception_ptr> errors(W);
    std::vector<std::thread> threads;
    for (size_t w = 0; w < W; ++w) {
        threads.emplace_back([&, w] {
            try {
                HP_CUDA(cudaSetDevice(ctx.device));
                for (size_t i = next++; i < tasks.size(); i = next++) {
                    fn(*wc[w], tasks[i]);
                    wc[w]->sync();
                }
            } catch (...) {
                errors[w] = std::current_exception();
                next = tasks.size();
            }
        });
    }
    for (std::thread &t: threads) t.join();
    for (size_t w = 0; w < W; ++w) wc[w]->arena.destroy();
    for (std::exception_ptr &e: errors)
        if (e) std::rethrow_exception(e);
}

// recursive_multisection_device (hierarchical_multisection.h:56-235), level
// by level: every subgraph of one hierarchy level is partitioned into the
// level's number of parts, then the next level's subgraphs are induced from
// those parts. Leaves write their parts, offset by the block-id path, into
// global_part.
void hm_solve(Ctx &ctx, const DGraph &g, const std::vector<u32> &hier, double eps, u64 seed, bool ultra,
              u32 *global_part, SolveStats *stats) {
    const u32 l = (u32) hier.size();
    std::vector<u32> index_vec = {1};
    for (u32 i = 0; i + 1 < l; ++i) index_vec.push_back(index_vec[i] * hier[i]);
    std::vector<u32> k_rem(l);
    u32 kp = 1;
    for (u32 i = 0; i < l; ++i) {
        k_rem[i] = kp * hier[i];
        kp *= hier[i];
    }
    const u32 global_k = kp;
    const s64 global_w = g.total_vw;
    const size_t mark = ctx.arena.front_mark();
    u32 *n_to_o = ctx.falloc<u32>(g.n);
    device_iota(ctx, n_to_o, g.n);
    std::vector<HmTask> cur(1);
    cur[0].g = g;
    cur[0].n_to_o = n_to_o;
    std::mutex stats_mu;
    for (u32 depth = 0; depth < l && !cur.empty(); ++depth) {
        const u32 level = l - 1 - depth;
        const u32 k_here = hier[level];
        const bool leaf = depth == l - 1;
        for (HmTask &t: cur) t.part = ctx.falloc<u32>(t.g.n);
        run_hm_tasks(ctx, cur, [&](Ctx &wc, HmTask &t) {
            const double imb = adaptive_imbalance(eps, global_w, global_k, t.g.total_vw, k_rem[l - 1 - depth], l - depth);
            SolveStats sub;
            solve_partition(wc, t.g, k_here, imb, ultra, seed, t.part, stats ? &sub : nullptr);
            if (leaf) {
                u32 offset = 0;
                for (u32 i = 0; i + 1 < l; ++i) offset += t.identifier[i] * index_vec[index_vec.size() - 1 - i];
                k_scatter_leaf<<<wc.grid(t.g.n, BLOCK), BLOCK, 0, wc.stream>>>(t.part, t.n_to_o, t.g.n, offset,
                                                                              global_part); note_launch();
                HP_LAUNCH_CHECK();
                wc.sync();
            }
            if (stats) {
                std::lock_guard<std::mutex> lock(stats_mu);
                stats->add(sub);
            }
        });
        if (leaf) break;
        std::vector<HmTask> next;
        for (HmTask &t: cur) {
            // the k_here subgraphs of this task in one pass over its graph
            std::vector<DGraph> subs;
            std::vector<u32 *> sub_n_to_o;
            graph_induced_all(ctx, t.g, t.part, k_here, t.n_to_o, subs, sub_n_to_o);
            for (u32 id = 0; id < k_here; ++id) {
                if (subs[id].n == 0) continue;
                HmTask c;
                c.g = subs[id];
                c.n_to_o = sub_n_to_o[id];
                c.identifier = t.identifier;
                c.identifier.push_back(id);
                next.push_back(std::move(c));
            }
        }
        cur = std::move(next);
    }
    ctx.sync();
    ctx.arena.front_release(mark);
}

} // namespace

s64 solve_mapping(Ctx &ctx, const DGraph &g, const std::vector<u32> &hier, const std::vector<s32> &dist, double eps,
                  int mode, u64 seed, u32 *part, SolveStats *stats) {
    const size_t front_mark = ctx.arena.front_mark();
    DistOracle D = make_dist_oracle(ctx, hier, dist);
    const u32 k = D.k;
    const u32 l = (u32) hier.size();
    s64 J = 0;
    if (g.n == 0) return 0;
    if (mode == 0) {
        // ProMapSolver::internal_solve (promap_solver.h:244-299)
        const s32 lmax = lmax_of(g.total_vw, k, eps);
        Hierarchy H;
        coarsen(ctx, g, k, H, stats);
        const DGraph &coarsest = H.graphs.back();
        auto t0 = Clock::now();
        HostCSR hc = download_sorted(ctx, coarsest);
        std::vector<u32> hpart;
        global_multisection(hc, hier, eps, seed, hpart);
        u32 *cpart = ctx.falloc<u32>(coarsest.n);
        HP_CUDA(cudaMemcpyAsync(cpart, hpart.data(), sizeof(u32) * coarsest.n, cudaMemcpyHostToDevice, ctx.stream));
        J = comm_cost_dev(ctx, coarsest, cpart, D);
        s32 *bw = ctx.falloc<s32>(k);
        block_weights(ctx, coarsest, cpart, k, bw);
        s32 maxw = max_block_weight(ctx, bw, k);
        if (stats) {
            stats->initial_ms += ms_since(t0);
            stats->initial_obj = J;
            stats->initial_maxw = maxw;
            stats->lmax = lmax;
        }
        uncoarsen(ctx, H, cpart, part, k, lmax, false, J, maxw, &D, stats);
        if (stats) {
            stats->final_obj = J;
            stats->final_maxw = maxw;
        }
    } else {
        // hierarchical_multisection (hierarchical_multisection.h:237-307)
        hm_solve(ctx, g, hier, eps, seed, mode == 2, part, stats);
        J = comm_cost_dev(ctx, g, part, D);
        if (stats) {
            s32 *bw = ctx.falloc<s32>(k);
            block_weights(ctx, g, part, k, bw);
            stats->final_obj = J;
            stats->final_maxw = max_block_weight(ctx, bw, k);
            stats->lmax = lmax_of(g.total_vw, k, eps);
        }
    }
    ctx.sync();
    ctx.arena.front_release(front_mark);
    return J;
}

} // namespace hp
