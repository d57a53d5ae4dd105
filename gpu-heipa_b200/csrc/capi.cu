// Implementation of the C ABI declared in include/gpuheipa.h.
#include "../../include/gpuheipa.h"

#include <algorithm>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <new>

#include "../host/generators.h"
#include "../host/initial_partition.h"
#include "../host/metis_io.h"
#include "service.cuh"
#include "solver.cuh"

struct hp_ctx {
    hp::Ctx c;
    hp::SolveStats last;
};

struct hp_graph {
    hp::DGraph g;
    size_t front_mark = 0;  // arena front before this graph was allocated
};

struct hp_jet {
    hp_ctx *ctx = nullptr;
    hp::JetLevel L;
    hp::DistOracle D;
    bool has_D = false;
    size_t back_mark = 0, front_mark = 0;
};

struct hp_host_graph {
    hp::HostCSR g;
};

struct hp_server {
    hp::Ctx c;  // owns the request buffer (its arena) and the worker contexts
    std::unique_ptr<hp::Service> svc;
    std::mutex mu;
    std::string last_error;
};

namespace {

template<typename F>
int guarded(hp_ctx *ctx, F &&f) {
    try {
        f();
        if (ctx) ctx->c.last_error.clear();
        return HP_OK;
    } catch (const hp::HpError &e) {
        if (ctx) ctx->c.last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        if (ctx) ctx->c.last_error = "host allocation failed";
        return HP_ERR_OOM;
    } catch (const std::exception &e) {
        if (ctx) ctx->c.last_error = e.what();
        return HP_ERR_ARG;
    }
}

template<typename F>
int guarded_host(F &&f) {
    try {
        f();
        return HP_OK;
    } catch (const hp::HpError &e) {
        return e.code;
    } catch (...) {
        return HP_ERR_ARG;
    }
}

std::vector<hp::u32> vec_u32(const uint32_t *p, uint32_t n) { return std::vector<hp::u32>(p, p + n); }
std::vector<hp::s32> vec_s32(const int32_t *p, uint32_t n) { return std::vector<hp::s32>(p, p + n); }

void check_hier(const uint32_t *hier, const int32_t *dist, uint32_t levels) {
    if (!hier || !dist || levels == 0) throw hp::HpError{HP_ERR_ARG, "hierarchy and distance are required"};
}

} // namespace

extern "C" {

int hp_ctx_create(int device, size_t arena_bytes, hp_ctx **out) {
    if (!out) return HP_ERR_ARG;
    *out = nullptr;
    hp_ctx *ctx = new (std::nothrow) hp_ctx();
    if (!ctx) return HP_ERR_OOM;
    int rc = guarded(ctx, [&] { ctx->c.init(device, arena_bytes); });
    if (rc != HP_OK) {
        ctx->c.destroy();
        delete ctx;
        return rc;
    }
    *out = ctx;
    return HP_OK;
}

int hp_ctx_destroy(hp_ctx *ctx) {
    if (!ctx) return HP_ERR_ARG;
    ctx->c.destroy();
    delete ctx;
    return HP_OK;
}

const char *hp_last_error(const hp_ctx *ctx) { return ctx ? ctx->c.last_error.c_str() : "null context"; }

size_t hp_arena_estimate(uint32_t n, uint64_t m, int has_ew, int has_vw) {
    return hp::arena_estimate(n, m, has_ew != 0, has_vw != 0);
}

size_t hp_arena_peak(const hp_ctx *ctx) { return ctx ? ctx->c.arena.peak() : 0; }

int hp_initial_partition(uint32_t n, const uint32_t *xadj, const uint32_t *adj, const int32_t *vw, const int32_t *ew,
                         uint32_t k, double imbalance, uint64_t seed, uint32_t *part) {
    if (!xadj || (n > 0 && !part) || k == 0 || k > hp::MAX_K) return HP_ERR_ARG;
    const uint64_t m = xadj[n];
    if (m > 0 && !adj) return HP_ERR_ARG;
    if (m > 0x7FFFFFFFull || n > 0x7FFFFFFFu) return HP_ERR_ARG;  // the partitioner indexes with int
    hp::HostCSR g;
    g.n = n;
    g.m = (uint32_t) m;
    g.xadj.assign(xadj, xadj + n + 1);
    for (uint32_t u = 0; u < n; ++u)
        if (xadj[u + 1] < xadj[u]) return HP_ERR_GRAPH;
    for (uint32_t u = 0; u < n; ++u)
        for (uint32_t j = xadj[u]; j < xadj[u + 1]; ++j)
            if (adj[j] >= n || adj[j] == u) return HP_ERR_GRAPH;
    g.adj.assign(adj, adj + m);
    if (ew) g.ew.assign(ew, ew + m);
    if (vw) g.vw.assign(vw, vw + n);
    try {
        std::vector<uint32_t> out;
        hp::initial_kway(g, k, imbalance, seed, out);
        std::copy(out.begin(), out.end(), part);
    } catch (const std::bad_alloc &) {
        return HP_ERR_OOM;
    }
    return HP_OK;
}

int hp_graph_upload(hp_ctx *ctx, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj, const int32_t *ew,
                    const int32_t *vw, hp_graph **out) {
    if (!ctx || !out) return HP_ERR_ARG;
    *out = nullptr;
    hp_graph *h = new (std::nothrow) hp_graph();
    if (!h) return HP_ERR_OOM;
    h->front_mark = ctx->c.arena.front_mark();
    int rc = guarded(ctx, [&] { h->g = hp::graph_upload(ctx->c, n, m, xadj, adj, ew, vw); });
    if (rc != HP_OK) {
        ctx->c.arena.front_release(h->front_mark);
        delete h;
        return rc;
    }
    *out = h;
    return HP_OK;
}

int hp_graph_free(hp_ctx *ctx, hp_graph *g) {
    if (!ctx || !g) return HP_ERR_ARG;
    ctx->c.arena.front_release(g->front_mark);
    delete g;
    return HP_OK;
}

int hp_graph_info(const hp_graph *g, uint32_t *n, uint64_t *m, int64_t *total_vw) {
    if (!g) return HP_ERR_ARG;
    if (n) *n = g->g.n;
    if (m) *m = g->g.m;
    if (total_vw) *total_vw = g->g.total_vw;
    return HP_OK;
}

int hp_graph_download(hp_ctx *ctx, const hp_graph *g, uint32_t *xadj, uint32_t *adj, int32_t *ew, int32_t *vw) {
    if (!ctx || !g) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        std::vector<hp::u32> tx, ta;
        std::vector<hp::s32> te;
        if (!xadj) {
            tx.resize((size_t) g->g.n + 1);
            xadj = tx.data();
        }
        if (!adj) {
            ta.resize(g->g.m);
            adj = ta.data();
        }
        if (!ew) {
            te.resize(g->g.m);
            ew = te.data();
        }
        hp::graph_download(ctx->c, g->g, xadj, adj, ew, vw);
    });
}

int hp_match(hp_ctx *ctx, const hp_graph *g, uint32_t *mapping, uint32_t *n_coarse) {
    if (!ctx || !g || !mapping) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        hp::ScratchScope ss(ctx->c.arena);
        hp::u32 *d = ctx->c.balloc<hp::u32>(g->g.n);
        hp::u32 nc = hp::match_graph(ctx->c, g->g, d);
        HP_CUDA(cudaMemcpyAsync(mapping, d, sizeof(hp::u32) * g->g.n, cudaMemcpyDeviceToHost, ctx->c.stream));
        ctx->c.sync();
        if (n_coarse) *n_coarse = nc;
    });
}

int hp_contract(hp_ctx *ctx, const hp_graph *g, const uint32_t *mapping, uint32_t n_coarse, hp_graph **out) {
    if (!ctx || !g || !mapping || !out) return HP_ERR_ARG;
    *out = nullptr;
    for (uint32_t u = 0; u < g->g.n; ++u)
        if (mapping[u] >= n_coarse) {
            ctx->c.last_error = "mapping value out of range";
            return HP_ERR_ARG;
        }
    hp_graph *h = new (std::nothrow) hp_graph();
    if (!h) return HP_ERR_OOM;
    h->front_mark = ctx->c.arena.front_mark();
    int rc = guarded(ctx, [&] {
        hp::u32 *d = ctx->c.falloc<hp::u32>(g->g.n);
        HP_CUDA(cudaMemcpyAsync(d, mapping, sizeof(hp::u32) * g->g.n, cudaMemcpyHostToDevice, ctx->c.stream));
        h->g = hp::contract_graph(ctx->c, g->g, d, n_coarse);
        ctx->c.sync();
    });
    if (rc != HP_OK) {
        ctx->c.arena.front_release(h->front_mark);
        delete h;
        return rc;
    }
    *out = h;
    return HP_OK;
}

int hp_jet_refine(hp_ctx *ctx, const hp_graph *g, uint32_t k, int32_t lmax, int ultra, uint32_t level,
                  uint32_t *part, int64_t *obj, int32_t *maxw, const uint32_t *hier, const int32_t *dist,
                  uint32_t levels) {
    if (!ctx || !g || !part || !obj || !maxw || k == 0) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        const size_t fm = ctx->c.arena.front_mark();
        hp::ScratchScope ss(ctx->c.arena);
        hp::DistOracle D;
        if (hier) {
            check_hier(hier, dist, levels);
            D = hp::make_dist_oracle(ctx->c, vec_u32(hier, levels), vec_s32(dist, levels));
            if (D.k != k) throw hp::HpError{HP_ERR_ARG, "k must equal the product of the hierarchy"};
        }
        for (uint32_t u = 0; u < g->g.n; ++u)
            if (part[u] >= k) throw hp::HpError{HP_ERR_ARG, "partition label out of range"};
        hp::u32 *d = ctx->c.balloc<hp::u32>(g->g.n);
        HP_CUDA(cudaMemcpyAsync(d, part, sizeof(hp::u32) * g->g.n, cudaMemcpyHostToDevice, ctx->c.stream));
        hp::s64 o = *obj;
        hp::s32 mw = *maxw;
        hp::jet_refine(ctx->c, g->g, d, k, lmax, ultra != 0, level, o, mw, hier ? &D : nullptr);
        HP_CUDA(cudaMemcpyAsync(part, d, sizeof(hp::u32) * g->g.n, cudaMemcpyDeviceToHost, ctx->c.stream));
        ctx->c.sync();
        *obj = o;
        *maxw = mw;
        ctx->c.arena.front_release(fm);
    });
}

int hp_jet_begin(hp_ctx *ctx, const hp_graph *g, uint32_t k, int32_t lmax, const uint32_t *part,
                 const uint32_t *hier, const int32_t *dist, uint32_t levels, hp_jet **out) {
    if (!ctx || !g || !part || !out || k == 0) return HP_ERR_ARG;
    *out = nullptr;
    hp_jet *j = new (std::nothrow) hp_jet();
    if (!j) return HP_ERR_OOM;
    j->ctx = ctx;
    j->front_mark = ctx->c.arena.front_mark();
    j->back_mark = ctx->c.arena.back_mark();
    int rc = guarded(ctx, [&] {
        if (hier) {
            check_hier(hier, dist, levels);
            j->D = hp::make_dist_oracle(ctx->c, vec_u32(hier, levels), vec_s32(dist, levels));
            j->has_D = true;
            if (j->D.k != k) throw hp::HpError{HP_ERR_ARG, "k must equal the product of the hierarchy"};
        }
        for (uint32_t u = 0; u < g->g.n; ++u)
            if (part[u] >= k) throw hp::HpError{HP_ERR_ARG, "partition label out of range"};
        hp::u32 *d = ctx->c.balloc<hp::u32>(g->g.n);
        HP_CUDA(cudaMemcpyAsync(d, part, sizeof(hp::u32) * g->g.n, cudaMemcpyHostToDevice, ctx->c.stream));
        j->L.setup(ctx->c, g->g, k, lmax, j->has_D ? &j->D : nullptr, d);
        ctx->c.sync();
    });
    if (rc != HP_OK) {
        ctx->c.arena.back_release(j->back_mark);
        ctx->c.arena.front_release(j->front_mark);
        delete j;
        return rc;
    }
    *out = j;
    return HP_OK;
}

static int jet_moves_out(hp_jet *j, uint32_t *moves, uint32_t *count) {
    hp::Ctx &c = j->ctx->c;
    const hp::DevStatus &st = c.read_status();
    if (st.err) throw hp::HpError{HP_ERR_DEVICE, "Jet kernel reported error bits " + std::to_string(st.err)};
    const hp::u32 nm = st.cnt[hp::ST_MOVES];
    if (count) *count = nm;
    if (moves && nm) {
        HP_CUDA(cudaMemcpyAsync(moves, j->L.moves, sizeof(hp::u32) * nm, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        std::sort(moves, moves + nm);
    }
    return HP_OK;
}

int hp_jet_lp(hp_jet *j, uint32_t ratio_pct, uint32_t *moves, uint32_t *count) {
    if (!j) return HP_ERR_ARG;
    return guarded(j->ctx, [&] {
        j->L.lp(ratio_pct);
        jet_moves_out(j, moves, count);
    });
}

int hp_jet_weak(hp_jet *j, uint32_t *moves, uint32_t *count) {
    if (!j) return HP_ERR_ARG;
    return guarded(j->ctx, [&] {
        j->L.weak();
        jet_moves_out(j, moves, count);
    });
}

int hp_jet_strong(hp_jet *j, uint32_t *moves, uint32_t *count) {
    if (!j) return HP_ERR_ARG;
    return guarded(j->ctx, [&] {
        j->L.strong();
        jet_moves_out(j, moves, count);
    });
}

int hp_jet_perform(hp_jet *j, int64_t *obj, int32_t *maxw) {
    if (!j) return HP_ERR_ARG;
    return guarded(j->ctx, [&] {
        j->L.perform();
        const hp::DevStatus &st = j->ctx->c.read_status();
        if (st.err) throw hp::HpError{HP_ERR_DEVICE, "Jet kernel reported error bits " + std::to_string(st.err)};
        const hp::s64 d = st.sum[hp::SUM_DELTA];
        if (obj) *obj += j->has_D ? d : d / 2;
        if (maxw) *maxw = st.imax[hp::MAX_BW];
    });
}

int hp_jet_state(hp_jet *j, uint32_t *map, int32_t *bw, uint32_t *dest_part, int32_t *gain1, uint32_t *lock,
                 uint32_t *dest_cache, int32_t *gain_cache) {
    if (!j) return HP_ERR_ARG;
    return guarded(j->ctx, [&] {
        hp::Ctx &c = j->ctx->c;
        const size_t n = j->L.g.n;
        auto cp = [&](void *dst, const void *src, size_t bytes) {
            if (dst) HP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c.stream));
        };
        cp(map, j->L.map, 4 * n);
        cp(bw, j->L.bw, 4 * (size_t) j->L.k);
        cp(dest_part, j->L.dest_part, 4 * n);
        cp(gain1, j->L.gain1, 4 * n);
        cp(lock, j->L.lock, 4 * n);
        cp(dest_cache, j->L.dest_cache, 4 * n);
        cp(gain_cache, j->L.gain_cache, 4 * n);
        c.sync();
    });
}

int hp_jet_end(hp_jet *j) {
    if (!j) return HP_ERR_ARG;
    j->ctx->c.arena.back_release(j->back_mark);
    j->ctx->c.arena.front_release(j->front_mark);
    delete j;
    return HP_OK;
}

int hp_edge_cut(hp_ctx *ctx, const hp_graph *g, const uint32_t *part, int64_t *cut) {
    if (!ctx || !g || !part || !cut) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        hp::ScratchScope ss(ctx->c.arena);
        hp::u32 *d = ctx->c.balloc<hp::u32>(g->g.n);
        HP_CUDA(cudaMemcpyAsync(d, part, sizeof(hp::u32) * g->g.n, cudaMemcpyHostToDevice, ctx->c.stream));
        *cut = hp::edge_cut_dev(ctx->c, g->g, d);
    });
}

int hp_comm_cost(hp_ctx *ctx, const hp_graph *g, const uint32_t *part, const uint32_t *hier, const int32_t *dist,
                 uint32_t levels, int64_t *J) {
    if (!ctx || !g || !part || !J) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        check_hier(hier, dist, levels);
        const size_t fm = ctx->c.arena.front_mark();
        hp::ScratchScope ss(ctx->c.arena);
        hp::DistOracle D = hp::make_dist_oracle(ctx->c, vec_u32(hier, levels), vec_s32(dist, levels));
        hp::u32 *d = ctx->c.balloc<hp::u32>(g->g.n);
        HP_CUDA(cudaMemcpyAsync(d, part, sizeof(hp::u32) * g->g.n, cudaMemcpyHostToDevice, ctx->c.stream));
        *J = hp::comm_cost_dev(ctx->c, g->g, d, D);
        ctx->c.arena.front_release(fm);
    });
}

int hp_partition_graph(hp_ctx *ctx, const hp_graph *g, uint32_t k, double imbalance, int ultra, uint64_t seed,
                       uint32_t *part, int64_t *cut) {
    if (!ctx || !g || !part || k == 0) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        const size_t fm = ctx->c.arena.front_mark();
        hp::u32 *d = ctx->c.falloc<hp::u32>(g->g.n);
        ctx->last = hp::SolveStats();
        hp::s64 c = hp::solve_partition(ctx->c, g->g, k, imbalance, ultra != 0, seed, d, &ctx->last);
        HP_CUDA(cudaMemcpyAsync(part, d, sizeof(hp::u32) * g->g.n, cudaMemcpyDeviceToHost, ctx->c.stream));
        ctx->c.sync();
        ctx->c.arena.front_release(fm);
        if (cut) *cut = c;
    });
}

int hp_partition(hp_ctx *ctx, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj, const int32_t *ew,
                 const int32_t *vw, uint32_t k, double imbalance, int ultra, uint64_t seed, uint32_t *part,
                 int64_t *cut) {
    if (!ctx || !part || k == 0) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        const size_t fm = ctx->c.arena.front_mark();
        try {
            hp::DGraph g = hp::graph_upload(ctx->c, n, m, xadj, adj, ew, vw);
            hp::u32 *d = ctx->c.falloc<hp::u32>(n);
            ctx->last = hp::SolveStats();
            hp::s64 c = hp::solve_partition(ctx->c, g, k, imbalance, ultra != 0, seed, d, &ctx->last);
            HP_CUDA(cudaMemcpyAsync(part, d, sizeof(hp::u32) * n, cudaMemcpyDeviceToHost, ctx->c.stream));
            ctx->c.sync();
            if (cut) *cut = c;
        } catch (...) {
            ctx->c.arena.front_release(fm);
            throw;
        }
        ctx->c.arena.front_release(fm);
    });
}

int hp_map_graph(hp_ctx *ctx, const hp_graph *g, const uint32_t *hier, const int32_t *dist, uint32_t levels,
                 double imbalance, int mode, uint64_t seed, uint32_t *part, int64_t *J) {
    if (!ctx || !g || !part || mode < 0 || mode > 2) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        check_hier(hier, dist, levels);
        const size_t fm = ctx->c.arena.front_mark();
        hp::u32 *d = ctx->c.falloc<hp::u32>(g->g.n);
        ctx->last = hp::SolveStats();
        hp::s64 j = hp::solve_mapping(ctx->c, g->g, vec_u32(hier, levels), vec_s32(dist, levels), imbalance, mode,
                                      seed, d, &ctx->last);
        HP_CUDA(cudaMemcpyAsync(part, d, sizeof(hp::u32) * g->g.n, cudaMemcpyDeviceToHost, ctx->c.stream));
        ctx->c.sync();
        ctx->c.arena.front_release(fm);
        if (J) *J = j;
    });
}

int hp_map(hp_ctx *ctx, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj, const int32_t *ew,
           const int32_t *vw, const uint32_t *hier, const int32_t *dist, uint32_t levels, double imbalance, int mode,
           uint64_t seed, uint32_t *part, int64_t *J) {
    if (!ctx || !part || mode < 0 || mode > 2) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        check_hier(hier, dist, levels);
        const size_t fm = ctx->c.arena.front_mark();
        try {
            hp::DGraph g = hp::graph_upload(ctx->c, n, m, xadj, adj, ew, vw);
            hp::u32 *d = ctx->c.falloc<hp::u32>(n);
            ctx->last = hp::SolveStats();
            hp::s64 j = hp::solve_mapping(ctx->c, g, vec_u32(hier, levels), vec_s32(dist, levels), imbalance, mode,
                                          seed, d, &ctx->last);
            HP_CUDA(cudaMemcpyAsync(part, d, sizeof(hp::u32) * n, cudaMemcpyDeviceToHost, ctx->c.stream));
            ctx->c.sync();
            if (J) *J = j;
        } catch (...) {
            ctx->c.arena.front_release(fm);
            throw;
        }
        ctx->c.arena.front_release(fm);
    });
}

namespace {

// Device bytes one request may use (input graph, hierarchy, Jet scratch);
// rounded up by the service.
size_t request_bytes(uint32_t n, uint64_t m, const int32_t *ew, const int32_t *vw) {
    return hp::request_estimate(n, m, ew != nullptr, vw != nullptr);
}

std::function<hp::s64(hp::Ctx &)> partition_job(uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj,
                                                 const int32_t *ew, const int32_t *vw, uint32_t k, double imbalance,
                                                 int ultra, uint64_t seed, uint32_t *part) {
    return [=](hp::Ctx &c) -> hp::s64 {
        hp::DGraph g = hp::graph_upload(c, n, m, xadj, adj, ew, vw);
        hp::u32 *d = c.falloc<hp::u32>(n);
        const hp::s64 cut = hp::solve_partition(c, g, k, imbalance, ultra != 0, seed, d, nullptr);
        HP_CUDA(cudaMemcpyAsync(part, d, sizeof(hp::u32) * n, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        return cut;
    };
}

std::function<hp::s64(hp::Ctx &)> mapping_job(uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj,
                                               const int32_t *ew, const int32_t *vw, std::vector<hp::u32> hier,
                                               std::vector<hp::s32> dist, double imbalance, int mode, uint64_t seed,
                                               uint32_t *part) {
    return [=](hp::Ctx &c) -> hp::s64 {
        hp::DGraph g = hp::graph_upload(c, n, m, xadj, adj, ew, vw);
        hp::u32 *d = c.falloc<hp::u32>(n);
        const hp::s64 J = hp::solve_mapping(c, g, hier, dist, imbalance, mode, seed, d, nullptr);
        HP_CUDA(cudaMemcpyAsync(part, d, sizeof(hp::u32) * n, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        return J;
    };
}

}  // namespace

int hp_partition_batch(hp_ctx *ctx, hp_batch_item *items, uint32_t count, uint32_t workers) {
    if (!ctx || (count && !items)) return HP_ERR_ARG;
    for (uint32_t i = 0; i < count; ++i)
        if (!items[i].part || items[i].k == 0) return HP_ERR_ARG;
    int first_error = HP_OK;
    const int rc = guarded(ctx, [&] {
        hp::ScratchScope ss(ctx->c.arena);
        const size_t free_bytes = ctx->c.arena.back_mark() - ctx->c.arena.front_mark();
        char *base = ctx->c.balloc<char>(free_bytes);
        std::vector<hp::u64> ids(count);
        {
            hp::Service svc(ctx->c, base, free_bytes, workers ? workers : 8);
            for (uint32_t i = 0; i < count; ++i) {
                hp_batch_item &it = items[i];
                auto job = std::make_shared<hp::Job>();
                job->bytes = request_bytes(it.n, it.m, it.ew, it.vw);
                job->run = partition_job(it.n, it.m, it.xadj, it.adj, it.ew, it.vw, it.k, it.imbalance, it.ultra,
                                         it.seed, it.part);
                ids[i] = svc.submit(job);
            }
            for (uint32_t i = 0; i < count; ++i) {
                std::shared_ptr<hp::Job> j = svc.wait(ids[i]);
                items[i].status = j->status;
                items[i].cut = j->objective;
                if (j->status != HP_OK && first_error == HP_OK) {
                    first_error = j->status;
                    ctx->c.last_error = "batch item " + std::to_string(i) + ": " + j->error;
                }
            }
        }
    });
    if (rc != HP_OK) return rc;
    return first_error;
}

int hp_server_create(int device, size_t buffer_bytes, uint32_t workers, hp_server **out) {
    if (!out || buffer_bytes == 0) return HP_ERR_ARG;
    *out = nullptr;
    hp_server *s = new (std::nothrow) hp_server();
    if (!s) return HP_ERR_OOM;
    int rc = guarded_host([&] {
        s->c.init(device, buffer_bytes);
        s->svc.reset(new hp::Service(s->c, s->c.arena.base(), s->c.arena.capacity(), workers ? workers : 8));
    });
    if (rc != HP_OK) {
        s->svc.reset();
        s->c.destroy();
        delete s;
        return rc;
    }
    *out = s;
    return HP_OK;
}

int hp_server_destroy(hp_server *s) {
    if (!s) return HP_ERR_ARG;
    s->svc.reset();  // finishes every queued request, then stops the workers
    s->c.destroy();
    delete s;
    return HP_OK;
}

const char *hp_server_last_error(hp_server *s) { return s ? s->last_error.c_str() : "null server"; }

int hp_server_submit_partition(hp_server *s, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj,
                               const int32_t *ew, const int32_t *vw, uint32_t k, double imbalance, int ultra,
                               uint64_t seed, uint32_t *part, uint64_t *request) {
    if (!s || !xadj || (m && !adj) || !part || !request || k == 0) return HP_ERR_ARG;
    return guarded_host([&] {
        auto job = std::make_shared<hp::Job>();
        job->bytes = request_bytes(n, m, ew, vw);
        job->run = partition_job(n, m, xadj, adj, ew, vw, k, imbalance, ultra, seed, part);
        *request = s->svc->submit(job);
    });
}

int hp_server_submit_map(hp_server *s, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj,
                         const int32_t *ew, const int32_t *vw, const uint32_t *hier, const int32_t *dist,
                         uint32_t levels, double imbalance, int mode, uint64_t seed, uint32_t *part,
                         uint64_t *request) {
    if (!s || !xadj || (m && !adj) || !part || !request || mode < 0 || mode > 2) return HP_ERR_ARG;
    return guarded_host([&] {
        check_hier(hier, dist, levels);
        auto job = std::make_shared<hp::Job>();
        job->bytes = request_bytes(n, m, ew, vw);
        job->run = mapping_job(n, m, xadj, adj, ew, vw, vec_u32(hier, levels), vec_s32(dist, levels), imbalance, mode,
                               seed, part);
        *request = s->svc->submit(job);
    });
}

int hp_server_poll(hp_server *s, uint64_t request, int *done) {
    if (!s || !done) return HP_ERR_ARG;
    *done = s->svc->is_done(request) ? 1 : 0;
    return HP_OK;
}

int hp_server_wait(hp_server *s, uint64_t request, int64_t *objective, double *latency_ms, double *run_ms) {
    if (!s) return HP_ERR_ARG;
    std::shared_ptr<hp::Job> j = s->svc->wait(request);
    if (!j) return HP_ERR_ARG;
    if (objective) *objective = j->objective;
    if (latency_ms) *latency_ms = j->t_end - j->t_submit;
    if (run_ms) *run_ms = j->t_end - j->t_start;
    if (j->status != HP_OK) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->last_error = j->error;
    }
    return j->status;
}

int hp_last_solve_stats(const hp_ctx *ctx, double *ms5, int64_t *initial_obj, int32_t *lmax, uint32_t *levels) {
    if (!ctx) return HP_ERR_ARG;
    const hp::SolveStats &s = ctx->last;
    if (ms5) {
        ms5[0] = s.coarsening_ms;
        ms5[1] = s.contraction_ms;
        ms5[2] = s.initial_ms;
        ms5[3] = s.uncontraction_ms;
        ms5[4] = s.refinement_ms;
    }
    if (initial_obj) *initial_obj = s.initial_obj;
    if (lmax) *lmax = s.lmax;
    if (levels) *levels = s.levels;
    return HP_OK;
}

int hp_last_solve_maxw(const hp_ctx *ctx, int32_t *initial_maxw, int32_t *final_maxw) {
    if (!ctx) return HP_ERR_ARG;
    if (initial_maxw) *initial_maxw = ctx->last.initial_maxw;
    if (final_maxw) *final_maxw = ctx->last.final_maxw;
    return HP_OK;
}

int hp_last_solve_level(const hp_ctx *ctx, uint32_t index, uint32_t *n, uint64_t *m) {
    if (!ctx || index >= ctx->last.level_n.size()) return HP_ERR_ARG;
    if (n) *n = ctx->last.level_n[index];
    if (m) *m = ctx->last.level_m[index];
    return HP_OK;
}

int hp_tune(hp_ctx *ctx, const char *name, int64_t value) {
    if (!ctx || !name || value < 0) return HP_ERR_ARG;
    hp::Tunables &t = ctx->c.tune;
    const std::string nm(name);
    if (nm == "jet_graph_max_m") t.jet_graph_max_m = (uint64_t) value;
    else if (nm == "order_small_n") t.order_small_n = (uint32_t) std::min<int64_t>(value, 0xFFFFFFFFll);
    else if (nm == "match_coop_max_n") t.match_coop_max_n = (uint32_t) std::min<int64_t>(value, 0xFFFFFFFFll);
    else if (nm == "match_coop_max_m") t.match_coop_max_m = (uint64_t) value;
    else if (nm == "jet_fused_max_n") t.jet_fused_max_n = (uint32_t) std::min<int64_t>(value, 0xFFFFFFFFll);
    else if (nm == "jet_fused_max_m") t.jet_fused_max_m = (uint64_t) value;
    else if (nm == "jet_coop_max_n") t.jet_coop_max_n = (uint32_t) std::min<int64_t>(value, 0xFFFFFFFFll);
    else if (nm == "jet_coop_max_m") t.jet_coop_max_m = (uint64_t) value;
    else if (nm == "jet_coop_max_deg") t.jet_coop_max_deg = (uint32_t) std::min<int64_t>(value, 0xFFFFFFFFll);
    else if (nm == "jet_coop_rows") t.jet_coop_rows = (uint32_t) std::min<int64_t>(value, 0xFFFFFFFFll);
    else if (nm == "jet_hub_deg") t.jet_hub_deg = (uint32_t) std::min<int64_t>(value, 0xFFFFFFFFll);
    else if (nm == "jet_chunk_mode" && value <= 2) t.jet_chunk_mode = (uint32_t) value;
    else if (nm == "jet_hub_conn" && value <= 1) t.jet_hub_conn = (uint32_t) value;
    else if (nm == "jet_hub_track_pct") t.jet_hub_track_pct = (uint32_t) std::min<int64_t>(value, 1000000);
    else if (nm == "jet_inval_all_pct" && value >= 1 && value <= 100) t.jet_inval_all_pct = (uint32_t) value;
    else if (nm == "jet_vec_loads" && value <= 1) t.jet_vec_loads = (uint32_t) value;
    else {
        ctx->c.last_error = "unknown tunable " + nm;
        return HP_ERR_ARG;
    }
    return HP_OK;
}

int hp_instrument(hp_ctx *ctx, int enable) {
    if (!ctx) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->c.sync();
        ctx->c.instr.clear();
        ctx->c.instr.enabled = enable != 0;
    });
}

int hp_kernel_timing(hp_ctx *ctx, const char *name, uint64_t *launches, double *ms, double *bytes) {
    if (!ctx || !name) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->c.sync();
        ctx->c.instr.resolve();
        uint64_t l = 0;
        double t = 0, b = 0;
        for (const auto &x: ctx->c.instr.totals)
            if (x.name == name) {
                l = x.launches;
                t = x.ms;
                b = x.bytes;
            }
        if (launches) *launches = l;
        if (ms) *ms = t;
        if (bytes) *bytes = b;
    });
}

int hp_kernel_log(hp_ctx *ctx, uint64_t index, char *name, size_t name_len, double *ms, double *bytes) {
    if (!ctx) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        if (index == 0) {
            ctx->c.sync();
            ctx->c.instr.resolve();
        }
        const auto &log = ctx->c.instr.log;
        if (index >= log.size()) throw hp::HpError{HP_ERR_ARG, "kernel log index past the end"};
        const auto &r = log[index];
        if (name && name_len) {
            const size_t k = std::min(name_len - 1, r.name.size());
            std::memcpy(name, r.name.data(), k);
            name[k] = 0;
        }
        if (ms) *ms = r.ms;
        if (bytes) *bytes = r.bytes;
    });
}

int hp_event_record(hp_ctx *ctx, int slot) {
    if (!ctx) return HP_ERR_ARG;
    return guarded(ctx, [&] { HP_CUDA(cudaEventRecord(ctx->c.event(slot), ctx->c.stream)); });
}

int hp_event_elapsed(hp_ctx *ctx, int slot_a, int slot_b, float *ms) {
    if (!ctx || !ms) return HP_ERR_ARG;
    return guarded(ctx, [&] {
        cudaEvent_t b = ctx->c.event(slot_b);
        HP_CUDA(cudaEventSynchronize(b));
        HP_CUDA(cudaEventElapsedTime(ms, ctx->c.event(slot_a), b));
    });
}

uint64_t hp_kernel_launches(void) { return hp::g_kernel_launches.load(); }

int hp_profile(hp_ctx *ctx, int enable) {
    if (!ctx) return HP_ERR_ARG;
    ctx->c.prof.enabled = enable != 0;
    ctx->c.prof.clear();
    return HP_OK;
}

int hp_profile_entry(const hp_ctx *ctx, uint32_t index, char *name, size_t name_len, double *ms, uint64_t *count) {
    if (!ctx || index >= ctx->c.prof.totals.size()) return HP_ERR_ARG;
    const auto &e = ctx->c.prof.totals[index];
    if (name && name_len) {
        std::strncpy(name, e.first.c_str(), name_len - 1);
        name[name_len - 1] = 0;
    }
    if (ms) *ms = e.second;
    if (count) *count = ctx->c.prof.counts[index].second;
    return HP_OK;
}

int hp_read_metis(const char *path, hp_host_graph **out) {
    if (!path || !out) return HP_ERR_ARG;
    *out = nullptr;
    hp_host_graph *h = new (std::nothrow) hp_host_graph();
    if (!h) return HP_ERR_OOM;
    std::string err;
    if (hp::read_metis(path, h->g, err) != 0) {
        delete h;
        return HP_ERR_IO;
    }
    *out = h;
    return HP_OK;
}

int hp_gen_grid(uint32_t w, uint32_t h, int32_t w_lo, int32_t w_hi, uint64_t seed, hp_host_graph **out) {
    if (!out) return HP_ERR_ARG;
    return guarded_host([&] { *out = new hp_host_graph{hp::gen_grid(w, h, w_lo, w_hi, seed)}; });
}

int hp_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, int32_t w_lo, int32_t w_hi,
                uint64_t seed, int explicit_vw, hp_host_graph **out) {
    if (!out || scale > 31) return HP_ERR_ARG;
    return guarded_host([&] {
        *out = new hp_host_graph{hp::gen_rmat(scale, edge_factor, a, b, c, w_lo, w_hi, seed, explicit_vw != 0)};
    });
}

int hp_gen_rgg3d(uint32_t n, double mean_degree, int32_t w_lo, int32_t w_hi, uint64_t seed, int explicit_vw,
                 hp_host_graph **out) {
    if (!out || n < 2) return HP_ERR_ARG;
    return guarded_host(
        [&] { *out = new hp_host_graph{hp::gen_rgg3d(n, mean_degree, w_lo, w_hi, seed, explicit_vw != 0)}; });
}

int hp_host_graph_info(const hp_host_graph *g, uint32_t *n, uint64_t *m, int *has_ew, int *has_vw) {
    if (!g) return HP_ERR_ARG;
    if (n) *n = g->g.n;
    if (m) *m = g->g.m;
    if (has_ew) *has_ew = !g->g.ew.empty();
    if (has_vw) *has_vw = !g->g.vw.empty();
    return HP_OK;
}

int hp_host_graph_copy(const hp_host_graph *g, uint32_t *xadj, uint32_t *adj, int32_t *ew, int32_t *vw) {
    if (!g) return HP_ERR_ARG;
    const hp::HostCSR &h = g->g;
    if (xadj) std::copy(h.xadj.begin(), h.xadj.end(), xadj);
    if (adj) std::copy(h.adj.begin(), h.adj.end(), adj);
    if (ew) {
        if (h.ew.empty()) std::fill(ew, ew + h.m, 1);
        else std::copy(h.ew.begin(), h.ew.end(), ew);
    }
    if (vw) {
        if (h.vw.empty()) std::fill(vw, vw + h.n, 1);
        else std::copy(h.vw.begin(), h.vw.end(), vw);
    }
    return HP_OK;
}

int hp_host_graph_free(hp_host_graph *g) {
    delete g;
    return HP_OK;
}

int hp_write_metis(const char *path, uint32_t n, uint64_t m, const uint32_t *xadj, const uint32_t *adj,
                   const int32_t *ew, const int32_t *vw) {
    if (!path || !xadj || (m && !adj)) return HP_ERR_ARG;
    return guarded_host([&] {
        hp::HostCSR g;
        g.n = n;
        g.m = (hp::u32) m;
        g.xadj.assign(xadj, xadj + n + 1);
        g.adj.assign(adj, adj + m);
        if (ew) g.ew.assign(ew, ew + m);
        if (vw) g.vw.assign(vw, vw + n);
        std::string err;
        if (hp::write_metis(path, g, vw != nullptr, ew != nullptr, err) != 0) throw hp::HpError{HP_ERR_IO, err};
    });
}

int hp_write_partition(const char *path, const uint32_t *part, uint32_t n) {
    if (!path || (n && !part)) return HP_ERR_ARG;
    std::string err;
    return hp::write_partition(path, part, n, err) == 0 ? HP_OK : HP_ERR_IO;
}

} // extern "C"
