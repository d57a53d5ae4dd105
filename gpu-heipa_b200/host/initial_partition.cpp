// Host-side initial partitioning of the coarsest graph: the reference's
// METIS-derived k-way partitioner (restated in metis_kway.cpp) and the
// hierarchy recursion of the IM initial mapping. See initial_partition.h.
#include "initial_partition.h"

#include <algorithm>
#include <cmath>
#include <numeric>

#include "metis_kway.h"

namespace hp {

void initial_kway(const HostCSR &hg, u32 k, double eps, u64 seed, std::vector<u32> &part) {
    part.assign(hg.n, 0);
    if (k <= 1 || hg.n == 0) return;
    // kway_core.h:1548-1571: the imbalance is narrowed to float and the seed
    // to int before ModifiedMetis::partition
    metis_kway(hg.n, hg.xadj.data(), hg.adj.data(), hg.vw.empty() ? nullptr : hg.vw.data(),
               hg.ew.empty() ? nullptr : hg.ew.data(), (int) k, (float) eps, (int) seed, part.data());
}

double adaptive_imbalance(double global_eps, s64 global_w, u32 global_k, s64 local_w, u32 local_k_rem, u64 depth) {
    double local = (1.0 + global_eps) * ((double) ((u64) local_k_rem * (u64) global_w) /
                                         (double) ((u64) global_k * (u64) local_w));
    return std::pow(local, 1.0 / (double) depth) - 1.0;
}

void sort_rows(HostCSR &g) {
    std::vector<std::pair<u32, s32> > row;
    for (u32 u = 0; u < g.n; ++u) {
        row.clear();
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) row.emplace_back(g.adj[j], g.ew.empty() ? 1 : g.ew[j]);
        std::sort(row.begin(), row.end());
        u32 j = g.xadj[u];
        for (auto &p: row) {
            g.adj[j] = p.first;
            if (!g.ew.empty()) g.ew[j] = p.second;
            ++j;
        }
    }
}

HostCSR induced_subgraph(const HostCSR &g, const std::vector<u32> &part, u32 id, std::vector<u32> &n_to_o) {
    std::vector<u32> local(g.n, SENTINEL);
    n_to_o.clear();
    for (u32 u = 0; u < g.n; ++u)
        if (part[u] == id) {
            local[u] = (u32) n_to_o.size();
            n_to_o.push_back(u);
        }
    HostCSR r;
    r.n = (u32) n_to_o.size();
    r.xadj.assign(r.n + 1, 0);
    r.vw.resize(r.n);
    for (u32 i = 0; i < r.n; ++i) {
        u32 u = n_to_o[i];
        r.vw[i] = g.vw.empty() ? 1 : g.vw[u];
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            u32 v = g.adj[j];
            if (part[v] != id) continue;
            r.adj.push_back(local[v]);
            r.ew.push_back(g.ew.empty() ? 1 : g.ew[j]);
        }
        r.xadj[i + 1] = (u32) r.adj.size();
    }
    r.m = (u32) r.adj.size();
    return r;
}

namespace {
void gms_recurse(const HostCSR &g, const std::vector<u32> &n_to_o, const std::vector<u32> &hierarchy, u32 level,
                 std::vector<u32> &identifier, const std::vector<u32> &index_vec, const std::vector<u32> &k_rem,
                 double eps, s64 global_w, u32 global_k, u64 seed, std::vector<u32> &global_part) {
    const u32 l = (u32) hierarchy.size();
    const u32 k_here = hierarchy[level];
    const u64 depth = identifier.size();
    const s64 local_w = g.total_vw();
    double imb = local_w > 0 ? adaptive_imbalance(eps, global_w, global_k, local_w, k_rem[l - 1 - depth], l - depth)
                             : eps;
    std::vector<u32> tmp;
    initial_kway(g, k_here, imb, seed, tmp);
    if (depth == l - 1) {
        u32 offset = 0;
        for (u32 i = 0; i + 1 < l; ++i) offset += identifier[i] * index_vec[index_vec.size() - 1 - i];
        for (u32 u = 0; u < g.n; ++u) global_part[n_to_o[u]] = offset + tmp[u];
        return;
    }
    for (u32 id = 0; id < k_here; ++id) {
        std::vector<u32> sub_n_to_o;
        HostCSR sub = induced_subgraph(g, tmp, id, sub_n_to_o);
        for (u32 &x: sub_n_to_o) x = n_to_o[x];
        identifier.push_back(id);
        gms_recurse(sub, sub_n_to_o, hierarchy, level - 1, identifier, index_vec, k_rem, eps, global_w, global_k, seed,
                    global_part);
        identifier.pop_back();
    }
}
} // namespace

void global_multisection(const HostCSR &g, const std::vector<u32> &hierarchy, double eps, u64 seed,
                         std::vector<u32> &part) {
    const u32 l = (u32) hierarchy.size();
    part.assign(g.n, 0);
    if (l == 0 || g.n == 0) return;
    std::vector<u32> index_vec = {1};
    for (u32 i = 0; i + 1 < l; ++i) index_vec.push_back(index_vec[i] * hierarchy[i]);
    std::vector<u32> k_rem(l);
    u32 p = 1;
    for (u32 i = 0; i < l; ++i) {
        k_rem[i] = p * hierarchy[i];
        p *= hierarchy[i];
    }
    std::vector<u32> n_to_o(g.n);
    std::iota(n_to_o.begin(), n_to_o.end(), 0u);
    std::vector<u32> identifier;
    gms_recurse(g, n_to_o, hierarchy, l - 1, identifier, index_vec, k_rem, eps, g.total_vw(), p, seed, part);
}

} // namespace hp
