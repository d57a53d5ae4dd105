// Host initial partitioner: multilevel recursive bisection + greedy k-way
// refinement. See initial_partition.h for the contract.
#include "initial_partition.h"

#include <algorithm>
#include <cmath>
#include <numeric>

#include <omp.h>

namespace hp {
namespace {

struct IGraph {
    u32 n = 0;
    std::vector<u32> xadj, adj;
    std::vector<s32> ew, vw;
    s64 W = 0;
};

IGraph to_igraph(const HostCSR &g) {
    IGraph r;
    r.n = g.n;
    r.xadj.assign(g.xadj.begin(), g.xadj.end());
    r.adj.assign(g.adj.begin(), g.adj.end());
    if (g.ew.empty()) r.ew.assign(g.m, 1);
    else r.ew.assign(g.ew.begin(), g.ew.end());
    if (g.vw.empty()) r.vw.assign(g.n, 1);
    else r.vw.assign(g.vw.begin(), g.vw.end());
    r.W = 0;
    for (s32 w: r.vw) r.W += w;
    if (r.xadj.empty()) r.xadj.assign(1, 0);
    return r;
}

// Indexed binary max-heap on s64 keys; ties go to the lower vertex id.
struct MaxHeap {
    std::vector<u32> heap;
    std::vector<s32> pos;
    std::vector<s64> key;

    void init(u32 n) {
        heap.clear();
        pos.assign(n, -1);
        key.assign(n, 0);
    }
    bool above(u32 a, u32 b) const { return key[a] > key[b] || (key[a] == key[b] && a < b); }
    void swap_at(size_t i, size_t j) {
        std::swap(heap[i], heap[j]);
        pos[heap[i]] = (s32) i;
        pos[heap[j]] = (s32) j;
    }
    void up(size_t i) {
        while (i > 0) {
            size_t p = (i - 1) / 2;
            if (!above(heap[i], heap[p])) break;
            swap_at(i, p);
            i = p;
        }
    }
    void down(size_t i) {
        for (;;) {
            size_t l = 2 * i + 1, r = l + 1, b = i;
            if (l < heap.size() && above(heap[l], heap[b])) b = l;
            if (r < heap.size() && above(heap[r], heap[b])) b = r;
            if (b == i) break;
            swap_at(i, b);
            i = b;
        }
    }
    bool contains(u32 v) const { return pos[v] >= 0; }
    bool empty() const { return heap.empty(); }
    u32 top() const { return heap[0]; }
    void push(u32 v, s64 k) {
        key[v] = k;
        pos[v] = (s32) heap.size();
        heap.push_back(v);
        up(heap.size() - 1);
    }
    void update(u32 v, s64 k) {
        s64 old = key[v];
        key[v] = k;
        if (k > old) up((size_t) pos[v]);
        else down((size_t) pos[v]);
    }
    void remove(u32 v) {
        size_t i = (size_t) pos[v];
        size_t last = heap.size() - 1;
        if (i != last) {
            swap_at(i, last);
            heap.pop_back();
            pos[v] = -1;
            up(i);
            down(i);
        } else {
            heap.pop_back();
            pos[v] = -1;
        }
    }
};

// Heavy-edge matching + contraction for the bisection hierarchy.
IGraph coarsen_hem(const IGraph &g, Rng64 &rng, s64 maxvw, std::vector<u32> &cmap) {
    const u32 n = g.n;
    std::vector<u32> order(n);
    std::iota(order.begin(), order.end(), 0u);
    for (u32 i = n; i > 1; --i) std::swap(order[i - 1], order[rng.below(i)]);
    std::vector<u32> match(n, SENTINEL);
    for (u32 u: order) {
        if (match[u] != SENTINEL) continue;
        u32 best = u;
        s32 bw = 0;
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            u32 v = g.adj[j];
            if (v == u || match[v] != SENTINEL) continue;
            if ((s64) g.vw[u] + g.vw[v] > maxvw) continue;
            if (g.ew[j] > bw) {
                bw = g.ew[j];
                best = v;
            }
        }
        match[u] = best;
        match[best] = u;
    }
    cmap.assign(n, SENTINEL);
    u32 nc = 0;
    for (u32 u = 0; u < n; ++u) {
        if (cmap[u] != SENTINEL) continue;
        cmap[u] = nc;
        cmap[match[u]] = nc;
        ++nc;
    }
    IGraph c;
    c.n = nc;
    c.W = g.W;
    c.vw.assign(nc, 0);
    c.xadj.assign(nc + 1, 0);
    std::vector<s32> acc(nc, 0);
    std::vector<u32> touched;
    std::vector<u32> first(nc, SENTINEL);
    // members of each coarse vertex in ascending fine id
    std::vector<u32> mem0(nc, SENTINEL), mem1(nc, SENTINEL);
    for (u32 u = 0; u < n; ++u) {
        u32 cu = cmap[u];
        c.vw[cu] += g.vw[u];
        if (mem0[cu] == SENTINEL) mem0[cu] = u;
        else mem1[cu] = u;
    }
    for (u32 cu = 0; cu < nc; ++cu) {
        touched.clear();
        for (u32 mi = 0; mi < 2; ++mi) {
            u32 u = mi == 0 ? mem0[cu] : mem1[cu];
            if (u == SENTINEL) continue;
            for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
                u32 cv = cmap[g.adj[j]];
                if (cv == cu) continue;
                if (acc[cv] == 0) touched.push_back(cv);
                acc[cv] += g.ew[j];
            }
        }
        std::sort(touched.begin(), touched.end());
        for (u32 cv: touched) {
            c.adj.push_back(cv);
            c.ew.push_back(acc[cv]);
            acc[cv] = 0;
        }
        c.xadj[cu + 1] = (u32) c.adj.size();
    }
    return c;
}

s64 overload(const s64 pw[2], const s64 maxw[2]) {
    return std::max<s64>(0, pw[0] - maxw[0]) + std::max<s64>(0, pw[1] - maxw[1]);
}

// Greedy graph growing: side 0 is grown from the seed vertex `start` (drawn
// at random by the caller, start < n) until it reaches target0.
void grow_bisection(const IGraph &g, s64 target0, u32 start, std::vector<u8> &side) {
    const u32 n = g.n;
    side.assign(n, 1);
    if (n == 0) return;
    std::vector<s64> gain(n, 0);
    for (u32 u = 0; u < n; ++u) {
        s64 s = 0;
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) s += g.ew[j];
        gain[u] = -s;
    }
    MaxHeap heap;
    heap.init(n);
    s64 w0 = 0;
    u32 scan = start;
    heap.push(start, gain[start]);
    u32 added = 0;
    while (w0 < target0 && added < n) {
        if (heap.empty()) {
            // disconnected remainder: continue from the next unassigned vertex
            u32 v = SENTINEL;
            for (u32 t = 0; t < n; ++t) {
                u32 c = (scan + t) % n;
                if (side[c] == 1) {
                    v = c;
                    break;
                }
            }
            if (v == SENTINEL) break;
            scan = v;
            heap.push(v, gain[v]);
        }
        u32 v = heap.top();
        heap.remove(v);
        side[v] = 0;
        w0 += g.vw[v];
        ++added;
        for (u32 j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
            u32 u = g.adj[j];
            if (side[u] != 1) continue;
            gain[u] += 2 * (s64) g.ew[j];
            if (heap.contains(u)) heap.update(u, gain[u]);
            else heap.push(u, gain[u]);
        }
    }
}

// 2-way FM refinement with balance constraints; returns the resulting cut.
s64 fm_refine(const IGraph &g, std::vector<u8> &side, s64 pw[2], const s64 maxw[2], int passes) {
    const u32 n = g.n;
    std::vector<s64> ext(n, 0), intl(n, 0);
    s64 cut = 0;
    for (u32 u = 0; u < n; ++u) {
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            if (side[g.adj[j]] != side[u]) ext[u] += g.ew[j];
            else intl[u] += g.ew[j];
        }
        cut += ext[u];
    }
    cut /= 2;
    MaxHeap heap[2];
    std::vector<u8> locked(n, 0);
    std::vector<u32> log;
    const u32 limit = std::max<u32>(64, n / 16);
    for (int pass = 0; pass < passes; ++pass) {
        heap[0].init(n);
        heap[1].init(n);
        std::fill(locked.begin(), locked.end(), 0);
        bool unbalanced = overload(pw, maxw) > 0;
        for (u32 u = 0; u < n; ++u)
            if (ext[u] > 0 || unbalanced) heap[side[u]].push(u, ext[u] - intl[u]);
        log.clear();
        s64 best_cut = cut, best_ov = overload(pw, maxw);
        size_t best_len = 0;
        u32 streak = 0;
        for (;;) {
            int from = -1;
            if (pw[0] > maxw[0]) from = 0;
            else if (pw[1] > maxw[1]) from = 1;
            // drop infeasible tops lazily by trying both sides
            u32 cand[2] = {SENTINEL, SENTINEL};
            for (int s = 0; s < 2; ++s) {
                if (heap[s].empty()) continue;
                u32 v = heap[s].top();
                if (pw[1 - s] + g.vw[v] <= maxw[1 - s] || from == s) cand[s] = v;
            }
            if (from == -1) {
                if (cand[0] == SENTINEL && cand[1] == SENTINEL) break;
                if (cand[0] == SENTINEL) from = 1;
                else if (cand[1] == SENTINEL) from = 0;
                else from = heap[0].above(cand[0], cand[1]) ? 0 : 1;
            } else if (cand[from] == SENTINEL) {
                break;
            }
            u32 v = cand[from];
            heap[from].remove(v);
            locked[v] = 1;
            s64 gv = ext[v] - intl[v];
            cut -= gv;
            pw[from] -= g.vw[v];
            pw[1 - from] += g.vw[v];
            side[v] = (u8) (1 - from);
            std::swap(ext[v], intl[v]);
            for (u32 j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
                u32 u = g.adj[j];
                s64 w = g.ew[j];
                if (side[u] == side[v]) {
                    ext[u] -= w;
                    intl[u] += w;
                } else {
                    ext[u] += w;
                    intl[u] -= w;
                }
                if (locked[u]) continue;
                s64 gu = ext[u] - intl[u];
                if (heap[side[u]].contains(u)) heap[side[u]].update(u, gu);
                else if (ext[u] > 0) heap[side[u]].push(u, gu);
            }
            log.push_back(v);
            s64 ov = overload(pw, maxw);
            if (ov < best_ov || (ov == best_ov && cut < best_cut)) {
                best_ov = ov;
                best_cut = cut;
                best_len = log.size();
                streak = 0;
            } else if (++streak > limit) {
                break;
            }
        }
        // roll back to the best prefix
        for (size_t i = log.size(); i > best_len; --i) {
            u32 v = log[i - 1];
            int s = side[v];
            s64 gv = ext[v] - intl[v];
            cut -= gv;
            pw[s] -= g.vw[v];
            pw[1 - s] += g.vw[v];
            side[v] = (u8) (1 - s);
            std::swap(ext[v], intl[v]);
            for (u32 j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
                u32 u = g.adj[j];
                s64 w = g.ew[j];
                if (side[u] == side[v]) {
                    ext[u] -= w;
                    intl[u] += w;
                } else {
                    ext[u] += w;
                    intl[u] -= w;
                }
            }
        }
        if (best_len == 0) break;
    }
    return cut;
}

void side_weights(const IGraph &g, const std::vector<u8> &side, s64 pw[2]) {
    pw[0] = pw[1] = 0;
    for (u32 u = 0; u < g.n; ++u) pw[side[u]] += g.vw[u];
}

constexpr int BISECTION_TRIES = 8;
thread_local int t_threads = BISECTION_TRIES;  // set_initial_partition_threads

// Multilevel bisection with side 0 targeting `target0`.
void multilevel_bisect(const IGraph &g, s64 target0, double ub, Rng64 &rng, std::vector<u8> &side) {
    const s64 maxw[2] = {(s64) std::floor((double) target0 * ub), (s64) std::floor((double) (g.W - target0) * ub)};
    std::vector<IGraph> levels;
    std::vector<std::vector<u32> > cmaps;
    const IGraph *cur = &g;
    const u32 threshold = 64;
    while (cur->n > threshold) {
        std::vector<u32> cmap;
        s64 maxvw = std::max<s64>(1, (s64) (1.5 * (double) g.W / (double) threshold));
        IGraph c = coarsen_hem(*cur, rng, maxvw, cmap);
        if ((double) c.n > 0.9 * (double) cur->n) break;
        levels.push_back(std::move(c));
        cmaps.push_back(std::move(cmap));
        cur = &levels.back();
    }
    // initial bisection on the coarsest level: best of several grown tries.
    // The seed vertices are drawn in order first; the tries are independent
    // and run on up to t_threads host threads, and the best one is chosen in
    // try order, so the result does not depend on the threads.
    const int tries = BISECTION_TRIES;
    if (cur->n == 0) {
        side.assign(g.n, 1);
        return;
    }
    u32 starts[tries];
    for (int t = 0; t < tries; ++t) starts[t] = rng.below(cur->n);
    std::vector<u8> try_side[tries];
    s64 try_cut[tries], try_ov[tries];
    const int nt = std::max(1, std::min(tries, t_threads));
#pragma omp parallel for num_threads(nt) schedule(static, 1) if (nt > 1)
    for (int t = 0; t < tries; ++t) {
        grow_bisection(*cur, target0, starts[t], try_side[t]);
        s64 pw[2];
        side_weights(*cur, try_side[t], pw);
        try_cut[t] = fm_refine(*cur, try_side[t], pw, maxw, 4);
        try_ov[t] = overload(pw, maxw);
    }
    int bt = 0;
    for (int t = 1; t < tries; ++t)
        if (try_ov[t] < try_ov[bt] || (try_ov[t] == try_ov[bt] && try_cut[t] < try_cut[bt])) bt = t;
    std::vector<u8> best_side;
    best_side.swap(try_side[bt]);
    // project and refine
    for (size_t li = levels.size(); li > 0; --li) {
        const IGraph &fine = (li >= 2) ? levels[li - 2] : g;
        const std::vector<u32> &cmap = cmaps[li - 1];
        std::vector<u8> fs(fine.n);
        for (u32 u = 0; u < fine.n; ++u) fs[u] = best_side[cmap[u]];
        s64 pw[2];
        side_weights(fine, fs, pw);
        fm_refine(fine, fs, pw, maxw, 4);
        best_side.swap(fs);
    }
    side.swap(best_side);
}

IGraph sub_igraph(const IGraph &g, const std::vector<u8> &side, u8 s, std::vector<u32> &ids) {
    std::vector<u32> local(g.n, SENTINEL);
    ids.clear();
    for (u32 u = 0; u < g.n; ++u)
        if (side[u] == s) {
            local[u] = (u32) ids.size();
            ids.push_back(u);
        }
    IGraph r;
    r.n = (u32) ids.size();
    r.xadj.assign(r.n + 1, 0);
    r.vw.resize(r.n);
    r.W = 0;
    for (u32 i = 0; i < r.n; ++i) {
        u32 u = ids[i];
        r.vw[i] = g.vw[u];
        r.W += g.vw[u];
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            u32 v = g.adj[j];
            if (side[v] != s) continue;
            r.adj.push_back(local[v]);
            r.ew.push_back(g.ew[j]);
        }
        r.xadj[i + 1] = (u32) r.adj.size();
    }
    return r;
}

void recursive_bisect(const IGraph &g, const std::vector<u32> &ids, u32 k, u32 first, double ub, Rng64 &rng,
                      std::vector<u32> &part) {
    if (k == 1 || g.n == 0) {
        for (u32 i = 0; i < g.n; ++i) part[ids[i]] = first;
        return;
    }
    const u32 k0 = k / 2, k1 = k - k0;
    const s64 target0 = (s64) ((double) g.W * (double) k0 / (double) k + 0.5);
    std::vector<u8> side;
    multilevel_bisect(g, target0, ub, rng, side);
    for (int s = 0; s < 2; ++s) {
        std::vector<u32> sub_ids;
        IGraph sub = sub_igraph(g, side, (u8) s, sub_ids);
        for (u32 &x: sub_ids) x = ids[x];
        recursive_bisect(sub, sub_ids, s == 0 ? k0 : k1, s == 0 ? first : first + k0, ub, rng, part);
    }
}

// Greedy k-way pass: first restores balance, then takes positive-gain moves.
void kway_refine(const IGraph &g, u32 k, s64 lmax, std::vector<u32> &part, int passes) {
    std::vector<s64> bw(k, 0);
    for (u32 u = 0; u < g.n; ++u) bw[part[u]] += g.vw[u];
    std::vector<s64> conn(k, 0);
    std::vector<u32> touched;
    for (int pass = 0; pass < passes; ++pass) {
        u32 moved = 0;
        for (u32 u = 0; u < g.n; ++u) {
            const u32 own = part[u];
            touched.clear();
            for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
                u32 b = part[g.adj[j]];
                if (conn[b] == 0) touched.push_back(b);
                conn[b] += g.ew[j];
            }
            const s64 own_conn = conn[own];
            const s64 w = g.vw[u];
            u32 best = SENTINEL;
            s64 best_gain = 0;
            if (bw[own] > lmax) {
                // balance move: best adjacent block that fits, else lightest block
                for (u32 b: touched) {
                    if (b == own || bw[b] + w > lmax) continue;
                    s64 gn = conn[b] - own_conn;
                    if (best == SENTINEL || gn > best_gain || (gn == best_gain && bw[b] < bw[best])) {
                        best = b;
                        best_gain = gn;
                    }
                }
                if (best == SENTINEL) {
                    u32 light = 0;
                    for (u32 b = 1; b < k; ++b)
                        if (bw[b] < bw[light]) light = b;
                    if (light != own && bw[light] + w <= lmax) best = light;
                }
            } else {
                for (u32 b: touched) {
                    if (b == own || bw[b] + w > lmax) continue;
                    s64 gn = conn[b] - own_conn;
                    if (gn > best_gain || (gn == best_gain && gn > 0 && bw[b] < bw[best])) {
                        best = b;
                        best_gain = gn;
                    }
                }
                if (best_gain <= 0) best = SENTINEL;
            }
            for (u32 b: touched) conn[b] = 0;
            if (best != SENTINEL) {
                bw[own] -= w;
                bw[best] += w;
                part[u] = best;
                ++moved;
            }
        }
        if (moved == 0) break;
    }
}

} // namespace

void set_initial_partition_threads(int threads) { t_threads = threads; }

void initial_kway(const HostCSR &hg, u32 k, double eps, u64 seed, std::vector<u32> &part) {
    part.assign(hg.n, 0);
    if (k <= 1 || hg.n == 0) return;
    IGraph g = to_igraph(hg);
    Rng64 rng(seed ^ 0x5EEDC0FFEEull);
    const double depth = std::ceil(std::log2((double) k));
    const double ub = std::pow(1.0 + std::max(0.0, eps), 1.0 / std::max(1.0, depth));
    std::vector<u32> ids(g.n);
    std::iota(ids.begin(), ids.end(), 0u);
    recursive_bisect(g, ids, k, 0, ub, rng, part);
    const s64 lmax = (s64) std::ceil((1.0 + eps) * ((double) g.W / (double) k));
    kway_refine(g, k, lmax, part, 8);
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
