// ORACLE — test infrastructure only (see oracle.h). CPU restatement of the
// reference's partitioning path with deterministic rules where the reference
// races. Every function cites the reference lines it follows; paths are
// relative to the GPU-HeiPa source tree.
//
// Deterministic rules used where the reference is race- or order-dependent
// (the CUDA implementation follows the same rules):
//  R1 matching commit (two_hop_matching.h:313-333): when several proposers
//     target the same receiver in one sub-round, the smallest proposer id wins.
//  R2 leaf/twin/relative pairing (two_hop_matching.h:205-253, 485-515): the
//     candidates are grouped by exact digest value and paired in ascending
//     vertex id within each group ((1st,2nd), (3rd,4th), ...).
//  R3 relative digest ties (two_hop_matching.h:545-565): min degree, then max
//     edge weight, then lowest neighbour id.
//  R4 best-block ties (jet_label_propagation.h:207-222, 657-670;
//     promap_jet_label_propagation.h:240-250): lowest block id.
//  R5 rebalance mini-bucket order (jet_label_propagation.h:439, 684): vertices
//     in one mini-bucket are ordered by vertex id (instead of atomic order).
//  R6 strong-rebalance fallback (jet_label_propagation.h:568-583): vertices
//     whose chunk does not hold half their weight take fallback slots in
//     ascending vertex id order.
//  R7 block-connectivity rows hold exactly the blocks with positive
//     connection (the reference may keep stale zero-weight entries).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include <omp.h>
#include <parallel/algorithm>

#include "../gpu-heipa_b200/host/hp_types.h"
#include "../gpu-heipa_b200/host/initial_partition.h"

using namespace hp;

namespace {

inline s32 EW(const HostCSR &g, u32 j) { return g.ew.empty() ? 1 : g.ew[j]; }
inline s32 VW(const HostCSR &g, u32 u) { return g.vw.empty() ? 1 : g.vw[u]; }
inline s32 wadd(s32 a, s32 b) { return (s32) ((u32) a + (u32) b); }
inline s32 wsub(s32 a, s32 b) { return (s32) ((u32) a - (u32) b); }
inline s32 wmul(s32 a, s32 b) { return (s32) ((u32) a * (u32) b); }
inline u32 deg(const HostCSR &g, u32 u) { return g.xadj[u + 1] - g.xadj[u]; }

// The indices i in [0, n) with pred(i), ascending, selected on all host
// threads (pred must be a pure function of i). Every loop below that the
// reference runs as a filter or stable compaction uses it, so the order of
// the result is the same as a one-thread scan.
template<typename P>
std::vector<u32> par_select(u32 n, P pred) {
    const int T = omp_get_max_threads();
    std::vector<size_t> cnt((size_t) T + 1, 0);
    std::vector<u32> out;
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const u32 lo = (u32) ((u64) n * (u64) t / (u64) nt), hi = (u32) ((u64) n * (u64) (t + 1) / (u64) nt);
        size_t c = 0;
        for (u32 i = lo; i < hi; ++i) c += pred(i) ? 1 : 0;
        cnt[(size_t) t + 1] = c;
#pragma omp barrier
#pragma omp single
        {
            for (int i = 0; i < nt; ++i) cnt[(size_t) i + 1] += cnt[(size_t) i];
            out.resize(cnt[(size_t) nt]);
        }
        size_t o = cnt[(size_t) t];
        for (u32 i = lo; i < hi; ++i)
            if (pred(i)) out[o++] = i;
    }
    return out;
}

// Relaxed atomic accesses for the few words that concurrent iterations of a
// parallel loop share (results do not depend on the interleaving).
inline u32 ld_relaxed(const u32 *p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline void st_relaxed(u32 *p, u32 v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
inline void atomic_min_u32(u32 *p, u32 v) {
    u32 cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (v < cur && !__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
}

constexpr u32 N_MAX_ITERATIONS = 12;      // jet_label_propagation.h:36
constexpr u32 N_MAX_WEAK_ITERATIONS = 2;  // jet_label_propagation.h:37
constexpr u32 MAX_SECTIONS = 128;         // jet_label_propagation.h:41
constexpr u32 MAX_BUCKETS = 50;           // jet_label_propagation.h:42
constexpr u32 MATCH_SEED = 12345u;        // two_hop_matching.h:590

u32 xorshift32(u32 x) {
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    return x;
}

u32 rotl32(u32 x, int r) { return (x << r) | (x >> (32 - r)); }

// MurmurHash3_x86_32 of one little-endian 4-byte block (Kokkos pod_hash<u32>).
u32 murmur3_u32(u32 key, u32 seed) {
    const u32 c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    u32 h = seed;
    u32 k = key;
    k *= c1;
    k = rotl32(k, 15);
    k *= c2;
    h ^= k;
    h = rotl32(h, 13);
    h = h * 5u + 0xe6546b64u;
    h ^= 4u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// jet_label_propagation.h:147-180 as an exact integer rule: with g = -gx/vwgt,
// g >= 1 -> 25 + min{k : 1.5^k >= g}, capped at 49; g < 1 -> 25 - min{k :
// 1.5^k >= 1/g}, floored at 2.
u32 gain_bucket(s32 gx, s32 vwgt) {
    if (gx > 0) return 0;
    if (gx == 0) return 1;
    unsigned __int128 a = (unsigned __int128) (-(s64) gx);
    unsigned __int128 b = (unsigned __int128) (vwgt < 1 ? 1 : vwgt);
    if (a >= b) {
        u32 k = 0;
        unsigned __int128 p2 = 1, p3 = 1;
        while (k < 24 && a * p2 > b * p3) {
            ++k;
            p2 *= 2;
            p3 *= 3;
        }
        return 25 + k;
    } else {
        u32 k = 0;
        unsigned __int128 p2 = 1, p3 = 1;
        while (k < 23 && b * p2 > a * p3) {
            ++k;
            p2 *= 2;
            p3 *= 3;
        }
        return 25 - k;
    }
}

u32 gain_bucket_float(s32 gx, s32 vwgt) {
    if (gx > 0) return 0;
    if (gx == 0) return 1;
    const float g = (float) (-gx) / (float) vwgt;
    int b = 25;
    const float INV = 1.0f / 0.5849625007211562f;
    const float EPS = 1e-6f;
    if (g < 1.0f) {
        const float x = (-std::log2(g)) * INV;
        const int k = (int) std::ceil(x - EPS);
        b -= k;
        if (b < 2) b = 2;
    } else {
        const float x = std::log2(g) * INV;
        const int k = (int) std::ceil(x - EPS);
        b += k;
        if (b > 49) b = 49;
    }
    return (u32) b;
}

// ---------------------------------------------------------------------------
// Coarsening: two_hop_matching.h:93-650
// ---------------------------------------------------------------------------

// pick_neighbor_flat two_hop_matching.h:102-141 (the team variant :143-188
// selects the same vertex for positive weights).
u32 pick(const HostCSR &g, const std::vector<u32> &vcmap, u32 u, u32 seed, bool initial) {
    const bool uniform = g.ew.empty();
    u32 h = SENTINEL;
    u32 r = xorshift32(u ^ seed);
    s32 max_ewt = 0;
    u32 tiebreaker = 0;
    for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
        u32 v = g.adj[j];
        if (!(initial || vcmap[v] == SENTINEL)) continue;
        if (!uniform) {
            s32 w = g.ew[j];
            if (max_ewt < w) {
                max_ewt = w;
                h = v;
                tiebreaker = xorshift32(v + r);
                continue;
            }
            if (max_ewt != w) continue;
        }
        u32 tb = xorshift32(v + r);
        if (tb >= tiebreaker) {
            h = v;
            tiebreaker = tb;
        }
    }
    return h;
}

// matchHash two_hop_matching.h:205-253 under rule R2.
template<typename D>
void pair_by_digest(const std::vector<u32> &cands, const std::vector<D> &dig, std::vector<u32> &vcmap) {
    // (digest, index) pairs are unique, so any sort gives the stable order
    std::vector<std::pair<D, u32> > kv(cands.size());
    for (size_t i = 0; i < cands.size(); ++i) kv[i] = {dig[i], (u32) i};
    __gnu_parallel::sort(kv.begin(), kv.end());
    std::vector<u32> idx(cands.size());
    for (size_t i = 0; i < cands.size(); ++i) idx[i] = kv[i].second;
    size_t i = 0;
    while (i < idx.size()) {
        size_t j = i;
        while (j < idx.size() && dig[idx[j]] == dig[idx[i]]) ++j;
        for (size_t p = i; p + 1 < j; p += 2) {
            u32 a = cands[idx[p]], b = cands[idx[p + 1]];
            u32 cv = a < b ? a : b;
            vcmap[a] = cv;
            vcmap[b] = cv;
        }
        i = j;
    }
}

u32 count_unmapped(const std::vector<u32> &vcmap) {
    u64 c = 0;
#pragma omp parallel for schedule(static) reduction(+ : c)
    for (s64 i = 0; i < (s64) vcmap.size(); ++i) c += vcmap[(size_t) i] == SENTINEL;
    return (u32) c;
}

u32 match(const HostCSR &g, std::vector<u32> &mapping) {
    const u32 n = g.n;
    std::vector<u32> vcmap(n, SENTINEL), hn(n, SENTINEL);
    const u32 seed = MATCH_SEED;
    const bool uniform = g.ew.empty();
    // initial pick: two_hop_matching.h:276-304
#pragma omp parallel for schedule(dynamic, 1024)
    for (s64 ii = 0; ii < (s64) n; ++ii) {  // reads vcmap, writes hn[i] only
        const u32 i = (u32) ii;
        if (uniform) {
            u32 d = deg(g, i);
            if (d == 0) continue;
            hn[i] = g.adj[g.xadj[i] + (xorshift32(i ^ seed) % d)];
        } else {
            hn[i] = pick(g, vcmap, i, seed, true);
        }
    }
    // main loop: two_hop_matching.h:306-392
    std::vector<u32> list(n);
    std::iota(list.begin(), list.end(), 0u);
    std::vector<u32> claim(n, SENTINEL);
    u32 round = 0;
    while (!list.empty()) {
        const u32 round_seed = seed ^ (round * 0x9e3779b1u);
        const s64 L = (s64) list.size();
        for (u32 r = 0; r < 4; ++r) {
#pragma omp parallel for schedule(static)
            for (s64 li = 0; li < L; ++li) {  // commit_p1 (writes vcmap[u] of its own u only)
                const u32 u = list[(size_t) li];
                u32 v = hn[u];
                if (v == SENTINEL || vcmap[u] != SENTINEL) continue;
                bool cond = r > 0 ? (murmur3_u32(u + r, 0) < murmur3_u32(v + r, 0)) : (u < v);
                if (!cond) vcmap[u] = SENTINEL - 1;
            }
            // commit_p2, rule R1: the smallest proposer of each receiver wins.
            // Proposers (vcmap SENTINEL) and receivers (SENTINEL - 1) are
            // disjoint and each proposer targets one receiver, so the pairs
            // do not depend on the order in which they are written.
#pragma omp parallel for schedule(static)
            for (s64 li = 0; li < L; ++li) {
                const u32 u = list[(size_t) li];
                u32 v = hn[u];
                if (v == SENTINEL || vcmap[u] != SENTINEL) continue;
                if (vcmap[v] != SENTINEL - 1) continue;
                atomic_min_u32(&claim[v], u);
            }
#pragma omp parallel for schedule(static)
            for (s64 li = 0; li < L; ++li) {
                const u32 u = list[(size_t) li];
                u32 v = hn[u];
                if (v == SENTINEL || ld_relaxed(&vcmap[u]) != SENTINEL || ld_relaxed(&claim[v]) != u) continue;
                u32 cv = u < v ? u : v;
                st_relaxed(&vcmap[v], cv);
                vcmap[u] = cv;
            }
#pragma omp parallel for schedule(static)
            for (s64 li = 0; li < L; ++li) {
                const u32 u = list[(size_t) li];
                u32 v = hn[u];
                if (v != SENTINEL && ld_relaxed(&claim[v]) != SENTINEL) st_relaxed(&claim[v], SENTINEL);
            }
#pragma omp parallel for schedule(static)
            for (s64 li = 0; li < L; ++li) {  // commit_p3
                const u32 u = list[(size_t) li];
                if (vcmap[u] == SENTINEL - 1) vcmap[u] = SENTINEL;
            }
        }
#pragma omp parallel for schedule(dynamic, 1024)
        for (s64 li = 0; li < (s64) list.size(); ++li) {  // re-pick (reads vcmap, writes hn[u] only)
            const u32 u = list[(size_t) li];
            if (vcmap[u] != SENTINEL || hn[u] == SENTINEL || vcmap[hn[u]] == SENTINEL) continue;
            hn[u] = pick(g, vcmap, u, round_seed, false);
        }
        std::vector<u32> keep = par_select((u32) list.size(), [&](u32 li) {  // compact
            const u32 u = list[li];
            return vcmap[u] == SENTINEL && hn[u] != SENTINEL;
        });
        for (u32 &x: keep) x = list[x];
        list.swap(keep);
        ++round;
    }
    u32 unmapped = count_unmapped(vcmap);
    // leaf matching: two_hop_matching.h:395-425
    if ((u64) unmapped * 4 > (u64) n) {
        std::vector<u32> c, d;
        for (u32 i = 0; i < n; ++i)
            if (vcmap[i] == SENTINEL && deg(g, i) == 1) {
                c.push_back(i);
                d.push_back(g.adj[g.xadj[i]]);
            }
        pair_by_digest(c, d, vcmap);
        unmapped = count_unmapped(vcmap);
    }
    // twin matching: two_hop_matching.h:427-524
    if ((u64) unmapped * 4 > (u64) n) {
        std::vector<u32> c = par_select(n, [&](u32 i) { return vcmap[i] == SENTINEL; });
        std::vector<u64> d(c.size());
#pragma omp parallel for schedule(dynamic, 1024)
        for (s64 ci = 0; ci < (s64) c.size(); ++ci) {
            const u32 i = c[(size_t) ci];
            u64 h = 0;
            for (u32 j = g.xadj[i]; j < g.xadj[i + 1]; ++j) {
                u64 y = murmur3_u32(g.adj[j], 0);
                h += y * y + y;
            }
            d[(size_t) ci] = h;
        }
        pair_by_digest(c, d, vcmap);
        unmapped = count_unmapped(vcmap);
    }
    // relative matching: two_hop_matching.h:526-571, rule R3
    if ((u64) unmapped * 4 > (u64) n) {
        std::vector<u32> c = par_select(n, [&](u32 i) { return vcmap[i] == SENTINEL; });
        std::vector<u32> d(c.size());
#pragma omp parallel for schedule(dynamic, 1024)
        for (s64 ci = 0; ci < (s64) c.size(); ++ci) {
            const u32 i = c[(size_t) ci];
            u32 h = SENTINEL;
            s32 max_wgt = 0;
            u32 min_deg = SENTINEL;
            for (u32 j = g.xadj[i]; j < g.xadj[i + 1]; ++j) {
                u32 v = g.adj[j];
                u32 vd = deg(g, v);
                s32 w = EW(g, j);
                if (min_deg > vd) {
                    min_deg = vd;
                    max_wgt = w;
                    h = v;
                } else if (min_deg == vd && (max_wgt < w || (max_wgt == w && v < h))) {
                    h = v;
                    max_wgt = w;
                }
            }
            d[(size_t) ci] = h;
        }
        pair_by_digest(c, d, vcmap);
    }
    // coarse ids: two_hop_matching.h:611-641
    for (u32 i = 0; i < n; ++i)
        if (vcmap[i] == SENTINEL) vcmap[i] = i;
    mapping.assign(n, 0);
    std::vector<u32> rank(n, SENTINEL);
    u32 nc = 0;
    for (u32 i = 0; i < n; ++i)
        if (vcmap[i] == i) rank[i] = nc++;
    for (u32 i = 0; i < n; ++i) mapping[i] = rank[vcmap[i]];
    return nc;
}

// graph.h:127-390: coarse vertex weight = sum of member weights; coarse edge
// weight = sum over fine edges between the two clusters; no self loops.
// Rows are emitted sorted by neighbour id.
HostCSR contract(const HostCSR &g, const std::vector<u32> &mapping, u32 nc) {
    HostCSR c;
    c.n = nc;
    c.vw.assign(nc, 0);
    for (u32 u = 0; u < g.n; ++u) c.vw[mapping[u]] = wadd(c.vw[mapping[u]], VW(g, u));
    std::vector<u32> moff(nc + 1, 0), mem(g.n);
    for (u32 u = 0; u < g.n; ++u) ++moff[mapping[u] + 1];
    for (u32 i = 0; i < nc; ++i) moff[i + 1] += moff[i];
    {
        std::vector<u32> cur(moff.begin(), moff.end() - 1);
        for (u32 u = 0; u < g.n; ++u) mem[cur[mapping[u]]++] = u;
    }
    // coarse rows on all threads, each with its own accumulator: every
    // thread writes the sorted rows of its coarse vertices into its own
    // buffer, then the rows are copied to their offsets
    c.xadj.assign(nc + 1, 0);
    const int T = omp_get_max_threads();
    std::vector<std::vector<u32> > badj((size_t) T);
    std::vector<std::vector<s32> > bew((size_t) T);
    std::vector<u64> where(nc);  // (thread << 40) | offset in that thread's buffer
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        std::vector<s32> acc(nc, 0);
        std::vector<u8> seen(nc, 0);
        std::vector<u32> touched;
        std::vector<u32> &ba = badj[(size_t) t];
        std::vector<s32> &be = bew[(size_t) t];
#pragma omp for schedule(dynamic, 256)
        for (s64 ci = 0; ci < (s64) nc; ++ci) {
            const u32 cu = (u32) ci;
            touched.clear();
            for (u32 q = moff[cu]; q < moff[cu + 1]; ++q) {
                u32 u = mem[q];
                for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
                    u32 cv = mapping[g.adj[j]];
                    if (cv == cu) continue;
                    if (!seen[cv]) {
                        seen[cv] = 1;
                        touched.push_back(cv);
                    }
                    acc[cv] = wadd(acc[cv], EW(g, j));
                }
            }
            std::sort(touched.begin(), touched.end());
            where[cu] = ((u64) t << 40) | (u64) ba.size();
            c.xadj[cu + 1] = (u32) touched.size();
            for (u32 cv: touched) {
                ba.push_back(cv);
                be.push_back(acc[cv]);
                acc[cv] = 0;
                seen[cv] = 0;
            }
        }
    }
    for (u32 i = 0; i < nc; ++i) c.xadj[i + 1] += c.xadj[i];
    c.m = c.xadj[nc];
    c.adj.resize(c.m);
    c.ew.resize(c.m);
#pragma omp parallel for schedule(dynamic, 1024)
    for (s64 ci = 0; ci < (s64) nc; ++ci) {
        const u32 cu = (u32) ci;
        const size_t t = (size_t) (where[cu] >> 40), off = (size_t) (where[cu] & ((1ull << 40) - 1));
        const u32 len = c.xadj[cu + 1] - c.xadj[cu];
        std::copy_n(badj[t].data() + off, len, c.adj.data() + c.xadj[cu]);
        std::copy_n(bew[t].data() + off, len, c.ew.data() + c.xadj[cu]);
    }
    return c;
}

// ---------------------------------------------------------------------------
// Distance oracle and objectives
// ---------------------------------------------------------------------------

// distance_oracle_matrix.h:64-81
std::vector<s32> distance_matrix(const std::vector<u32> &hier, const std::vector<s32> &dist) {
    u32 k = 1;
    for (u32 a: hier) k *= a;
    std::vector<s32> D((size_t) k * k, 0);
    const u32 l = (u32) hier.size();
    for (u32 i = 0; i < k; ++i)
        for (u32 j = 0; j < k; ++j) {
            if (i == j) continue;
            u32 level = 0, group = 1;
            for (; level < l; ++level) {
                group *= hier[level];
                if (i / group == j / group) break;
            }
            D[(size_t) i * k + j] = dist[level];
        }
    return D;
}

s64 edge_cut(const HostCSR &g, const std::vector<u32> &part) {
    s64 s = 0;
    for (u32 u = 0; u < g.n; ++u)
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j)
            if (part[u] != part[g.adj[j]]) s += EW(g, j);
    return s / 2;
}

s64 comm_cost(const HostCSR &g, const std::vector<u32> &part, const std::vector<s32> &D, u32 k) {
    s64 s = 0;
    for (u32 u = 0; u < g.n; ++u)
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j)
            s += (s64) EW(g, j) * D[(size_t) part[u] * k + part[g.adj[j]]];
    return s;
}

s32 lmax_of(s64 W, u32 k, double eps) { return (s32) std::ceil((1.0 + eps) * ((double) W / (double) k)); }

// ---------------------------------------------------------------------------
// Jet refinement: jet_label_propagation.h and promap_jet_label_propagation.h
// ---------------------------------------------------------------------------

// Connectivity row of one vertex (rule R7: the blocks adjacent to u with
// their connection weight, in first-seen order; every consumer breaks ties
// by the lowest block id explicitly). One per thread: the per-vertex
// loops of the Jet steps below read only state that the loop does not write,
// so they run on all host threads with the same results as one thread.
struct Conn {
    std::vector<s32> acc;
    std::vector<u32> touched;
    void build(const HostCSR &g, const std::vector<u32> &map, u32 u) {
        for (u32 b: touched) acc[b] = 0;
        touched.clear();
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            u32 b = map[g.adj[j]];
            if (acc[b] == 0) touched.push_back(b);
            acc[b] = wadd(acc[b], EW(g, j));
        }
    }
    s32 of(u32 b) const { return acc[b]; }
};

struct Jet {
    const HostCSR *g = nullptr;
    u32 n = 0, k = 0;
    s32 lmax = 0;
    s32 g_weight = 0;
    bool promap = false;
    std::vector<s32> D;  // k*k when promap
    std::vector<u32> map, dest_cache, dest_part, lock;
    std::vector<s32> bw, gain_cache, gain1;
    std::vector<Conn> conns;  // one per host thread
    std::vector<u8> moving;   // perform_moves scratch, all zero between calls

    s32 dist(u32 a, u32 b) const { return D[(size_t) a * k + b]; }
    Conn &conn(u32 u) {
        Conn &c = conns[(size_t) omp_get_thread_num()];
        c.build(*g, map, u);
        return c;
    }
};

void jet_init(Jet &J, const HostCSR &g, u32 k, s32 lmax, const u32 *part) {
    J.g = &g;
    J.n = g.n;
    J.k = k;
    J.lmax = lmax;
    s64 W = g.total_vw();
    J.g_weight = (s32) W;
    J.map.assign(part, part + g.n);
    J.bw.assign(k, 0);
    for (u32 u = 0; u < g.n; ++u) J.bw[J.map[u]] = wadd(J.bw[J.map[u]], VW(g, u));
    J.dest_cache.assign(g.n, NULL_PART);
    J.gain_cache.assign(g.n, 0);
    J.dest_part.assign(g.n, NO_MOVE);
    J.lock.assign(g.n, 0);
    J.gain1.assign(g.n, 0);
    J.moving.assign(g.n, 0);
    J.conns.assign((size_t) omp_get_max_threads(), Conn{});
    for (Conn &c: J.conns) c.acc.assign(k, 0);
}

// jet_lp jet_label_propagation.h:182-354 (edge cut) and ProMap_jet_lp
// promap_jet_label_propagation.h:206-330 (J gains).
std::vector<u32> jet_lp(Jet &J, u32 ratio_pct) {
    const HostCSR &g = *J.g;
    const u32 n = J.n;
#pragma omp parallel for schedule(dynamic, 1024)
    for (s64 ui = 0; ui < (s64) n; ++ui) {  // best_block
        const u32 u = (u32) ui;
        if (J.dest_cache[u] != NULL_PART) {
            J.dest_part[u] = J.dest_cache[u];
            continue;
        }
        const Conn &C = J.conn(u);
        const u32 o = J.map[u];
        u32 best = NO_MOVE;
        s32 gain = 0;
        if (!J.promap) {
            const s32 own = C.of(o);
            s32 bc = 0;
            for (u32 b: C.touched) {
                if (b == o) continue;
                s32 c = C.of(b);
                if (c > bc || (c == bc && best != NO_MOVE && b < best)) {  // rule R4
                    bc = c;
                    best = b;
                }
            }
            if (best != NO_MOVE) {
                if (bc >= own || (s64) own - (s64) bc < ((s64) ratio_pct * (s64) own) / 100) gain = wsub(bc, own);
                else best = NO_MOVE;
            }
        } else {
            s32 bd = -1;
            for (u32 b: C.touched) {
                if (b == o) continue;
                s32 delta = 0;
                for (u32 id: C.touched) delta = wadd(delta, wmul(C.of(id), wsub(J.dist(o, id), J.dist(b, id))));
                if (delta > bd || (delta == bd && best != NO_MOVE && b < best)) {  // rule R4
                    bd = delta;
                    best = b;
                }
            }
            if (best != NO_MOVE) gain = bd;
        }
        J.gain_cache[u] = gain;
        J.dest_cache[u] = best;
        J.dest_part[u] = best;
    }
    std::vector<u8> viable(n);
#pragma omp parallel for schedule(static)
    for (s64 ui = 0; ui < (s64) n; ++ui) {  // filter potentially viable moves
        const u32 u = (u32) ui;
        viable[u] = J.dest_part[u] != NO_MOVE && J.lock[u] == 0;
        if (viable[u]) {
            J.gain1[u] = J.gain_cache[u];
        } else {
            J.gain1[u] = GAIN_MIN;
            J.lock[u] = 0;
        }
    }
    std::vector<u32> cands = par_select(n, [&](u32 u) { return viable[u] != 0; });
#pragma omp parallel for schedule(dynamic, 1024)
    for (s64 ci = 0; ci < (s64) cands.size(); ++ci) {  // afterburner (writes lock[u] only)
        const u32 u = cands[(size_t) ci];
        const s32 ug = J.gain1[u];
        const u32 ou = J.map[u], nu = J.dest_part[u];
        s32 change = 0;
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            u32 v = g.adj[j];
            s32 vg = J.gain1[v];
            bool first = vg > ug || (vg == ug && v < u);
            if (!first) continue;
            u32 nv = J.dest_part[v], ov = J.map[v];
            s32 w = EW(g, j);
            if (!J.promap) {
                s32 t = (s32) (nv == nu) - (s32) (nv == ou) + (s32) (ov == ou) - (s32) (ov == nu);
                change = wadd(change, wmul(w, t));
            } else {
                s32 before_u = wsub(J.dist(ou, ov), J.dist(nu, ov));
                s32 after_u = wsub(J.dist(ou, nv), J.dist(nu, nv));
                change = wadd(change, wmul(w, wsub(after_u, before_u)));
            }
        }
        if (wadd(ug, change) >= 0) J.lock[u] = 1;
    }
    std::vector<u32> moves = par_select((u32) cands.size(), [&](u32 ci) { return J.lock[cands[ci]] != 0; });
    for (u32 &x: moves) x = cands[x];
    return moves;
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

// Bucket bookkeeping shared by both rebalancers (rule R5): candidates ordered
// by (key, vertex id). prefix[i] = weight of all candidates before i in that
// order; B(x) = weight of candidates with key < x.
struct BucketOrder {
    std::vector<u32> keys_sorted;
    std::vector<s64> prefix_sorted;  // exclusive prefix in sorted order
    std::vector<s64> prefix;         // per candidate index
    void build(const std::vector<u32> &keys, const std::vector<s32> &w) {
        const size_t c = keys.size();
        // (key, candidate index) is unique, so sorting it gives the stable
        // order by key
        std::vector<u64> kv(c);
#pragma omp parallel for schedule(static)
        for (s64 i = 0; i < (s64) c; ++i) kv[(size_t) i] = ((u64) keys[(size_t) i] << 32) | (u64) i;
        __gnu_parallel::sort(kv.begin(), kv.end());
        keys_sorted.resize(c);
        prefix_sorted.resize(c + 1);
        prefix.resize(c);
        s64 run = 0;
        for (size_t i = 0; i < c; ++i) {
            const u32 id = (u32) kv[i];
            keys_sorted[i] = (u32) (kv[i] >> 32);
            prefix_sorted[i] = run;
            prefix[id] = run;
            run += w[id];
        }
        prefix_sorted[c] = run;
    }
    s64 B(u64 x) const {
        size_t pos = std::lower_bound(keys_sorted.begin(), keys_sorted.end(), x,
                                      [](u32 a, u64 b) { return (u64) a < b; }) - keys_sorted.begin();
        return prefix_sorted[pos];
    }
};

// The flagged vertices in ascending id with their keys and weights.
void collect_candidates(const HostCSR &g, const std::vector<u8> &is_cand, const std::vector<u32> &keyv,
                        std::vector<u32> &cands, std::vector<u32> &keys, std::vector<s32> &wts) {
    cands = par_select(g.n, [&](u32 u) { return is_cand[u] != 0; });
    keys.resize(cands.size());
    wts.resize(cands.size());
#pragma omp parallel for schedule(static)
    for (s64 i = 0; i < (s64) cands.size(); ++i) {
        keys[(size_t) i] = keyv[cands[(size_t) i]];
        wts[(size_t) i] = VW(g, cands[(size_t) i]);
    }
}

// rebalance_weak jet_label_propagation.h:592-751 (ProMap variant
// promap_jet_label_propagation.h:554-717 computes the same move set).
std::vector<u32> rebalance_weak(Jet &J) {
    const HostCSR &g = *J.g;
    const u32 n = J.n, k = J.k;
    const s32 lmax = J.lmax;
    const s32 opt = (J.g_weight + (s32) (k - 1)) / (s32) k;
    s32 max_b_w = (s32) ((99 * (s64) lmax) / 100);
    if (max_b_w < lmax - 100) max_b_w = lmax - 100;
    u32 sections, width;
    sections_of(n, k, sections, width);
    std::vector<u32> under;
    for (u32 b = 0; b < k; ++b)
        if (J.bw[b] < max_b_w) under.push_back(b);
    // per vertex (all threads): target and mini-bucket key; then the
    // candidates in ascending vertex id
    std::vector<u32> keyv(n);
    std::vector<u8> is_cand(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (s64 ui = 0; ui < (s64) n; ++ui) {
        const u32 u = (u32) ui;
        const u32 o = J.map[u];
        u32 best = o;
        s32 gn = 0;
        const s32 vw = VW(g, u);
        if (J.bw[o] > lmax && 2 * (s64) vw < 3 * ((s64) J.bw[o] - (s64) opt)) {
            const Conn &C = J.conn(u);
            s32 best_w = 0;
            const s32 own = C.of(o);
            for (u32 b: C.touched) {
                s32 c = C.of(b);
                if (J.bw[b] < max_b_w && (c > best_w || (c == best_w && best != o && b < best))) {  // rule R4
                    best = b;
                    best_w = c;
                }
            }
            gn = wsub(best_w, own);
            if (best_w <= 0) {
                if (!under.empty()) best = under[u % (u32) under.size()];
                gn = -own;
            }
        }
        J.dest_part[u] = best;
        if (o != best) {
            u32 gt = gain_bucket(gn, vw);
            keyv[u] = (MAX_BUCKETS * o + gt) * sections + (u % sections);
            is_cand[u] = 1;
        }
    }
    std::vector<u32> cands, keys;
    std::vector<s32> wts;
    collect_candidates(g, is_cand, keyv, cands, keys, wts);
    BucketOrder bo;
    bo.build(keys, wts);
    std::vector<u32> moves = par_select((u32) cands.size(), [&](u32 i) {
        u32 u = cands[i], o = J.map[u];
        s64 score = bo.prefix[i] - bo.B((u64) o * width);
        s64 limit = (s64) J.bw[o] - lmax;
        return score < limit;
    });
    for (u32 &x: moves) x = cands[x];
    return moves;
}

// rebalance_strong jet_label_propagation.h:356-590 (ProMap variant
// promap_jet_label_propagation.h:332-552 computes the same move set).
std::vector<u32> rebalance_strong(Jet &J) {
    const HostCSR &g = *J.g;
    const u32 n = J.n, k = J.k;
    const s32 lmax = J.lmax;
    const s32 opt = (J.g_weight + (s32) (k - 1)) / (s32) k;
    const s32 max_b_w = std::max<s32>(opt + 1, (s32) ((99 * (s64) lmax) / 100));
    u32 sections, width;
    sections_of(n, k, sections, width);
    s32 max_vwgt = INT32_MIN;  // find max size :377-385 (Max reducer identity)
    for (u32 b = 0; b < k; ++b)
        if (J.bw[b] < max_b_w && max_b_w - J.bw[b] > max_vwgt) max_vwgt = max_b_w - J.bw[b];
    std::vector<u32> keyv(n);
    std::vector<u8> is_cand(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (s64 ui = 0; ui < (s64) n; ++ui) {  // score_candidates :404-442
        const u32 u = (u32) ui;
        const u32 o = J.map[u];
        const s32 ow = J.bw[o];
        const s32 vw = VW(g, u);
        if (ow > lmax && (s64) vw <= 2 * (s64) max_vwgt && (s64) vw < 2 * ((s64) ow - (s64) opt)) {
            const Conn &C = J.conn(u);
            const s32 own = C.of(o);
            s32 count = 0, sum = 0;
            for (u32 b: C.touched) {
                if (b == o) continue;
                if (J.bw[b] < max_b_w) {
                    sum = wadd(sum, C.of(b));
                    ++count;
                }
            }
            if (count == 0) count = 1;
            s32 gn = wsub(sum / count, own);
            u32 gt = gain_bucket(gn, std::min<s32>(vw, ow - lmax));
            keyv[u] = (MAX_BUCKETS * o + gt) * sections + (u % sections) + 1;
            is_cand[u] = 1;
        }
    }
    std::vector<u32> cands, keys;
    std::vector<s32> wts;
    collect_candidates(g, is_cand, keyv, cands, keys, wts);
    BucketOrder bo;
    bo.build(keys, wts);
    std::vector<s64> evict_adjust(k, 0);
    std::vector<u32> moves;
    std::vector<s64> mscore;
    std::vector<s64> scores(cands.size());
#pragma omp parallel for schedule(static)
    for (s64 i = 0; i < (s64) cands.size(); ++i)
        scores[(size_t) i] = bo.prefix[(size_t) i] - bo.B((u64) J.map[cands[(size_t) i]] * width);
    for (size_t i = 0; i < cands.size(); ++i) {  // filter_scores :490-509
        u32 u = cands[i], o = J.map[u];
        s64 score = scores[i];
        s64 limit = (s64) J.bw[o] - lmax;
        if (score < limit) {
            if (score + VW(g, u) >= limit) evict_adjust[o] = score + VW(g, u);
            moves.push_back(u);
            mscore.push_back(bo.prefix[i]);
        }
    }
    // cookie cutter :524-551
    std::vector<s64> evict_start(k + 1, 0);
    s64 run = 0;
    for (u32 p = 0; p < k; ++p) {
        s64 add = evict_adjust[p];
        if (add == 0) add = bo.B((u64) (p + 1) * width) - bo.B((u64) p * width);
        evict_adjust[p] = bo.B((u64) p * width) - run;
        run += add;
    }
    s64 max_v = run;
    s64 run2 = 0;
    for (u32 p = 0; p < k; ++p) {
        if (max_b_w > J.bw[p]) run2 += (s64) max_b_w - J.bw[p];
        evict_start[p + 1] = run2;
    }
    // adjust_scores :560-584, rule R6
    for (size_t i = 0; i < moves.size(); ++i) {
        u32 u = moves[i], o = J.map[u];
        const s64 vw = VW(g, u);
        s64 tg = mscore[i] - evict_adjust[o];
        s32 id = 0;
        bool done = false;
        while (id < (s32) k) {
            while (id <= (s32) k && evict_start[id] <= tg) ++id;
            --id;
            if (id < (s32) k && vw / 2 <= evict_start[id + 1] - tg) {
                J.dest_part[u] = (u32) id;
                done = true;
                break;
            }
            if (id < (s32) k) {
                tg = max_v;
                max_v += vw;
            }
        }
        if (!done) J.dest_part[u] = o;
    }
    return moves;
}

// perform_moves jet_label_propagation.h:753-924 / ProMap_perform_moves
// promap_jet_label_propagation.h:1103-1216. The objective change is computed
// exactly from the old and new labels of both endpoints (directed sum; edge
// cut = directed/2, J = directed).
void perform_moves(Jet &J, const std::vector<u32> &moves, s64 &obj, s32 &maxw) {
    const HostCSR &g = *J.g;
    std::vector<u8> &moving = J.moving;
    const s64 M = (s64) moves.size();
#pragma omp parallel for schedule(static)
    for (s64 mi = 0; mi < M; ++mi) {
        const u32 u = moves[(size_t) mi];
        if (J.dest_part[u] != J.map[u]) moving[u] = 1;
    }
    s64 d = 0;  // exact integer sum: the same in any order
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : d)
    for (s64 mi = 0; mi < (s64) moves.size(); ++mi) {
        const u32 u = moves[(size_t) mi];
        if (!moving[u]) continue;
        const u32 ou = J.map[u], nu = J.dest_part[u];
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            u32 v = g.adj[j];
            u32 ov = J.map[v], nv = moving[v] ? J.dest_part[v] : ov;
            s64 w = EW(g, j);
            s64 c;
            if (!J.promap) c = w * ((s64) (nu != nv) - (s64) (ou != ov));
            else c = w * ((s64) J.dist(nu, nv) - (s64) J.dist(ou, ov));
            d += moving[v] ? c : 2 * c;
        }
    }
    obj += J.promap ? d : d / 2;
    // block weights: per-thread wrapping s32 deltas (the sum is the same in
    // any order); labels: one vertex per iteration
    const int T = omp_get_max_threads();
    std::vector<s32> bwd((size_t) T * J.k, 0);
#pragma omp parallel num_threads(T)
    {
        s32 *dk = bwd.data() + (size_t) omp_get_thread_num() * J.k;
#pragma omp for schedule(static)
        for (s64 mi = 0; mi < M; ++mi) {
            const u32 u = moves[(size_t) mi];
            const u32 ou = J.map[u], nu = J.dest_part[u];
            const s32 w = VW(g, u);
            dk[ou] = wsub(dk[ou], w);
            dk[nu] = wadd(dk[nu], w);
            J.map[u] = nu;
            J.dest_part[u] = ou;
            J.dest_cache[u] = NULL_PART;
            moving[u] = 0;
        }
    }
    for (int t = 0; t < T; ++t)
        for (u32 b = 0; b < J.k; ++b) J.bw[b] = wadd(J.bw[b], bwd[(size_t) t * J.k + b]);
#pragma omp parallel for schedule(dynamic, 256)
    for (s64 mi = 0; mi < (s64) moves.size(); ++mi) {
        const u32 u = moves[(size_t) mi];
        for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            u32 *dc = &J.dest_cache[g.adj[j]];
            if (ld_relaxed(dc) != NULL_PART) st_relaxed(dc, NULL_PART);  // skip shared lines already reset
        }
    }
    maxw = 0;
    for (u32 b = 0; b < J.k; ++b) maxw = std::max(maxw, J.bw[b]);
}

// jet_refine jet_label_propagation.h:926-1033 / ProMap_jet_refine
// promap_jet_label_propagation.h:1218-1311.
void jet_refine(const HostCSR &g, u32 k, s32 lmax, bool ultra, u32 level, std::vector<u32> &part, s64 &obj, s32 &maxw,
                const std::vector<s32> *D) {
    Jet J;
    jet_init(J, g, k, lmax, part.data());
    if (D) {
        J.promap = true;
        J.D = *D;
    }
    s64 best_obj = obj;
    s32 best_max = maxw;
    std::vector<u32> ratios;
    if (ultra && !J.promap) ratios = {85, 80, 75, 70, 65, 60, 55, 50, 45, 40, 35, 30, 25, 20, 15, 10, 5};
    else ratios = {level == 0 ? 25u : 75u};
    for (u32 ratio: ratios) {
        u32 balance_iteration = 0, iteration = 0;
        while (iteration < N_MAX_ITERATIONS) {
            iteration += 1;
            std::vector<u32> moves;
            if (!J.promap) {
                if (maxw <= lmax) {
                    moves = jet_lp(J, ratio);
                    balance_iteration = 0;
                    if (moves.empty()) break;
                } else {
                    if (balance_iteration < N_MAX_WEAK_ITERATIONS) {
                        moves = rebalance_weak(J);
                        if (moves.empty()) {
                            balance_iteration = N_MAX_WEAK_ITERATIONS;
                            continue;
                        }
                    } else {
                        moves = rebalance_strong(J);
                        if (moves.empty()) break;
                    }
                    balance_iteration++;
                }
            } else {
                if (maxw <= lmax) {
                    moves = jet_lp(J, ratio);
                    balance_iteration = 0;
                } else {
                    balance_iteration++;
                    if (balance_iteration < N_MAX_WEAK_ITERATIONS) moves = rebalance_weak(J);
                    else moves = rebalance_strong(J);
                }
                if (moves.empty()) continue;
            }
            perform_moves(J, moves, obj, maxw);
            const bool leq = J.promap ? (maxw < best_max) : (maxw <= best_max);
            if (best_max > lmax && maxw < best_max) {
                part = J.map;
                best_obj = obj;
                best_max = maxw;
                iteration = 0;
            } else if (obj < best_obj && (maxw <= lmax || leq)) {
                if (1000 * obj < 999 * best_obj) iteration = 0;  // PHI = 0.999
                part = J.map;
                best_obj = obj;
                best_max = maxw;
            }
        }
    }
    obj = best_obj;
    maxw = best_max;
}

std::vector<u32> project(const std::vector<u32> &coarse_part, const std::vector<u32> &mapping) {
    std::vector<u32> p(mapping.size());
    for (size_t u = 0; u < mapping.size(); ++u) p[u] = coarse_part[mapping[u]];
    return p;
}

s32 max_block(const HostCSR &g, const std::vector<u32> &part, u32 k) {
    std::vector<s32> bw(k, 0);
    for (u32 u = 0; u < g.n; ++u) bw[part[u]] = wadd(bw[part[u]], VW(g, u));
    s32 m = 0;
    for (s32 w: bw) m = std::max(m, w);
    return m;
}

// The initial partitioner: the reference's own ModifiedMetis::partition
// (kway_core.h:1527-1571) compiled from its sources into
// oracle/_ref/libkway_ref.so when that library was built (oracle.py installs
// it here), else the product's restatement of it (host/metis_kway.cpp).
typedef void (*RefKwayFn)(uint32_t, const uint32_t *, const uint32_t *, const int32_t *, const int32_t *, int, double,
                          uint64_t, uint32_t *);
RefKwayFn g_ref_kway = nullptr;

void oracle_kway(const HostCSR &g, u32 k, double eps, u64 seed, std::vector<u32> &part) {
    if (!g_ref_kway || k <= 1 || g.n == 0) {
        initial_kway(g, k, eps, seed, part);
        return;
    }
    std::vector<s32> vw(g.n), ew(g.m);
    for (u32 u = 0; u < g.n; ++u) vw[u] = VW(g, u);
    for (u32 j = 0; j < g.m; ++j) ew[j] = EW(g, j);
    part.assign(g.n, 0);
    g_ref_kway(g.n, g.xadj.data(), g.adj.data(), vw.data(), ew.data(), (int) k, eps, seed, part.data());
}

// recursive_partition global_multisection.h:132-220: partition into the
// current level's k, then recurse into every block's induced subgraph (empty
// subgraphs are skipped; the reference would divide by zero there).
void ims_recurse(const HostCSR &g, const std::vector<u32> &n_to_o, const std::vector<u32> &hier, u32 level,
                 std::vector<u32> &identifier, const std::vector<u32> &index_vec, const std::vector<u32> &k_rem,
                 double eps, s64 global_w, u32 global_k, u64 seed, std::vector<u32> &global_part) {
    const u32 l = (u32) hier.size();
    const u32 k_here = hier[level];
    const u64 depth = identifier.size();
    const s64 local_w = g.total_vw();
    const double imb =
        local_w > 0 ? adaptive_imbalance(eps, global_w, global_k, local_w, k_rem[l - 1 - depth], l - depth) : eps;
    std::vector<u32> tmp;
    oracle_kway(g, k_here, imb, seed, tmp);
    if (depth == l - 1) {
        u32 offset = 0;
        for (u32 i = 0; i + 1 < l; ++i) offset += identifier[i] * index_vec[index_vec.size() - 1 - i];
        for (u32 u = 0; u < g.n; ++u) global_part[n_to_o[u]] = offset + tmp[u];
        return;
    }
    for (u32 id = 0; id < k_here; ++id) {
        std::vector<u32> sub_n_to_o;
        HostCSR sub = induced_subgraph(g, tmp, id, sub_n_to_o);
        if (sub.n == 0) continue;
        for (u32 &x: sub_n_to_o) x = n_to_o[x];
        identifier.push_back(id);
        ims_recurse(sub, sub_n_to_o, hier, level - 1, identifier, index_vec, k_rem, eps, global_w, global_k, seed,
                    global_part);
        identifier.pop_back();
    }
}

// global_multisection_host global_multisection.h:222-257.
void ims_initial(const HostCSR &g, const std::vector<u32> &hier, double eps, u64 seed, std::vector<u32> &part) {
    const u32 l = (u32) hier.size();
    part.assign(g.n, 0);
    if (l == 0 || g.n == 0) return;
    std::vector<u32> index_vec = {1};
    for (u32 i = 0; i + 1 < l; ++i) index_vec.push_back(index_vec[i] * hier[i]);
    std::vector<u32> k_rem(l);
    u32 p = 1;
    for (u32 i = 0; i < l; ++i) {
        k_rem[i] = p * hier[i];
        p *= hier[i];
    }
    std::vector<u32> n_to_o(g.n);
    std::iota(n_to_o.begin(), n_to_o.end(), 0u);
    std::vector<u32> identifier;
    ims_recurse(g, n_to_o, hier, l - 1, identifier, index_vec, k_rem, eps, g.total_vw(), p, seed, part);
}

// Solver::internal_solve solver.h:340-400 (and the device constructor
// :144-246 used by hierarchical multisection).
s64 partition_graph(const HostCSR &g, u32 k, double eps, bool ultra, u64 seed, std::vector<u32> &part) {
    part.assign(g.n, 0);
    if (k <= 1) return 0;
    const s32 lmax = lmax_of(g.total_vw(), k, eps);
    std::vector<HostCSR> graphs;
    std::vector<std::vector<u32> > maps;
    const HostCSR *cur = &g;
    while (cur->n > 8 * k) {  // solver.h:343-347
        std::vector<u32> mapping;
        u32 nc = match(*cur, mapping);
        if ((u64) nc * 100 > (u64) cur->n * 99) break;  // shrank by less than 1%: stop coarsening
        graphs.push_back(contract(*cur, mapping, nc));
        maps.push_back(std::move(mapping));
        cur = &graphs.back();
    }
    HostCSR coarsest = *cur;
    sort_rows(coarsest);
    std::vector<u32> cpart;
    oracle_kway(coarsest, k, eps, seed, cpart);
    s64 cut = edge_cut(*cur, cpart);
    s32 maxw = max_block(*cur, cpart, k);
    for (size_t l = maps.size(); l > 0; --l) {
        const HostCSR &fine = (l >= 2) ? graphs[l - 2] : g;
        cpart = project(cpart, maps[l - 1]);
        jet_refine(fine, k, lmax, ultra, (u32) (l - 1), cpart, cut, maxw, nullptr);
    }
    part.swap(cpart);
    return cut;
}

// recursive_multisection_device hierarchical_multisection.h:56-235
void hm_recurse(const HostCSR &g, const std::vector<u32> &n_to_o, const std::vector<u32> &hier, u32 level,
                std::vector<u32> &identifier, const std::vector<u32> &index_vec, const std::vector<u32> &k_rem,
                double eps, s64 global_w, u32 global_k, u64 seed, bool ultra, std::vector<u32> &global_part) {
    const u32 l = (u32) hier.size();
    const u32 k_here = hier[level];
    const u64 depth = identifier.size();
    const double imb = adaptive_imbalance(eps, global_w, global_k, g.total_vw(), k_rem[l - 1 - depth], l - depth);
    std::vector<u32> tmp;
    partition_graph(g, k_here, imb, ultra, seed, tmp);
    if (depth == l - 1) {
        u32 offset = 0;
        for (u32 i = 0; i + 1 < l; ++i) offset += identifier[i] * index_vec[index_vec.size() - 1 - i];
        for (u32 u = 0; u < g.n; ++u) global_part[n_to_o[u]] = offset + tmp[u];
        return;
    }
    for (u32 id = 0; id < k_here; ++id) {
        std::vector<u32> sub_n_to_o;
        HostCSR sub = induced_subgraph(g, tmp, id, sub_n_to_o);
        if (sub.n == 0) continue;
        for (u32 &x: sub_n_to_o) x = n_to_o[x];
        identifier.push_back(id);
        hm_recurse(sub, sub_n_to_o, hier, level - 1, identifier, index_vec, k_rem, eps, global_w, global_k, seed, ultra,
                   global_part);
        identifier.pop_back();
    }
}

const HostCSR &G(const void *g) { return *(const HostCSR *) g; }

} // namespace

extern "C" {

uint32_t or_xorshift32(uint32_t x) { return xorshift32(x); }
int or_threads() { return omp_get_max_threads(); }
uint32_t or_murmur3_u32(uint32_t key, uint32_t seed) { return murmur3_u32(key, seed); }
uint32_t or_gain_bucket(int32_t gx, int32_t vwgt) { return gain_bucket(gx, vwgt); }
uint32_t or_gain_bucket_float(int32_t gx, int32_t vwgt) { return gain_bucket_float(gx, vwgt); }

void *or_graph_new(uint32_t n, uint32_t m, const uint32_t *xadj, const uint32_t *adj, const int32_t *ew,
                   const int32_t *vw) {
    HostCSR *g = new HostCSR();
    g->n = n;
    g->m = m;
    g->xadj.assign(xadj, xadj + n + 1);
    g->adj.assign(adj, adj + m);
    if (ew) g->ew.assign(ew, ew + m);
    if (vw) g->vw.assign(vw, vw + n);
    return g;
}
void or_graph_free(void *g) { delete (HostCSR *) g; }
uint32_t or_graph_n(const void *g) { return G(g).n; }
uint32_t or_graph_m(const void *g) { return G(g).m; }
int or_graph_has_ew(const void *g) { return !G(g).ew.empty(); }
int or_graph_has_vw(const void *g) { return !G(g).vw.empty(); }
void or_graph_get(const void *gp, uint32_t *xadj, uint32_t *adj, int32_t *ew, int32_t *vw) {
    const HostCSR &g = G(gp);
    if (xadj) std::copy(g.xadj.begin(), g.xadj.end(), xadj);
    if (adj) std::copy(g.adj.begin(), g.adj.end(), adj);
    if (ew) {
        if (g.ew.empty()) std::fill(ew, ew + g.m, 1);
        else std::copy(g.ew.begin(), g.ew.end(), ew);
    }
    if (vw) {
        if (g.vw.empty()) std::fill(vw, vw + g.n, 1);
        else std::copy(g.vw.begin(), g.vw.end(), vw);
    }
}

uint32_t or_match(const void *g, uint32_t *mapping_out) {
    std::vector<u32> mapping;
    u32 nc = match(G(g), mapping);
    std::copy(mapping.begin(), mapping.end(), mapping_out);
    return nc;
}

void *or_contract(const void *g, const uint32_t *mapping, uint32_t n_c) {
    std::vector<u32> mp(mapping, mapping + G(g).n);
    return new HostCSR(contract(G(g), mp, n_c));
}

int64_t or_edge_cut(const void *g, const uint32_t *part) {
    std::vector<u32> p(part, part + G(g).n);
    return edge_cut(G(g), p);
}

int64_t or_comm_cost(const void *g, const uint32_t *part, const uint32_t *hier, const int32_t *dist, uint32_t l) {
    std::vector<u32> h(hier, hier + l);
    std::vector<s32> d(dist, dist + l);
    u32 k = 1;
    for (u32 a: h) k *= a;
    std::vector<u32> p(part, part + G(g).n);
    return comm_cost(G(g), p, distance_matrix(h, d), k);
}

void or_distance_matrix(const uint32_t *hier, const int32_t *dist, uint32_t l, int32_t *out) {
    std::vector<u32> h(hier, hier + l);
    std::vector<s32> d(dist, dist + l);
    std::vector<s32> D = distance_matrix(h, d);
    std::copy(D.begin(), D.end(), out);
}

void *or_jet_new(const void *g, uint32_t k, int32_t lmax, const uint32_t *part, const uint32_t *hier,
                 const int32_t *dist, uint32_t l) {
    Jet *J = new Jet();
    jet_init(*J, G(g), k, lmax, part);
    if (hier) {
        J->promap = true;
        J->D = distance_matrix(std::vector<u32>(hier, hier + l), std::vector<s32>(dist, dist + l));
    }
    return J;
}
void or_jet_free(void *st) { delete (Jet *) st; }

static uint32_t copy_moves(const std::vector<u32> &mv, uint32_t *out) {
    if (out) std::copy(mv.begin(), mv.end(), out);
    return (uint32_t) mv.size();
}
uint32_t or_jet_lp(void *st, uint32_t ratio_pct, uint32_t *moves_out) {
    return copy_moves(jet_lp(*(Jet *) st, ratio_pct), moves_out);
}
uint32_t or_jet_weak(void *st, uint32_t *moves_out) { return copy_moves(rebalance_weak(*(Jet *) st), moves_out); }
uint32_t or_jet_strong(void *st, uint32_t *moves_out) { return copy_moves(rebalance_strong(*(Jet *) st), moves_out); }
void or_jet_perform(void *st, const uint32_t *moves, uint32_t count, int64_t *obj_inout, int32_t *maxw_out) {
    std::vector<u32> mv(moves, moves + count);
    s64 obj = *obj_inout;
    s32 mw = 0;
    perform_moves(*(Jet *) st, mv, obj, mw);
    *obj_inout = obj;
    *maxw_out = mw;
}
void or_jet_state(const void *stp, uint32_t *map, int32_t *bw, uint32_t *dest_part, int32_t *gain1, uint32_t *lock,
                  uint32_t *dest_cache, int32_t *gain_cache) {
    const Jet &J = *(const Jet *) stp;
    if (map) std::copy(J.map.begin(), J.map.end(), map);
    if (bw) std::copy(J.bw.begin(), J.bw.end(), bw);
    if (dest_part) std::copy(J.dest_part.begin(), J.dest_part.end(), dest_part);
    if (gain1) std::copy(J.gain1.begin(), J.gain1.end(), gain1);
    if (lock) std::copy(J.lock.begin(), J.lock.end(), lock);
    if (dest_cache) std::copy(J.dest_cache.begin(), J.dest_cache.end(), dest_cache);
    if (gain_cache) std::copy(J.gain_cache.begin(), J.gain_cache.end(), gain_cache);
}

void or_jet_refine(const void *g, uint32_t k, int32_t lmax, int ultra, uint32_t level, uint32_t *part_inout,
                   int64_t *obj_inout, int32_t *maxw_inout, const uint32_t *hier, const int32_t *dist, uint32_t l) {
    std::vector<u32> part(part_inout, part_inout + G(g).n);
    s64 obj = *obj_inout;
    s32 mw = *maxw_inout;
    std::vector<s32> D;
    if (hier) D = distance_matrix(std::vector<u32>(hier, hier + l), std::vector<s32>(dist, dist + l));
    jet_refine(G(g), k, lmax, ultra != 0, level, part, obj, mw, hier ? &D : nullptr);
    std::copy(part.begin(), part.end(), part_inout);
    *obj_inout = obj;
    *maxw_inout = mw;
}

int64_t or_partition(const void *g, uint32_t k, double eps, int ultra, uint64_t seed, uint32_t *part_out) {
    std::vector<u32> part;
    s64 cut = partition_graph(G(g), k, eps, ultra != 0, seed, part);
    std::copy(part.begin(), part.end(), part_out);
    return cut;
}

int64_t or_map_hm(const void *gp, const uint32_t *hier, const int32_t *dist, uint32_t l, double eps, int ultra,
                  uint64_t seed, uint32_t *part_out) {
    const HostCSR &g = G(gp);
    std::vector<u32> h(hier, hier + l);
    std::vector<s32> d(dist, dist + l);
    std::vector<u32> index_vec = {1};
    for (u32 i = 0; i + 1 < l; ++i) index_vec.push_back(index_vec[i] * h[i]);
    std::vector<u32> k_rem(l);
    u32 p = 1;
    for (u32 i = 0; i < l; ++i) {
        k_rem[i] = p * h[i];
        p *= h[i];
    }
    std::vector<u32> n_to_o(g.n);
    std::iota(n_to_o.begin(), n_to_o.end(), 0u);
    std::vector<u32> part(g.n, 0), identifier;
    hm_recurse(g, n_to_o, h, l - 1, identifier, index_vec, k_rem, eps, g.total_vw(), p, seed, ultra != 0, part);
    std::copy(part.begin(), part.end(), part_out);
    return comm_cost(g, part, distance_matrix(h, d), p);
}

int64_t or_map_im(const void *gp, const uint32_t *hier, const int32_t *dist, uint32_t l, double eps, uint64_t seed,
                  uint32_t *part_out) {
    const HostCSR &g = G(gp);
    std::vector<u32> h(hier, hier + l);
    std::vector<s32> d(dist, dist + l);
    u32 k = 1;
    for (u32 a: h) k *= a;
    std::vector<s32> D = distance_matrix(h, d);
    const s32 lmax = lmax_of(g.total_vw(), k, eps);
    std::vector<HostCSR> graphs;
    std::vector<std::vector<u32> > maps;
    const HostCSR *cur = &g;
    while (cur->n > 8 * k) {  // promap_solver.h:247-251
        std::vector<u32> mapping;
        u32 nc = match(*cur, mapping);
        if ((u64) nc * 100 > (u64) cur->n * 99) break;  // shrank by less than 1%
        graphs.push_back(contract(*cur, mapping, nc));
        maps.push_back(std::move(mapping));
        cur = &graphs.back();
    }
    HostCSR coarsest = *cur;
    sort_rows(coarsest);
    std::vector<u32> cpart;
    ims_initial(coarsest, h, eps, seed, cpart);  // promap_solver.h:391-409
    s64 J = comm_cost(*cur, cpart, D, k);
    s32 maxw = max_block(*cur, cpart, k);
    for (size_t lv = maps.size(); lv > 0; --lv) {
        const HostCSR &fine = (lv >= 2) ? graphs[lv - 2] : g;
        cpart = project(cpart, maps[lv - 1]);
        jet_refine(fine, k, lmax, false, (u32) (lv - 1), cpart, J, maxw, &D);
    }
    std::copy(cpart.begin(), cpart.end(), part_out);
    return J;
}

int32_t or_lmax(int64_t total_weight, uint32_t k, double eps) { return lmax_of(total_weight, k, eps); }

void or_set_ref_kway(void *fn) { g_ref_kway = (RefKwayFn) fn; }
int or_uses_ref_kway(void) { return g_ref_kway != nullptr; }

void or_initial_kway(const void *g, uint32_t k, double eps, uint64_t seed, uint32_t *part_out) {
    std::vector<u32> part;
    oracle_kway(G(g), k, eps, seed, part);
    std::copy(part.begin(), part.end(), part_out);
}

} // extern "C"
