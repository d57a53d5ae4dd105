// Restatement of the reference's host initial partitioner
// (src/initial_partitioning/kway_partitioner/kway_core.h and the kway_*.h
// helpers it includes); see metis_kway.h. Each function names the reference
// function it follows. Ties, float expressions and the order of random draws
// are kept as in the reference, because the partition has to come out the
// same; the data structures are this file's own.
#include "metis_kway.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <utility>
#include <vector>

namespace hp {

// ---- the C library's rand() sequence ------------------------------------------

void LibcRand::seed_with(u32 seed) {
    if (seed == 0) seed = 1;
    s32 word = (s32) seed;
    r_[0] = word;
    for (int i = 1; i < 31; ++i) {
        // r[i] = 16807 * r[i-1] mod (2^31 - 1), by Schrage's method
        const long hi = word / 127773, lo = word % 127773;
        long w = 16807 * lo - 2836 * hi;
        if (w < 0) w += 2147483647;
        word = (s32) w;
        r_[i] = word;
    }
    f_ = 3;
    b_ = 0;
    for (int i = 0; i < 310; ++i) next();
}

int LibcRand::next() {
    const u32 v = (u32) r_[f_] + (u32) r_[b_];
    r_[f_] = (s32) v;
    if (++f_ == 31) {
        f_ = 0;
        ++b_;
    } else if (++b_ == 31) {
        b_ = 0;
    }
    return (int) (v >> 1);
}

namespace {

constexpr int BND_REFINE = 1;   // kway_utility.h:35
constexpr int BND_BALANCE = 2;  // kway_utility.h:36
constexpr int OPT_REFINE = 1;   // kway_utility.h:39
constexpr int OPT_BALANCE = 2;  // kway_utility.h:40
constexpr int FREE = -1;        // unmatched (kway_utility.h:42)

// Graph of the partitioner (kway_graph.h): int arrays, the vertex weight
// total `w` and the running cut of the current bisection or partition.
struct KGraph {
    int n = -1, m = -1, w = -1;
    std::vector<int> vw, xadj, adj, ew;
    int cut = -1;
    KGraph() = default;
    KGraph(int n_, int m_, int w_ = 0) : n(n_), m(m_), w(w_), vw(n_), xadj(n_ + 1), adj(m_), ew(m_), cut(0) {}
    void reshape(int n_, int m_, int w_ = -1) {
        n = n_;
        m = m_;
        w = w_;
        vw.resize(n_);
        xadj.resize(n_ + 1);
        adj.resize(m_);
        ew.resize(m_);
    }
};

// Boundary vertex set with O(1) insert and swap-remove (kway_boundary.h); the
// order of `val` is observable (it is permuted and scanned).
struct BndSet {
    int cnt = 0;
    std::vector<int> pos, val;
    explicit BndSet(int n = 0) : cnt(0), pos(n, -1), val(n) {}
    void add(int v) {
        val[cnt] = v;
        pos[v] = cnt++;
    }
    void remove(int v) {
        const int last = val[--cnt];
        val[pos[v]] = last;
        pos[last] = pos[v];
        pos[v] = -1;
    }
    bool has(int v) const { return pos[v] != -1; }
    void clear() {
        cnt = 0;
        std::fill(pos.begin(), pos.end(), -1);
    }
};

// Internal / external edge weight per vertex for a bisection (BisectInfo).
struct Side2 {
    std::vector<int> in, ex;
    explicit Side2(int n = 0) : in(n), ex(n) {}
};

// Per-vertex block connectivity for the k-way refinement (kway_block_conn.h):
// dense weights per (vertex, block), the list of connected blocks in
// insertion order with swap-remove, internal and external weight, and a second
// copy of the per-vertex counters for projection.
class KConn {
public:
    KConn(int n, int k)
        : n_(n), k_(k), cnt_(n, 0), cnt2_(n, 0), in_(n, 0), in2_(n, 0), ex_(n, 0), ex2_(n, 0),
          w_((size_t) n * k, 0), at_((size_t) n * k, -1), ids_((size_t) n * k, -1) {}
    void update(int v, int id, int delta) {
        if (delta == 0) return;
        const size_t o = (size_t) v * k_ + id;
        const int before = w_[o];
        const int after = before + delta;
        w_[o] = after;
        if (before == 0 && after > 0) {  // a new connection
            const int p = cnt_[v]++;
            at_[o] = p;
            ids_[(size_t) v * k_ + p] = id;
            return;
        }
        if (before > 0 && after == 0) {  // a connection disappears
            const int p = at_[o];
            const int last = cnt_[v] - 1;
            if (p != last) {
                const int last_id = ids_[(size_t) v * k_ + last];
                ids_[(size_t) v * k_ + p] = last_id;
                at_[(size_t) v * k_ + last_id] = p;
            }
            ids_[(size_t) v * k_ + last] = -1;
            at_[o] = -1;
            --cnt_[v];
        }
    }
    int get(int v, int id) const { return w_[(size_t) v * k_ + id]; }
    void clear() {
        std::fill(cnt_.begin(), cnt_.end(), 0);
        std::fill(cnt2_.begin(), cnt2_.end(), 0);
        std::fill(w_.begin(), w_.end(), 0);
        std::fill(at_.begin(), at_.end(), -1);
        std::fill(ids_.begin(), ids_.end(), -1);
        std::fill(in_.begin(), in_.end(), 0);
        std::fill(in2_.begin(), in2_.end(), 0);
        std::fill(ex_.begin(), ex_.end(), 0);
        std::fill(ex2_.begin(), ex2_.end(), 0);
    }
    void swap_copies() {
        cnt_.swap(cnt2_);
        in_.swap(in2_);
        ex_.swap(ex2_);
    }
    int ex_copy(int v) const { return ex2_[v]; }
    int in(int v) const { return in_[v]; }
    int ex(int v) const { return ex_[v]; }
    int nconn(int v) const { return cnt_[v]; }
    void add_in(int v, int x) { in_[v] += x; }
    void add_ex(int v, int x) { ex_[v] += x; }
    void set_in(int v, int x) { in_[v] = x; }
    void set_ex(int v, int x) { ex_[v] = x; }
    int conn_id(int v, int i) const { return ids_[(size_t) v * k_ + i]; }
    int conn_w(int v, int i) const { return get(v, conn_id(v, i)); }

private:
    int n_, k_;
    std::vector<int> cnt_, cnt2_, in_, in2_, ex_, ex2_, w_, at_, ids_;
};

// Binary max-heap of (key, vertex) with a position index (kway_prio_queue.h,
// kway_indexed_prio_queue.h). A key moves up only past strictly smaller
// parents and down only below strictly larger children (the right child only
// when strictly larger than the left), which fixes the order among equal keys.
template<typename K>
class MaxHeap {
public:
    explicit MaxHeap(size_t cap) : size_(0), h_(cap), at_(cap, -1) {}
    bool empty() const { return size_ == 0; }
    bool contains(int v) const { return v >= 0 && (size_t) v < at_.size() && at_[v] != -1; }
    void clear() {
        for (long i = (long) size_ - 1; i >= 0; --i) at_[h_[i].v] = -1;
        size_ = 0;
    }
    void insert(int v, K key) {
        long i = (long) size_++;
        up(i, key);
        put(i, v, key);
    }
    void erase(int v) {
        long i = at_[v];
        at_[v] = -1;
        if (--size_ == 0 || h_[size_].v == v) return;
        const int lv = h_[size_].v;
        const K lk = h_[size_].key;
        if (lk > h_[i].key) up(i, lk);
        else down(i, lk);
        put(i, lv, lk);
    }
    void update(int v, K key) {
        long i = at_[v];
        const K old = h_[i].key;
        if (key == old) return;
        if (key > old) up(i, key);
        else down(i, key);
        put(i, v, key);
    }
    int pop() {
        const int top = h_[0].v;
        at_[top] = -1;
        if (--size_ == 0) return top;
        const int lv = h_[size_].v;
        const K lk = h_[size_].key;
        long i = 0;
        down(i, lk);
        put(i, lv, lk);
        return top;
    }

private:
    struct Item {
        K key;
        int v;
    };
    size_t size_;
    std::vector<Item> h_;
    std::vector<long> at_;
    void up(long &i, const K &key) {
        while (i > 0) {
            const long p = (i - 1) >> 1;
            if (!(key > h_[p].key)) break;
            h_[i] = h_[p];
            at_[h_[i].v] = i;
            i = p;
        }
    }
    void down(long &i, const K &key) {
        for (;;) {
            const long l = 2 * i + 1;
            if (l >= (long) size_) break;
            long c = l;
            if (h_[l].key > key) {
                if (l + 1 < (long) size_ && h_[l + 1].key > h_[l].key) c = l + 1;
            } else if (l + 1 < (long) size_ && h_[l + 1].key > key) {
                c = l + 1;
            } else {
                break;
            }
            h_[i] = h_[c];
            at_[h_[i].v] = i;
            i = c;
        }
    }
    void put(long i, int v, const K &key) {
        h_[i].key = key;
        h_[i].v = v;
        at_[v] = i;
    }
};

// permute (kway_utility.h:58-75): nshuffles random 4-element block swaps, or
// n random pair swaps for n < 10.
void shuffle(int n, std::vector<int> &p, int nshuffles, LibcRand &R) {
    if (n < 10) {
        for (int i = 0; i < n; ++i) {
            const int a = R.next() % n;
            const int b = R.next() % n;
            std::swap(p[a], p[b]);
        }
        return;
    }
    for (int i = 0; i < nshuffles; ++i) {
        const int v = R.next() % (n - 3);
        const int u = R.next() % (n - 3);
        std::swap(p[v + 0], p[u + 2]);
        std::swap(p[v + 1], p[u + 3]);
        std::swap(p[v + 2], p[u + 0]);
        std::swap(p[v + 3], p[u + 1]);
    }
}

// counting_sort (kway_utility.h:77-92): stable by key in the order of tperm.
void bucket_order(int n, int maxkey, const std::vector<int> &keys, const std::vector<int> &tperm,
                  std::vector<int> &perm) {
    std::vector<int> start(maxkey + 2, 0);
    for (int i = 0; i < n; ++i) ++start[keys[i]];
    for (int i = 1; i < maxkey + 1; ++i) start[i] += start[i - 1];
    for (int i = maxkey + 1; i > 0; --i) start[i] = start[i - 1];
    start[0] = 0;
    for (int ii = 0; ii < n; ++ii) {
        const int i = tperm[ii];
        perm[start[keys[i]]++] = i;
    }
}

// Match_2HopAny (kway_core.h:285-327): unmatched vertices of degree < max_deg
// that share a neighbour are paired, from the ends of each neighbour's list.
int pair_two_hop_any(const KGraph &g, std::vector<int> &match, std::vector<int> &cmap, int cn, int &unmatched,
                     int max_deg, const std::vector<int> &perm) {
    std::vector<int> off(g.n + 1, 0);
    for (int v = 0; v < g.n; ++v)
        if (match[v] == FREE && g.xadj[v + 1] - g.xadj[v] < max_deg)
            for (int j = g.xadj[v]; j < g.xadj[v + 1]; ++j) off[g.adj[j]]++;
    for (int i = 1; i < g.n; ++i) off[i] += off[i - 1];
    for (int i = g.n; i > 0; --i) off[i] = off[i - 1];
    off[0] = 0;
    std::vector<int> lst(off[g.n]);
    for (int pi = 0; pi < g.n; ++pi) {
        const int i = perm[pi];
        if (match[i] == FREE && g.xadj[i + 1] - g.xadj[i] < max_deg)
            for (int j = g.xadj[i]; j < g.xadj[i + 1]; ++j) lst[off[g.adj[j]]++] = i;
    }
    for (int i = g.n; i > 0; --i) off[i] = off[i - 1];
    off[0] = 0;
    for (int pi = 0; pi < g.n; ++pi) {
        const int i = perm[pi];
        if (off[i + 1] - off[i] < 2) continue;
        for (int hi = off[i + 1], lo = off[i]; lo < hi; ++lo) {
            if (match[lst[lo]] != FREE) continue;
            for (--hi; hi > lo; --hi) {
                if (match[lst[hi]] == FREE) {
                    cmap[lst[lo]] = cmap[lst[hi]] = cn++;
                    match[lst[lo]] = lst[hi];
                    match[lst[hi]] = lst[lo];
                    unmatched -= 2;
                    break;
                }
            }
        }
    }
    return cn;
}

struct NeighbourhoodKey {
    int key;
    int vertex;
};

int by_neighbourhood_key(const void *a, const void *b) {
    const NeighbourhoodKey *x = (const NeighbourhoodKey *) a, *y = (const NeighbourhoodKey *) b;
    return (x->key > y->key) - (x->key < y->key);
}

// Match_2HopAll (kway_core.h:329-387): unmatched vertices with identical
// neighbourhoods are paired (candidates ordered by a neighbourhood checksum
// with the C library's qsort, as the reference orders them).
int pair_two_hop_all(const KGraph &g, std::vector<int> &match, std::vector<int> &cmap, int cn, int &unmatched,
                     int max_deg, const std::vector<int> &perm) {
    const int mask = INT32_MAX / max_deg;
    int nc = 0;
    std::vector<NeighbourhoodKey> keys(unmatched);
    for (int pi = 0; pi < g.n; ++pi) {
        const int i = perm[pi];
        const int d = g.xadj[i + 1] - g.xadj[i];
        if (match[i] == FREE && d > 1 && d < max_deg) {
            int s = 0;
            for (int j = g.xadj[i]; j < g.xadj[i + 1]; ++j) s += g.adj[j] % mask;
            keys[nc].vertex = i;
            keys[nc].key = (s % mask) * max_deg + d;
            ++nc;
        }
    }
    std::qsort(keys.data(), nc, sizeof(NeighbourhoodKey), by_neighbourhood_key);
    std::vector<int> mark(g.n, 0);
    for (int pi = 0; pi < nc; ++pi) {
        const int i = keys[pi].vertex;
        if (match[i] != FREE) continue;
        for (int j = g.xadj[i]; j < g.xadj[i + 1]; ++j) mark[g.adj[j]] = i;
        for (int pk = pi + 1; pk < nc; ++pk) {
            const int k = keys[pk].vertex;
            if (match[k] != FREE) continue;
            if (keys[pi].key != keys[pk].key) break;
            if (g.xadj[i + 1] - g.xadj[i] != g.xadj[k + 1] - g.xadj[k]) break;
            int jj = g.xadj[k];
            for (; jj < g.xadj[k + 1]; ++jj)
                if (mark[g.adj[jj]] != i) break;
            if (jj == g.xadj[k + 1]) {
                cmap[i] = cmap[k] = cn++;
                match[i] = k;
                match[k] = i;
                unmatched -= 2;
                break;
            }
        }
    }
    return cn;
}

// Match_2Hop (kway_core.h:389-397). The unmatched count is passed by value,
// as in the reference: the later passes see the count after the first two.
int pair_two_hop(const KGraph &g, std::vector<int> &match, std::vector<int> &cmap, int cn, int unmatched,
                 const std::vector<int> &perm) {
    cn = pair_two_hop_any(g, match, cmap, cn, unmatched, 2, perm);
    cn = pair_two_hop_all(g, match, cmap, cn, unmatched, 64, perm);
    if (unmatched > 1.5 * 0.10 * g.n) cn = pair_two_hop_any(g, match, cmap, cn, unmatched, 3, perm);
    if (unmatched > 2.0 * 0.10 * g.n) cn = pair_two_hop_any(g, match, cmap, cn, unmatched, g.n, perm);
    return cn;
}

// heavy_edge_matching (kway_core.h:399-476): vertices in random order within
// sqrt-degree buckets, each matched to its heaviest free neighbour within the
// weight limit; isolated vertices pair with the next free vertex; two-hop
// passes when more than 10% stay unmatched. Returns the coarse vertex count;
// cmap holds coarse ids in vertex order.
int heavy_edge_match(const KGraph &g, std::vector<int> &match, std::vector<int> &cmap, int max_vw, LibcRand &R) {
    std::vector<int> perm(g.n), tperm(g.n), deg(g.n);
    std::fill_n(match.data(), g.n, FREE);
    for (int i = 0; i < g.n; ++i) tperm[i] = i;
    shuffle(g.n, tperm, g.n / 8, R);
    const int avgdeg = 4.0 * (g.xadj[g.n] / g.n);
    for (int i = 0; i < g.n; ++i) {
        const int b = std::sqrt(1 + g.xadj[i + 1] - g.xadj[i]);
        deg[i] = b > avgdeg ? avgdeg : b;
    }
    bucket_order(g.n, avgdeg, deg, tperm, perm);
    int unmatched = 0, cn = 0, last_free = 0;
    for (int pi = 0; pi < g.n; ++pi) {
        const int i = perm[pi];
        if (match[i] != FREE) continue;
        int best = i;
        if (g.vw[i] < max_vw) {
            if (g.xadj[i] == g.xadj[i + 1]) {
                last_free = (pi > last_free ? pi : last_free) + 1;
                for (; last_free < g.n; ++last_free) {
                    const int j = perm[last_free];
                    if (match[j] == FREE) {
                        best = j;
                        break;
                    }
                }
            } else {
                int bw = -1;
                for (int j = g.xadj[i]; j < g.xadj[i + 1]; ++j) {
                    const int k = g.adj[j];
                    if (match[k] == FREE && bw < g.ew[j] && g.vw[i] + g.vw[k] <= max_vw) {
                        best = k;
                        bw = g.ew[j];
                    }
                }
                if (best == i && 2 * g.vw[i] < max_vw) {
                    ++unmatched;
                    best = FREE;
                }
            }
        }
        if (best != FREE) {
            cmap[i] = cmap[best] = cn++;
            match[i] = best;
            match[best] = i;
        }
    }
    if (unmatched > 0.10 * g.n) cn = pair_two_hop(g, match, cmap, cn, unmatched, perm);
    cn = 0;
    for (int i = 0; i < g.n; ++i) {
        if (match[i] == FREE) {
            match[i] = i;
            cmap[i] = cn++;
        } else if (i <= match[i]) {
            cmap[i] = cmap[match[i]] = cn++;
        }
    }
    return cn;
}

// coarse_graph (kway_core.h:478-595): one coarse row per matched pair, in
// first-occurrence order of the coarse neighbours; a small hash table for
// short rows (the coarse vertex's own id is kept in slot 0 while aggregating
// and replaced by the last entry at the end), a dense index otherwise.
KGraph contract_pairs(const KGraph &g, const std::vector<int> &match, const std::vector<int> &cmap, int cn) {
    constexpr int mask = (1 << 13) - 1;
    KGraph c(cn, g.m + 1);
    c.cut = -1;
    std::vector<int> slot(mask + 1, -1), dense(cn, -1);
    int cv = 0, ce = 0;
    c.xadj[0] = 0;
    for (int v = 0; v < g.n; ++v) {
        const int u = match[v];
        if (u < v) continue;
        c.vw[cv] = g.vw[v];
        if (v != u) c.vw[cv] += g.vw[u];
        const int dv = g.xadj[v + 1] - g.xadj[v], du = g.xadj[u + 1] - g.xadj[u];
        const int base = ce;
        int ne = 0;
        if (dv + du < (mask >> 2)) {
            slot[cv & mask] = 0;
            c.adj[base] = cv;
            ne = 1;
            auto add_row = [&](int x) {
                for (int j = g.xadj[x]; j < g.xadj[x + 1]; ++j) {
                    const int cn_id = cmap[g.adj[j]];
                    int h = cn_id & mask;
                    while (slot[h] != -1 && c.adj[base + slot[h]] != cn_id) h = (h + 1) & mask;
                    const int p = slot[h];
                    if (p == -1) {
                        c.adj[base + ne] = cn_id;
                        c.ew[base + ne] = g.ew[j];
                        slot[h] = ne++;
                    } else {
                        c.ew[base + p] += g.ew[j];
                    }
                }
            };
            add_row(v);
            if (v != u) add_row(u);
            for (int j = ne - 1; j >= 0; --j) {
                const int cn_id = c.adj[base + j];
                int h = cn_id & mask;
                while (c.adj[base + slot[h]] != cn_id) h = (h + 1) & mask;
                slot[h] = -1;
            }
            --ne;
            c.adj[base] = c.adj[base + ne];
            c.ew[base] = c.ew[base + ne];
        } else {
            auto add_row = [&](int x) {
                for (int j = g.xadj[x]; j < g.xadj[x + 1]; ++j) {
                    const int cn_id = cmap[g.adj[j]];
                    const int p = dense[cn_id];
                    if (p == -1) {
                        c.adj[base + ne] = cn_id;
                        c.ew[base + ne] = g.ew[j];
                        dense[cn_id] = ne++;
                    } else {
                        c.ew[base + p] += g.ew[j];
                    }
                }
            };
            add_row(v);
            if (v != u) {
                add_row(u);
                const int self = dense[cv];
                if (self != -1) {
                    --ne;
                    c.adj[base + self] = c.adj[base + ne];
                    c.ew[base + self] = c.ew[base + ne];
                    dense[cv] = -1;
                }
            }
            for (int j = 0; j < ne; ++j) dense[c.adj[base + j]] = -1;
        }
        ce += ne;
        c.xadj[++cv] = ce;
    }
    c.n = cv;
    c.m = ce;
    c.w = g.w;
    return c;
}

// balance_bisection_boundary (kway_core.h:136-219).
void balance_from_boundary(KGraph &g, Side2 &s, BndSet &bnd, std::vector<int> &pw, const std::vector<float> &tw,
                           std::vector<int> &side, LibcRand &R) {
    std::vector<int> moved(g.n, -1), perm(g.n);
    int target[2];
    target[0] = (int) g.w * tw[0];
    target[1] = g.w - target[0];
    const int mindiff = std::abs(target[0] - pw[0]);
    const int from = pw[0] < target[0] ? 1 : 0;
    const int to = (from + 1) % 2;
    MaxHeap<int> q(g.n);
    for (int i = 0; i < bnd.cnt; ++i) perm[i] = i;
    shuffle(bnd.cnt, perm, bnd.cnt / 5, R);
    for (int i = 0; i < bnd.cnt; ++i) {
        const int v = bnd.val[perm[i]];
        if (side[v] == from && g.vw[v] <= mindiff) q.insert(v, s.ex[v] - s.in[v]);
    }
    int cut = g.cut;
    for (int step = 0; step < g.n; ++step) {
        if (q.empty()) break;
        const int x = q.pop();
        if (pw[to] + g.vw[x] > target[to]) break;
        cut -= s.ex[x] - s.in[x];
        pw[to] += g.vw[x];
        pw[from] -= g.vw[x];
        side[x] = to;
        moved[x] = step;
        std::swap(s.in[x], s.ex[x]);
        if (s.ex[x] == 0 && g.xadj[x] < g.xadj[x + 1]) bnd.remove(x);
        for (int j = g.xadj[x]; j < g.xadj[x + 1]; ++j) {
            const int k = g.adj[j];
            const int d = to == side[k] ? g.ew[j] : -g.ew[j];
            s.in[k] += d;
            s.ex[k] -= d;
            const bool cand = moved[k] == -1 && side[k] == from && g.vw[k] <= mindiff;
            if (bnd.has(k)) {
                if (s.ex[k] == 0) {
                    bnd.remove(k);
                    if (cand) q.erase(k);
                } else if (cand) {
                    q.update(k, s.ex[k] - s.in[k]);
                }
            } else if (s.ex[k] > 0) {
                bnd.add(k);
                if (cand) q.insert(k, s.ex[k] - s.in[k]);
            }
        }
    }
    g.cut = cut;
}

// balance_bisection_general (kway_core.h:221-283).
void balance_from_all(KGraph &g, Side2 &s, BndSet &bnd, std::vector<int> &pw, const std::vector<float> &tw,
                      std::vector<int> &side, LibcRand &R) {
    std::vector<int> moved(g.n, -1), perm(g.n);
    int target[2];
    target[0] = (int) g.w * tw[0];
    target[1] = g.w - target[0];
    const int mindiff = std::abs(target[0] - pw[0]);
    const int from = pw[0] < target[0] ? 1 : 0;
    const int to = (from + 1) % 2;
    MaxHeap<int> q(g.n);
    for (int i = 0; i < g.n; ++i) perm[i] = i;
    shuffle(g.n, perm, g.n / 5, R);
    for (int ii = 0; ii < g.n; ++ii) {
        const int i = perm[ii];
        if (side[i] == from && g.vw[i] <= mindiff) q.insert(i, s.ex[i] - s.in[i]);
    }
    int cut = g.cut;
    for (int step = 0; step < g.n; ++step) {
        if (q.empty()) break;
        const int x = q.pop();
        if (pw[to] + g.vw[x] > target[to]) break;
        cut -= s.ex[x] - s.in[x];
        pw[to] += g.vw[x];
        pw[from] -= g.vw[x];
        side[x] = to;
        moved[x] = step;
        std::swap(s.in[x], s.ex[x]);
        if (s.ex[x] == 0 && bnd.has(x) && g.xadj[x] < g.xadj[x + 1]) bnd.remove(x);
        if (s.ex[x] > 0 && !bnd.has(x)) bnd.add(x);
        for (int j = g.xadj[x]; j < g.xadj[x + 1]; ++j) {
            const int k = g.adj[j];
            const int d = to == side[k] ? g.ew[j] : -g.ew[j];
            s.in[k] += d;
            s.ex[k] -= d;
            if (moved[k] == -1 && side[k] == from && g.vw[k] <= mindiff) q.update(k, s.ex[k] - s.in[k]);
            const bool was = bnd.has(k);
            if (s.ex[k] == 0 && was) bnd.remove(k);
            if (s.ex[k] > 0 && !was) bnd.add(k);
        }
    }
    g.cut = cut;
}

// FM_2WayCutRefine (kway_core.h:597-741): max_iter passes of boundary FM with
// one queue per side, moving from the heavier side, rolled back to the best
// prefix of moves.
void fm_two_way(KGraph &g, BndSet &bnd, Side2 &s, std::vector<int> &pw, const std::vector<float> &tw,
                std::vector<int> &side, int max_iter, LibcRand &R) {
    std::vector<int> moved(g.n, -1), swaps(g.n), perm(g.n);
    int target[2];
    target[0] = g.w * tw[0];
    target[1] = g.w - target[0];
    const int limit = (((0.01 * g.n) > (15) ? (0.01 * g.n) : (15)) < (100) ? ((0.01 * g.n) > (15) ? (0.01 * g.n) : (15))
                                                                            : (100));
    const int avgvw = ((pw[0] + pw[1]) / 20) < (2 * (pw[0] + pw[1]) / g.n) ? ((pw[0] + pw[1]) / 20)
                                                                           : (2 * (pw[0] + pw[1]) / g.n);
    MaxHeap<int> q0(g.n), q1(g.n);
    MaxHeap<int> *q[2] = {&q0, &q1};
    const int origdiff = std::abs(target[0] - pw[0]);
    for (int pass = 0; pass < max_iter; ++pass) {
        q[0]->clear();
        q[1]->clear();
        int best_at = -1, newcut = g.cut, mincut = g.cut;
        const int initcut = g.cut;
        int mindiff = std::abs(target[0] - pw[0]);
        for (int i = 0; i < bnd.cnt; ++i) perm[i] = i;
        shuffle(bnd.cnt, perm, bnd.cnt, R);
        for (int ii = 0; ii < bnd.cnt; ++ii) {
            const int v = bnd.val[perm[ii]];
            q[side[v]]->insert(v, s.ex[v] - s.in[v]);
        }
        int nsw = 0;
        for (; nsw < g.n; ++nsw) {
            const int from = (target[0] - pw[0] < target[1] - pw[1] ? 0 : 1);
            const int to = (from + 1) % 2;
            if (q[from]->empty()) break;
            const int x = q[from]->pop();
            newcut -= s.ex[x] - s.in[x];
            pw[to] += g.vw[x];
            pw[from] -= g.vw[x];
            if ((newcut < mincut && std::abs(target[0] - pw[0]) <= origdiff + avgvw) ||
                (newcut == mincut && std::abs(target[0] - pw[0]) < mindiff)) {
                mincut = newcut;
                mindiff = std::abs(target[0] - pw[0]);
                best_at = nsw;
            } else if (nsw - best_at > limit) {
                newcut += s.ex[x] - s.in[x];
                pw[from] += g.vw[x];
                pw[to] -= g.vw[x];
                break;
            }
            side[x] = to;
            moved[x] = nsw;
            swaps[nsw] = x;
            std::swap(s.in[x], s.ex[x]);
            if (s.ex[x] == 0 && g.xadj[x] < g.xadj[x + 1]) bnd.remove(x);
            for (int j = g.xadj[x]; j < g.xadj[x + 1]; ++j) {
                const int k = g.adj[j];
                const int d = to == side[k] ? g.ew[j] : -g.ew[j];
                s.in[k] += d;
                s.ex[k] -= d;
                if (bnd.has(k)) {
                    if (s.ex[k] == 0) {
                        bnd.remove(k);
                        if (moved[k] == -1) q[side[k]]->erase(k);
                    } else if (moved[k] == -1) {
                        q[side[k]]->update(k, s.ex[k] - s.in[k]);
                    }
                } else if (s.ex[k] > 0) {
                    bnd.add(k);
                    if (moved[k] == -1) q[side[k]]->insert(k, s.ex[k] - s.in[k]);
                }
            }
        }
        for (int i = 0; i < nsw; ++i) moved[swaps[i]] = -1;
        for (--nsw; nsw > best_at; --nsw) {  // roll back past the best prefix
            const int x = swaps[nsw];
            const int to = (side[x] + 1) % 2;
            side[x] = to;
            std::swap(s.in[x], s.ex[x]);
            if (s.ex[x] == 0 && bnd.has(x) && g.xadj[x] < g.xadj[x + 1]) bnd.remove(x);
            else if (s.ex[x] > 0 && !bnd.has(x)) bnd.add(x);
            pw[to] += g.vw[x];
            pw[(to + 1) % 2] -= g.vw[x];
            for (int j = g.xadj[x]; j < g.xadj[x + 1]; ++j) {
                const int k = g.adj[j];
                const int d = to == side[k] ? g.ew[j] : -g.ew[j];
                s.in[k] += d;
                s.ex[k] -= d;
                if (bnd.has(k) && s.ex[k] == 0) bnd.remove(k);
                if (!bnd.has(k) && s.ex[k] > 0) bnd.add(k);
            }
        }
        g.cut = mincut;
        if (best_at <= 0 || mincut == initcut) break;
    }
}

// Project2WayPartition (kway_core.h:105-134): coarse sides to the fine
// graph; vertices of non-boundary coarse vertices are interior.
void project_two_way(const KGraph &g, Side2 &s, std::vector<int> &cmap, BndSet &bnd, const BndSet &cbnd,
                     std::vector<int> &side, const std::vector<int> &cside) {
    for (int i = 0; i < g.n; ++i) {
        const int j = cmap[i];
        side[i] = cside[j];
        cmap[i] = cbnd.pos[j];
    }
    for (int i = 0; i < g.n; ++i) {
        int in = 0, ex = 0;
        if (cmap[i] == -1) {
            for (int j = g.xadj[i]; j < g.xadj[i + 1]; ++j) in += g.ew[j];
        } else {
            const int me = side[i];
            for (int j = g.xadj[i]; j < g.xadj[i + 1]; ++j) {
                if (me == side[g.adj[j]]) in += g.ew[j];
                else ex += g.ew[j];
            }
        }
        s.in[i] = in;
        s.ex[i] = ex;
        if (ex > 0 || g.xadj[i] == g.xadj[i + 1]) bnd.add(i);
    }
}

// ComputeLoadImbalanceDiff (kway_core.h:863-873).
float imbalance_excess(const KGraph &g, int k, const std::vector<int> &pw, float ub) {
    float mx = -1.0f;
    for (int j = 0; j < k; ++j) {
        const float cur = pw[j] * ((float) k / g.w) - ub;
        if (cur > mx) mx = cur;
    }
    return mx;
}

// ComputeLoadImbalance (kway_core.h:852-861).
float imbalance_of(const KGraph &g, int k, const std::vector<int> &pw) {
    float mx = 1.0;
    for (int j = 0; j < k; ++j) {
        const float cur = pw[j] * ((float) k / g.w);
        if (cur > mx) mx = cur;
    }
    return mx;
}

// ComputeLoadImbalanceDiffWeighted (kway_core.h:890-900).
float imbalance_excess_2(const KGraph &g, const std::vector<int> &pw, const std::vector<float> &tw, float ub) {
    float mx = -1.0f;
    for (int i = 0; i < 2; ++i) {
        const float cur = pw[i] * (1.0f / (g.w * tw[i])) - ub;
        if (cur > mx) mx = cur;
    }
    return mx;
}

// balance_bisection (kway_core.h:875-884).
void balance_two_way(KGraph &g, BndSet &bnd, Side2 &s, const std::vector<float> &tw, std::vector<int> &pw,
                     std::vector<int> &side, float ub, LibcRand &R) {
    if (imbalance_excess(g, 2, pw, ub) <= 0) return;
    if (fabsf(tw[0] * g.w - pw[0]) < 3 * g.w / g.n) return;
    if (bnd.cnt > 0) balance_from_boundary(g, s, bnd, pw, tw, side, R);
    else balance_from_all(g, s, bnd, pw, tw, side, R);
}

// Compute2WayPartitionParams (kway_core.h:1064-1095).
void two_way_params(KGraph &g, BndSet &bnd, std::vector<int> &pw, const std::vector<int> &side, Side2 &s) {
    std::fill_n(pw.data(), 2, 0);
    bnd.clear();
    int cut = 0;
    for (int i = 0; i < g.n; ++i) pw[side[i]] += g.vw[i];
    for (int i = 0; i < g.n; ++i) {
        const int a = g.xadj[i], b = g.xadj[i + 1], me = side[i];
        int in = 0, ex = 0;
        for (int j = a; j < b; ++j) {
            if (me == side[g.adj[j]]) in += g.ew[j];
            else ex += g.ew[j];
        }
        s.in[i] = in;
        s.ex[i] = ex;
        if (ex > 0 || a == b) {
            bnd.add(i);
            cut += ex;
        }
    }
    g.cut = cut / 2;
}

// bisection (kway_core.h:1097-1185): max_tries graph-growing bisections from
// random seeds (breadth-first until side 1 falls to its bound), each balanced
// and refined by FM; the best cut is kept.
void grow_bisection(KGraph &g, BndSet &bnd, float ub, const std::vector<float> &tw, std::vector<int> &pw,
                    std::vector<int> &side, Side2 &s, int max_tries, int max_iter, LibcRand &R) {
    std::vector<int> trial(g.n), fifo(g.n), seen(g.n);
    const int maxw = ub * g.w * tw[1];
    const int minw = (1.0 / ub) * g.w * tw[1];
    int bestcut = 0;
    for (int t = 0; t < max_tries; ++t) {
        std::fill_n(trial.data(), g.n, 1);
        std::fill(seen.begin(), seen.end(), 0);
        int w[2];
        w[1] = g.w;
        w[0] = 0;
        fifo[0] = R.next() % g.n;
        seen[fifo[0]] = 1;
        int head = 0, tail = 1, left = g.n - 1, drain = 0;
        for (;;) {
            int v = 0;
            if (head == tail) {
                if (left == 0 || drain) break;
                int r = R.next() % left;
                for (v = 0; v < g.n; ++v) {
                    if (seen[v] == 0) {
                        if (r == 0) break;
                        --r;
                    }
                }
                fifo[0] = v;
                seen[v] = 1;
                head = 0;
                tail = 1;
                --left;
            }
            v = fifo[head++];
            if (w[0] > 0 && w[1] - g.vw[v] < minw) {
                drain = 1;
                continue;
            }
            trial[v] = 0;
            w[0] += g.vw[v];
            w[1] -= g.vw[v];
            if (w[1] <= maxw) break;
            drain = 0;
            for (int j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
                const int u = g.adj[j];
                if (seen[u] == 0) {
                    fifo[tail++] = u;
                    seen[u] = 1;
                    --left;
                }
            }
        }
        if (w[1] == 0) trial[R.next() % g.n] = 1;
        if (w[0] == 0) trial[R.next() % g.n] = 0;
        two_way_params(g, bnd, pw, trial, s);
        balance_two_way(g, bnd, s, tw, pw, trial, ub, R);
        fm_two_way(g, bnd, s, pw, tw, trial, max_iter, R);
        if (t == 0 || bestcut > g.cut) {
            bestcut = g.cut;
            std::copy_n(trial.data(), g.n, side.data());
            if (bestcut == 0) break;
        }
    }
    g.cut = bestcut;
}

// split_graph (kway_core.h:1187-1265): the two sides as graphs of their own
// (vertices in order; rows of interior vertices copied, boundary rows
// filtered), with the original labels carried along.
void split_two(const KGraph &g, const BndSet &bnd, const std::vector<int> &label, const std::vector<int> &side,
               KGraph &lg, std::vector<int> &llab, KGraph &rg, std::vector<int> &rlab) {
    int ns[2] = {0, 0}, ms[2] = {0, 0}, ws[2] = {0, 0};
    std::vector<int> rename(g.n);
    for (int i = 0; i < g.n; ++i) {
        const int p = side[i];
        rename[i] = ns[p]++;
        ws[p] += g.vw[i];
        ms[p] += g.xadj[i + 1] - g.xadj[i];
    }
    lg.reshape(ns[0], ms[0], ws[0]);
    rg.reshape(ns[1], ms[1], ws[1]);
    llab.resize(ns[0]);
    rlab.resize(ns[1]);
    KGraph *out[2] = {&lg, &rg};
    ns[0] = ns[1] = ms[0] = ms[1] = 0;
    lg.xadj[0] = rg.xadj[0] = 0;
    for (int i = 0; i < g.n; ++i) {
        const int p = side[i];
        KGraph &o = *out[p];
        if (!bnd.has(i)) {
            for (int j = g.xadj[i]; j < g.xadj[i + 1]; ++j) {
                o.adj[ms[p] + (j - g.xadj[i])] = g.adj[j];
                o.ew[ms[p] + (j - g.xadj[i])] = g.ew[j];
            }
            ms[p] += g.xadj[i + 1] - g.xadj[i];
        } else {
            int l = ms[p];
            for (int j = g.xadj[i]; j < g.xadj[i + 1]; ++j) {
                const int k = g.adj[j];
                if (side[k] == p) {
                    o.adj[l] = k;
                    o.ew[l++] = g.ew[j];
                }
            }
            ms[p] = l;
        }
        o.vw[ns[p]] = g.vw[i];
        if (p == 0) llab[ns[p]] = label[i];
        else rlab[ns[p]] = label[i];
        o.xadj[++ns[p]] = ms[p];
    }
    for (int p = 0; p < 2; ++p) {
        KGraph &o = *out[p];
        const int e = o.xadj[ns[p]];
        for (int i = 0; i < e; ++i) o.adj[i] = rename[o.adj[i]];
    }
    lg.m = ms[0];
    rg.m = ms[1];
}

// multilevel_bisection (kway_core.h:1267-1361). `side` and `spare` (and
// `bnd` and `bnd2`) are exchanged level by level as in the reference; the
// result ends in `side`.
void multilevel_two_way(KGraph &g, BndSet &bnd, std::vector<int> &side, const std::vector<float> &tw, int max_tries,
                        int threshold, float ub, int max_iter, BndSet &bnd2, std::vector<int> &spare, LibcRand &R) {
    int bestobj = 0, curobj = 0;
    float bestbal = 0.0, curbal = 0.0;
    if (g.n == 0) return;
    std::vector<int> pw(2);
    Side2 s(g.n);
    std::vector<int> match(g.n);
    int *const side_orig = side.data();
    std::vector<int> best;
    if (max_tries > 1) best.resize(g.n);
    for (int t = 0; t < max_tries; ++t) {
        std::vector<KGraph> levels;
        std::vector<std::vector<int> > cmaps;
        levels.push_back(g);
        const int maxvw = 1.5 * levels.back().w / threshold;
        do {
            KGraph &fine = levels.back();
            cmaps.emplace_back(fine.n);
            std::vector<int> &cm = cmaps.back();
            const int cn = heavy_edge_match(fine, match, cm, maxvw, R);
            KGraph coarse = contract_pairs(fine, match, cm, cn);
            levels.push_back(std::move(coarse));
        } while (levels.back().n > threshold && levels.back().n < 0.85 * levels[levels.size() - 2].n &&
                 levels.back().m > levels.back().n / 2);
        const int nlevels = (int) levels.size() - 1;
        bnd.cnt = 0;
        grow_bisection(levels.back(), bnd, ub, tw, pw, side, s, 2, max_iter, R);
        two_way_params(levels.back(), bnd, pw, side, s);
        for (int level = nlevels; level > 0; --level) {
            KGraph &coarse = levels[level];
            std::vector<int> &cm = cmaps[level - 1];
            balance_two_way(coarse, bnd, s, tw, pw, side, ub, R);
            fm_two_way(coarse, bnd, s, pw, tw, side, max_iter, R);
            KGraph &fine = levels[level - 1];
            bnd2.clear();
            project_two_way(fine, s, cm, bnd2, bnd, spare, side);
            fine.cut = coarse.cut;
            std::swap(bnd, bnd2);
            std::swap(side, spare);
        }
        balance_two_way(levels[0], bnd, s, tw, pw, side, ub, R);
        fm_two_way(levels[0], bnd, s, pw, tw, side, max_iter, R);
        g.cut = levels[0].cut;
        curobj = g.cut;
        curbal = imbalance_excess_2(g, pw, tw, ub);
        if (t == 0 || (curbal <= 0.0005 && bestobj > curobj) || (bestbal > 0.0005 && curbal < bestbal)) {
            bestobj = curobj;
            bestbal = curbal;
            if (t < max_tries - 1) std::copy_n(side.data(), g.n, best.data());
        }
        if (bestobj == 0) break;
    }
    if (bestobj != curobj) {
        std::copy_n(best.data(), g.n, side.data());
        two_way_params(g, bnd, pw, side, s);
    }
    if (side.data() != side_orig) std::copy_n(side.data(), g.n, side_orig);
}

// recursive_bisection (kway_core.h:1363-1390): bisect with target weights
// from tw, write the blocks of this level, split and recurse on both halves
// with renormalised targets.
void recursive_two_way(KGraph &g, BndSet &bnd, int k, const std::vector<int> &label, std::vector<int> &part,
                       float *tw, int first, int max_tries, int threshold, float ub, int max_iter, BndSet &bnd2,
                       std::vector<int> &side, std::vector<int> &spare, LibcRand &R) {
    std::vector<float> tw2(2);
    tw2[0] = std::accumulate(tw, tw + (k >> 1), 0.0f);
    tw2[1] = 1.0 - tw2[0];
    multilevel_two_way(g, bnd, side, tw2, max_tries, threshold, ub, max_iter, bnd2, spare, R);
    for (int i = 0; i < g.n; ++i) part[label[i]] = side[i] + first;
    KGraph lg, rg;
    std::vector<int> llab, rlab;
    if (k > 2) split_two(g, bnd, label, side, lg, llab, rg, rlab);
    const float wsum = std::accumulate(tw, tw + (k >> 1), 0.0f);
    std::transform(tw, tw + (k >> 1), tw, [wsum](float x) { return x / wsum; });
    std::transform(tw + (k >> 1), tw + k, tw + (k >> 1), [wsum](float x) { return x / (1.0f - wsum); });
    if (k > 3) {
        recursive_two_way(lg, bnd, (k >> 1), llab, part, tw, first, max_tries, threshold, ub, max_iter, bnd2, side,
                          spare, R);
        recursive_two_way(rg, bnd, k - (k >> 1), rlab, part, tw + (k >> 1), first + (k >> 1), max_tries, threshold,
                          ub, max_iter, bnd2, side, spare, R);
    } else if (k == 3) {
        recursive_two_way(rg, bnd, k - (k >> 1), rlab, part, tw + (k >> 1), first + (k >> 1), max_tries, threshold,
                          ub, max_iter, bnd2, side, spare, R);
    }
}

// recursive_bisection_head (kway_core.h:1392-1414): restarts the random
// sequence at 4321, as the reference does.
void recursive_kway(KGraph &g, int k, float ub, int max_tries, std::vector<int> &part, LibcRand &R) {
    std::fill_n(part.data(), g.n, 0);
    if (k == 1) return;
    R.seed_with(4321);
    ub += 0.0000499f;
    std::vector<float> tw(k, 1.0f / k);
    std::vector<int> label(g.n);
    for (int i = 0; i < g.n; ++i) label[i] = i;
    BndSet bnd(g.n), bnd2(g.n);
    std::vector<int> side(g.n), spare(g.n);
    recursive_two_way(g, bnd, k, label, part, tw.data(), 0, max_tries, 50, ub, 3, bnd2, side, spare, R);
}

// ComputeKWayPartitionParams (kway_core.h:743-784).
void kway_params(KGraph &g, BndSet &bnd, int k, std::vector<int> &pw, const std::vector<int> &part, KConn &C) {
    std::fill_n(pw.data(), k, 0);
    bnd.clear();
    C.clear();
    int cut = 0;
    for (int u = 0; u < g.n; ++u) pw[part[u]] += g.vw[u];
    for (int u = 0; u < g.n; ++u) {
        const int me = part[u];
        for (int j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            if (me == part[g.adj[j]]) C.add_in(u, g.ew[j]);
            else C.add_ex(u, g.ew[j]);
        }
        if (C.ex(u) == 0) continue;
        cut += C.ex(u);
        for (int j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
            const int other = part[g.adj[j]];
            if (me == other) continue;
            C.update(u, other, g.ew[j]);
        }
        if (C.ex(u) >= C.in(u)) bnd.add(u);
    }
    g.cut = cut / 2;
}

// ProjectKWayPartition (kway_core.h:786-840): projects the coarse blocks and
// rebuilds the connectivity of fine vertices whose coarse vertex had external
// weight (the others are interior).
void project_kway(KGraph &g, BndSet &bnd, std::vector<int> &cmap, std::vector<int> &part, KGraph &coarse,
                  const std::vector<int> &cpart, KConn &C) {
    for (int u = 0; u < g.n; ++u) {
        const int v = cmap[u];
        part[u] = cpart[v];
        cmap[u] = C.ex_copy(v);
    }
    C.clear();
    const int coarse_cut = coarse.cut;
    coarse.reshape(0, 0);
    bnd.clear();
    for (int i = 0; i < g.n; ++i) {
        const int a = g.xadj[i], b = g.xadj[i + 1];
        if (cmap[i] == 0) {
            int in = 0;
            for (int j = a; j < b; ++j) in += g.ew[j];
            C.set_in(i, in);
        } else {
            const int me = part[i];
            int in = 0, ex = 0;
            for (int j = a; j < b; ++j) {
                const int other = part[g.adj[j]];
                if (me == other) {
                    in += g.ew[j];
                } else {
                    ex += g.ew[j];
                    C.update(i, other, g.ew[j]);
                }
            }
            C.set_in(i, in);
            C.set_ex(i, ex);
            if (ex > 0 && ex - in >= 0) bnd.add(i);
        }
    }
    g.cut = coarse_cut;
}

// compute_boundary (kway_core.h:842-850).
void kway_boundary(const KGraph &g, BndSet &bnd, int type, const KConn &C) {
    bnd.clear();
    for (int u = 0; u < g.n; ++u)
        if (C.ex(u) > 0 && (type != BND_REFINE || C.ex(u) >= C.in(u))) bnd.add(u);
}

// is_balanced (kway_core.h:886-888).
bool balanced(const KGraph &g, int k, const std::vector<int> &pw, float ub, float slack) {
    return imbalance_excess(g, k, pw, ub) <= slack;
}

// UpdateAdjacentVertexInfoAndBND (kway_core.h:49-79).
void neighbour_moved(int v, int v_id, int from, int to, int w, KConn &C, BndSet &bnd, int type) {
    if (v_id == from) {
        C.add_ex(v, w);
        C.add_in(v, -w);
        if (type == BND_REFINE) {
            if (C.ex(v) - C.in(v) >= 0 && !bnd.has(v)) bnd.add(v);
        } else if (C.ex(v) > 0 && !bnd.has(v)) {
            bnd.add(v);
        }
    } else if (v_id == to) {
        C.add_in(v, w);
        C.add_ex(v, -w);
        if (type == BND_REFINE) {
            if (C.ex(v) - C.in(v) < 0 && bnd.has(v)) bnd.remove(v);
        } else if (C.ex(v) <= 0 && bnd.has(v)) {
            bnd.remove(v);
        }
    }
    if (v_id != from) C.update(v, from, -w);
    if (v_id != to) C.update(v, to, w);
}

// UpdateMovedVertexInfoAndBND (kway_core.h:81-103).
void vertex_moved(int u, int from, int to, KConn &C, BndSet &bnd, std::vector<int> &part, int type) {
    part[u] = to;
    const int w_to = C.get(u, to);
    C.add_ex(u, C.in(u) - w_to);
    const int old_in = C.in(u);
    C.set_in(u, w_to);
    C.update(u, to, -w_to);
    C.update(u, from, old_in);
    if (type == BND_REFINE) {
        if (bnd.has(u) && C.ex(u) - C.in(u) < 0) bnd.remove(u);
        if (!bnd.has(u) && C.ex(u) - C.in(u) >= 0) bnd.add(u);
    } else {
        if (bnd.has(u) && C.ex(u) <= 0) bnd.remove(u);
        if (!bnd.has(u) && C.ex(u) > 0) bnd.add(u);
    }
}

inline float rgain_of(const KConn &C, int u) {
    return (C.nconn(u) > 0 ? 1.0f * C.ex(u) / std::sqrt(static_cast<float>(C.nconn(u))) : 0.0f) - C.in(u);
}

// Greedy_KWayCutOptimize (kway_core.h:902-1062): greedy k-way refinement (or
// balancing) over the boundary, vertices taken by a float priority.
void greedy_kway(KGraph &g, BndSet &bnd, int k, float ub, std::vector<int> &pw, std::vector<int> &part, int max_iter,
                 int mode, KConn &C, LibcRand &R) {
    const int type = mode == OPT_REFINE ? BND_REFINE : BND_BALANCE;
    if (mode != OPT_BALANCE) {
        const float cur = imbalance_of(g, k, pw);
        ub = (ub > cur) ? ub : cur;
    }
    const int maxpw = (1.0f / k) * g.w * ub;
    const int minpw = (1.0f / k) * g.w * (1.0f / ub);
    std::vector<int> perm(g.n), moved(g.n, -1);
    MaxHeap<float> q(g.n);
    for (int pass = 0; pass < max_iter; ++pass) {
        if (mode == OPT_BALANCE) {
            bool stop = true;
            for (int i = 0; i < k; ++i)
                if (pw[i] > maxpw || pw[i] < minpw) {
                    stop = false;
                    break;
                }
            if (stop) break;
        }
        const int oldcut = g.cut;
        for (int i = 0; i < bnd.cnt; ++i) perm[i] = i;
        shuffle(bnd.cnt, perm, bnd.cnt / 4, R);
        for (int i = 0; i < bnd.cnt; ++i) {
            const int u = bnd.val[perm[i]];
            q.insert(u, rgain_of(C, u));
        }
        int nmoved = 0;
        while (!q.empty()) {
            const int u = q.pop();
            moved[u] = pass;
            const int from = part[u];
            const int uw = g.vw[u];
            int to, jj;
            if (mode == OPT_REFINE) {
                for (jj = C.nconn(u) - 1; jj >= 0; --jj) {
                    to = C.conn_id(u, jj);
                    if ((C.conn_w(u, jj) > C.in(u) && (pw[from] - uw >= minpw || pw[to] < pw[from] - uw) &&
                         (pw[to] + uw <= maxpw || pw[to] < pw[from] - uw)) ||
                        (C.conn_w(u, jj) == C.in(u) && pw[to] < pw[from] - uw))
                        break;
                }
                if (jj < 0) continue;
                for (int j = jj - 1; j >= 0; --j) {
                    to = C.conn_id(u, j);
                    if ((C.conn_w(u, j) > C.conn_w(u, jj) && (pw[from] - uw >= minpw || pw[to] < pw[from] - uw) &&
                         (pw[to] + uw <= maxpw || pw[to] < pw[from] - uw)) ||
                        (C.conn_w(u, j) == C.conn_w(u, jj) && pw[to] < pw[C.conn_id(u, jj)]))
                        jj = j;
                }
                to = C.conn_id(u, jj);
            } else {
                for (jj = C.nconn(u) - 1; jj >= 0; --jj) {
                    to = C.conn_id(u, jj);
                    if (from >= k || pw[to] < pw[from] - uw) break;
                }
                if (jj < 0) continue;
                for (int j = jj - 1; j >= 0; --j) {
                    to = C.conn_id(u, j);
                    if (pw[to] < pw[C.conn_id(u, jj)]) jj = j;
                }
                to = C.conn_id(u, jj);
            }
            g.cut -= C.conn_w(u, jj) - C.in(u);
            ++nmoved;
            pw[to] += uw;
            pw[from] -= uw;
            vertex_moved(u, from, to, C, bnd, part, type);
            for (int j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
                const int v = g.adj[j];
                const int w = g.ew[j];
                const int v_id = part[v];
                const int before = C.nconn(v);
                neighbour_moved(v, v_id, from, to, w, C, bnd, type);
                if (!(v_id == to || v_id == from || before != C.nconn(v))) continue;
                if (moved[v] == pass) continue;
                const float rg = rgain_of(C, v);
                const bool keep = type == BND_REFINE ? C.ex(v) - C.in(v) >= 0 : C.ex(v) > 0;
                if (q.contains(v)) {
                    if (keep) q.update(v, rg);
                    else q.erase(v);
                } else if (keep) {
                    q.insert(v, rg);
                }
            }
        }
        if (nmoved == 0 || (mode == OPT_REFINE && g.cut == oldcut)) break;
    }
}

// multilevel_partition (kway_core.h:1416-1525): coarsen to `threshold`
// vertices, recursive bisection of the coarsest graph, greedy k-way
// balancing and refinement on every level while projecting back.
int multilevel_kway(KGraph &g, int k, float ub, std::vector<int> &part, int threshold, int n_init, int max_tries,
                    int max_iter, LibcRand &R) {
    int curobj = 0, bestobj = 0;
    float curbal = 0.0f, bestbal = 0.0f;
    BndSet bnd(g.n);
    std::vector<int> pw(k), where1(g.n), where2(g.n), match(g.n);
    std::vector<KGraph> levels;
    std::vector<std::vector<int> > cmaps;
    KConn C(g.n, k);
    for (int t = 0; t < max_tries; ++t) {
        levels.clear();
        cmaps.clear();
        levels.push_back(g);
        const int maxvw = 1.5 * levels.back().w / threshold;
        do {
            KGraph &fine = levels.back();
            cmaps.emplace_back(fine.n);
            std::vector<int> &cm = cmaps.back();
            const int cn = heavy_edge_match(fine, match, cm, maxvw, R);
            KGraph coarse = contract_pairs(fine, match, cm, cn);
            levels.push_back(std::move(coarse));
        } while (levels.back().n > threshold && levels.back().n < 0.85 * levels[levels.size() - 2].n &&
                 levels.back().m > levels.back().n / 2);
        const float ub_level = (float) std::pow(ub, 1.0 / std::log(k));
        recursive_kway(levels.back(), k, ub_level, n_init, where1, R);
        const int nlevels = (int) cmaps.size();
        bnd.cnt = 0;
        kway_params(levels.back(), bnd, k, pw, where1, C);
        int cl = nlevels;
        for (int pass = 0; cl >= 0; ++pass) {
            KGraph &cg = levels[cl];
            if (2 * pass >= nlevels && !balanced(cg, k, pw, ub, .02f)) {
                kway_boundary(cg, bnd, BND_BALANCE, C);
                greedy_kway(cg, bnd, k, ub, pw, where1, 1, OPT_BALANCE, C, R);
                kway_boundary(cg, bnd, BND_REFINE, C);
            }
            greedy_kway(cg, bnd, k, ub, pw, where1, max_iter, OPT_REFINE, C, R);
            if (cl > 0) {
                KGraph &fine = levels[cl - 1];
                C.swap_copies();
                project_kway(fine, bnd, cmaps[cl - 1], where2, cg, where1, C);
                std::swap(where1, where2);
            }
            --cl;
        }
        g.cut = levels[0].cut;
        if (!balanced(levels[0], k, pw, ub, 0.0f)) {
            kway_boundary(levels[0], bnd, BND_BALANCE, C);
            greedy_kway(levels[0], bnd, k, ub, pw, where1, 3, OPT_BALANCE, C, R);
            kway_boundary(levels[0], bnd, BND_REFINE, C);
            greedy_kway(levels[0], bnd, k, ub, pw, where1, max_iter, OPT_REFINE, C, R);
        }
        g.cut = levels[0].cut;
        curobj = g.cut;
        curbal = imbalance_excess(g, k, pw, ub);
        if (t == 0 || (curbal <= 0.0005f && bestobj > curobj) || (bestbal > 0.0005f && curbal < bestbal)) {
            std::copy_n(where1.data(), g.n, part.data());
            bestobj = curobj;
            bestbal = curbal;
        }
        if (bestobj == 0) break;
    }
    return bestobj;
}

} // namespace

// partition (kway_core.h:1527-1545) on a copy of the caller's CSR
// (kway_core.h:1548-1571 builds the same int arrays).
void metis_kway(u32 n, const u32 *xadj, const u32 *adj, const s32 *vw, const s32 *ew, int k, float imbalance,
                int seed, u32 *part) {
    for (u32 u = 0; u < n; ++u) part[u] = 0;
    if (k == 1 || n == 0) return;
    s64 total = 0;
    for (u32 u = 0; u < n; ++u) total += vw ? vw[u] : 1;
    KGraph g((int) n, (int) xadj[n], (int) total);
    for (u32 u = 0; u <= n; ++u) g.xadj[u] = (int) xadj[u];
    for (u32 u = 0; u < n; ++u) g.vw[u] = vw ? vw[u] : 1;
    for (u32 j = 0; j < xadj[n]; ++j) {
        g.adj[j] = (int) adj[j];
        g.ew[j] = ew ? ew[j] : 1;
    }
    const int uf = static_cast<int>(imbalance * 1000.0f);
    float ub = 1.0f + 0.001f * uf;
    ub += 0.0000499f;
    LibcRand R((u32) seed);
    const int candidate = static_cast<int>((double) g.n / (40.0 * log2(k)));
    const int threshold = (candidate > 30 * k) ? candidate : 30 * k;
    std::vector<int> out(n, 0);
    multilevel_kway(g, k, ub, out, threshold, 1, 1, 3, R);
    for (u32 u = 0; u < n; ++u) part[u] = (u32) out[u];
}

} // namespace hp
