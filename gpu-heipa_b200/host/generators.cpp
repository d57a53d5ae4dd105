#include "generators.h"

#include <algorithm>
#include <cmath>
#include <parallel/algorithm>
#include <omp.h>

namespace hp {
namespace {

inline s32 pair_weight(u64 seed, u32 a, u32 b, s32 lo, s32 hi) {
    u32 x = a < b ? a : b, y = a < b ? b : a;
    u64 h = splitmix64(seed * 0x9E3779B97F4A7C15ull ^ (((u64) x << 32) | (u64) y));
    return lo + (s32) (h % (u64) (hi - lo + 1));
}

// Builds a symmetric CSR from sorted unique canonical keys (min << 32 | max).
HostCSR csr_from_keys(u32 n, const std::vector<u64> &keys, size_t nkeys, s32 w_lo, s32 w_hi, u64 wseed) {
    HostCSR g;
    g.n = n;
    g.xadj.assign((size_t) n + 1, 0);
    for (size_t i = 0; i < nkeys; ++i) {
        ++g.xadj[(keys[i] >> 32) + 1];
        ++g.xadj[(keys[i] & 0xFFFFFFFFull) + 1];
    }
    for (u32 u = 0; u < n; ++u) g.xadj[u + 1] += g.xadj[u];
    g.m = g.xadj[n];
    g.adj.resize(g.m);
    const bool weighted = w_hi > 0;
    if (weighted) g.ew.resize(g.m);
    std::vector<u32> cur(g.xadj.begin(), g.xadj.end() - 1);
    // keys sorted by (min, max): row u first receives all x < u (as the max of
    // key (x,u), in ascending x), then all y > u (ascending) -> sorted rows
    for (size_t i = 0; i < nkeys; ++i) {
        u32 a = (u32) (keys[i] >> 32), b = (u32) (keys[i] & 0xFFFFFFFFull);
        s32 w = weighted ? pair_weight(wseed, a, b, w_lo, w_hi) : 1;
        u32 pa = cur[a]++, pb = cur[b]++;
        g.adj[pa] = b;
        g.adj[pb] = a;
        if (weighted) {
            g.ew[pa] = w;
            g.ew[pb] = w;
        }
    }
    return g;
}

} // namespace

HostCSR gen_grid(u32 w, u32 h, s32 w_lo, s32 w_hi, u64 seed) {
    HostCSR g;
    g.n = w * h;
    g.xadj.assign((size_t) g.n + 1, 0);
    const bool weighted = w_hi > 0;
    for (u32 y = 0; y < h; ++y) {
        for (u32 x = 0; x < w; ++x) {
            u32 u = y * w + x;
            u32 nb[4];
            int c = 0;
            if (y > 0) nb[c++] = u - w;
            if (x > 0) nb[c++] = u - 1;
            if (x + 1 < w) nb[c++] = u + 1;
            if (y + 1 < h) nb[c++] = u + w;
            for (int i = 0; i < c; ++i) {
                g.adj.push_back(nb[i]);
                if (weighted) g.ew.push_back(pair_weight(seed, u, nb[i], w_lo, w_hi));
            }
            g.xadj[u + 1] = (u32) g.adj.size();
        }
    }
    g.m = (u32) g.adj.size();
    return g;
}

HostCSR gen_rmat(u32 scale, u32 edge_factor, double a, double b, double c, s32 w_lo, s32 w_hi, u64 seed,
                 bool explicit_vw) {
    const u32 n = 1u << scale;
    const u64 ne = (u64) edge_factor * (u64) n;
    std::vector<u32> perm(n);
    for (u32 i = 0; i < n; ++i) perm[i] = i;
    {
        Rng64 rng(seed ^ 0x7065726D75746521ull);
        for (u32 i = n; i > 1; --i) std::swap(perm[i - 1], perm[rng.below(i)]);
    }
    const double ta = a * 4294967296.0, tb = (a + b) * 4294967296.0, tc = (a + b + c) * 4294967296.0;
    std::vector<u64> keys(ne);
#pragma omp parallel for schedule(static)
    for (s64 i = 0; i < (s64) ne; ++i) {
        u64 st = splitmix64(seed ^ ((u64) i * 0xA24BAED4963EE407ull));
        u32 u = 0, v = 0;
        u64 bits = 0;
        for (u32 l = 0; l < scale; ++l) {
            if ((l & 1) == 0) {
                st += 0x9E3779B97F4A7C15ull;
                bits = splitmix64(st);
            }
            double r = (double) (u32) (bits >> ((l & 1) * 32));
            u32 ub, vb;
            if (r < ta) {
                ub = 0;
                vb = 0;
            } else if (r < tb) {
                ub = 0;
                vb = 1;
            } else if (r < tc) {
                ub = 1;
                vb = 0;
            } else {
                ub = 1;
                vb = 1;
            }
            u = (u << 1) | ub;
            v = (v << 1) | vb;
        }
        u32 pu = perm[u], pv = perm[v];
        if (pu == pv) keys[i] = ~0ull;
        else keys[i] = pu < pv ? (((u64) pu << 32) | pv) : (((u64) pv << 32) | pu);
    }
    __gnu_parallel::sort(keys.begin(), keys.end());
    size_t nk = 0;
    for (size_t i = 0; i < keys.size(); ++i) {
        if (keys[i] == ~0ull) break;
        if (nk == 0 || keys[nk - 1] != keys[i]) keys[nk++] = keys[i];
    }
    HostCSR g = csr_from_keys(n, keys, nk, w_lo, w_hi, seed ^ 0x77656967687473ull);
    if (explicit_vw) g.vw.assign(n, 1);
    return g;
}

double rgg3d_radius(u32 n, double mean_degree) {
    // expected degree in the unit cube: (n-1) * (4/3 pi r^3 - 3/2 pi r^4) + O(r^5)
    const double pi = 3.14159265358979323846;
    double r = std::cbrt(mean_degree / ((double) (n - 1) * 4.0 / 3.0 * pi));
    for (int it = 0; it < 50; ++it) {
        double f = (double) (n - 1) * (4.0 / 3.0 * pi * r * r * r - 1.5 * pi * r * r * r * r) - mean_degree;
        double df = (double) (n - 1) * (4.0 * pi * r * r - 6.0 * pi * r * r * r);
        r -= f / df;
    }
    return r;
}

HostCSR gen_rgg3d(u32 n, double mean_degree, s32 w_lo, s32 w_hi, u64 seed, bool explicit_vw) {
    const double r = rgg3d_radius(n, mean_degree);
    const double r2 = r * r;
    std::vector<float> px(n), py(n), pz(n);
#pragma omp parallel for schedule(static)
    for (s64 i = 0; i < (s64) n; ++i) {
        u64 h = splitmix64(seed ^ ((u64) i * 0xD6E8FEB86659FD93ull));
        u64 h2 = splitmix64(h);
        px[i] = (float) ((double) (h >> 11) * (1.0 / 9007199254740992.0));
        py[i] = (float) ((double) (h2 >> 11) * (1.0 / 9007199254740992.0));
        pz[i] = (float) ((double) (splitmix64(h2) >> 11) * (1.0 / 9007199254740992.0));
    }
    const u32 G = std::max<u32>(1, (u32) std::floor(1.0 / r));
    const u64 ncell = (u64) G * G * G;
    auto cell_of = [&](u32 i, u32 &cx, u32 &cy, u32 &cz) {
        cx = std::min<u32>(G - 1, (u32) (px[i] * (float) G));
        cy = std::min<u32>(G - 1, (u32) (py[i] * (float) G));
        cz = std::min<u32>(G - 1, (u32) (pz[i] * (float) G));
    };
    std::vector<u32> cstart(ncell + 1, 0), order(n);
    for (u32 i = 0; i < n; ++i) {
        u32 cx, cy, cz;
        cell_of(i, cx, cy, cz);
        ++cstart[((u64) cz * G + cy) * G + cx + 1];
    }
    for (u64 c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    {
        std::vector<u32> cur(cstart.begin(), cstart.end() - 1);
        for (u32 i = 0; i < n; ++i) {
            u32 cx, cy, cz;
            cell_of(i, cx, cy, cz);
            order[cur[((u64) cz * G + cy) * G + cx]++] = i;
        }
    }
    auto visit = [&](u32 i, auto &&fn) {
        u32 cx, cy, cz;
        cell_of(i, cx, cy, cz);
        for (int dz = -1; dz <= 1; ++dz) {
            s64 z = (s64) cz + dz;
            if (z < 0 || z >= G) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                s64 y = (s64) cy + dy;
                if (y < 0 || y >= G) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    s64 x = (s64) cx + dx;
                    if (x < 0 || x >= G) continue;
                    u64 c = ((u64) z * G + (u64) y) * G + (u64) x;
                    for (u32 t = cstart[c]; t < cstart[c + 1]; ++t) {
                        u32 j = order[t];
                        if (j == i) continue;
                        double ddx = (double) px[i] - px[j], ddy = (double) py[i] - py[j], ddz = (double) pz[i] - pz[j];
                        if (ddx * ddx + ddy * ddy + ddz * ddz < r2) fn(j);
                    }
                }
            }
        }
    };
    HostCSR g;
    g.n = n;
    g.xadj.assign((size_t) n + 1, 0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (s64 i = 0; i < (s64) n; ++i) {
        u32 cnt = 0;
        visit((u32) i, [&](u32) { ++cnt; });
        g.xadj[i + 1] = cnt;
    }
    for (u32 u = 0; u < n; ++u) g.xadj[u + 1] += g.xadj[u];
    g.m = g.xadj[n];
    g.adj.resize(g.m);
    const bool weighted = w_hi > 0;
    if (weighted) g.ew.resize(g.m);
    const u64 wseed = seed ^ 0x77656967687473ull;
#pragma omp parallel for schedule(dynamic, 4096)
    for (s64 i = 0; i < (s64) n; ++i) {
        u32 p = g.xadj[i];
        visit((u32) i, [&](u32 j) { g.adj[p++] = j; });
        std::sort(g.adj.begin() + g.xadj[i], g.adj.begin() + g.xadj[i + 1]);
        if (weighted)
            for (u32 t = g.xadj[i]; t < g.xadj[i + 1]; ++t) g.ew[t] = pair_weight(wseed, (u32) i, g.adj[t], w_lo, w_hi);
    }
    if (explicit_vw) g.vw.assign(n, 1);
    return g;
}

} // namespace hp
