#include "metis_io.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <charconv>
#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace hp {
namespace {

struct Mapped {
    const char *data = nullptr;
    size_t size = 0;
    int fd = -1;
    ~Mapped() {
        if (data && size) munmap((void *) data, size);
        if (fd >= 0) close(fd);
    }
};

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// Parses an unsigned decimal at p (after skipping blanks); returns false if
// no digit is present before end of line.
inline bool parse_u64(const char *&p, const char *end, u64 &out) {
    while (p < end && is_space(*p)) ++p;
    if (p >= end || *p < '0' || *p > '9') return false;
    u64 v = 0;
    while (p < end && *p >= '0' && *p <= '9') {
        v = v * 10 + (u64) (*p - '0');
        ++p;
    }
    out = v;
    return true;
}

inline void skip_line(const char *&p, const char *end) {
    while (p < end && *p != '\n') ++p;
    if (p < end) ++p;
}

// Vertex lines of the body, one after another (the reference's reader loop,
// host_graph.h:187-240): '%' lines are skipped, an empty line is a vertex
// without neighbours, lines after the n-th vertex are ignored. Reports the
// exact error of the first malformed line.
int parse_body_seq(const char *p, const char *end, HostCSR &g, u64 n, bool has_vw, bool has_ew,
                   std::string &err) {
    u64 cur = 0;
    u32 u = 0;
    while (u < g.n) {
        if (p >= end) {
            err = "unexpected end of file at vertex " + std::to_string(u + 1);
            return 1;
        }
        if (*p == '%') {
            skip_line(p, end);
            continue;
        }
        if (has_vw) {
            u64 w;
            if (!parse_u64(p, end, w)) {
                err = "missing vertex weight at vertex " + std::to_string(u + 1);
                return 1;
            }
            g.vw[u] = (s32) w;
        }
        for (;;) {
            u64 v;
            if (!parse_u64(p, end, v)) break;
            if (v == 0 || v > n) {
                err = "neighbour id out of range at vertex " + std::to_string(u + 1);
                return 1;
            }
            if (cur >= g.m) {
                err = "more edges than the header states";
                return 1;
            }
            g.adj[cur] = (u32) (v - 1);
            if (has_ew) {
                u64 w;
                if (!parse_u64(p, end, w)) {
                    err = "missing edge weight at vertex " + std::to_string(u + 1);
                    return 1;
                }
                g.ew[cur] = (s32) w;
            }
            ++cur;
        }
        while (p < end && is_space(*p)) ++p;
        if (p < end && *p != '\n') {
            err = "unexpected character at vertex " + std::to_string(u + 1);
            return 1;
        }
        if (p < end) ++p;
        g.xadj[++u] = (u32) cur;
    }
    if (cur != g.m) {
        err = "number of expected edges " + std::to_string(g.m) + " not equal to number of edges " +
              std::to_string(cur) + " found";
        return 1;
    }
    return 0;
}

inline const char *line_end(const char *p, const char *end) {
    const void *q = memchr(p, '\n', (size_t) (end - p));
    return q ? (const char *) q : end;
}

// Numeric tokens of one line, or -1 when the line holds anything but blanks
// and unsigned decimals.
inline long count_tokens(const char *p, const char *e) {
    long t = 0;
    while (p < e) {
        while (p < e && is_space(*p)) ++p;
        if (p >= e) break;
        if (*p < '0' || *p > '9') return -1;
        while (p < e && *p >= '0' && *p <= '9') ++p;
        if (p < e && !is_space(*p)) return -1;
        ++t;
    }
    return t;
}

constexpr size_t PAR_MIN_BYTES = 4u << 20;  // smaller bodies are parsed by one thread
constexpr size_t PAR_CHUNK_BYTES = 1u << 20;

// The same parse in chunks of whole lines on all host threads: pass 1 counts
// the vertex lines of each chunk and the numbers on each line, a prefix sum
// gives every line its vertex id and CSR offset, pass 2 parses the lines into
// place. Returns false on anything unusual (malformed line, missing lines,
// wrong edge count, id out of range); the caller then runs the sequential
// parse, which reports the exact error.
bool parse_body_par(const char *p, const char *end, HostCSR &g, u64 n, bool has_vw, bool has_ew) {
    const size_t bytes = (size_t) (end - p);
    const size_t threads = (size_t) omp_get_max_threads();
    const size_t T = std::max<size_t>(1, std::min<size_t>(threads * 4, bytes / PAR_CHUNK_BYTES));
    std::vector<const char *> cb(T + 1);
    cb[0] = p;
    cb[T] = end;
    for (size_t t = 1; t < T; ++t) {
        const char *q = std::max(cb[t - 1], p + bytes / T * t);
        q = line_end(q, end);
        cb[t] = q < end ? q + 1 : end;
    }
    // pass 1: numbers on each vertex line (-1: malformed), per chunk
    std::vector<std::vector<long> > toks(T);
#pragma omp parallel for schedule(dynamic, 1)
    for (long t = 0; t < (long) T; ++t) {
        std::vector<long> &v = toks[(size_t) t];
        v.reserve((size_t) (cb[t + 1] - cb[t]) / 8 + 1);
        for (const char *q = cb[t]; q < cb[t + 1];) {
            const char *e = line_end(q, cb[t + 1]);
            if (*q != '%') v.push_back(count_tokens(q, e));
            q = e + 1;
        }
    }
    // first vertex id of each chunk; entries per vertex -> offsets
    std::vector<u64> first(T + 1, 0);
    for (size_t t = 0; t < T; ++t) first[t + 1] = first[t] + toks[t].size();
    if (first[T] < n) return false;
    const long per = has_ew ? 2 : 1, lead = has_vw ? 1 : 0;
    g.xadj[0] = 0;
    u64 cur = 0;
    for (size_t t = 0; t < T && first[t] < n; ++t) {
        const std::vector<long> &v = toks[t];
        for (size_t i = 0; i < v.size() && first[t] + i < n; ++i) {
            const long c = v[i] - lead;
            if (v[i] < 0 || c < 0 || c % per != 0) return false;
            cur += (u64) (c / per);
            if (cur > g.m) return false;
            g.xadj[first[t] + i + 1] = (u32) cur;
        }
    }
    if (cur != g.m) return false;
    // pass 2: parse into place (every line is known to be well formed)
    bool bad = false;
#pragma omp parallel for schedule(dynamic, 1) reduction(|| : bad)
    for (long t = 0; t < (long) T; ++t) {
        u64 u = first[(size_t) t];
        for (const char *q = cb[t]; q < cb[t + 1] && u < n && !bad;) {
            const char *e = line_end(q, cb[t + 1]);
            if (*q != '%') {
                const char *r = q;
                u64 x = 0;
                if (has_vw) {
                    parse_u64(r, e, x);
                    g.vw[u] = (s32) x;
                }
                for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
                    parse_u64(r, e, x);
                    if (x == 0 || x > n) {
                        bad = true;
                        break;
                    }
                    g.adj[j] = (u32) (x - 1);
                    if (has_ew) {
                        parse_u64(r, e, x);
                        g.ew[j] = (s32) x;
                    }
                }
                ++u;
            }
            q = e + 1;
        }
    }
    return !bad;
}

} // namespace

int read_metis(const std::string &path, HostCSR &g, std::string &err) {
    Mapped mm;
    mm.fd = open(path.c_str(), O_RDONLY | O_CLOEXEC);
    if (mm.fd < 0) {
        err = "cannot open " + path;
        return 1;
    }
    struct stat st{};
    if (fstat(mm.fd, &st) != 0) {
        err = "cannot stat " + path;
        return 1;
    }
    mm.size = (size_t) st.st_size;
    if (mm.size == 0) {
        err = "empty file " + path;
        return 1;
    }
    void *addr = mmap(nullptr, mm.size, PROT_READ, MAP_PRIVATE | MAP_POPULATE, mm.fd, 0);
    if (addr == MAP_FAILED) {
        err = "cannot mmap " + path;
        mm.size = 0;
        return 1;
    }
    mm.data = (const char *) addr;
    madvise(addr, mm.size, MADV_SEQUENTIAL | MADV_WILLNEED);
    const char *p = mm.data, *end = mm.data + mm.size;

    while (p < end && *p == '%') skip_line(p, end);
    u64 n = 0, m_und = 0;
    if (!parse_u64(p, end, n) || !parse_u64(p, end, m_und)) {
        err = "malformed header";
        return 1;
    }
    bool has_vw = false, has_ew = false;
    {
        const char *q = p;
        while (q < end && is_space(*q)) ++q;
        if (q < end && *q >= '0' && *q <= '9') {
            const char *s = q;
            while (q < end && *q >= '0' && *q <= '9') ++q;
            std::string fmt(s, q);
            // right-aligned: last digit = edge weights, second to last = vertex weights
            if (fmt.size() >= 1) has_ew = fmt[fmt.size() - 1] == '1';
            if (fmt.size() >= 2) has_vw = fmt[fmt.size() - 2] == '1';
            if (fmt.size() >= 3 && fmt[fmt.size() - 3] == '1') {
                err = "vertex sizes (fmt 1xx) are not supported";
                return 1;
            }
            u64 ncon = 0;
            const char *r = q;
            if (parse_u64(r, end, ncon) && ncon > 1) {
                err = "multi-constraint graphs are not supported";
                return 1;
            }
        }
    }
    skip_line(p, end);
    if (n >= 0xFFFFFFFFull || 2 * m_und >= 0xFFFFFFFFull) {
        err = "graph too large for 32-bit ids/offsets";
        return 1;
    }
    g.n = (u32) n;
    g.m = (u32) (2 * m_und);
    g.xadj.assign(g.n + 1, 0);
    g.adj.resize(g.m);
    g.ew.clear();
    g.vw.clear();
    if (has_ew) g.ew.resize(g.m);
    if (has_vw) g.vw.resize(g.n);

    if ((size_t) (end - p) >= PAR_MIN_BYTES && omp_get_max_threads() > 1 &&
        parse_body_par(p, end, g, n, has_vw, has_ew))
        return 0;
    return parse_body_seq(p, end, g, n, has_vw, has_ew, err);
}

namespace {

// Formats items [0, count) in ranges (ends[i-1], ends[i]] on all host threads,
// a few ranges per thread at a time, and writes the texts in order, so the
// buffered text stays a few MB per thread.
template<typename Fmt>
bool write_ranges(FILE *f, const std::vector<u64> &ends, Fmt fmt) {
    const size_t R = ends.size();
    const size_t batch = (size_t) omp_get_max_threads() * 2;
    std::vector<std::string> bufs(std::min(batch, R));
    for (size_t r0 = 0; r0 < R; r0 += batch) {
        const size_t r1 = std::min(R, r0 + batch);
#pragma omp parallel for schedule(dynamic, 1)
        for (long r = (long) r0; r < (long) r1; ++r) {
            std::string &b = bufs[(size_t) r - r0];
            b.clear();
            fmt(r == 0 ? 0 : ends[(size_t) r - 1], ends[(size_t) r], b);
        }
        for (size_t r = r0; r < r1; ++r)
            if (fwrite(bufs[r - r0].data(), 1, bufs[r - r0].size(), f) != bufs[r - r0].size()) return false;
    }
    return true;
}

// Range ends over [0, n) with about `per` units each, by a prefix of units.
template<typename Units>
std::vector<u64> split_ranges(u64 n, u64 per, Units units) {
    std::vector<u64> ends;
    u64 acc = 0;
    for (u64 u = 0; u < n; ++u) {
        acc += units(u);
        if (acc >= per) {
            ends.push_back(u + 1);
            acc = 0;
        }
    }
    if (ends.empty() || ends.back() != n) ends.push_back(n);
    return ends;
}

} // namespace

int write_metis(const std::string &path, const HostCSR &g, bool write_vw, bool write_ew, std::string &err) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) {
        err = "cannot open " + path;
        return 1;
    }
    std::string head = std::to_string(g.n) + " " + std::to_string(g.m / 2);
    if (write_vw || write_ew) head += std::string(" 0") + (write_vw ? "1" : "0") + (write_ew ? "1" : "0");
    head += "\n";
    bool ok = fwrite(head.data(), 1, head.size(), f) == head.size();
    // about 2^18 entries (a few MB of text) per range
    const std::vector<u64> ends =
        split_ranges(g.n, 1u << 18, [&](u64 u) { return (u64) (g.xadj[u + 1] - g.xadj[u]) + 1; });
    ok = ok && write_ranges(f, ends, [&](u64 lo, u64 hi, std::string &buf) {
        char tmp[32];
        for (u64 u = lo; u < hi; ++u) {
            bool first = true;
            if (write_vw) {
                auto r = std::to_chars(tmp, tmp + 32, g.vw.empty() ? 1 : g.vw[u]);
                buf.append(tmp, r.ptr);
                first = false;
            }
            for (u32 j = g.xadj[u]; j < g.xadj[u + 1]; ++j) {
                if (!first) buf.push_back(' ');
                first = false;
                auto r = std::to_chars(tmp, tmp + 32, (u64) g.adj[j] + 1);
                buf.append(tmp, r.ptr);
                if (write_ew) {
                    buf.push_back(' ');
                    auto r2 = std::to_chars(tmp, tmp + 32, g.ew.empty() ? 1 : g.ew[j]);
                    buf.append(tmp, r2.ptr);
                }
            }
            buf.push_back('\n');
        }
    });
    if (fclose(f) != 0 || !ok) {
        err = "write failed " + path;
        return 1;
    }
    return 0;
}

int write_partition(const std::string &path, const u32 *part, u32 n, std::string &err) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) {
        err = "could not open " + path + " to write partition";
        return 1;
    }
    std::vector<u64> ends;
    for (u64 e = 1u << 18; e < n; e += 1u << 18) ends.push_back(e);
    ends.push_back(n);
    const bool ok = write_ranges(f, ends, [&](u64 lo, u64 hi, std::string &buf) {
        char tmp[16];
        for (u64 u = lo; u < hi; ++u) {
            auto r = std::to_chars(tmp, tmp + 16, part[u]);
            buf.append(tmp, r.ptr);
            buf.push_back('\n');
        }
    });
    if (fclose(f) != 0 || !ok) {
        err = "write failed " + path;
        return 1;
    }
    return 0;
}

int read_partition(const std::string &path, std::vector<u32> &part, std::string &err) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) {
        err = "cannot open partition file " + path;
        return 1;
    }
    part.clear();
    unsigned long v;
    while (fscanf(f, "%lu", &v) == 1) part.push_back((u32) v);
    fclose(f);
    return 0;
}

} // namespace hp
