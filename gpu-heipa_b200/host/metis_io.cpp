#include "metis_io.h"

#include <cstdio>
#include <cstring>
#include <charconv>
#include <fcntl.h>
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
    void *addr = mmap(nullptr, mm.size, PROT_READ, MAP_PRIVATE, mm.fd, 0);
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

int write_metis(const std::string &path, const HostCSR &g, bool write_vw, bool write_ew, std::string &err) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) {
        err = "cannot open " + path;
        return 1;
    }
    std::string buf;
    buf.reserve(1 << 22);
    buf += std::to_string(g.n) + " " + std::to_string(g.m / 2);
    if (write_vw || write_ew) buf += std::string(" 0") + (write_vw ? "1" : "0") + (write_ew ? "1" : "0");
    buf += "\n";
    char tmp[32];
    for (u32 u = 0; u < g.n; ++u) {
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
        if (buf.size() > (1u << 22)) {
            fwrite(buf.data(), 1, buf.size(), f);
            buf.clear();
        }
    }
    fwrite(buf.data(), 1, buf.size(), f);
    if (fclose(f) != 0) {
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
    std::string buf;
    buf.reserve(1 << 20);
    char tmp[16];
    for (u32 u = 0; u < n; ++u) {
        auto r = std::to_chars(tmp, tmp + 16, part[u]);
        buf.append(tmp, r.ptr);
        buf.push_back('\n');
        if (buf.size() > (1u << 20)) {
            fwrite(buf.data(), 1, buf.size(), f);
            buf.clear();
        }
    }
    fwrite(buf.data(), 1, buf.size(), f);
    if (fclose(f) != 0) {
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
