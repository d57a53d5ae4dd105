// Shared command-line handling of the GPU-HeiPa and GPU-HeiProMap tools:
// option tables with long/short keys and defaults, unknown arguments ignored
// (src/utility/configuration.h:50-127, promap_configuration.h:38-131), and
// the statistics block printed after a solve (solver.h:301-329,
// promap_solver.h:199-227). Unlike the reference, a bad option value or a
// failed call is reported on stderr with a non-zero exit status.
#pragma once

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "gpuheipa.h"

namespace cli {

struct Option {
    std::string large_key, small_key, description, default_val, input;
    bool is_set = false;
    bool is_switch = false;  // takes no value
};

class Options {
public:
    explicit Options(std::vector<Option> opts) : opts_(std::move(opts)) {}

    // Returns false when --help was given (the help text is printed).
    bool parse(int argc, char **argv) {
        for (int i = 1; i < argc; ++i)
            if (std::string(argv[i]) == "--help") {
                help(argv[0]);
                return false;
            }
        for (int i = 1; i < argc; ++i) {
            const std::string a = argv[i];
            for (Option &o: opts_) {
                if (a == o.large_key || (!o.small_key.empty() && a == o.small_key)) {
                    if (o.is_switch) {
                        o.input = "1";
                    } else {
                        if (i + 1 >= argc) fail("missing value for " + a);
                        o.input = argv[++i];
                    }
                    o.is_set = true;
                    break;
                }
            }
        }
        return true;
    }

    bool is_set(const std::string &key) const { return find(key).is_set; }

    std::string get(const std::string &key) const {
        const Option &o = find(key);
        return o.is_set ? o.input : o.default_val;
    }

    std::string require(const std::string &key) const {
        const Option &o = find(key);
        if (!o.is_set && o.default_val.empty()) fail("missing required option " + key);
        return get(key);
    }

    void help(const char *prog) const {
        std::cout << "Usage: " << prog << " [options]\n";
        for (const Option &o: opts_) {
            std::cout << "  " << o.large_key;
            if (!o.small_key.empty()) std::cout << ", " << o.small_key;
            std::cout << "\t" << o.description;
            if (!o.default_val.empty()) std::cout << " (default: " << o.default_val << ")";
            std::cout << "\n";
        }
    }

    [[noreturn]] static void fail(const std::string &msg) {
        std::cerr << "Error: " << msg << std::endl;
        std::exit(EXIT_FAILURE);
    }

private:
    const Option &find(const std::string &key) const {
        for (const Option &o: opts_)
            if (o.large_key == key || o.small_key == key) return o;
        fail("unknown option " + key);
    }
    std::vector<Option> opts_;
};

inline double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

inline uint64_t parse_u64(const std::string &s, const std::string &what) {
    try {
        size_t pos = 0;
        const unsigned long long v = std::stoull(s, &pos);
        if (pos != s.size()) throw std::invalid_argument(s);
        return v;
    } catch (...) {
        Options::fail("invalid value for " + what + ": " + s);
    }
}

inline double parse_f64(const std::string &s, const std::string &what) {
    try {
        size_t pos = 0;
        const double v = std::stod(s, &pos);
        if (pos != s.size()) throw std::invalid_argument(s);
        return v;
    } catch (...) {
        Options::fail("invalid value for " + what + ": " + s);
    }
}

// "a1:a2:...:al" -> values
inline std::vector<uint64_t> parse_colon_list(const std::string &s, const std::string &what) {
    std::vector<uint64_t> out;
    size_t start = 0;
    while (start <= s.size()) {
        const size_t end = s.find(':', start);
        const std::string tok = s.substr(start, end == std::string::npos ? std::string::npos : end - start);
        out.push_back(parse_u64(tok, what));
        if (end == std::string::npos) break;
        start = end + 1;
    }
    return out;
}

inline void check(int rc, hp_ctx *ctx, const std::string &what) {
    if (rc == HP_OK) return;
    std::cerr << "Error: " << what << " failed (status " << rc << ")";
    if (ctx) std::cerr << ": " << hp_last_error(ctx);
    std::cerr << std::endl;
    std::exit(EXIT_FAILURE);
}

struct BlockStats {
    int64_t empty = 0, overloaded = 0, sum_overload = 0;
};

// Empty / overloaded blocks and the total overload of a partition.
inline BlockStats block_stats(const std::vector<uint32_t> &part, const int32_t *vw, uint32_t k, int32_t lmax) {
    std::vector<int64_t> bw(k, 0);
    for (size_t u = 0; u < part.size(); ++u) bw[part[u]] += vw ? vw[u] : 1;
    BlockStats s;
    for (uint32_t b = 0; b < k; ++b) {
        if (bw[b] == 0) ++s.empty;
        if (bw[b] > lmax) {
            ++s.overloaded;
            s.sum_overload += bw[b] - lmax;
        }
    }
    return s;
}

inline void print_phase_times(const double ms[5]) {
    std::cout << "Coarsening        : " << ms[0] << "\n";
    std::cout << "Contraction       : " << ms[1] << "\n";
    std::cout << "Init. Part.       : " << ms[2] << "\n";
    std::cout << "Uncontraction     : " << ms[3] << "\n";
    std::cout << "Refinement        : " << ms[4] << "\n";
}

inline void print_levels(hp_ctx *ctx) {
    uint32_t n = 0;
    uint64_t m = 0;
    for (uint32_t i = 0; hp_last_solve_level(ctx, i, &n, &m) == HP_OK; ++i) std::cout << n << " " << m << "\n";
}

}  // namespace cli
