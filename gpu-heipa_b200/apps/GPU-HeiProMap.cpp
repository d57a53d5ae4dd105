// GPU-HeiProMap: process mapping of a METIS communication graph onto a
// hierarchy a1:...:al with distances d1:...:dl, on one GPU through the C ABI.
// Flags, defaults and stdout keys follow app/GPU-HeiProMap.cpp and
// src/utility/promap_configuration.h:38-131 (--graph/-g, --hierarchy/-h,
// --distance/-d, --imbalance/-e, --config/-c IM|HM|HM-ultra, --mapping/-m
// written only when given, --verbose-level); k = a1 * ... * al. --seed and
// --device are additions. J counts every directed entry (comm_cost.h:36-56).
#include <chrono>
#include <cstdint>
#include <iostream>
#include <string>
#include <vector>

#include "cli_common.h"

namespace {

std::string join(const std::vector<uint64_t> &v) {
    std::string s;
    for (size_t i = 0; i < v.size(); ++i) s += (i ? ":" : "") + std::to_string(v[i]);
    return s;
}

}  // namespace

int main(int argc, char **argv) {
    const auto t_start = std::chrono::steady_clock::now();
    std::ios::sync_with_stdio(false);
    cli::Options opt({
        {"--help", "", "Produces the help message", "", ""},
        {"--graph", "-g", "Filepath to the graph.", "", ""},
        {"--mapping", "-m", "Output filepath to the generated mapping.", "GPU-HeiProMap_par.txt", ""},
        {"--hierarchy", "-h", "Hierarchy in the form a1:a2:...:al .", "", ""},
        {"--distance", "-d", "Distance in the form d1:d2:...:dl .", "", ""},
        {"--imbalance", "-e", "Allowed imbalance (for example 0.03).", "0.03", ""},
        {"--config", "-c", "Algorithm Config {IM, HM, HM-ultra}.", "", ""},
        {"--verbose-level", "", "Whether to print.", "1", ""},
        {"--seed", "", "Seed of the initial partitioner.", "0", ""},
        {"--device", "", "CUDA device.", "0", ""},
        {"--deterministic", "", "Accepted for compatibility: every result is deterministic (same input, seed and "
                                "config give the same output).", "", "", false, true},
    });
    if (argc == 1) {
        opt.help(argv[0]);
        return EXIT_FAILURE;
    }
    if (!opt.parse(argc, argv)) return EXIT_SUCCESS;
    const std::string graph_in = opt.require("--graph");
    const std::vector<uint64_t> hier64 = cli::parse_colon_list(opt.require("--hierarchy"), "--hierarchy");
    const std::vector<uint64_t> dist64 = cli::parse_colon_list(opt.require("--distance"), "--distance");
    const double imbalance = cli::parse_f64(opt.get("--imbalance"), "--imbalance");
    const std::string config = opt.require("--config");
    const int verbose = (int) cli::parse_u64(opt.get("--verbose-level"), "--verbose-level");
    const uint64_t seed = cli::parse_u64(opt.get("--seed"), "--seed");
    const int device = (int) cli::parse_u64(opt.get("--device"), "--device");
    int mode = -1;
    if (config == "IM") mode = HP_MAP_IM;
    else if (config == "HM") mode = HP_MAP_HM;
    else if (config == "HM-ultra") mode = HP_MAP_HM_ULTRA;
    else cli::Options::fail("invalid config: " + config);
    if (hier64.size() != dist64.size()) cli::Options::fail("hierarchy and distance have different lengths");
    std::vector<uint32_t> hier;
    std::vector<int32_t> dist;
    uint64_t k = 1;
    for (size_t i = 0; i < hier64.size(); ++i) {
        if (hier64[i] == 0 || hier64[i] > 0xFFFFFFFFull || dist64[i] > 0x7FFFFFFFull)
            cli::Options::fail("invalid hierarchy or distance entry");
        hier.push_back((uint32_t) hier64[i]);
        dist.push_back((int32_t) dist64[i]);
        k *= hier64[i];
        if (k > 0xFFFFFFFFull) cli::Options::fail("hierarchy product too large");
    }

    hp_host_graph *hg = nullptr;
    cli::check(hp_read_metis(graph_in.c_str(), &hg), nullptr, "reading " + graph_in);
    uint32_t n = 0;
    uint64_t m = 0;
    int has_ew = 0, has_vw = 0;
    hp_host_graph_info(hg, &n, &m, &has_ew, &has_vw);
    std::vector<uint32_t> xadj(n + 1), adj(m);
    std::vector<int32_t> ew(has_ew ? m : 0), vw(has_vw ? n : 0);
    hp_host_graph_copy(hg, xadj.data(), adj.data(), has_ew ? ew.data() : nullptr, has_vw ? vw.data() : nullptr);
    hp_host_graph_free(hg);
    if (verbose >= 1) std::cout << "Read graph in     : " << cli::ms_since(t_start) << std::endl;

    const auto t_solve = std::chrono::steady_clock::now();
    hp_ctx *ctx = nullptr;
    cli::check(hp_ctx_create(device, hp_arena_estimate(n, m, has_ew, has_vw), &ctx), nullptr, "context creation");
    hp_graph *g = nullptr;
    cli::check(hp_graph_upload(ctx, n, m, xadj.data(), adj.data(), has_ew ? ew.data() : nullptr,
                               has_vw ? vw.data() : nullptr, &g),
               ctx, "graph upload");
    std::vector<uint32_t> part(n);
    int64_t J = 0;
    const auto t_map = std::chrono::steady_clock::now();
    cli::check(hp_map_graph(ctx, g, hier.data(), dist.data(), (uint32_t) hier.size(), imbalance, mode, seed,
                            part.data(), &J),
               ctx, "process mapping");
    const double map_ms = cli::ms_since(t_map);
    const double solve_ms = cli::ms_since(t_solve);

    double phase[5] = {0, 0, 0, 0, 0};
    int64_t initial_J = 0;
    int32_t lmax = 0, init_maxw = 0, final_maxw = 0;
    uint32_t levels = 0;
    hp_last_solve_stats(ctx, phase, &initial_J, &lmax, &levels);
    hp_last_solve_maxw(ctx, &init_maxw, &final_maxw);
    if (verbose >= 1) {
        const cli::BlockStats bs = cli::block_stats(part, has_vw ? vw.data() : nullptr, (uint32_t) k, lmax);
        double misc = map_ms;
        for (double x: phase) misc -= x;
        std::cout << "------- Info -------\n";
        std::cout << "Total solve time  : " << map_ms << "\n";
        std::cout << "#Vertices         : " << n << "\n";
        std::cout << "#Edges            : " << m / 2 << "\n";
        std::cout << "k                 : " << k << "\n";
        std::cout << "hierarchy         : " << join(hier64) << "\n";
        std::cout << "distances         : " << join(dist64) << "\n";
        std::cout << "imbalance         : " << imbalance << "\n";
        std::cout << "Lmax              : " << lmax << "\n";
        std::cout << "------- Stat -------\n";
        std::cout << "Init. comm-cost   : " << initial_J << "\n";
        std::cout << "Init. max block w : " << init_maxw << "\n";
        std::cout << "Final comm-cost   : " << J << "\n";
        std::cout << "Final max block w : " << final_maxw << "\n";
        std::cout << "#empty partitions : " << bs.empty << "\n";
        std::cout << "#oload partitions : " << bs.overloaded << "\n";
        std::cout << "Sum oload weights : " << bs.sum_overload << "\n";
        std::cout << "------- Time -------\n";
        cli::print_phase_times(phase);
        std::cout << "Misc              : " << misc << "\n";
        std::cout << "ALL               : " << map_ms << "\n";
        std::cout << "Solved in         : " << solve_ms << std::endl;
    }

    if (opt.is_set("--mapping")) {
        const auto t_w = std::chrono::steady_clock::now();
        cli::check(hp_write_partition(opt.get("--mapping").c_str(), part.data(), n), nullptr, "writing the mapping");
        if (verbose >= 1) std::cout << "Write partition in: " << cli::ms_since(t_w) << std::endl;
    }

    const auto t_d = std::chrono::steady_clock::now();
    hp_graph_free(ctx, g);
    hp_ctx_destroy(ctx);
    if (verbose >= 1) std::cout << "Destructed in     : " << cli::ms_since(t_d) << std::endl;
    if (verbose >= 1)
        std::cout << "Total Time spent in GPU-HeiProMap.cpp: " << cli::ms_since(t_start) / 1000.0 << " seconds."
                  << std::endl;
    return EXIT_SUCCESS;
}
