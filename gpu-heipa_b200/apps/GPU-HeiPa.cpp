// GPU-HeiPa: k-way graph partitioning of a METIS graph on one GPU through the
// C ABI. Flags, defaults and stdout keys follow app/GPU-HeiPa.cpp and
// src/utility/configuration.h:50-58 (--graph/-g, --k/-k, --imbalance/-e,
// --config/-c default|ultra, --mapping/-m written only when given,
// --verbose-level); --seed and --device are additions. The partition file has
// one block id per line (src/utility/util.h:288-329).
#include <chrono>
#include <cstdint>
#include <iostream>
#include <string>
#include <vector>

#include "cli_common.h"

int main(int argc, char **argv) {
    const auto t_start = std::chrono::steady_clock::now();
    std::ios::sync_with_stdio(false);
    cli::Options opt({
        {"--help", "", "Produces the help message", "", ""},
        {"--graph", "-g", "Filepath to the graph.", "", ""},
        {"--mapping", "-m", "Output filepath to the generated mapping.", "GPU-HeiPa_par.txt", ""},
        {"--k", "-k", "Number of blocks k", "", ""},
        {"--imbalance", "-e", "Allowed imbalance (for example 0.03).", "0.03", ""},
        {"--config", "-c", "Algorithm Config {default, ultra}.", "", ""},
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
    const uint64_t k = cli::parse_u64(opt.require("--k"), "--k");
    const double imbalance = cli::parse_f64(opt.get("--imbalance"), "--imbalance");
    const std::string config = opt.require("--config");
    const int verbose = (int) cli::parse_u64(opt.get("--verbose-level"), "--verbose-level");
    const uint64_t seed = cli::parse_u64(opt.get("--seed"), "--seed");
    const int device = (int) cli::parse_u64(opt.get("--device"), "--device");
    if (config != "default" && config != "ultra") cli::Options::fail("invalid config: " + config);
    if (k == 0 || k > 0xFFFFFFFFull) cli::Options::fail("invalid k");

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
    const auto t_up = std::chrono::steady_clock::now();
    hp_graph *g = nullptr;
    cli::check(hp_graph_upload(ctx, n, m, xadj.data(), adj.data(), has_ew ? ew.data() : nullptr,
                               has_vw ? vw.data() : nullptr, &g),
               ctx, "graph upload");
    const double upload_ms = cli::ms_since(t_up);
    std::vector<uint32_t> part(n);
    int64_t cut = 0;
    const auto t_part = std::chrono::steady_clock::now();
    cli::check(hp_partition_graph(ctx, g, (uint32_t) k, imbalance, config == "ultra", seed, part.data(), &cut), ctx,
               "partitioning");
    const double part_ms = cli::ms_since(t_part);
    const double solve_ms = cli::ms_since(t_solve);

    double phase[5] = {0, 0, 0, 0, 0};
    int64_t initial_cut = 0;
    int32_t lmax = 0, init_maxw = 0, final_maxw = 0;
    uint32_t levels = 0;
    hp_last_solve_stats(ctx, phase, &initial_cut, &lmax, &levels);
    hp_last_solve_maxw(ctx, &init_maxw, &final_maxw);
    if (verbose >= 1) {
        cli::print_levels(ctx);
        const cli::BlockStats bs = cli::block_stats(part, has_vw ? vw.data() : nullptr, (uint32_t) k, lmax);
        double misc = part_ms;
        for (double x: phase) misc -= x;
        std::cout << "------- Info -------\n";
        std::cout << "Graph             : " << graph_in << "\n";
        std::cout << "#Vertices         : " << n << "\n";
        std::cout << "#Edges            : " << m / 2 << "\n";
        std::cout << "k                 : " << k << "\n";
        std::cout << "imbalance         : " << imbalance << "\n";
        std::cout << "Lmax              : " << lmax << "\n";
        std::cout << "------- Stat -------\n";
        std::cout << "Init. edge-cut    : " << initial_cut << "\n";
        std::cout << "Init. max block w : " << init_maxw << "\n";
        std::cout << "Final edge-cut    : " << cut << "\n";
        std::cout << "Final max block w : " << final_maxw << "\n";
        std::cout << "#empty partitions : " << bs.empty << "\n";
        std::cout << "#oload partitions : " << bs.overloaded << "\n";
        std::cout << "Sum oload weights : " << bs.sum_overload << "\n";
        std::cout << "------- Time -------\n";
        std::cout << "Total solve time  : " << part_ms << "\n";
        cli::print_phase_times(phase);
        std::cout << "Down/Upload       : " << upload_ms << "\n";
        std::cout << "Misc              : " << misc << "\n";
        std::cout << "ALL               : " << part_ms + upload_ms << "\n";
        std::cout << "Solved in         : " << solve_ms << std::endl;
    }

    if (opt.is_set("--mapping")) {
        const auto t_w = std::chrono::steady_clock::now();
        cli::check(hp_write_partition(opt.get("--mapping").c_str(), part.data(), n), nullptr, "writing the partition");
        if (verbose >= 1) std::cout << "Write partition in: " << cli::ms_since(t_w) << std::endl;
    }

    const auto t_d = std::chrono::steady_clock::now();
    hp_graph_free(ctx, g);
    hp_ctx_destroy(ctx);
    if (verbose >= 1) std::cout << "Destructed in     : " << cli::ms_since(t_d) << std::endl;
    if (verbose >= 2)
        std::cout << "Total Time in GPU-HeiPa.cpp : " << cli::ms_since(t_start) / 1000.0 << " seconds." << std::endl;
    return EXIT_SUCCESS;
}
