// Drop-in for the reference CLI gpart_partition_standard
// (app/partition_main.cu:21-183): same argv, environment knobs, stdout keys,
// raw int32 label file and exit codes (0 ok, 1 failure with
// "gpart_partition: <message>" on stderr, 2 usage).  A thin client of the C ABI.
#include "gpart_b200.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {
void check(gp_status status) {
    if (status != GP_OK) throw std::runtime_error(gp_last_error());
}
int env_int(const char* name, int lo, int hi, const char* message) {
    const char* v = std::getenv(name);
    const int x = std::stoi(v);
    if (x < lo || x > hi) throw std::runtime_error(message);
    return x;
}
}  // namespace

int main(int argc, char** argv) {
    gp_context* ctx = nullptr;
    try {
        const auto wall_start = std::chrono::steady_clock::now();
        bool verify = false;
        int positional = argc;
        while (positional > 1 && std::string(argv[positional - 1]) == "--verify") {
            verify = true;
            --positional;
        }
        if (positional < 5 || positional > 7) {
            std::cerr << "Usage: " << argv[0] << " <indptr.bin> <indices.bin> <parts> <partition.out>"
                      << " [imbalance_ratio=1.03] [seed] [--verify]\n";
            return 2;
        }
        for (const char* retired : {"GPART_REFINE_MODE", "GPART_JOINT_ROUNDS", "GPART_JOINT_CONFLICT_ROUNDS",
                                    "GPART_JOINT_DEDUPLICATE", "GPART_JOINT_COMPLEMENT", "GPART_JOINT_DIAGNOSTICS",
                                    "GPART_SPARSE_DELTA", "GPART_REPAIR_ENUMERATION", "GPART_SPARSE_CUT_BOUND"})
            if (std::getenv(retired))
                throw std::invalid_argument(std::string(retired) + " was retired; unset it.");
        const int parts = std::stoi(argv[3]);
        const double imbalance = positional >= 6 ? std::stod(argv[5]) : 1.03;
        const auto seed = positional >= 7 ? static_cast<uint32_t>(std::stoul(argv[6])) : 0U;
        const auto load_start = std::chrono::steady_clock::now();
        // The int64 files go straight to the device: chunked reads into
        // pinned buffers overlapped with the copy and the narrowing.
        check(gp_context_create(0, &ctx));
        int64_t n = 0, m = 0;
        check(gp_load_csr_int64(ctx, argv[1], argv[2], &n, &m));
        uint64_t capacity = 0;
        check(gp_partition_capacity(static_cast<uint64_t>(n), parts, imbalance, &capacity));
        const auto load_end = std::chrono::steady_clock::now();
        std::cout << "vertices=" << n << " edge_entries=" << m << " device_count=1\n";
        std::cout << "verify=" << (verify ? 1 : 0) << '\n';
        uint32_t flags = verify ? GP_FLAG_VERIFY : 0u;
        if (const char* v = std::getenv("GPART_HEM_COARSEN"); v && std::string(v) == "0")
            check(gp_set_option(ctx, "seed_matching", 0));
        if (const char* v = std::getenv("GPART_REGRET_FORCE_FULL"); v && std::string(v) != "0")
            check(gp_set_option(ctx, "capacity_safe_fast_path", 0));
        const char* mode = std::getenv("GPART_COARSEN_MODE");
        const std::string coarsen_mode = mode ? mode : "regret";
        if (coarsen_mode != "regret") throw std::runtime_error("Only regret coarsening is maintained");
        if (std::getenv("GPART_HEM_DEGREE_LIMIT"))
            check(gp_set_option(ctx, "heavy_edge_degree_limit",
                                env_int("GPART_HEM_DEGREE_LIMIT", 2, 256, "GPART_HEM_DEGREE_LIMIT must be between 2 and 256")));
        if (std::getenv("GPART_FINE_FACTOR"))
            check(gp_set_option(ctx, "progressive_fine_factor", std::stoi(std::getenv("GPART_FINE_FACTOR"))));
        if (std::getenv("GPART_CAPACITY_GROWTH"))
            check(gp_set_option(ctx, "progressive_capacity_growth", std::stoi(std::getenv("GPART_CAPACITY_GROWTH"))));
        int beta = parts <= 8 ? std::max(64, (512 + parts - 1) / parts) : std::max(2, (32 + parts - 1) / parts);
        if (std::getenv("GPART_COARSE_BETA")) {
            beta = env_int("GPART_COARSE_BETA", 2, 256, "GPART_COARSE_BETA must be between 2 and 256");
            check(gp_set_option(ctx, "cluster_size_factor", beta));
        }
        std::cout << "pipeline_mode=incremental_bucket cluster_size_factor=" << beta
                  << " progressive_cluster_capacity=" << (parts >= 16) << " pack_isolated=1\n";
        std::cout << "seed_matching=" << !(std::getenv("GPART_HEM_COARSEN") && std::string(std::getenv("GPART_HEM_COARSEN")) == "0")
                  << " coarsen_mode=" << coarsen_mode << '\n';
        std::vector<int32_t> labels(static_cast<size_t>(n));
        gp_stats stats{};
        if (!std::getenv("GPART_LOG_LEVELS")) flags |= GP_FLAG_QUIET;
        check(gp_partition_loaded(ctx, parts, imbalance, seed, flags, labels.data(), &stats));
        const auto output_start = std::chrono::steady_clock::now();
        std::ofstream output(argv[4], std::ios::binary | std::ios::trunc);
        if (!output) throw std::runtime_error("cannot open partition output");
        output.write(reinterpret_cast<const char*>(labels.data()), static_cast<std::streamsize>(labels.size() * sizeof(int32_t)));
        output.close();
        if (!output) throw std::runtime_error("cannot write partition output");
        const auto output_end = std::chrono::steady_clock::now();
        std::cout << std::setprecision(10) << "final_edge_cut=" << stats.edge_cut << '\n'
                  << "final_max_part_weight=" << stats.max_part_weight << '\n'
                  << "final_imbalance=" << (n ? static_cast<double>(stats.max_part_weight) * parts / static_cast<double>(n) : 0.0)
                  << '\n';
        std::cout << std::setprecision(10)
                  << "partition_timing input_load_seconds=" << std::chrono::duration<double>(load_end - load_start).count()
                  << " coarsen_seconds=" << stats.coarsen_seconds << " initial_partition_seconds=" << stats.initial_seconds
                  << " uncoarsen_seconds=" << stats.uncoarsen_seconds << " input_prepare_seconds=" << stats.h2d_seconds
                  << " final_partition_d2h_seconds=" << stats.d2h_seconds
                  << " timing_scope=device_input_to_device_partition"
                  << " partition_output_seconds=" << std::chrono::duration<double>(output_end - output_start).count()
                  << " partition_total_seconds=" << stats.algorithm_seconds
                  << " algorithm_total_seconds=" << stats.algorithm_seconds
                  << " wall_total_seconds=" << std::chrono::duration<double>(output_end - wall_start).count() << '\n';
        gp_context_destroy(ctx);
        return 0;
    } catch (const std::exception& error) {
        if (ctx) gp_context_destroy(ctx);
        std::cerr << "gpart_partition: " << error.what() << '\n';
        return 1;
    }
}
