// Warm in-process timing harness for the reference partitioner (measurement
// infrastructure; the product never links or runs it).
//
// Generates the seeded R-MAT graph of the benchmark workload in this process
// (the counter-based generator described below; tests/test_ref_harness.py
// checks it against the library's generator byte for byte), then runs the
// reference's own public pipeline exactly as app/partition_main.cu:99-137
// does — validate_weighted_shape + make_device_weighted, coarsen,
// initial_partition_metis, uncoarsen, hierarchy release, label download —
// `warmup` + `steps` times in one process.  Per step it reports the three
// spans of the CLI's partition_timing line: input_prepare (validation +
// upload), algorithm_total (upload done -> scratch pool released, the CLI's
// timing scope) and final_partition_d2h.  The last stdout line is
//   REF_BENCH_JSON {...}
//
// usage: gpart_ref_bench rmat SCALE EF A B C GSEED K EPS SEED WARMUP STEPS
//        gpart_ref_bench write-rmat SCALE EF A B C GSEED indptr.i64 indices.i64
//
// R-MAT generator: sample i draws its SCALE quadrant choices from a splitmix64
// stream keyed by (GSEED, "RMAT", i); each u = 53-bit uniform picks
// (0,0) / (0,1) / (1,0) / (1,1) with probabilities A, B, C, 1-A-B-C, high bit
// first.  Both directions of every non-loop sample are kept, then sorted by
// (source, target) and deduplicated.
#include "coarsen.hpp"
#include "graph.hpp"
#include "graph_types.hpp"
#include "initial_partition.hpp"
#include "partition_capacity.hpp"
#include "uncoarsen.hpp"
#include "check.hpp"
#include "detail/scratch_pool.hpp"

#include <thrust/copy.h>
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <parallel/algorithm>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

std::uint64_t splitmix(std::uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

gpart::WeightedGraph rmat(int scale, int ef, double a, double b, double c, std::uint64_t gseed) {
    const std::int64_t n = std::int64_t{1} << scale;
    const std::int64_t samples = static_cast<std::int64_t>(ef) * n;
    const double pa = a, pab = a + b, pabc = a + b + c;
    const std::uint64_t stream_key = splitmix(gseed * 0x9E3779B97F4A7C15ULL + 0x524d4154ULL);
    std::vector<std::uint64_t> pairs(static_cast<std::size_t>(2 * samples), ~0ULL);
#pragma omp parallel for schedule(static)
    for (std::int64_t i = 0; i < samples; ++i) {
        std::uint64_t state = splitmix(stream_key + static_cast<std::uint64_t>(i) * 0xD1B54A32D192ED03ULL);
        std::uint64_t row = 0, col = 0;
        for (int level = scale - 1; level >= 0; --level) {
            state += 0x9E3779B97F4A7C15ULL;
            const double u = static_cast<double>(splitmix(state) >> 11) * 0x1.0p-53;
            const std::uint64_t bit = std::uint64_t{1} << level;
            if (u >= pabc) { row |= bit; col |= bit; }
            else if (u >= pab) row |= bit;
            else if (u >= pa) col |= bit;
        }
        if (row != col) {
            pairs[static_cast<std::size_t>(2 * i)] = (row << scale) | col;
            pairs[static_cast<std::size_t>(2 * i + 1)] = (col << scale) | row;
        }
    }
    __gnu_parallel::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    if (!pairs.empty() && pairs.back() == ~0ULL) pairs.pop_back();  // dropped self loops
    gpart::WeightedGraph g;
    g.offsets.assign(static_cast<std::size_t>(n + 1), 0);
    g.neighbors.resize(pairs.size());
    const std::uint64_t mask = (std::uint64_t{1} << scale) - 1;
    for (std::size_t e = 0; e < pairs.size(); ++e) {
        ++g.offsets[static_cast<std::size_t>((pairs[e] >> scale) + 1)];
        g.neighbors[e] = static_cast<gpart::GraphTypes::VertexT>(pairs[e] & mask);
    }
    for (std::int64_t v = 0; v < n; ++v) g.offsets[static_cast<std::size_t>(v + 1)] += g.offsets[static_cast<std::size_t>(v)];
    g.edge_weights.assign(pairs.size(), 1u);
    g.vertex_weights.assign(static_cast<std::size_t>(n), 1u);
    return g;
}

void write_int64(const std::string& path, const std::vector<std::int64_t>& values) {
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    if (!out) throw std::runtime_error("cannot open " + path);
    out.write(reinterpret_cast<const char*>(values.data()), static_cast<std::streamsize>(values.size() * 8));
    if (!out) throw std::runtime_error("cannot write " + path);
}

double seconds(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

}  // namespace

int main(int argc, char** argv) {
    try {
        const std::string mode = argc > 1 ? argv[1] : "";
        if (mode == "write-rmat" && argc == 10) {
            const auto g = rmat(std::stoi(argv[2]), std::stoi(argv[3]), std::stod(argv[4]), std::stod(argv[5]),
                                std::stod(argv[6]), std::stoull(argv[7]));
            write_int64(argv[8], std::vector<std::int64_t>(g.offsets.begin(), g.offsets.end()));
            write_int64(argv[9], std::vector<std::int64_t>(g.neighbors.begin(), g.neighbors.end()));
            std::cout << "vertices=" << g.vertices() << " edges=" << g.edges() << '\n';
            return 0;
        }
        if (mode != "rmat" || argc != 13) {
            std::cerr << "usage: gpart_ref_bench rmat SCALE EF A B C GSEED K EPS SEED WARMUP STEPS\n"
                         "       gpart_ref_bench write-rmat SCALE EF A B C GSEED indptr indices\n";
            return 2;
        }
        const int parts = std::stoi(argv[8]);
        const double imbalance = std::stod(argv[9]);
        const auto seed = static_cast<std::uint32_t>(std::stoul(argv[10]));
        const int warmup = std::stoi(argv[11]), steps = std::stoi(argv[12]);
        const auto gen_start = std::chrono::steady_clock::now();
        const auto graph = rmat(std::stoi(argv[2]), std::stoi(argv[3]), std::stod(argv[4]), std::stod(argv[5]),
                                std::stod(argv[6]), std::stoull(argv[7]));
        const double gen_seconds = seconds(gen_start, std::chrono::steady_clock::now());
        gpart::partition_capacity(static_cast<std::uint64_t>(graph.vertices()), parts, imbalance);
        // app/partition_main.cu:52-87 and :111-118 with no environment overrides.
        gpart::CoarsenOptions co;
        co.parts = parts;
        co.seed = seed;
        co.strict_verify = false;
        co.detailed_timings = false;
        co.seed_matching = true;
        co.capacity_safe_fast_path = true;
        co.heavy_edge_degree_limit = 64;
        co.cluster_size_factor = parts <= 8 ? std::max(64, (512 + parts - 1) / parts)
                                            : std::max(2, (32 + parts - 1) / parts);
        co.pack_isolated = true;
        co.progressive_cluster_capacity = parts >= 16;
        gpart::RefineOptions ro;
        ro.parts = parts;
        ro.allow_initial_imbalance = true;
        ro.imbalance_ratio = imbalance;
        ro.max_rounds = 32;
        ro.strict_verify = false;
        ro.refinement_growth_ratio = 2.0;
        std::vector<double> prepare, algorithm, download;
        std::uint64_t cut = 0;
        std::vector<gpart::GraphTypes::VertexT> partition;
        for (int step = 0; step < warmup + steps; ++step) {
            const auto prepare_start = std::chrono::steady_clock::now();
            gpart::validate_weighted_shape(graph, true);
            auto device_graph = gpart::make_device_weighted(graph);
            CUDA_CHECK(cudaDeviceSynchronize());
            const auto start = std::chrono::steady_clock::now();
            gpart::detail::ScratchPoolSession scratch_pool;
            auto hierarchy = gpart::coarsen(std::move(device_graph), co);
            CUDA_CHECK(cudaDeviceSynchronize());
            auto coarse = gpart::initial_partition_metis(hierarchy.levels.back(), parts, imbalance, seed, false);
            CUDA_CHECK(cudaDeviceSynchronize());
            auto result = gpart::uncoarsen(hierarchy, std::move(coarse), ro);
            CUDA_CHECK(cudaDeviceSynchronize());
            hierarchy.levels.clear();
            hierarchy.fine_to_coarse.clear();
            scratch_pool.finish();
            CUDA_CHECK(cudaDeviceSynchronize());
            const auto free_end = std::chrono::steady_clock::now();
            partition.resize(result.device_partition.size());
            thrust::copy(result.device_partition.begin(), result.device_partition.end(), partition.begin());
            const auto d2h_end = std::chrono::steady_clock::now();
            cut = result.final_cut;
            if (step >= warmup) {
                prepare.push_back(seconds(prepare_start, start));
                algorithm.push_back(seconds(start, free_end));
                download.push_back(seconds(free_end, d2h_end));
            }
        }
        auto list = [](const std::vector<double>& v) {
            std::ostringstream s;
            s.precision(9);
            s << '[';
            for (std::size_t i = 0; i < v.size(); ++i) s << (i ? "," : "") << v[i];
            s << ']';
            return s.str();
        };
        std::cout.precision(9);
        std::cout << "REF_BENCH_JSON {\"vertices\": " << graph.vertices() << ", \"edges\": " << graph.edges()
                  << ", \"generation_seconds\": " << gen_seconds << ", \"final_cut\": " << cut
                  << ", \"input_prepare_seconds\": " << list(prepare)
                  << ", \"algorithm_total_seconds\": " << list(algorithm)
                  << ", \"final_partition_d2h_seconds\": " << list(download) << "}" << std::endl;
        return 0;
    } catch (const std::exception& error) {
        std::cerr << "gpart_ref_bench: " << error.what() << '\n';
        return 1;
    }
}
