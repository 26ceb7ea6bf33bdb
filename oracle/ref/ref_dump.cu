// Dump harness for the reference partitioner (test infrastructure only).
//
// Links the reference's own coarsen / initial_partition_metis / uncoarsen
// objects and drives them exactly as app/partition_main.cu:52-126 does (same
// CoarsenOptions and RefineOptions, no environment overrides), but accepts
// optional uint32 vertex and edge weight files so weighted inputs can be fed
// to the reference too.  After each stage it writes the device state to a
// binary dump consumed by tests/golden/make_golden.py:
//
//   "GPDUMP01"
//   int32 levels
//   per level: int64 n, int64 m, uint64 maximum_degree, uint8 has_heavy_rows,
//              uint64 incident_weight_bound,
//              int32 offsets[n+1], int32 neighbors[m], uint32 edge_w[m],
//              uint32 vertex_w[n], then int32 map[n] unless it is the last level
//   int64 coarsest_n, int32 metis_labels[coarsest_n]
//   int64 n, int32 final_labels[n], uint64 final_cut, double algorithm_seconds
//
// usage: gpart_ref_dump indptr.i64 indices.i64 vw.u32|- ew.u32|- k eps seed out
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
#include <stdexcept>
#include <string>
#include <vector>

namespace {
template <typename T>
std::vector<T> read_file(const std::string& path) {
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) throw std::runtime_error("cannot open " + path);
    const auto bytes = static_cast<std::size_t>(in.tellg());
    if (bytes % sizeof(T)) throw std::runtime_error("bad size " + path);
    std::vector<T> out(bytes / sizeof(T));
    in.seekg(0);
    if (bytes) in.read(reinterpret_cast<char*>(out.data()), static_cast<std::streamsize>(bytes));
    return out;
}
template <typename T>
void put(std::ofstream& out, const T& value) { out.write(reinterpret_cast<const char*>(&value), sizeof(T)); }
template <typename T>
void put_vec(std::ofstream& out, const std::vector<T>& v) {
    if (!v.empty()) out.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}
}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc != 9) {
            std::cerr << "usage: gpart_ref_dump indptr indices vw|- ew|- k eps seed out\n";
            return 2;
        }
        const int parts = std::stoi(argv[5]);
        const double imbalance = std::stod(argv[6]);
        const auto seed = static_cast<std::uint32_t>(std::stoul(argv[7]));
        auto graph = gpart::load_weighted_graph(argv[1], argv[2]);
        if (std::string(argv[3]) != "-") {
            auto vw = read_file<std::uint32_t>(argv[3]);
            if (vw.size() != graph.vertex_weights.size()) throw std::runtime_error("vertex weight length");
            graph.vertex_weights = vw;
        }
        if (std::string(argv[4]) != "-") {
            auto ew = read_file<std::uint32_t>(argv[4]);
            if (ew.size() != graph.edge_weights.size()) throw std::runtime_error("edge weight length");
            graph.edge_weights = ew;
        }
        gpart::partition_capacity(
            [&] { std::uint64_t t = 0; for (auto w : graph.vertex_weights) t += w; return t; }(),
            parts, imbalance);
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
        gpart::validate_weighted_shape(graph, true);
        auto device_graph = gpart::make_device_weighted(graph);
        CUDA_CHECK(cudaDeviceSynchronize());
        const auto start = std::chrono::steady_clock::now();
        gpart::detail::ScratchPoolSession pool;
        auto hierarchy = gpart::coarsen(std::move(device_graph), co);
        CUDA_CHECK(cudaDeviceSynchronize());
        const auto coarsen_end = std::chrono::steady_clock::now();

        std::ofstream out(argv[8], std::ios::binary | std::ios::trunc);
        if (!out) throw std::runtime_error("cannot open dump");
        out.write("GPDUMP01", 8);
        const auto levels = static_cast<std::int32_t>(hierarchy.levels.size());
        put(out, levels);
        for (std::int32_t i = 0; i < levels; ++i) {
            const auto& level = hierarchy.levels[static_cast<std::size_t>(i)];
            auto host = gpart::copy_device_weighted(level);
            put(out, static_cast<std::int64_t>(host.vertices()));
            put(out, static_cast<std::int64_t>(host.edges()));
            put(out, static_cast<std::uint64_t>(level.maximum_degree));
            put(out, static_cast<std::uint8_t>(level.has_heavy_rows ? 1 : 0));
            put(out, static_cast<std::uint64_t>(level.incident_weight_bound));
            put_vec(out, host.offsets);
            put_vec(out, host.neighbors);
            put_vec(out, host.edge_weights);
            put_vec(out, host.vertex_weights);
            if (i + 1 < levels) {
                const auto& map = hierarchy.fine_to_coarse[static_cast<std::size_t>(i)];
                std::vector<std::int32_t> host_map(map.size());
                thrust::copy(map.begin(), map.end(), host_map.begin());
                put_vec(out, host_map);
            }
        }
        const auto coarse_dump_end = std::chrono::steady_clock::now();
        auto coarse = gpart::initial_partition_metis(hierarchy.levels.back(), parts, imbalance, seed, false);
        {
            std::vector<std::int32_t> labels(coarse.size());
            thrust::copy(coarse.begin(), coarse.end(), labels.begin());
            put(out, static_cast<std::int64_t>(labels.size()));
            put_vec(out, labels);
        }
        gpart::RefineOptions ro;
        ro.parts = parts;
        ro.allow_initial_imbalance = true;
        ro.imbalance_ratio = imbalance;
        ro.max_rounds = 32;
        ro.strict_verify = false;
        ro.refinement_growth_ratio = 2.0;
        auto result = gpart::uncoarsen(hierarchy, std::move(coarse), ro);
        CUDA_CHECK(cudaDeviceSynchronize());
        const auto end = std::chrono::steady_clock::now();
        hierarchy.levels.clear();
        hierarchy.fine_to_coarse.clear();
        pool.finish();
        std::vector<std::int32_t> labels(result.device_partition.size());
        thrust::copy(result.device_partition.begin(), result.device_partition.end(), labels.begin());
        put(out, static_cast<std::int64_t>(labels.size()));
        put_vec(out, labels);
        put(out, static_cast<std::uint64_t>(result.final_cut));
        // The dump itself is excluded from the reported time.
        const double seconds = std::chrono::duration<double>(coarsen_end - start).count() +
                               std::chrono::duration<double>(end - coarse_dump_end).count();
        put(out, seconds);
        out.close();
        std::cout << "ref_dump levels=" << levels << " final_cut=" << result.final_cut
                  << " seconds=" << seconds << '\n';
        return 0;
    } catch (const std::exception& error) {
        std::cerr << "gpart_ref_dump: " << error.what() << '\n';
        return 1;
    }
}
