// Single-level refinement harness for the reference partitioner (test
// infrastructure only).
//
// Runs the reference's own refinement of one graph from a given start
// labelling, with the RefineOptions of app/partition_main.cu:111-118 except
// for the round and exchange budgets, which the caller chooses.  The public
// refine_partition (include/refine.hpp:84-88) cannot be used: it copies the
// host labels with a device execution policy (ScratchBuffer::assign,
// include/detail/scratch_buffer.hpp:59-63, from src/refine.cu:337) and fails
// with cudaErrorInvalidValue.  So the graph goes through the resident
// refine_hierarchy_device (include/refine.hpp:94-97) as a one-level
// hierarchy, which runs the same run_incremental_refinement on it (the
// "coarsest" level of src/refine.cu:542-567).  That path reports its
// RefineStats only on its refine_coarsest stdout line, which this harness
// captures and parses.  The dump, consumed by tests/golden/make_golden.py:
//
//   "GPREF002"
//   int64 n, int32 labels[n]
//   int64 fields[16]: rounds, proposals, accepted, initial_cut, final_cut,
//         final_max_part_weight, admission_iterations, admission_fallbacks,
//         lp_cut_gain, lp_cut_loss, rebalance_cut_gain, rebalance_cut_loss,
//         checkpoint_updates, group_cut_gain, group_accepted,
//         frontier_vertices_initial  (-1: not reported by that line)
//
// usage: gpart_ref_refine indptr.i64 indices.i64 vw.u32|- ew.u32|- labels.i32
//                         k eps max_rounds exchange_rounds out
#include "graph.hpp"
#include "graph_types.hpp"
#include "hierarchy.hpp"
#include "refine.hpp"
#include "check.hpp"
#include "detail/scratch_pool.hpp"

#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
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
}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc != 11) {
            std::cerr << "usage: gpart_ref_refine indptr indices vw|- ew|- labels k eps max_rounds exchange_rounds out\n";
            return 2;
        }
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
        auto labels = read_file<gpart::GraphTypes::VertexT>(argv[5]);
        if (labels.size() != graph.vertex_weights.size()) throw std::runtime_error("label length");
        gpart::RefineOptions ro;  // app/partition_main.cu:111-118
        ro.parts = std::stoi(argv[6]);
        ro.imbalance_ratio = std::stod(argv[7]);
        ro.max_rounds = std::stoi(argv[8]);
        ro.exchange_rounds = std::stoi(argv[9]);
        ro.allow_initial_imbalance = true;
        ro.strict_verify = false;
        ro.refinement_growth_ratio = 2.0;
        gpart::validate_weighted_shape(graph, true);
        std::map<std::string, std::int64_t> line;
        std::vector<gpart::GraphTypes::VertexT> refined(labels.size());
        {
            gpart::detail::ScratchPoolSession pool;
            gpart::DeviceHierarchy hierarchy;
            hierarchy.levels.push_back(gpart::make_device_weighted(graph));
            thrust::device_vector<gpart::GraphTypes::VertexT> start(labels.begin(), labels.end());
            std::ostringstream captured;
            auto* previous = std::cout.rdbuf(captured.rdbuf());
            gpart::DeviceUncoarsenResult result;
            try {
                result = gpart::refine_hierarchy_device(hierarchy, std::move(start), ro);
                CUDA_CHECK(cudaDeviceSynchronize());
            } catch (...) {
                std::cout.rdbuf(previous);
                throw;
            }
            std::cout.rdbuf(previous);
            thrust::copy(result.device_partition.begin(), result.device_partition.end(), refined.begin());
            std::istringstream lines(captured.str());
            for (std::string text; std::getline(lines, text);) {
                if (text.rfind("refine_coarsest ", 0) != 0) continue;
                std::istringstream words(text);
                for (std::string word; words >> word;) {
                    const auto eq = word.find('=');
                    if (eq == std::string::npos) continue;
                    try {
                        line[word.substr(0, eq)] = std::stoll(word.substr(eq + 1));
                    } catch (...) {
                    }
                }
            }
            hierarchy.levels.clear();
            pool.finish();
        }
        if (!line.count("final_cut")) throw std::runtime_error("no refine_coarsest line");
        auto field = [&](const char* key) { return line.count(key) ? line[key] : std::int64_t{-1}; };
        std::ofstream out(argv[10], std::ios::binary | std::ios::trunc);
        if (!out) throw std::runtime_error("cannot open dump");
        out.write("GPREF002", 8);
        const std::int64_t n = static_cast<std::int64_t>(refined.size());
        out.write(reinterpret_cast<const char*>(&n), sizeof(n));
        out.write(reinterpret_cast<const char*>(refined.data()), static_cast<std::streamsize>(n * sizeof(refined[0])));
        const std::int64_t fields[16] = {
            field("rounds"), -1, -1, field("initial_cut"), field("final_cut"), -1, -1, -1,
            field("lp_cut_gain"), field("lp_cut_loss"), field("rebalance_cut_gain"), field("rebalance_cut_loss"), -1,
            field("group_cut_gain"), field("group_accepted"), field("frontier_vertices_initial")};
        out.write(reinterpret_cast<const char*>(fields), sizeof(fields));
        out.close();
        std::cout << "ref_refine n=" << n << " rounds=" << field("rounds") << " initial_cut=" << field("initial_cut")
                  << " final_cut=" << field("final_cut") << " rebalance_cut_gain=" << field("rebalance_cut_gain")
                  << " rebalance_cut_loss=" << field("rebalance_cut_loss") << '\n';
        return 0;
    } catch (const std::exception& error) {
        std::cerr << "gpart_ref_refine: " << error.what() << '\n';
        return 1;
    }
}
