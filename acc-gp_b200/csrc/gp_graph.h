// Device graph, hierarchy and per-call context shared by the pipeline files.
#pragma once
#include "gp_device.cuh"

#include <vector>

namespace gp {

constexpr int kInvalid = 0x7fffffff;  // SCLP_INVALID (src/coarsen.cu:292)

// A CSR level on the device (DeviceWeightedGraph, include/graph.hpp:148-171).
// ew == nullptr means unit edge weights.  The three metadata fields follow
// the reference's meaning exactly: maximum_degree is a bound (exact after an
// aggregation pass), incident_bound bounds every row's weight sum.
// Rows longer than kHeavyRow entries are split into chunks of at most
// kChunk entries so that row-parallel kernels give them many blocks instead
// of one serial warp (R-MAT hubs have 10^5 neighbours).
constexpr int kHeavyRow = 2048;
constexpr int kChunk = 2048;

struct DGraph {
    i64 n = 0, m = 0;
    int* off = nullptr;
    int* nbr = nullptr;
    u32* ew = nullptr;
    u32* vw = nullptr;
    bool implicit_unit = false;
    u64 maximum_degree = ~0ULL;
    bool has_heavy_rows = true;
    u64 incident_bound = ~0ULL;
    // Heavy rows (ascending) and their chunks; built by build_chunks().
    int* heavy = nullptr;
    i64 heavy_count = 0;
    int* chunk_row = nullptr;
    int* chunk_hidx = nullptr;  // index of the chunk's row in `heavy`
    int* chunk_begin = nullptr;
    int* heavy_chunk0 = nullptr;  // first chunk of each heavy row (chunks of a row are consecutive)
    i64 chunks = 0;
    i64 heavy_entries = 0;  // CSR entries in heavy rows
    int heavy_min = kHeavyRow;  // rows longer than this are the heavy (chunked) rows
};

// Chunk-parallel loop body helpers: the chunk's edge range.
__device__ __forceinline__ int chunk_end(const DGraph& g, int chunk, int row) {
    const int end = g.chunk_begin[chunk] + kChunk;
    const int row_end = g.off[row + 1];
    return end < row_end ? end : row_end;
}

struct Hierarchy {
    std::vector<DGraph> levels;  // level 0 is the input
    std::vector<int*> maps;      // maps[i]: level i -> level i+1
};

// Thread-mapping thresholds.  They decide which kernel and how many threads
// handle a row, never a value: every choice computes the same exact integer
// sums, so results do not depend on them and gp_autotune may set them per
// workload.  The defaults are the fixed values this library was tuned with.
struct Mapping {
    int medium_degree = 256;    // coarsening: rows of 9..this, a warp and a 512-slot shared hash (<= 256)
    int large_narrow = 1024;    // coarsening: large rows up to this use a half-size shared table
    int build_short = 64;       // refinement: cache-build rows up to this, 8 lanes per row
    int rebuild_divisor = 100;  // refinement: rebuild the cache when moved entries exceed (n k size + 8 m) / this
    int on_demand_degree = 32;  // refinement: no cache when the maximum degree is at most this (0: never)
    // Refinement rows above these entry counts go through the block-per-chunk
    // kernels (2048-entry chunks) instead of a warp: on levels of at most
    // 65,536 vertices, at most 2^20 vertices, and larger ones.
    int refine_heavy_small = 256;
    int refine_heavy_mid = 512;
    int refine_heavy_large = 2048;
};

// Coarsening options, app/partition_main.cu:52-87 with no environment overrides.
struct CoarsenOptions {
    int parts = 4;
    u32 seed = 0;
    double stop_ratio = 0.90;
    int max_levels = 24;
    int cluster_size_factor = 256;
    bool pack_isolated = true;
    bool progressive = false;
    int fine_factor = 64, growth = 8;
    bool seed_matching = true, fast_path = true;
    int heavy_limit = 64;
    bool log = true;
    bool verify = false;  // GP_FLAG_VERIFY: strict per-level checks
    Mapping mapping;
};

// Device-resident scalars read back in batches through pinned memory.
constexpr int kScalars = 512;  // >= 2 * kMaxParts + headroom

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    Arena persist;  // hierarchy storage for one call
    Arena scratch;  // stack-disciplined temporaries
    u64* dev_scalars = nullptr;
    u64* host_scalars = nullptr;  // pinned
    cudaEvent_t ev[8] = {};
    // Kept host copies (GP_FLAG_KEEP_HIERARCHY).
    struct HostLevel {
        i64 n = 0, m = 0;
        std::vector<int> off, nbr, map;
        std::vector<u32> ew, vw;
        u64 meta[4] = {0, 0, 0, 0};
    };
    std::vector<HostLevel> kept;
    std::vector<int> initial_labels;

    // Copy `count` device scalars to the host and wait for them.
    const u64* read_scalars(int count) {
        GP_CUDA(cudaMemcpyAsync(host_scalars, dev_scalars, sizeof(u64) * count, cudaMemcpyDeviceToHost, stream));
        GP_CUDA(cudaStreamSynchronize(stream));
        return host_scalars;
    }
    void clear_scalars(int count) {
        GP_CUDA(cudaMemsetAsync(dev_scalars, 0, sizeof(u64) * count, stream));
    }
};

// Entry points of the pipeline stages.
// Rows longer than heavy_min entries become g's heavy rows, listed with their
// kChunk-entry chunks in `storage` (the context's persist arena by default).
void build_chunks(Context& ctx, DGraph& g, int heavy_min = kHeavyRow, Arena* storage = nullptr);
Hierarchy coarsen(Context& ctx, const DGraph& input, const CoarsenOptions& o);
void keep_levels(Context& ctx, const Hierarchy& h);

struct RefineOutcome {
    u64 cut = 0;
    u64 max_load = 0;
    int levels_refined = 0;
};
// Round budgets of one level's refinement (RefineOptions::max_rounds and
// exchange_rounds, include/refine.hpp:13-26; the pipeline uses 32 and 2).
struct RefineBudget {
    int rounds = 32;
    int exchange_rounds = 2;
};
// What one level's refinement did (the RefineStats fields of
// include/refine.hpp:28-53 that describe the moves, not the layout).
struct LevelStats {
    int rounds = 0, admission_iterations = 0, checkpoint_updates = 0;
    bool repair_failed = false;
    u64 proposals = 0, accepted = 0, initial_cut = 0, final_cut = 0, final_max_load = 0;
    u64 lp_gain = 0, lp_loss = 0, rebalance_gain = 0, rebalance_loss = 0, group_gain = 0, group_accepted = 0;
};
// Refines from the coarsest level down to level 0 (refine_hierarchy_impl,
// src/refine.cu:483-730); `labels` (device, level-0 sized) receives the result.
RefineOutcome uncoarsen(Context& ctx, Hierarchy& h, const std::vector<int>& coarse_labels, int k, double eps,
                        int* labels, bool log, bool verify, const Mapping& mapping);

// Refines one graph from `labels` (device, n entries, values in [0,k)) in
// place: refine_partition (src/refine.cu:470-481) on a device-resident graph
// whose metadata coarsen() has filled.  The part loads are measured first.
LevelStats refine_single(Context& ctx, const DGraph& g, int* labels, int k, double eps, const RefineBudget& budget,
                         bool log, bool verify, const Mapping& mapping);

// Device edge cut of labels (directed sum / 2); throws on an odd sum.
u64 device_cut(Context& ctx, const DGraph& g, const int* labels);

// GP_FLAG_VERIFY checks (gp_verify.cu); failures throw with `status` or GP_INTERNAL.
void verify_csr(Context& ctx, const DGraph& g, bool allow_self_loops, gp_status status);
void verify_level(Context& ctx, const DGraph& fine, const DGraph& coarse, const int* map, u64 cluster_cap);

}  // namespace gp
