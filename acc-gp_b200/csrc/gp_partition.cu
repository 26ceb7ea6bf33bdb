// C ABI and pipeline driver: upload -> coarsen -> METIS -> uncoarsen -> labels
// (the sequence app/partition_main.cu:99-137 runs), on one CUDA stream.
#include "gp_graph.h"
#include "gp_metis.h"
#include "gp_primitives.cuh"

#include <algorithm>
#include <cstdlib>
#include <cxxabi.h>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>

struct gp_context {
    gp::Context ctx;
    gp::KernelProfiler profiler;
    gp::CoarsenOptions defaults;  // overridable per context, see gp_set_option
    bool seed_matching = true, fast_path = true;
    int cluster_size_factor = 0, fine_factor = 64, growth = 8, heavy_limit = 64;
    gp::Mapping mapping;  // thread-mapping thresholds (gp_set_option, gp_autotune)
    gp::WorkerPool* pool = nullptr;  // batch workers, created on first use
    // gp_load_csr_int64: the loaded graph's device arrays (their own arena,
    // kept across partitions), the pinned staging buffers and their events.
    gp::Arena input;
    gp::DGraph loaded;
    int* loaded_labels = nullptr;
    bool has_loaded = false;
    long long* pinned[2] = {nullptr, nullptr};
    cudaEvent_t staged[2] = {nullptr, nullptr};
};

namespace gp {

WorkerPool*& worker_pool(gp_context* ctx) { return ctx->pool; }
int context_device(const gp_context* ctx) { return ctx->ctx.device; }
size_t context_reserved(const gp_context* ctx) { return ctx->ctx.persist.reserved() + ctx->ctx.scratch.reserved(); }
void context_trim(gp_context* ctx) {
    cudaSetDevice(ctx->ctx.device);
    cudaStreamSynchronize(ctx->ctx.stream);
    ctx->ctx.persist.reset_device();
    ctx->ctx.scratch.reset_device();
}
void copy_options(const gp_context* from, gp_context* to) {
    to->seed_matching = from->seed_matching;
    to->fast_path = from->fast_path;
    to->cluster_size_factor = from->cluster_size_factor;
    to->fine_factor = from->fine_factor;
    to->growth = from->growth;
    to->mapping = from->mapping;
    to->heavy_limit = from->heavy_limit;
}

thread_local KernelProfiler* g_profiler = nullptr;

bool KernelProfiler::matches(const void* kernel) {
    for (auto& entry : cache)
        if (entry.first == kernel) return entry.second;
    const char* name = nullptr;
    bool hit = false;
    if (cudaFuncGetName(&name, kernel) == cudaSuccess && name) {
        // Match the pattern against the symbol and its demangled form.
        hit = std::strstr(name, pattern.c_str()) != nullptr;
        int status = 0;
        char* readable = abi::__cxa_demangle(name, nullptr, nullptr, &status);
        if (readable) {
            hit = hit || std::strstr(readable, pattern.c_str()) != nullptr;
            std::free(readable);
        }
    }
    cache.emplace_back(kernel, hit);
    return hit;
}
void KernelProfiler::before(cudaStream_t s) {
    if (used == events.size()) {
        cudaEvent_t a, b;
        GP_CUDA(cudaEventCreate(&a));
        GP_CUDA(cudaEventCreate(&b));
        events.emplace_back(a, b);
    }
    GP_CUDA(cudaEventRecord(events[used].first, s));
}
void KernelProfiler::after(cudaStream_t s) {
    GP_CUDA(cudaEventRecord(events[used].second, s));
    ++used;
}

namespace {

// load_weighted_graph's narrowing (src/graph.cpp:70-107) of one chunk of
// the int64 files, values copied to int32 at out[0..count).  The first
// failing position (first_index + i) of each check is kept with atomicMin:
// bad[0] an offset negative or below its predecessor (`previous` is the value
// before the chunk), bad[1] an offset above int32, bad[2] a neighbor outside
// [0, n).
__global__ void k_narrow(i64 count, const long long* in, int* out, bool neighbors, long long n, long long previous,
                         u64 first_index, u64* bad) {
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const long long x = in[i];
        const u64 at = first_index + static_cast<u64>(i);
        if (neighbors) {
            if (x < 0 || x >= n) atomicMin(bad + 2, at);
        } else {
            const long long before = i ? in[i - 1] : previous;
            if (x < 0 || x < before) atomicMin(bad, at);
            else if (x > 0x7fffffffLL) atomicMin(bad + 1, at);
        }
        out[i] = static_cast<int>(x);
    }
}

__global__ void k_fill_ones(i64 n, u32* p) {
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<i64>(gridDim.x) * blockDim.x)
        p[i] = 1u;
}

// Shape and range checks of a device CSR (validate_weighted_shape,
// src/graph.cpp:118-155), as two flat grid-stride sweeps so that long rows
// do not serialise.  Scalars: 0 bad offsets, 1 bad neighbour, 2 zero vertex
// weight, 3 total vertex weight, 4 directed edge-weight sum.
__global__ void k_validate_vertices(i64 n, i64 m, const int* off, const u32* vw, u64* sc) {
    u64 total = 0;
    u32 bad = 0, zero = 0;
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int b = off[v], e = off[v + 1];
        bad |= b > e || b < 0 || e > m || (v == 0 && b != 0) || (v == n - 1 && e != m);
        const u32 w = vw ? vw[v] : 1u;
        zero |= w == 0;
        total += w;
    }
    total = warp_sum(total);
    bad = __any_sync(0xffffffffu, bad);
    zero = __any_sync(0xffffffffu, zero);
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicOr(sc + 0, 1ULL);
        if (zero) atomicOr(sc + 2, 1ULL);
        if (total) atomicAdd(sc + 3, total);
    }
}
__global__ void k_validate_edges(i64 n, i64 m, const int* nbr, const u32* ew, u64* sc) {
    u64 directed = 0;
    u32 bad = 0;
    for (i64 e = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; e < m; e += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int u = nbr[e];
        bad |= u < 0 || u >= n;
        directed += ew ? ew[e] : 1u;
    }
    directed = warp_sum(directed);
    bad = __any_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicOr(sc + 1, 1ULL);
        if (directed) atomicAdd(sc + 4, directed);
    }
}

HostCsr download(Context& ctx, const DGraph& g) {
    HostCsr h;
    h.n = g.n;
    h.off.resize(g.n + 1);
    h.nbr.resize(g.m);
    h.ew.resize(g.m);
    h.vw.resize(g.n);
    cudaStream_t s = ctx.stream;
    GP_CUDA(cudaMemcpyAsync(h.off.data(), g.off, sizeof(int) * (g.n + 1), cudaMemcpyDeviceToHost, s));
    if (g.m) GP_CUDA(cudaMemcpyAsync(h.nbr.data(), g.nbr, sizeof(int) * g.m, cudaMemcpyDeviceToHost, s));
    if (g.ew && g.m) GP_CUDA(cudaMemcpyAsync(h.ew.data(), g.ew, sizeof(u32) * g.m, cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaMemcpyAsync(h.vw.data(), g.vw, sizeof(u32) * g.n, cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    if (!g.ew) std::fill(h.ew.begin(), h.ew.end(), 1u);
    return h;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    GP_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

// Compulsory HBM traffic of the V-cycle (the roofline model): per coarsened
// level 2 CSR sweeps + writing the next level; per refined level one sweep
// plus the projection.
u64 algorithmic_bytes(const Hierarchy& h) {
    u64 bytes = 0;
    for (size_t i = 0; i < h.levels.size(); ++i) {
        const DGraph& g = h.levels[i];
        const u64 n = static_cast<u64>(g.n), m = static_cast<u64>(g.m);
        const u64 sweep = 4 * (n + 1) + 4 * m + (g.ew ? 4 * m : 0) + 4 * m + 4 * n;
        if (i + 1 < h.levels.size()) {
            const DGraph& c = h.levels[i + 1];
            bytes += 2 * sweep + 4 * (static_cast<u64>(c.n) + 1) + 8 * static_cast<u64>(c.m) + 4 * static_cast<u64>(c.n) + 4 * n;
        }
        bytes += sweep + 12 * n;
    }
    return bytes;
}

// The input graph on the device: host arrays copied into the persist arena
// (or caller device arrays used in place), unit vertex weights materialised,
// then the shape checks of validate_weighted_shape (src/graph.cpp:118-155)
// on the device, which also give the total vertex weight and the directed
// edge-weight sum.  Records ev[0] (before the copies) and ev[1] (after).
struct Input {
    DGraph g;
    u64 total = 0, directed = 0;
};
Input prepare_input(Context& ctx, const gp_csr* in, bool device_input) {
    if (in->n <= 0) fail(GP_INVALID_ARGUMENT, "empty CSR indptr");
    if (in->n > std::numeric_limits<int>::max() || in->m > std::numeric_limits<int>::max() || in->m < 0)
        fail(GP_INVALID_ARGUMENT, "graph exceeds supported 32-bit CSR limits; dataset excluded");
    if (!device_input) {
        // O(1) shape checks here; monotone offsets, neighbour ranges and
        // positive weights are checked on the device after the upload (the
        // same messages), not by a serial scan of the host arrays.
        if (!in->offsets || (in->m > 0 && !in->neighbors)) fail(GP_INVALID_ARGUMENT, "graph arrays must not be NULL");
        if (in->offsets[0] != 0 || in->offsets[in->n] != in->m) fail(GP_INVALID_ARGUMENT, "invalid weighted CSR shape");
    }
    cudaStream_t s = ctx.stream;
    const i64 n = in->n, m = in->m;
    Input out;
    DGraph& g = out.g;
    g.n = n;
    g.m = m;
    GP_CUDA(cudaEventRecord(ctx.ev[0], s));
    if (device_input) {
        g.off = const_cast<int*>(in->offsets);
        g.nbr = const_cast<int*>(in->neighbors);
        g.ew = const_cast<u32*>(in->edge_weights);
        g.vw = const_cast<u32*>(in->vertex_weights);
    } else {
        g.off = ctx.persist.alloc<int>(n + 1);
        g.nbr = ctx.persist.alloc<int>(m);
        GP_CUDA(cudaMemcpyAsync(g.off, in->offsets, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
        if (m) GP_CUDA(cudaMemcpyAsync(g.nbr, in->neighbors, sizeof(int) * m, cudaMemcpyHostToDevice, s));
        if (in->edge_weights) {
            g.ew = ctx.persist.alloc<u32>(m);
            if (m) GP_CUDA(cudaMemcpyAsync(g.ew, in->edge_weights, sizeof(u32) * m, cudaMemcpyHostToDevice, s));
        }
        if (in->vertex_weights) {
            g.vw = ctx.persist.alloc<u32>(n);
            GP_CUDA(cudaMemcpyAsync(g.vw, in->vertex_weights, sizeof(u32) * n, cudaMemcpyHostToDevice, s));
        }
    }
    if (!g.vw) {
        g.vw = ctx.persist.alloc<u32>(n);
        launch(k_fill_ones, std::min(blocks_for(n, 256), 148 * 8), 256, 0, s, n, g.vw);
    }
    g.implicit_unit = g.ew == nullptr;
    GP_CUDA(cudaEventRecord(ctx.ev[1], s));
    ctx.clear_scalars(5);
    launch(k_validate_vertices, std::min(blocks_for(n, 256), 148 * 16), 256, 0, s, n, m, g.off, g.vw, ctx.dev_scalars);
    launch(k_validate_edges, std::min(blocks_for(m, 256), 148 * 16), 256, 0, s, n, m, g.nbr, g.ew, ctx.dev_scalars);
    const u64* vs = ctx.read_scalars(5);
    if (vs[0]) fail(GP_INVALID_ARGUMENT, "weighted CSR offsets are not monotone");
    if (vs[1]) fail(GP_INVALID_ARGUMENT, "weighted CSR contains an invalid neighbor");
    if (vs[2]) fail(GP_INVALID_ARGUMENT, "vertex weights must be positive");
    out.total = vs[3];
    out.directed = vs[4];
    return out;
}

}  // namespace

// Kept hierarchies of resident graphs (see gp_internal.h).  An entry owns the
// arena its levels live in; entries in use by a call are never dropped.
struct HierarchyCache {
    struct Key {
        uint64_t graph;
        int k;
        uint32_t seed, flags;
        bool operator<(const Key& o) const {
            return std::tie(graph, k, seed, flags) < std::tie(o.graph, o.k, o.seed, o.flags);
        }
    };
    struct Entry {
        Arena storage;
        Hierarchy h;
        u64 total = 0, directed = 0;
        int users = 0;
        u64 last_use = 0;
    };
    int device = 0;
    uint64_t budget = 0;
    std::mutex mu;
    std::map<Key, std::unique_ptr<Entry>> entries;
    u64 clock = 0;

    Entry* find(const Key& key) {
        std::lock_guard<std::mutex> lock(mu);
        auto it = entries.find(key);
        if (it == entries.end()) return nullptr;
        ++it->second->users;
        it->second->last_use = ++clock;
        return it->second.get();
    }
    // Keeps a complete `fresh` entry, in use by the caller, and drops least
    // recently used idle entries while the total exceeds the budget.  When
    // another call kept the same key first, `fresh` is still the caller's
    // and is freed at its release.  Returns the caller's entry.
    Entry* insert(const Key& key, std::unique_ptr<Entry> fresh) {
        std::lock_guard<std::mutex> lock(mu);
        fresh->users = 1;
        fresh->last_use = ++clock;
        Entry* out = fresh.get();
        if (entries.count(key)) retired.push_back(std::move(fresh));
        else entries.emplace(key, std::move(fresh));
        evict();
        return out;
    }
    void release(Entry* e) {
        std::lock_guard<std::mutex> lock(mu);
        --e->users;
        evict();
        free_retired();
    }
    uint64_t bytes() const {
        uint64_t b = 0;
        for (auto& kv : entries) b += kv.second->storage.reserved();
        return b;
    }

private:
    std::vector<std::unique_ptr<Entry>> retired;  // duplicates, freed once idle
    void evict() {
        while (bytes() > budget) {
            auto victim = entries.end();
            for (auto it = entries.begin(); it != entries.end(); ++it)
                if (!it->second->users && (victim == entries.end() || it->second->last_use < victim->second->last_use))
                    victim = it;
            if (victim == entries.end()) break;  // everything is in use
            cudaSetDevice(device);
            entries.erase(victim);
        }
    }
    void free_retired() {
        for (auto& e : retired) if (e && !e->users) { cudaSetDevice(device); e.reset(); }
        retired.erase(std::remove(retired.begin(), retired.end(), nullptr), retired.end());
    }
};

namespace {

gp_status run(gp_context* handle, const gp_csr* in, bool device_input, int k, double eps, uint32_t seed,
              uint32_t flags, int* labels_out, void* user_stream, gp_stats* stats, HierarchyCache* cache = nullptr,
              uint64_t graph_key = 0) {
    Context& ctx = handle->ctx;
    if (!in || !labels_out) fail(GP_INVALID_ARGUMENT, "graph and labels must not be NULL");
    if (k < 2 || k > kMaxParts || !std::isfinite(eps) || eps < 1.0) fail(GP_INVALID_ARGUMENT, "invalid partition capacity options");
    if (in->n <= 0) fail(GP_INVALID_ARGUMENT, "empty CSR indptr");
    GP_CUDA(cudaSetDevice(ctx.device));
    cudaStream_t s = ctx.stream;
    cudaStream_t caller = static_cast<cudaStream_t>(user_stream);
    if (caller) {  // order after the caller's producers
        GP_CUDA(cudaEventRecord(ctx.ev[7], caller));
        GP_CUDA(cudaStreamWaitEvent(s, ctx.ev[7], 0));
    }
    const u64 launches0 = g_launches;
    ctx.persist.release({0, 0});
    ctx.scratch.release({0, 0});
    ctx.persist.reset_peak();
    ctx.scratch.reset_peak();
    const i64 n = in->n;
    // A kept hierarchy of a resident graph, or a fresh one.
    HierarchyCache::Entry* kept = nullptr;
    struct Release {
        HierarchyCache* cache;
        HierarchyCache::Entry*& entry;
        ~Release() { if (cache && entry) cache->release(entry); }
    } release{cache, kept};
    const HierarchyCache::Key key{graph_key, k, seed, flags & GP_FLAG_NO_SEED_MATCHING};
    if (cache) kept = cache->find(key);
    Input input;
    const bool reused = kept != nullptr;
    // On a miss with a cache, the input's own arrays (unit vertex weights) and
    // the levels go to a new entry's arena: it stands in for the persist
    // arena until the hierarchy is complete.
    std::unique_ptr<HierarchyCache::Entry> fresh;
    struct Borrow {
        Arena& persist;
        Arena* lent = nullptr;
        void end() { if (lent) persist.swap(*lent); lent = nullptr; }
        ~Borrow() { end(); }
    } borrow{ctx.persist};
    if (reused) {  // validated and measured when it was kept
        GP_CUDA(cudaEventRecord(ctx.ev[0], s));
        GP_CUDA(cudaEventRecord(ctx.ev[1], s));
        input.g = kept->h.levels.front();
        input.total = kept->total;
        input.directed = kept->directed;
    } else {
        if (cache) {
            fresh = std::make_unique<HierarchyCache::Entry>();
            ctx.persist.swap(fresh->storage);
            borrow.lent = &fresh->storage;
        }
        input = prepare_input(ctx, in, device_input);
    }
    DGraph& g = input.g;
    const u64 total = input.total, directed = input.directed;
    uint64_t capacity = 0;
    if (gp_status st = capacity_of(total, k, eps, &capacity); st != GP_OK) fail(st, last_error());

    CoarsenOptions o;
    o.parts = k;
    o.seed = seed;
    o.cluster_size_factor = handle->cluster_size_factor
        ? handle->cluster_size_factor
        : (k <= 8 ? std::max(64, (512 + k - 1) / k) : std::max(2, (32 + k - 1) / k));
    o.pack_isolated = true;
    o.progressive = k >= 16;
    o.fine_factor = handle->fine_factor;
    o.growth = handle->growth;
    o.heavy_limit = handle->heavy_limit;
    o.seed_matching = handle->seed_matching && !(flags & GP_FLAG_NO_SEED_MATCHING);
    o.fast_path = handle->fast_path;
    o.log = !(flags & GP_FLAG_QUIET);
    o.verify = (flags & GP_FLAG_VERIFY) != 0;
    o.mapping = handle->mapping;
    // --verify: the input must be bidirectional with equal reverse weights
    // (validate_weighted_csr, src/graph.cpp:157-182).
    if (o.verify && !reused) verify_csr(ctx, g, true, GP_INVALID_ARGUMENT);
    Hierarchy h = reused ? kept->h : coarsen(ctx, g, o);
    if (fresh) {  // the entry is complete: the persist arena is the call's own again
        borrow.end();
        fresh->h = h;
        fresh->total = total;
        fresh->directed = directed;
        kept = cache->insert(key, std::move(fresh));
    }
    GP_CUDA(cudaEventRecord(ctx.ev[2], s));
    if (flags & GP_FLAG_KEEP_HIERARCHY) keep_levels(ctx, h);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (flags & GP_FLAG_COARSEN_ONLY) {
        GP_CUDA(cudaStreamSynchronize(s));
        if (stats) {
            stats->levels = static_cast<int32_t>(h.levels.size());
            stats->coarsest_vertices = static_cast<int32_t>(h.levels.back().n);
            stats->coarsen_seconds = elapsed(ctx.ev[1], ctx.ev[2]) * 1e-3;
            stats->kernel_launches = g_launches - launches0;
        }
        return GP_OK;
    }
    const auto t_init = std::chrono::steady_clock::now();
    HostCsr coarsest = download(ctx, h.levels.back());
    std::vector<int> coarse_labels;
    std::string error;
    if (gp_status st = metis_initial_partition(coarsest, k, eps, seed, coarse_labels, error); st != GP_OK) fail(st, error);
    const double init_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_init).count();
    ctx.initial_labels = coarse_labels;
    GP_CUDA(cudaEventRecord(ctx.ev[3], s));
    int* labels_dev = device_input ? labels_out : ctx.persist.alloc<int>(n);
    RefineOutcome r = uncoarsen(ctx, h, coarse_labels, k, eps, labels_dev, o.log, o.verify, o.mapping);
    GP_CUDA(cudaEventRecord(ctx.ev[4], s));
    if (directed & 1ULL) fail(GP_INTERNAL, "symmetric graph has odd directed edge weight");
    if (!device_input)
        GP_CUDA(cudaMemcpyAsync(labels_out, labels_dev, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaEventRecord(ctx.ev[5], s));
    GP_CUDA(cudaEventSynchronize(ctx.ev[5]));
    if (caller) {
        GP_CUDA(cudaEventRecord(ctx.ev[6], s));
        GP_CUDA(cudaStreamWaitEvent(caller, ctx.ev[6], 0));
    }
    if (stats) {
        stats->edge_cut = r.cut;
        stats->max_part_weight = r.max_load;
        stats->capacity = capacity;
        stats->levels = static_cast<int32_t>(h.levels.size());
        stats->coarsest_vertices = static_cast<int32_t>(h.levels.back().n);
        stats->coarsen_seconds = elapsed(ctx.ev[1], ctx.ev[2]) * 1e-3;
        stats->initial_seconds = init_seconds;
        stats->uncoarsen_seconds = elapsed(ctx.ev[3], ctx.ev[4]) * 1e-3;
        stats->algorithm_seconds = elapsed(ctx.ev[1], ctx.ev[4]) * 1e-3;
        stats->h2d_seconds = device_input ? 0.0 : elapsed(ctx.ev[0], ctx.ev[1]) * 1e-3;
        stats->d2h_seconds = device_input ? 0.0 : elapsed(ctx.ev[4], ctx.ev[5]) * 1e-3;
        stats->kernel_launches = g_launches - launches0;
        stats->algorithmic_bytes = algorithmic_bytes(h);
        stats->device_peak_bytes = ctx.persist.peak() + ctx.scratch.peak();
        stats->hierarchy_reused = reused ? 1u : 0u;
    }
    return GP_OK;
}

// refine_partition (src/refine.cu:470-481, include/refine.hpp:84-88): one
// graph refined from the caller's labels with the pipeline's refinement and
// the caller's round budgets.
gp_status run_refine(gp_context* handle, const gp_csr* in, int k, double eps, int rounds, int exchange_rounds,
                     uint32_t flags, int* labels, gp_refine_stats* out) {
    Context& ctx = handle->ctx;
    if (!in || !labels) fail(GP_INVALID_ARGUMENT, "graph and labels must not be NULL");
    if (k < 2 || k > kMaxParts || rounds < 0 || rounds > 64 || exchange_rounds < 0 || exchange_rounds > 8 ||
        !std::isfinite(eps) || eps < 1.0 || in->n <= 0)
        fail(GP_INVALID_ARGUMENT, "invalid refinement options");
    for (i64 v = 0; v < in->n; ++v)
        if (labels[v] < 0 || labels[v] >= k) fail(GP_INVALID_ARGUMENT, "refinement partition has an invalid part id");
    GP_CUDA(cudaSetDevice(ctx.device));
    cudaStream_t s = ctx.stream;
    const u64 launches0 = g_launches;
    ctx.persist.release({0, 0});
    ctx.scratch.release({0, 0});
    Input input = prepare_input(ctx, in, false);
    uint64_t capacity = 0;
    if (gp_status st = capacity_of(input.total, k, eps, &capacity); st != GP_OK) fail(st, last_error());
    if (flags & GP_FLAG_REQUIRE_BALANCED) {  // allow_initial_imbalance = false
        std::vector<u64> loads(static_cast<size_t>(k), 0);
        for (i64 v = 0; v < in->n; ++v) loads[labels[v]] += in->vertex_weights ? in->vertex_weights[v] : 1u;
        if (*std::max_element(loads.begin(), loads.end()) > capacity)
            fail(GP_INVALID_ARGUMENT, "initial refinement partition is imbalanced");
    }
    CoarsenOptions o;  // metadata of the input level only (no coarsening)
    o.parts = k;
    o.max_levels = 0;
    o.log = false;
    o.verify = (flags & GP_FLAG_VERIFY) != 0;
    o.mapping = handle->mapping;
    if (o.verify) verify_csr(ctx, input.g, true, GP_INVALID_ARGUMENT);
    Hierarchy h = coarsen(ctx, input.g, o);
    int* dev_labels = ctx.persist.alloc<int>(in->n);
    GP_CUDA(cudaMemcpyAsync(dev_labels, labels, sizeof(int) * in->n, cudaMemcpyHostToDevice, s));
    RefineBudget budget;
    budget.rounds = rounds;
    budget.exchange_rounds = exchange_rounds;
    GP_CUDA(cudaEventRecord(ctx.ev[2], s));
    const LevelStats st = refine_single(ctx, h.levels[0], dev_labels, k, eps, budget, !(flags & GP_FLAG_QUIET),
                                        o.verify, handle->mapping);
    GP_CUDA(cudaEventRecord(ctx.ev[3], s));
    if (st.repair_failed) fail(GP_CAPACITY_INFEASIBLE, "initial refinement capacity repair failed");
    if (o.verify && device_cut(ctx, h.levels[0], dev_labels) != st.final_cut)
        fail(GP_INTERNAL, "final cut differs from CSR scan");
    GP_CUDA(cudaMemcpyAsync(labels, dev_labels, sizeof(int) * in->n, cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->rounds = st.rounds;
        out->admission_iterations = st.admission_iterations;
        out->checkpoint_updates = st.checkpoint_updates;
        out->proposals = st.proposals;
        out->accepted = st.accepted;
        out->initial_cut = st.initial_cut;
        out->final_cut = st.final_cut;
        out->final_max_part_weight = st.final_max_load;
        out->capacity = capacity;
        out->lp_cut_gain = st.lp_gain;
        out->lp_cut_loss = st.lp_loss;
        out->rebalance_cut_gain = st.rebalance_gain;
        out->rebalance_cut_loss = st.rebalance_loss;
        out->group_cut_gain = st.group_gain;
        out->group_accepted = st.group_accepted;
        out->seconds = elapsed(ctx.ev[2], ctx.ev[3]) * 1e-3;
        out->kernel_launches = g_launches - launches0;
    }
    return GP_OK;
}

template <class F>
gp_status guarded(F&& f) {
    try {
        return f();
    } catch (const Failure& e) {
        set_error(e.what());
        return e.status;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return GP_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_error(e.what());
        return GP_INTERNAL;
    }
}

}  // namespace
}  // namespace gp

namespace gp {
Context& context_of(gp_context* ctx) { return ctx->ctx; }

HierarchyCache* hierarchy_cache_create(int device, uint64_t budget_bytes) {
    auto* c = new HierarchyCache;
    c->device = device;
    c->budget = budget_bytes;
    return c;
}
void hierarchy_cache_destroy(HierarchyCache* cache) {
    if (!cache) return;
    cudaSetDevice(cache->device);
    delete cache;
}
uint64_t hierarchy_cache_bytes(const HierarchyCache* cache) {
    if (!cache) return 0;
    auto* c = const_cast<HierarchyCache*>(cache);
    std::lock_guard<std::mutex> lock(c->mu);
    return c->bytes();
}
gp_status partition_resident(gp_context* ctx, HierarchyCache* cache, uint64_t graph_key, const gp_csr* device_graph,
                             int32_t k, double epsilon, uint32_t seed, uint32_t flags, int32_t* labels_device,
                             gp_stats* stats) {
    if (!ctx) { set_error("context is NULL"); return GP_INVALID_ARGUMENT; }
    return guarded([&] {
        return run(ctx, device_graph, true, k, epsilon, seed, flags, labels_device, nullptr, stats, cache, graph_key);
    });
}
}  // namespace gp

using namespace gp;

extern "C" {

gp_status gp_context_create(int device, gp_context** out) {
    return guarded([&]() -> gp_status {
        if (!out) fail(GP_INVALID_ARGUMENT, "out is NULL");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            cudaGetLastError();
            fail(GP_NO_DEVICE, "no CUDA device is available");
        }
        if (device < 0 || device >= count) fail(GP_INVALID_ARGUMENT, "device ordinal out of range");
        GP_CUDA(cudaSetDevice(device));
        auto* h = new gp_context;
        Context& c = h->ctx;
        c.device = device;
        try {
            GP_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
            GP_CUDA(cudaMalloc(&c.dev_scalars, sizeof(u64) * kScalars));
            GP_CUDA(cudaMallocHost(&c.host_scalars, sizeof(u64) * kScalars));
            for (auto& e : c.ev) GP_CUDA(cudaEventCreate(&e));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return GP_OK;
    });
}

void gp_context_destroy(gp_context* h) {
    if (!h) return;
    destroy_worker_pool(h->pool);
    h->pool = nullptr;
    Context& c = h->ctx;
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    h->input.reset_device();
    for (auto& p : h->pinned) if (p) cudaFreeHost(p);
    for (auto& e : h->staged) if (e) cudaEventDestroy(e);
    if (h->profiler.device_bytes) {
        cudaSetDevice(c.device);
        cudaFree(h->profiler.device_bytes);
    }
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    c.persist.reset_device();
    c.scratch.reset_device();
    if (c.dev_scalars) cudaFree(c.dev_scalars);
    if (c.host_scalars) cudaFreeHost(c.host_scalars);
    for (auto& e : c.ev) if (e) cudaEventDestroy(e);
    if (c.stream) cudaStreamDestroy(c.stream);
    delete h;
}

gp_status gp_partition(gp_context* ctx, const gp_csr* graph, int32_t k, double epsilon, uint32_t seed,
                       uint32_t flags, int32_t* labels_out, gp_stats* stats) {
    if (!ctx) { set_error("context is NULL"); return GP_INVALID_ARGUMENT; }
    return guarded([&] { return run(ctx, graph, false, k, epsilon, seed, flags, labels_out, nullptr, stats); });
}

gp_status gp_partition_device(gp_context* ctx, const gp_csr* graph, int32_t k, double epsilon, uint32_t seed,
                              uint32_t flags, int32_t* labels_out_device, void* stream, gp_stats* stats) {
    if (!ctx) { set_error("context is NULL"); return GP_INVALID_ARGUMENT; }
    return guarded([&] { return run(ctx, graph, true, k, epsilon, seed, flags, labels_out_device, stream, stats); });
}

gp_status gp_refine(gp_context* ctx, const gp_csr* graph, int32_t k, double epsilon, int32_t max_rounds,
                    int32_t exchange_rounds, uint32_t flags, int32_t* labels, gp_refine_stats* stats) {
    if (!ctx) { set_error("context is NULL"); return GP_INVALID_ARGUMENT; }
    return guarded([&] { return run_refine(ctx, graph, k, epsilon, max_rounds, exchange_rounds, flags, labels, stats); });
}

// load_weighted_graph + make_device_weighted (src/graph.cpp:47-116,205-218)
// in one pass: each file is read in chunks of kLoadChunk int64 values into
// one of two pinned buffers while the other chunk is copied to the device and
// narrowed there, so the disk read, the copy and the narrowing overlap.
constexpr int64_t kLoadChunk = int64_t{1} << 23;  // 64 MB of int64 per buffer
gp_status gp_load_csr_int64(gp_context* ctx, const char* indptr_path, const char* indices_path, int64_t* n_out,
                            int64_t* m_out) {
    if (!ctx || !indptr_path || !indices_path) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    int64_t n = 0, m = 0;
    if (gp_status st = gp_read_csr_int64(indptr_path, indices_path, &n, &m, nullptr, nullptr); st != GP_OK) return st;
    return guarded([&]() -> gp_status {
        ctx->has_loaded = false;
        FILE* a = std::fopen(indptr_path, "rb");
        if (!a) fail(GP_IO_ERROR, std::string("cannot open ") + indptr_path);
        long long ends[2] = {0, 0};
        const bool ends_ok = std::fread(&ends[0], 8, 1, a) == 1 && std::fseek(a, -8, SEEK_END) == 0 &&
                             std::fread(&ends[1], 8, 1, a) == 1 && std::fseek(a, 0, SEEK_SET) == 0;
        if (!ends_ok) { std::fclose(a); fail(GP_IO_ERROR, std::string("cannot read ") + indptr_path); }
        if (ends[0] != 0 || ends[1] != m) { std::fclose(a); fail(GP_INVALID_ARGUMENT, "CSR offsets do not match indices"); }
        FILE* b = std::fopen(indices_path, "rb");
        if (!b) { std::fclose(a); fail(GP_IO_ERROR, std::string("cannot open ") + indices_path); }
        struct Files { FILE* a; FILE* b; ~Files() { std::fclose(a); std::fclose(b); } } files{a, b};
        Context& c = ctx->ctx;
        GP_CUDA(cudaSetDevice(c.device));
        cudaStream_t s = c.stream;
        for (int i = 0; i < 2; ++i) {
            if (!ctx->pinned[i]) GP_CUDA(cudaMallocHost(&ctx->pinned[i], sizeof(long long) * kLoadChunk));
            if (!ctx->staged[i]) GP_CUDA(cudaEventCreateWithFlags(&ctx->staged[i], cudaEventDisableTiming));
        }
        GP_CUDA(cudaStreamSynchronize(s));
        ctx->input.release({0, 0});
        DGraph g;
        g.n = n;
        g.m = m;
        g.off = ctx->input.alloc<int>(n + 1);
        g.nbr = ctx->input.alloc<int>(m);
        int* labels = ctx->input.alloc<int>(n);
        long long* staging[2] = {ctx->input.alloc<long long>(kLoadChunk), ctx->input.alloc<long long>(kLoadChunk)};
        GP_CUDA(cudaMemsetAsync(c.dev_scalars, 0xff, 3 * sizeof(u64), s));
        int chunk = 0;
        auto stream_file = [&](FILE* f, const char* path, int64_t count, int* out, bool neighbors) {
            long long previous = 0;
            for (int64_t done = 0; done < count; ++chunk) {
                const int buf = chunk & 1;
                const int64_t take = std::min(kLoadChunk, count - done);
                // The buffer's previous copy must have left it before it is refilled.
                if (chunk >= 2) GP_CUDA(cudaEventSynchronize(ctx->staged[buf]));
                if (std::fread(ctx->pinned[buf], 8, static_cast<size_t>(take), f) != static_cast<size_t>(take))
                    fail(GP_IO_ERROR, std::string("cannot read ") + path);
                GP_CUDA(cudaMemcpyAsync(staging[buf], ctx->pinned[buf], sizeof(long long) * take, cudaMemcpyHostToDevice, s));
                GP_CUDA(cudaEventRecord(ctx->staged[buf], s));
                launch(k_narrow, std::min(blocks_for(take, 256), 148 * 8), 256, 0, s, take,
                       static_cast<const long long*>(staging[buf]), out + done, neighbors, static_cast<long long>(n),
                       previous, static_cast<u64>(done), c.dev_scalars);
                previous = ctx->pinned[buf][take - 1];
                done += take;
            }
        };
        stream_file(a, indptr_path, n + 1, g.off, false);
        stream_file(b, indices_path, m, g.nbr, true);
        // The reference stops at the first failing offset, then at the first
        // failing neighbor.
        const u64* bad = c.read_scalars(3);
        if (bad[0] != ~0ULL && bad[0] <= bad[1]) fail(GP_INVALID_ARGUMENT, "CSR offsets are not monotone");
        if (bad[1] != ~0ULL) fail(GP_INVALID_ARGUMENT, "graph exceeds supported 32-bit CSR limits; dataset excluded");
        if (bad[2] != ~0ULL) fail(GP_INVALID_ARGUMENT, "CSR contains an invalid neighbor");
        ctx->loaded = g;
        ctx->loaded_labels = labels;
        ctx->has_loaded = true;
        if (n_out) *n_out = n;
        if (m_out) *m_out = m;
        return GP_OK;
    });
}

gp_status gp_partition_loaded(gp_context* ctx, int32_t k, double epsilon, uint32_t seed, uint32_t flags,
                              int32_t* labels_out, gp_stats* stats) {
    if (!ctx || !labels_out) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    if (!ctx->has_loaded) { set_error("no graph loaded; call gp_load_csr_int64 first"); return GP_INVALID_ARGUMENT; }
    return guarded([&]() -> gp_status {
        Context& c = ctx->ctx;
        const DGraph& g = ctx->loaded;
        GP_CUDA(cudaSetDevice(c.device));
        int* labels_dev = ctx->loaded_labels;
        const gp_csr dg{g.n, g.m, g.off, g.nbr, nullptr, nullptr};
        gp_stats local{};
        gp_stats* st = stats ? stats : &local;
        const gp_status status = run(ctx, &dg, true, k, epsilon, seed, flags, labels_dev, nullptr, st);
        if (status == GP_OK && !(flags & GP_FLAG_COARSEN_ONLY)) {
            GP_CUDA(cudaEventRecord(c.ev[5], c.stream));
            GP_CUDA(cudaMemcpyAsync(labels_out, labels_dev, sizeof(int) * g.n, cudaMemcpyDeviceToHost, c.stream));
            GP_CUDA(cudaEventRecord(c.ev[6], c.stream));
            GP_CUDA(cudaStreamSynchronize(c.stream));
            st->d2h_seconds = elapsed(c.ev[5], c.ev[6]) * 1e-3;
        }
        return status;
    });
}

// Coordinate search over the mapping thresholds, each candidate timed by the
// best of `repeats` partitions of the same device-resident graph.
gp_status gp_autotune(gp_context* ctx, const gp_csr* graph, int32_t k, double epsilon, uint32_t seed, int32_t repeats,
                      gp_tuning* out) {
    if (!ctx || !graph || !out || repeats < 1) { set_error("NULL argument or repeats < 1"); return GP_INVALID_ARGUMENT; }
    if (graph->n <= 0 || graph->n > std::numeric_limits<int>::max() || graph->m < 0 ||
        graph->m > std::numeric_limits<int>::max() || !graph->offsets || (graph->m && !graph->neighbors)) {
        set_error("invalid graph");
        return GP_INVALID_ARGUMENT;
    }
    struct Buffers {
        void* p[5] = {};
        ~Buffers() { for (void* q : p) if (q) cudaFree(q); }
    } buf;
    return guarded([&]() -> gp_status {
        Context& c = ctx->ctx;
        GP_CUDA(cudaSetDevice(c.device));
        const i64 n = graph->n, m = graph->m;
        GP_CUDA(cudaMalloc(&buf.p[0], sizeof(int) * (n + 1)));
        GP_CUDA(cudaMalloc(&buf.p[1], sizeof(int) * std::max<i64>(m, 1)));
        GP_CUDA(cudaMalloc(&buf.p[4], sizeof(int) * n));
        GP_CUDA(cudaMemcpy(buf.p[0], graph->offsets, sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
        if (m) GP_CUDA(cudaMemcpy(buf.p[1], graph->neighbors, sizeof(int) * m, cudaMemcpyHostToDevice));
        if (graph->vertex_weights) {
            GP_CUDA(cudaMalloc(&buf.p[2], sizeof(u32) * n));
            GP_CUDA(cudaMemcpy(buf.p[2], graph->vertex_weights, sizeof(u32) * n, cudaMemcpyHostToDevice));
        }
        if (graph->edge_weights && m) {
            GP_CUDA(cudaMalloc(&buf.p[3], sizeof(u32) * m));
            GP_CUDA(cudaMemcpy(buf.p[3], graph->edge_weights, sizeof(u32) * m, cudaMemcpyHostToDevice));
        }
        const gp_csr dg{n, m, static_cast<int*>(buf.p[0]), static_cast<int*>(buf.p[1]), static_cast<u32*>(buf.p[2]),
                        static_cast<u32*>(buf.p[3])};
        int* labels_dev = static_cast<int*>(buf.p[4]);
        std::vector<int> reference(static_cast<size_t>(n)), labels(static_cast<size_t>(n));
        int trials = 0;
        // Best algorithm time of `repeats` partitions; the labels must not change.
        auto time_setting = [&](bool first) {
            double best = std::numeric_limits<double>::infinity();
            for (int r = 0; r < repeats + (first ? 1 : 0); ++r) {  // the very first partition only warms up
                gp_stats st{};
                if (gp_status s = run(ctx, &dg, true, k, epsilon, seed, GP_FLAG_QUIET, labels_dev, nullptr, &st); s != GP_OK)
                    fail(s, last_error());
                GP_CUDA(cudaMemcpy(labels.data(), labels_dev, sizeof(int) * n, cudaMemcpyDeviceToHost));
                if (first && r == 0) { reference = labels; continue; }
                if (labels != reference) fail(GP_INTERNAL, "mapping thresholds changed the partition");
                best = std::min(best, st.algorithm_seconds * 1e3);
                ++trials;
            }
            return best;
        };
        struct Restore {  // a failed search leaves the thresholds it started from
            gp_context* ctx;
            Mapping start;
            bool done = false;
            ~Restore() { if (!done) ctx->mapping = start; }
        } restore{ctx, ctx->mapping};
        const double default_ms = time_setting(true);
        double best_ms = default_ms;
        using Field = int Mapping::*;
        struct Knob { Field field; std::vector<int> values; };
        const Knob knobs[] = {
            {&Mapping::medium_degree, {64, 128, 256}},
            {&Mapping::large_narrow, {512, 1024, 2048}},
            {&Mapping::build_short, {32, 64, 128}},
            {&Mapping::rebuild_divisor, {25, 50, 100, 200, 400}},
            {&Mapping::on_demand_degree, {0, 32}},
            {&Mapping::refine_heavy_small, {128, 256, 512}},
            {&Mapping::refine_heavy_mid, {256, 512, 1024}},
            {&Mapping::refine_heavy_large, {1024, 2048, 4096}},
        };
        for (const Knob& knob : knobs) {
            const int kept = ctx->mapping.*knob.field;
            int chosen = kept;
            for (int value : knob.values) {
                if (value == kept) continue;
                ctx->mapping.*knob.field = value;
                const double ms = time_setting(false);
                if (ms < 0.99 * best_ms) { best_ms = ms; chosen = value; }
            }
            ctx->mapping.*knob.field = chosen;
        }
        restore.done = true;
        *out = gp_tuning{ctx->mapping.medium_degree, ctx->mapping.large_narrow, ctx->mapping.build_short,
                         ctx->mapping.rebuild_divisor, ctx->mapping.on_demand_degree, default_ms, best_ms, trials,
                         ctx->mapping.refine_heavy_small, ctx->mapping.refine_heavy_mid,
                         ctx->mapping.refine_heavy_large};
        return GP_OK;
    });
}

gp_status gp_set_option(gp_context* ctx, const char* name, int64_t value) {
    if (!ctx || !name) { set_error("context/name is NULL"); return GP_INVALID_ARGUMENT; }
    const std::string key(name);
    if (key == "seed_matching") ctx->seed_matching = value != 0;
    else if (key == "capacity_safe_fast_path") ctx->fast_path = value != 0;
    else if (key == "cluster_size_factor" && (value == 0 || (value >= 2 && value <= 256))) ctx->cluster_size_factor = static_cast<int>(value);
    else if (key == "progressive_fine_factor" && value >= 2 && value <= (1 << 20)) ctx->fine_factor = static_cast<int>(value);
    else if (key == "progressive_capacity_growth" && value >= 2 && value <= 16) ctx->growth = static_cast<int>(value);
    else if (key == "heavy_edge_degree_limit" && value >= 2 && value <= 256) ctx->heavy_limit = static_cast<int>(value);
    else if (key == "medium_degree" && value >= 8 && value <= 256) ctx->mapping.medium_degree = static_cast<int>(value);
    else if (key == "large_narrow" && value >= 256 && value <= 2048) ctx->mapping.large_narrow = static_cast<int>(value);
    else if (key == "build_short" && value >= 8 && value <= 2048) ctx->mapping.build_short = static_cast<int>(value);
    else if (key == "rebuild_divisor" && value >= 1 && value <= 100000) ctx->mapping.rebuild_divisor = static_cast<int>(value);
    else if (key == "on_demand_degree" && value >= 0 && value <= 32) ctx->mapping.on_demand_degree = static_cast<int>(value);
    else if (key == "refine_heavy_small" && value >= 64 && value <= 8192) ctx->mapping.refine_heavy_small = static_cast<int>(value);
    else if (key == "refine_heavy_mid" && value >= 64 && value <= 8192) ctx->mapping.refine_heavy_mid = static_cast<int>(value);
    else if (key == "refine_heavy_large" && value >= 64 && value <= 8192) ctx->mapping.refine_heavy_large = static_cast<int>(value);
    else if (key == "arena_chunk_mb" && value >= 1 && value <= (int64_t{1} << 24)) {
        ctx->ctx.persist.set_chunk_bytes(static_cast<size_t>(value) << 20);
        ctx->ctx.scratch.set_chunk_bytes(static_cast<size_t>(value) << 20);
    }
    else { set_error("unknown option or value out of range: " + key); return GP_INVALID_ARGUMENT; }
    return GP_OK;
}

gp_status gp_profile_begin(gp_context* ctx, const char* kernel_substring) {
    if (!ctx || !kernel_substring) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    ctx->profiler.pattern = kernel_substring;
    ctx->profiler.cache.clear();
    ctx->profiler.used = 0;
    ctx->profiler.bytes = 0;
    ctx->profiler.last_timed = false;
    return guarded([&]() -> gp_status {
        GP_CUDA(cudaSetDevice(ctx->ctx.device));
        if (!ctx->profiler.device_bytes) GP_CUDA(cudaMalloc(&ctx->profiler.device_bytes, sizeof(unsigned long long)));
        GP_CUDA(cudaMemset(ctx->profiler.device_bytes, 0, sizeof(unsigned long long)));
        g_profiler = &ctx->profiler;
        return GP_OK;
    });
}

gp_status gp_profile_end(gp_context* ctx, uint64_t* launches, double* total_ms, double* algorithmic_bytes) {
    if (!ctx) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    return guarded([&]() -> gp_status {
        g_profiler = nullptr;
        auto& p = ctx->profiler;
        double ms = 0;
        for (size_t i = 0; i < p.used; ++i) {
            GP_CUDA(cudaEventSynchronize(p.events[i].second));
            float t = 0;
            GP_CUDA(cudaEventElapsedTime(&t, p.events[i].first, p.events[i].second));
            ms += t;
        }
        if (launches) *launches = p.used;
        if (total_ms) *total_ms = ms;
        unsigned long long device_bytes = 0;
        if (p.device_bytes)
            GP_CUDA(cudaMemcpy(&device_bytes, p.device_bytes, sizeof(device_bytes), cudaMemcpyDeviceToHost));
        if (algorithmic_bytes) *algorithmic_bytes = p.bytes + static_cast<double>(device_bytes);
        p.used = 0;
        p.bytes = 0;
        return GP_OK;
    });
}

gp_status gp_level_count(gp_context* ctx, int32_t* levels) {
    if (!ctx || !levels) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    *levels = static_cast<int32_t>(ctx->ctx.kept.size());
    return GP_OK;
}

gp_status gp_level_size(gp_context* ctx, int32_t level, int64_t* n, int64_t* m) {
    if (!ctx || level < 0 || level >= static_cast<int32_t>(ctx->ctx.kept.size())) { set_error("no such level"); return GP_INVALID_ARGUMENT; }
    if (n) *n = ctx->ctx.kept[level].n;
    if (m) *m = ctx->ctx.kept[level].m;
    return GP_OK;
}

gp_status gp_level_copy(gp_context* ctx, int32_t level, int32_t* offsets, int32_t* neighbors, uint32_t* edge_weights,
                        uint32_t* vertex_weights, int32_t* map, uint64_t* metadata) {
    if (!ctx || level < 0 || level >= static_cast<int32_t>(ctx->ctx.kept.size())) { set_error("no such level"); return GP_INVALID_ARGUMENT; }
    const auto& L = ctx->ctx.kept[level];
    if (offsets) std::copy(L.off.begin(), L.off.end(), offsets);
    if (neighbors) std::copy(L.nbr.begin(), L.nbr.end(), neighbors);
    if (edge_weights) std::copy(L.ew.begin(), L.ew.end(), edge_weights);
    if (vertex_weights) std::copy(L.vw.begin(), L.vw.end(), vertex_weights);
    if (map && !L.map.empty()) std::copy(L.map.begin(), L.map.end(), map);
    if (metadata) std::copy(L.meta, L.meta + 4, metadata);
    return GP_OK;
}

gp_status gp_write_kept_hierarchy(gp_context* ctx, const char* path) {
    if (!ctx) { set_error("context is NULL"); return GP_INVALID_ARGUMENT; }
    const auto& kept = ctx->ctx.kept;
    std::vector<gp_level> levels(kept.size());
    for (size_t i = 0; i < kept.size(); ++i) {
        const auto& L = kept[i];
        levels[i].graph = gp_csr{L.n, L.m, L.off.data(), L.nbr.data(), L.vw.data(), L.ew.data()};
        levels[i].map = L.map.empty() ? nullptr : L.map.data();
    }
    return gp_write_hierarchy(levels.data(), static_cast<int32_t>(levels.size()), path);
}

gp_status gp_initial_labels(gp_context* ctx, int32_t* labels, int64_t capacity) {
    if (!ctx || !labels) { set_error("NULL argument"); return GP_INVALID_ARGUMENT; }
    const auto& v = ctx->ctx.initial_labels;
    if (static_cast<int64_t>(v.size()) > capacity) { set_error("buffer too small"); return GP_INVALID_ARGUMENT; }
    std::copy(v.begin(), v.end(), labels);
    return GP_OK;
}

}  // extern "C"
