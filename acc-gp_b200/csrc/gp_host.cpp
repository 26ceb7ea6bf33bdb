// Host-side utilities behind the C ABI: error reporting, partition capacity,
// the int64 on-disk CSR format, the independent verifier and the seeded
// synthetic generators.  Nothing here touches the GPU.
#include "gp_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>
#include <omp.h>

namespace gp {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& message) { g_last_error = message; }
const char* last_error() { return g_last_error.c_str(); }

// partition_capacity (include/partition_capacity.hpp:14-25): floor of
// total*eps/k in long double, rejected when it cannot hold ceil(total/k).
gp_status capacity_of(uint64_t total, int k, double eps, uint64_t* out) {
    if (k < 2 || k > kMaxParts || !std::isfinite(eps) || eps < 1.0) {
        set_error("invalid partition capacity options");
        return GP_INVALID_ARGUMENT;
    }
    const long double raw = static_cast<long double>(total) * eps / k;
    if (!std::isfinite(raw) || raw >= static_cast<long double>(std::numeric_limits<uint64_t>::max())) {
        set_error("partition capacity exceeds uint64");
        return GP_INVALID_ARGUMENT;
    }
    const auto capacity = static_cast<uint64_t>(std::floor(raw));
    if (capacity < total / static_cast<unsigned>(k) + (total % static_cast<unsigned>(k) != 0)) {
        set_error("integer partition capacity cannot hold total weight");
        return GP_CAPACITY_INFEASIBLE;
    }
    *out = capacity;
    return GP_OK;
}

gp_status validate_host_csr(const gp_csr* g, bool need_positive_vw) {
    if (!g || g->n < 0 || g->m < 0 || (!g->offsets && g->n >= 0)) {
        set_error("graph is NULL or has negative sizes");
        return GP_INVALID_ARGUMENT;
    }
    if (g->n > std::numeric_limits<int32_t>::max() || g->m > std::numeric_limits<int32_t>::max()) {
        set_error("graph exceeds supported 32-bit CSR limits; dataset excluded");
        return GP_INVALID_ARGUMENT;
    }
    if (g->m > 0 && !g->neighbors) { set_error("neighbors is NULL"); return GP_INVALID_ARGUMENT; }
    if (g->offsets[0] != 0 || g->offsets[g->n] != g->m) {
        set_error("invalid weighted CSR shape");
        return GP_INVALID_ARGUMENT;
    }
    for (int64_t v = 0; v < g->n; ++v)
        if (g->offsets[v] > g->offsets[v + 1]) {
            set_error("weighted CSR offsets are not monotone");
            return GP_INVALID_ARGUMENT;
        }
    unsigned bad = 0;
    const int64_t n = g->n;
    for (int64_t e = 0; e < g->m; ++e) bad |= static_cast<unsigned>(g->neighbors[e] < 0 || g->neighbors[e] >= n);
    if (bad) { set_error("weighted CSR contains an invalid neighbor"); return GP_INVALID_ARGUMENT; }
    if (need_positive_vw && g->vertex_weights)
        for (int64_t v = 0; v < n; ++v)
            if (!g->vertex_weights[v]) { set_error("vertex weights must be positive"); return GP_INVALID_ARGUMENT; }
    return GP_OK;
}

}  // namespace gp

using namespace gp;

extern "C" {

const char* gp_last_error(void) { return gp::last_error(); }
const char* gp_version(void) { return "gpart_b200 1.0 (sm_100a)"; }

gp_status gp_partition_capacity(uint64_t total, int32_t k, double epsilon, uint64_t* capacity) {
    if (!capacity) { set_error("capacity is NULL"); return GP_INVALID_ARGUMENT; }
    return capacity_of(total, k, epsilon, capacity);
}

// load_weighted_graph (src/graph.cpp:47-116): int64 indptr/indices, the same
// range and monotonicity checks, narrowed to int32.
gp_status gp_read_csr_int64(const char* indptr_path, const char* indices_path, int64_t* n_out,
                            int64_t* m_out, int32_t* offsets, int32_t* neighbors) {
    auto count = [](const char* path, int64_t& elements) -> gp_status {
        std::ifstream in(path, std::ios::binary | std::ios::ate);
        if (!in) { set_error(std::string("cannot open ") + path); return GP_IO_ERROR; }
        const auto bytes = static_cast<int64_t>(in.tellg());
        if (bytes < 0 || bytes % 8) { set_error(std::string("invalid binary size ") + path); return GP_IO_ERROR; }
        elements = bytes / 8;
        return GP_OK;
    };
    int64_t offset_count = 0, edge_count = 0;
    if (auto s = count(indptr_path, offset_count); s != GP_OK) return s;
    if (auto s = count(indices_path, edge_count); s != GP_OK) return s;
    if (offset_count < 1) { set_error("empty CSR indptr"); return GP_INVALID_ARGUMENT; }
    const int64_t n = offset_count - 1;
    if (n > std::numeric_limits<int32_t>::max() || edge_count > std::numeric_limits<int32_t>::max()) {
        set_error("graph exceeds supported 32-bit CSR limits; dataset excluded");
        return GP_INVALID_ARGUMENT;
    }
    if (n_out) *n_out = n;
    if (m_out) *m_out = edge_count;
    if (!offsets && !neighbors) return GP_OK;
    if (!offsets || !neighbors) { set_error("offsets and neighbors must both be given"); return GP_INVALID_ARGUMENT; }
    std::vector<int64_t> disk(static_cast<size_t>(offset_count));
    {
        std::ifstream in(indptr_path, std::ios::binary);
        in.read(reinterpret_cast<char*>(disk.data()), static_cast<std::streamsize>(offset_count * 8));
        if (!in) { set_error(std::string("cannot read ") + indptr_path); return GP_IO_ERROR; }
    }
    if (disk.front() != 0 || disk.back() != edge_count) { set_error("CSR offsets do not match indices"); return GP_INVALID_ARGUMENT; }
    for (int64_t i = 0; i < offset_count; ++i) {
        if (disk[i] < 0 || (i > 0 && disk[i] < disk[i - 1])) { set_error("CSR offsets are not monotone"); return GP_INVALID_ARGUMENT; }
        offsets[i] = static_cast<int32_t>(disk[i]);
    }
    std::ifstream in(indices_path, std::ios::binary);
    if (!in) { set_error(std::string("cannot open ") + indices_path); return GP_IO_ERROR; }
    constexpr int64_t chunk = 1 << 20;
    std::vector<int64_t> raw(chunk);
    for (int64_t done = 0; done < edge_count;) {
        const int64_t take = std::min(chunk, edge_count - done);
        in.read(reinterpret_cast<char*>(raw.data()), static_cast<std::streamsize>(take * 8));
        if (!in) { set_error(std::string("cannot read ") + indices_path); return GP_IO_ERROR; }
        unsigned bad = 0;
        for (int64_t i = 0; i < take; ++i) {
            bad |= static_cast<unsigned>(raw[i] < 0 || raw[i] >= n);
            neighbors[done + i] = static_cast<int32_t>(raw[i]);
        }
        if (bad) { set_error("CSR contains an invalid neighbor"); return GP_INVALID_ARGUMENT; }
        done += take;
    }
    return GP_OK;
}

gp_status gp_write_csr_int64(const char* indptr_path, const char* indices_path, const gp_csr* g) {
    if (auto s = validate_host_csr(g, false); s != GP_OK) return s;
    std::ofstream a(indptr_path, std::ios::binary | std::ios::trunc), b(indices_path, std::ios::binary | std::ios::trunc);
    if (!a || !b) { set_error("cannot open CSR output"); return GP_IO_ERROR; }
    std::vector<int64_t> buf(1 << 20);
    auto dump = [&](std::ofstream& out, const int32_t* src, int64_t count) {
        for (int64_t done = 0; done < count;) {
            const int64_t take = std::min<int64_t>(static_cast<int64_t>(buf.size()), count - done);
            for (int64_t i = 0; i < take; ++i) buf[i] = src[done + i];
            out.write(reinterpret_cast<const char*>(buf.data()), static_cast<std::streamsize>(take * 8));
            done += take;
        }
    };
    dump(a, g->offsets, g->n + 1);
    dump(b, g->neighbors, g->m);
    if (!a || !b) { set_error("cannot write CSR output"); return GP_IO_ERROR; }
    return GP_OK;
}

// write_hierarchy (include/hierarchy.hpp:38-123): checks first, then the
// int32 stream into a temporary that is renamed into place.
gp_status gp_write_hierarchy(const gp_level* levels, int32_t count, const char* path) {
    if (!path) { set_error("path is NULL"); return GP_INVALID_ARGUMENT; }
    if (!levels || count < 1) { set_error("cannot write an incomplete hierarchy"); return GP_INVALID_ARGUMENT; }
    constexpr int64_t kMax = std::numeric_limits<int32_t>::max();
    for (int32_t i = 0; i < count; ++i) {
        const gp_csr& g = levels[i].graph;
        if (i + 1 < count && !levels[i].map) { set_error("cannot write an incomplete hierarchy"); return GP_INVALID_ARGUMENT; }
        if (g.n < 0 || g.m < 0 || g.n > kMax || g.m > kMax) {
            set_error("hierarchy export requires 32-bit dimensions");
            return GP_INVALID_ARGUMENT;
        }
        if (!g.offsets || (g.m && !g.neighbors)) { set_error("cannot write an incomplete hierarchy"); return GP_INVALID_ARGUMENT; }
        for (int64_t v = 0; v <= g.n; ++v)
            if (g.offsets[v] < 0) { set_error("hierarchy row offset exceeds int32"); return GP_INVALID_ARGUMENT; }
        if (g.edge_weights)
            for (int64_t e = 0; e < g.m; ++e)
                if (g.edge_weights[e] > static_cast<uint32_t>(kMax)) {
                    set_error("hierarchy edge weight exceeds int32");
                    return GP_INVALID_ARGUMENT;
                }
        if (g.vertex_weights)
            for (int64_t v = 0; v < g.n; ++v)
                if (g.vertex_weights[v] > static_cast<uint32_t>(kMax)) {
                    set_error("hierarchy vertex weight exceeds int32");
                    return GP_INVALID_ARGUMENT;
                }
        if (i > 0)
            for (int64_t v = 0; v < levels[i - 1].graph.n; ++v)
                if (levels[i - 1].map[v] < 0 || levels[i - 1].map[v] >= g.n) {
                    set_error("hierarchy map contains an invalid coarse id");
                    return GP_INVALID_ARGUMENT;
                }
    }
    const std::string temporary = std::string(path) + ".tmp";
    std::ofstream out(temporary, std::ios::binary | std::ios::trunc);
    if (!out) { set_error("cannot open hierarchy temporary file"); return GP_IO_ERROR; }
    auto put = [&](const void* data, int64_t ints) {
        out.write(static_cast<const char*>(data), static_cast<std::streamsize>(ints * 4));
    };
    std::vector<int32_t> ones;
    auto unit = [&](int64_t len) -> const int32_t* {
        if (static_cast<int64_t>(ones.size()) < len) ones.assign(static_cast<size_t>(len), 1);
        return ones.data();
    };
    put(&count, 1);
    for (int32_t i = 0; i < count; ++i) {
        const gp_csr& g = levels[i].graph;
        const int32_t dims[2] = {static_cast<int32_t>(g.n), static_cast<int32_t>(g.m)};
        put(dims, 2);
        put(g.offsets, g.n + 1);
        if (g.m) put(g.neighbors, g.m);
        put(g.edge_weights ? static_cast<const void*>(g.edge_weights) : unit(g.m), g.m);
        put(g.vertex_weights ? static_cast<const void*>(g.vertex_weights) : unit(g.n), g.n);
        if (i > 0) put(levels[i - 1].map, levels[i - 1].graph.n);
    }
    out.flush();
    const bool written = static_cast<bool>(out);
    out.close();
    if (!written) {
        std::remove(temporary.c_str());
        set_error("failed while writing hierarchy");
        return GP_IO_ERROR;
    }
    if (std::rename(temporary.c_str(), path) != 0) {
        std::remove(temporary.c_str());
        set_error("cannot commit hierarchy output");
        return GP_IO_ERROR;
    }
    return GP_OK;
}

// host_cut (src/graph.cpp:184-203).
gp_status gp_edge_cut(const gp_csr* g, const int32_t* labels, uint64_t* cut) {
    if (auto s = validate_host_csr(g, false); s != GP_OK) return s;
    if (!labels || !cut) { set_error("labels/cut is NULL"); return GP_INVALID_ARGUMENT; }
    uint64_t directed = 0;
#pragma omp parallel for reduction(+ : directed) schedule(dynamic, 4096)
    for (int64_t v = 0; v < g->n; ++v)
        for (int64_t e = g->offsets[v]; e < g->offsets[v + 1]; ++e)
            if (labels[v] != labels[g->neighbors[e]]) directed += g->edge_weights ? g->edge_weights[e] : 1u;
    if (directed & 1ULL) { set_error("weighted CSR cut is not symmetric"); return GP_INTERNAL; }
    *cut = directed / 2;
    return GP_OK;
}

// The independent verifier of tools/verify_csr.cpp:37-110, generalised to
// vertex/edge weights and a caller-chosen epsilon; capacity is the same
// floor(total*eps/k) the partitioner enforces.
gp_status gp_verify(const gp_csr* g, const int32_t* labels, int32_t k, double epsilon,
                    int32_t check_symmetry, uint64_t* cut_out, uint64_t* loads_out,
                    int32_t* capacity_ok, char* json, size_t json_capacity) {
    if (auto s = validate_host_csr(g, false); s != GP_OK) return s;
    if (!labels || k < 2 || k > kMaxParts) { set_error("invalid k or labels"); return GP_INVALID_ARGUMENT; }
    const int64_t n = g->n;
    std::vector<uint64_t> loads(static_cast<size_t>(k), 0);
    uint64_t total = 0;
    for (int64_t v = 0; v < n; ++v) {
        if (labels[v] < 0 || labels[v] >= k) { set_error("invalid label"); return GP_INVALID_ARGUMENT; }
        const uint64_t w = g->vertex_weights ? g->vertex_weights[v] : 1u;
        loads[static_cast<size_t>(labels[v])] += w;
        total += w;
    }
    uint64_t cut = 0, nonloop = 0;
    int unsorted = 0, asym = 0;
#pragma omp parallel for reduction(+ : cut, nonloop) reduction(| : unsorted) schedule(dynamic, 1024)
    for (int64_t v = 0; v < n; ++v)
        for (int64_t e = g->offsets[v]; e < g->offsets[v + 1]; ++e) {
            const int32_t u = g->neighbors[e];
            const uint64_t w = g->edge_weights ? g->edge_weights[e] : 1u;
            nonloop += (u != v) ? w : 0;
            cut += labels[v] != labels[u] ? w : 0;
            if (e > g->offsets[v] && g->neighbors[e - 1] > u) unsorted = 1;
        }
    if (check_symmetry) {
        if (unsorted) { set_error("symmetry check requires sorted rows"); return GP_INVALID_ARGUMENT; }
#pragma omp parallel for reduction(| : asym) schedule(dynamic, 256)
        for (int64_t v = 0; v < n; ++v)
            for (int64_t e = g->offsets[v]; e < g->offsets[v + 1];) {
                const int32_t u = g->neighbors[e];
                int64_t end = e + 1;
                uint64_t w = g->edge_weights ? g->edge_weights[e] : 1u;
                while (end < g->offsets[v + 1] && g->neighbors[end] == u) { w += g->edge_weights ? g->edge_weights[end] : 1u; ++end; }
                if (u != v) {
                    const int32_t* lo = std::lower_bound(g->neighbors + g->offsets[u], g->neighbors + g->offsets[u + 1], static_cast<int32_t>(v));
                    const int32_t* hi = std::upper_bound(lo, g->neighbors + g->offsets[u + 1], static_cast<int32_t>(v));
                    uint64_t back = 0;
                    for (const int32_t* p = lo; p < hi; ++p) back += g->edge_weights ? g->edge_weights[p - g->neighbors] : 1u;
                    if (hi - lo != end - e || back != w) asym = 1;
                }
                e = end;
            }
        if (asym) { set_error("asymmetric edge multiplicity or weight"); return GP_INVALID_ARGUMENT; }
    }
    if ((cut & 1ULL) || (nonloop & 1ULL)) { set_error("odd undirected edge/cut count"); return GP_INTERNAL; }
    cut /= 2;
    nonloop /= 2;
    uint64_t capacity = 0;
    if (auto s = capacity_of(total, k, epsilon, &capacity); s != GP_OK) return s;
    const uint64_t maximum = *std::max_element(loads.begin(), loads.end());
    if (cut_out) *cut_out = cut;
    if (loads_out) std::copy(loads.begin(), loads.end(), loads_out);
    if (capacity_ok) *capacity_ok = maximum <= capacity;
    if (json && json_capacity) {
        std::ostringstream out;
        out.precision(17);
        out << "{\"vertices\":" << n << ",\"undirected_edges\":" << nonloop << ",\"cut\":" << cut
            << ",\"cut_ratio\":" << (nonloop ? static_cast<double>(cut) / nonloop : 0) << ",\"loads\":[";
        for (int p = 0; p < k; ++p) out << (p ? "," : "") << loads[static_cast<size_t>(p)];
        out << "],\"max_load\":" << maximum << ",\"max_load_ratio\":"
            << (total ? static_cast<double>(maximum) * k / total : 0) << ",\"capacity\":" << capacity
            << ",\"capacity_ok\":" << (maximum <= capacity ? "true" : "false") << "}";
        const auto text = out.str();
        std::snprintf(json, json_capacity, "%s", text.c_str());
    }
    return GP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Seeded synthetic inputs.  Every random value is a pure function of
// (seed, stream, counter) through the splitmix64 finaliser, so the graphs are
// identical on every host and independent of thread count.
// ---------------------------------------------------------------------------
namespace {

inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
inline uint64_t keyed(uint64_t seed, uint64_t stream, uint64_t counter) {
    return mix64(mix64(seed * 0x9E3779B97F4A7C15ULL + stream) + counter * 0xD1B54A32D192ED03ULL);
}

// Parallel LSD radix sort of 64-bit keys restricted to `bits` low bits.
void radix_sort_u64(std::vector<uint64_t>& keys, int bits) {
    const size_t count = keys.size();
    std::vector<uint64_t> other(count);
    constexpr int kDigit = 11;
    const int threads = std::max(1, omp_get_max_threads());
    std::vector<size_t> hist(static_cast<size_t>(threads) << kDigit);
    for (int shift = 0; shift < bits; shift += kDigit) {
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(threads)
        {
            const int t = omp_get_thread_num();
            const size_t lo = count * t / threads, hi = count * (t + 1) / threads;
            size_t* h = hist.data() + (static_cast<size_t>(t) << kDigit);
            for (size_t i = lo; i < hi; ++i) ++h[(keys[i] >> shift) & ((1u << kDigit) - 1)];
#pragma omp barrier
#pragma omp single
            {
                size_t running = 0;
                for (size_t d = 0; d < (1u << kDigit); ++d)
                    for (int u = 0; u < threads; ++u) {
                        size_t& slot = hist[(static_cast<size_t>(u) << kDigit) + d];
                        const size_t c = slot;
                        slot = running;
                        running += c;
                    }
            }
            for (size_t i = lo; i < hi; ++i) other[h[(keys[i] >> shift) & ((1u << kDigit) - 1)]++] = keys[i];
        }
        keys.swap(other);
    }
}

struct RmatKey {
    int scale, ef;
    double a, b, c;
    uint64_t seed;
    bool operator<(const RmatKey& o) const {
        return std::tie(scale, ef, a, b, c, seed) < std::tie(o.scale, o.ef, o.a, o.b, o.c, o.seed);
    }
};
struct RmatGraph { std::vector<int32_t> offsets, neighbors; };
std::mutex g_rmat_mutex;
std::map<RmatKey, RmatGraph> g_rmat_cache;

RmatGraph build_rmat(const RmatKey& key) {
    const int s = key.scale;
    const int64_t n = int64_t{1} << s;
    const int64_t samples = static_cast<int64_t>(key.ef) * n;
    const double ta = key.a, tb = key.a + key.b, tc = key.a + key.b + key.c;
    std::vector<uint64_t> edges(static_cast<size_t>(2 * samples));
    std::vector<uint8_t> keep(static_cast<size_t>(samples));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < samples; ++i) {
        uint64_t state = keyed(key.seed, 0x524d4154ULL, static_cast<uint64_t>(i));
        uint64_t src = 0, dst = 0;
        for (int l = 0; l < s; ++l) {
            state += 0x9E3779B97F4A7C15ULL;
            const double u = static_cast<double>(mix64(state) >> 11) * 0x1.0p-53;
            const uint64_t bit = uint64_t{1} << (s - 1 - l);
            if (u < ta) {
            } else if (u < tb) {
                dst |= bit;
            } else if (u < tc) {
                src |= bit;
            } else {
                src |= bit;
                dst |= bit;
            }
        }
        keep[i] = src != dst;
        edges[2 * i] = (src << s) | dst;
        edges[2 * i + 1] = (dst << s) | src;
    }
    // Drop self loops before sorting.
    size_t w = 0;
    for (int64_t i = 0; i < samples; ++i)
        if (keep[i]) { edges[w++] = edges[2 * i]; edges[w++] = edges[2 * i + 1]; }
    edges.resize(w);
    radix_sort_u64(edges, 2 * s);
    edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
    RmatGraph g;
    g.offsets.assign(static_cast<size_t>(n + 1), 0);
    g.neighbors.resize(edges.size());
    const uint64_t mask = (uint64_t{1} << s) - 1;
    for (size_t i = 0; i < edges.size(); ++i) {
        ++g.offsets[static_cast<size_t>((edges[i] >> s) + 1)];
        g.neighbors[i] = static_cast<int32_t>(edges[i] & mask);
    }
    for (int64_t v = 0; v < n; ++v) g.offsets[static_cast<size_t>(v + 1)] += g.offsets[static_cast<size_t>(v)];
    return g;
}

}  // namespace

extern "C" {

gp_status gp_generate_grid2d(int32_t width, int32_t height, int64_t* n_out, int64_t* m_out,
                             int32_t* offsets, int32_t* neighbors) {
    if (width < 1 || height < 1 || static_cast<int64_t>(width) * height > std::numeric_limits<int32_t>::max()) {
        set_error("invalid grid size");
        return GP_INVALID_ARGUMENT;
    }
    const int64_t n = static_cast<int64_t>(width) * height;
    const int64_t m = 2 * (static_cast<int64_t>(width - 1) * height + static_cast<int64_t>(height - 1) * width);
    if (n_out) *n_out = n;
    if (m_out) *m_out = m;
    if (!offsets || !neighbors) return GP_OK;
    int64_t e = 0;
    for (int32_t y = 0; y < height; ++y)
        for (int32_t x = 0; x < width; ++x) {
            const int64_t v = static_cast<int64_t>(y) * width + x;
            offsets[v] = static_cast<int32_t>(e);
            if (y > 0) neighbors[e++] = static_cast<int32_t>(v - width);
            if (x > 0) neighbors[e++] = static_cast<int32_t>(v - 1);
            if (x + 1 < width) neighbors[e++] = static_cast<int32_t>(v + 1);
            if (y + 1 < height) neighbors[e++] = static_cast<int32_t>(v + width);
        }
    offsets[n] = static_cast<int32_t>(e);
    return GP_OK;
}

gp_status gp_generate_mesh3d(int32_t X, int32_t Y, int32_t Z, int32_t weighted, uint64_t seed,
                             int64_t* n_out, int64_t* m_out, int32_t* offsets, int32_t* neighbors,
                             uint32_t* vertex_weights, uint32_t* edge_weights) {
    if (X < 1 || Y < 1 || Z < 1 || static_cast<int64_t>(X) * Y * Z > std::numeric_limits<int32_t>::max() / 8) {
        set_error("invalid mesh size");
        return GP_INVALID_ARGUMENT;
    }
    const int64_t n = static_cast<int64_t>(X) * Y * Z;
    const int64_t m = 2 * (static_cast<int64_t>(X - 1) * Y * Z + static_cast<int64_t>(Y - 1) * X * Z +
                           static_cast<int64_t>(Z - 1) * X * Y);
    if (n_out) *n_out = n;
    if (m_out) *m_out = m;
    if (!offsets || !neighbors) return GP_OK;
    const int64_t XY = static_cast<int64_t>(X) * Y;
    int64_t e = 0;
    for (int64_t v = 0; v < n; ++v) {
        const int64_t x = v % X, y = (v / X) % Y, z = v / XY;
        offsets[v] = static_cast<int32_t>(e);
        if (z > 0) neighbors[e++] = static_cast<int32_t>(v - XY);
        if (y > 0) neighbors[e++] = static_cast<int32_t>(v - X);
        if (x > 0) neighbors[e++] = static_cast<int32_t>(v - 1);
        if (x + 1 < X) neighbors[e++] = static_cast<int32_t>(v + 1);
        if (y + 1 < Y) neighbors[e++] = static_cast<int32_t>(v + X);
        if (z + 1 < Z) neighbors[e++] = static_cast<int32_t>(v + XY);
    }
    offsets[n] = static_cast<int32_t>(e);
    if (weighted) {
        gp_csr g{n, m, offsets, neighbors, nullptr, nullptr};
        return gp_generate_weights(&g, seed, 1, 4, 1, 16, vertex_weights, edge_weights);
    }
    if (vertex_weights) std::fill(vertex_weights, vertex_weights + n, 1u);
    if (edge_weights) std::fill(edge_weights, edge_weights + m, 1u);
    return GP_OK;
}

gp_status gp_generate_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                           uint64_t seed, int64_t* n_out, int64_t* m_out, int32_t* offsets,
                           int32_t* neighbors) {
    if (scale < 1 || scale > 26 || edge_factor < 1 || edge_factor > 64 || a < 0 || b < 0 || c < 0 ||
        a + b + c > 1.0) {
        set_error("invalid R-MAT parameters");
        return GP_INVALID_ARGUMENT;
    }
    const RmatKey key{scale, edge_factor, a, b, c, seed};
    std::lock_guard<std::mutex> lock(g_rmat_mutex);
    auto it = g_rmat_cache.find(key);
    if (it == g_rmat_cache.end()) {
        g_rmat_cache.clear();  // keep at most one cached graph
        it = g_rmat_cache.emplace(key, build_rmat(key)).first;
    }
    const auto& g = it->second;
    if (static_cast<int64_t>(g.neighbors.size()) > std::numeric_limits<int32_t>::max()) {
        set_error("R-MAT graph exceeds 32-bit CSR limits");
        return GP_INVALID_ARGUMENT;
    }
    if (n_out) *n_out = static_cast<int64_t>(g.offsets.size()) - 1;
    if (m_out) *m_out = static_cast<int64_t>(g.neighbors.size());
    if (offsets) std::copy(g.offsets.begin(), g.offsets.end(), offsets);
    if (neighbors) std::copy(g.neighbors.begin(), g.neighbors.end(), neighbors);
    if (offsets && neighbors) g_rmat_cache.clear();
    return GP_OK;
}

gp_status gp_generate_weights(const gp_csr* g, uint64_t seed, uint32_t vw_lo, uint32_t vw_hi,
                              uint32_t ew_lo, uint32_t ew_hi, uint32_t* vertex_weights,
                              uint32_t* edge_weights) {
    if (auto s = validate_host_csr(g, false); s != GP_OK) return s;
    if (vw_lo < 1 || vw_hi < vw_lo || ew_lo < 1 || ew_hi < ew_lo) { set_error("invalid weight range"); return GP_INVALID_ARGUMENT; }
    const int64_t n = g->n;
    if (vertex_weights) {
#pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < n; ++v)
            vertex_weights[v] = vw_lo + static_cast<uint32_t>(keyed(seed, 0x5657ULL, static_cast<uint64_t>(v)) %
                                                              (static_cast<uint64_t>(vw_hi) - vw_lo + 1));
    }
    if (edge_weights) {
#pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t v = 0; v < n; ++v)
            for (int64_t e = g->offsets[v]; e < g->offsets[v + 1]; ++e) {
                const uint64_t u = static_cast<uint64_t>(g->neighbors[e]);
                const uint64_t lo = std::min<uint64_t>(u, static_cast<uint64_t>(v));
                const uint64_t hi = std::max<uint64_t>(u, static_cast<uint64_t>(v));
                edge_weights[e] = ew_lo + static_cast<uint32_t>(keyed(seed, 0x4557ULL, (lo << 32) | hi) %
                                                               (static_cast<uint64_t>(ew_hi) - ew_lo + 1));
            }
    }
    return GP_OK;
}

}  // extern "C"
