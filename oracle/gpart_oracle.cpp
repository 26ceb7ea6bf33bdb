// CPU oracle of the Acc-GPart partitioner (test infrastructure only; see
// gpart_oracle.h).  Serial C++17 restatement of the reference's rules.  Every
// function cites the reference lines it restates; reference paths are
// relative to the Acc-GPart source tree.
#include "gpart_oracle.h"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>
#include <cstdio>
#include <cstdlib>

// Declarations of the METIS 5.1 API as shipped with the CUDA toolkit
// (64-bit idx_t, 32-bit real_t; option slots probed at run time).
extern "C" {
typedef int64_t idx_t;
typedef float real_t;
int METIS_SetDefaultOptions(idx_t* options);
int METIS_PartGraphKway(idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, real_t*,
                        real_t*, idx_t*, idx_t*, idx_t*);
}

namespace {

using u64 = uint64_t;
using i64 = int64_t;
using u32 = uint32_t;
constexpr int kMaxParts = 128;
constexpr int32_t kInvalid = 0x7fffffff;
constexpr int kMetisOptions = 40, kMetisSeed = 8, kMetisNumbering = 17, kMetisOk = 1;

struct Fail : std::runtime_error {
    int status;
    Fail(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};
[[noreturn]] void fail(int status, const std::string& m) { throw Fail(status, m); }

thread_local std::string g_error;

// mix32 of src/coarsen.cu:173-179 (also seed_matching.cuh:7, refine.cu:50).
inline u32 mix32(u32 x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    return x ^ (x >> 16);
}

struct Graph {
    i64 n = 0, m = 0;
    std::vector<int32_t> off, nbr;
    std::vector<u32> ew, vw;  // always materialised
    bool implicit_unit = false;
    u64 maximum_degree = UINT64_MAX;  // DeviceWeightedGraph metadata, include/graph.hpp:148-171
    bool has_heavy_rows = true;
    u64 incident_weight_bound = UINT64_MAX;
    i64 deg(i64 v) const { return off[v + 1] - off[v]; }
};

// partition_capacity (include/partition_capacity.hpp:14-25).
u64 partition_capacity(u64 total, int parts, double eps) {
    if (parts < 2 || parts > kMaxParts || !std::isfinite(eps) || eps < 1.0) fail(1, "invalid partition capacity options");
    const long double raw = static_cast<long double>(total) * eps / parts;
    if (!std::isfinite(raw) || raw >= static_cast<long double>(UINT64_MAX)) fail(1, "partition capacity exceeds uint64");
    const u64 c = static_cast<u64>(std::floor(raw));
    if (c < total / static_cast<unsigned>(parts) + (total % parts != 0)) fail(2, "integer partition capacity cannot hold total weight");
    return c;
}

// ---------------------------------------------------------------- coarsening

struct Options {  // app/partition_main.cu:52-87 with no environment overrides
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
};

struct Workspace {  // SclpWorkspace::Impl state, src/coarsen.cu:299-396
    bool positive = false, unit = false, sorted_unique = false, invariants_known = false;
    i64 original_vertices = 0;
    u64 maximum_row_weight = 0, total_vw = 0, max_vw = 0;
    std::vector<u64> row_bounds;
};

struct Aggregate {
    std::vector<int32_t> map;
    std::vector<u32> cvw;
    i64 nc = 0;
    u64 max_w = 0, capacity = 0, stats_max_degree = 0;
    bool stats_heavy = false;
};

// record_bound_kernel + metadata (src/coarsen.cu:51-99, 1807-1848).
void level0_metadata(Graph& g, Workspace& ws) {
    u64 maxb = 0, maxraw = 0;
    bool unsorted = false, zero = false, nonunit = false;
    ws.row_bounds.assign(static_cast<size_t>(g.n), 0);
    for (i64 v = 0; v < g.n; ++v) {
        u64 d = 0;
        for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
            const u64 w = g.ew[e];
            d = ~0ULL - d < w ? ~0ULL : d + w;
            if (e > g.off[v] && g.nbr[e] <= g.nbr[e - 1]) unsorted = true;
            zero |= w == 0;
            nonunit |= w != 1;
        }
        ws.row_bounds[v] = d;
        maxb = std::max(maxb, d);
        maxraw = std::max<u64>(maxraw, static_cast<u64>(g.deg(v)));
    }
    ws.original_vertices = g.n;
    ws.maximum_row_weight = maxb;
    g.incident_weight_bound = maxb;
    ws.sorted_unique = !unsorted;
    ws.positive = !zero;
    ws.unit = !nonunit;
    g.maximum_degree = maxraw;
    g.has_heavy_rows = maxraw >= 4096;
}

struct Prop {
    std::vector<int32_t> target;  // proposals
    std::vector<u64> gain, regret;
    std::vector<u32> tie;
};

// form_exact_proposals (src/coarsen.cu:739-970): roles, exact per-cluster
// affinities (aggregation.cuh:180-511 in all degree classes) and decoding
// (aggregation.cuh:513-557).  Every class computes the same per-(v,cluster)
// sums, so one serial scan per row reproduces all of them.
void form_proposals(const Graph& g, const std::vector<int32_t>& clusters, const std::vector<u64>& cw,
                    std::vector<uint8_t>& roles, u64 capacity, u32 seed, int level, int round,
                    bool filter_roles, u32 threshold, bool need_regret, Prop& out,
                    std::vector<u64>& acc, std::vector<int32_t>& touched) {
    const i64 n = g.n;
    const u32 role_salt = seed ^ (static_cast<u32>(level) * 0x9e3779b9U) ^ (static_cast<u32>(round) * 0x85ebca6bU) ^ 0x27d4eb2dU;
    const u32 tie_salt = seed ^ (static_cast<u32>(level) * 0xc2b2ae35U) ^ (static_cast<u32>(round) * 0x165667b1U) ^ 0xd3a2646cU;
    // residual_freeze_roles (singleton_growth.cuh:27-40)
    for (i64 v = 0; v < n; ++v)
        roles[v] = clusters[v] == v && cw[v] == static_cast<u64>(g.vw[v]) &&
                   (!filter_roles || mix32(static_cast<u32>(v) ^ role_salt) < threshold);
    const bool second_on = filter_roles && need_regret;
    auto admissible = [&](int32_t s, int32_t t) {  // SclpResidualPolicy::admissible
        const u64 base = cw[t];
        return base != 0 && base <= capacity && cw[s] <= capacity - base;
    };
    out.target.assign(static_cast<size_t>(n), kInvalid);
    out.gain.assign(static_cast<size_t>(n), 0);
    out.tie.assign(static_cast<size_t>(n), 0);
    out.regret.assign(static_cast<size_t>(n), 0);
    for (i64 v = 0; v < n; ++v) {
        const int32_t src = clusters[v];
        if (!roles[src]) continue;  // filter_sources; decode's role check
        touched.clear();
        for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
            const int32_t u = g.nbr[e];
            if (u == v) continue;
            const int32_t c = clusters[u];
            if (acc[c] == UINT64_MAX) { acc[c] = 0; touched.push_back(c); }
            acc[c] += g.ew[e];
        }
        u64 current = 0, best = 0, tie = 0, second = 0;
        for (int32_t c : touched) {
            const u64 conn = acc[c];
            acc[c] = UINT64_MAX;
            if (c == src) { current = conn; continue; }
            if (filter_roles && (roles[c] || !admissible(src, c))) continue;
            const u64 key = (static_cast<u64>(mix32(static_cast<u32>(v) ^ mix32(static_cast<u32>(c)) ^ tie_salt)) << 32) |
                            (0xffffffffULL - static_cast<u32>(c));
            const bool better = conn > best || (conn == best && conn != 0 && key > tie);
            if (better) {
                second = std::max(second, best);
                best = conn;
                tie = key;
            } else second = std::max(second, conn);
        }
        const u64 role_gain = best > current ? best - current : 0;
        if (!role_gain) continue;
        const auto target = static_cast<int32_t>(0xffffffffULL - (tie & 0xffffffffULL));
        if (target < 0 || target == src) continue;
        out.target[v] = target;
        out.gain[v] = best - current;
        if (second_on) out.regret[v] = best - second;
        out.tie[v] = static_cast<u32>(tie >> 32);
    }
}

// Stable order of proposals by (target asc, key desc, tie desc, vertex asc):
// build_admission_order (src/coarsen.cu:666-718) with the radix key of
// capacity_admission.hpp:14-35 (the gain field holds every gain exactly).
std::vector<int32_t> admission_order(const std::vector<int32_t>& target, const std::vector<u64>& key,
                                     const std::vector<u32>& tie) {
    std::vector<int32_t> order;
    for (size_t v = 0; v < target.size(); ++v)
        if (target[v] != kInvalid) order.push_back(static_cast<int32_t>(v));
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        if (target[a] != target[b]) return target[a] < target[b];
        if (key[a] != key[b]) return key[a] > key[b];
        return tie[a] > tie[b];
    });
    return order;
}

// seed matching (seed_matching.cuh:12-91; call site src/coarsen.cu:505-535).
i64 seed_matching(const Graph& g, u64 capacity, u32 salt, std::vector<int32_t>& roots, std::vector<u64>& cw) {
    const i64 n = g.n;
    std::vector<int32_t> choice(static_cast<size_t>(n), -1);
    for (i64 v = 0; v < n; ++v) {
        if (g.deg(v) > 1024) continue;
        const u64 weight = g.vw[v];
        int32_t best = -1;
        u32 bw = 0, bh = 0;
        for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
            const int32_t u = g.nbr[e];
            if (u == v || weight > capacity || static_cast<u64>(g.vw[u]) > capacity - weight) continue;
            const int32_t lo = std::min<int32_t>(static_cast<int32_t>(v), u), hi = std::max<int32_t>(static_cast<int32_t>(v), u);
            const u32 h = mix32(static_cast<u32>(lo) ^ mix32(static_cast<u32>(hi) ^ salt));
            const u32 w = g.ew[e];
            if (best < 0 || w > bw || (w == bw && (h > bh || (h == bh && u > best)))) { best = u; bw = w; bh = h; }
        }
        choice[v] = best;
    }
    std::vector<int32_t> matched(static_cast<size_t>(n), -1);
    for (i64 v = 0; v < n; ++v) {
        const int32_t u = choice[v];
        if (u > v && choice[u] == v) { matched[v] = u; matched[u] = static_cast<int32_t>(v); }
    }
    i64 clusters = 0;
    roots.resize(static_cast<size_t>(n));
    cw.assign(static_cast<size_t>(n), 0);
    for (i64 v = 0; v < n; ++v) {
        const int32_t p = matched[v];
        roots[v] = p < 0 ? static_cast<int32_t>(v) : std::min<int32_t>(static_cast<int32_t>(v), p);
        clusters += roots[v] == v;
    }
    for (i64 v = 0; v < n; ++v) cw[roots[v]] += g.vw[v];
    return clusters;
}

// aggregate_typed (src/coarsen.cu:467-1380).
Aggregate aggregate(const Graph& g, Workspace& ws, int parts, u32 seed, int level, int factor,
                    bool pack_isolated, bool matching, bool fast_path) {
    const i64 n = g.n;
    if (!ws.invariants_known) {
        ws.total_vw = 0;
        ws.max_vw = 0;
        for (u32 w : g.vw) { ws.total_vw += w; ws.max_vw = std::max<u64>(ws.max_vw, w); }
        ws.invariants_known = true;
    }
    const u64 total = ws.total_vw, maxv = ws.max_vw;
    const u64 denom = static_cast<u64>(factor) * static_cast<u64>(parts);
    Aggregate out;
    out.capacity = std::max(maxv, total / denom + (total % denom != 0));
    const u64 C = out.capacity;
    std::vector<int32_t> clusters(static_cast<size_t>(n));
    std::vector<u64> cw;
    i64 cluster_count = n;
    if (matching) {
        cluster_count = seed_matching(g, C, seed ^ (static_cast<u32>(level) * 0x9e3779b9U), clusters, cw);
    } else {
        std::iota(clusters.begin(), clusters.end(), 0);
        cw.assign(g.vw.begin(), g.vw.end());
    }
    // degree classes (aggregation.cuh:5-71, src/coarsen.cu:547-579)
    if (g.maximum_degree <= 8) {
        out.stats_max_degree = g.maximum_degree;
        out.stats_heavy = false;
    } else {
        u64 md = 0;
        bool heavy = false;
        for (i64 v = 0; v < n; ++v) { md = std::max<u64>(md, static_cast<u64>(g.deg(v))); heavy |= g.deg(v) >= 4096; }
        out.stats_max_degree = md;
        out.stats_heavy = heavy;
    }
    std::vector<uint8_t> roles(static_cast<size_t>(n));
    std::vector<u64> acc(static_cast<size_t>(n), UINT64_MAX);
    std::vector<int32_t> touched;
    Prop prop;
    const i64 desired = (n + 1) / 2;
    u64 bound = matching ? (maxv > C / 2 ? C : 2 * maxv) : maxv;
    auto count_clusters = [&]() { i64 c = 0; for (u64 w : cw) c += w != 0; return c; };
    for (int round = 0; round < 4; ++round) {  // src/coarsen.cu:982-1128
        if (static_cast<double>(cluster_count) <= 0.60 * n) break;
        const i64 removable = std::max<i64>(0, cluster_count - desired);
        const double fraction = std::min(0.50, static_cast<double>(removable) / static_cast<double>(cluster_count));
        const auto threshold = static_cast<u32>(fraction * 4294967296.0);
        const u64 room = C - bound;
        const u64 degree = out.stats_max_degree;
        const bool all_fit = fast_path && (degree == 0 || bound <= room / maxv / degree);
        const u64 next_bound = all_fit ? bound + bound * degree * maxv : C;
        form_proposals(g, clusters, cw, roles, C, seed, level, round, true, threshold, !all_fit, prop, acc, touched);
        const i64 before = cluster_count;
        if (all_fit) {  // residual_commit_all (singleton_growth.cuh:45-60)
            for (i64 v = 0; v < n; ++v) {
                const int32_t t = prop.target[v];
                if (t == kInvalid) continue;
                clusters[v] = t;
                cw[v] = 0;
                cw[t] += g.vw[v];
            }
        } else {
            const auto order = admission_order(prop.target, prop.regret, prop.tie);
            // inclusive_scan_by_key + sclp_commit_kernel (aggregation.cuh:624-652)
            std::vector<char> accept(order.size(), 0);
            u64 prefix = 0;
            for (size_t i = 0; i < order.size(); ++i) {
                const int32_t v = order[i], t = prop.target[v];
                if (i == 0 || prop.target[order[i - 1]] != t) prefix = 0;
                prefix += g.vw[v];
                const u64 base = cw[t];
                accept[i] = base <= C && prefix <= C - base;
            }
            for (size_t i = 0; i < order.size(); ++i) {
                if (!accept[i]) continue;
                const int32_t v = order[i], t = prop.target[v], s = clusters[v];
                cw[s] -= g.vw[v];
                cw[t] += g.vw[v];
                clusters[v] = t;
            }
        }
        cluster_count = count_clusters();
        if (cluster_count > before) fail(5, "residual singleton merge accounting failed");
        bound = next_bound;
        if (static_cast<double>(cluster_count) <= 0.60 * n) break;
    }
    if (pack_isolated) {  // src/coarsen.cu:1130-1161, aggregation.cuh:713-745
        std::vector<int32_t> iso;
        for (i64 v = 0; v < n; ++v)
            if (g.off[v] == g.off[v + 1]) iso.push_back(static_cast<int32_t>(v));
        if (iso.size() > 1) {
            std::vector<u64> pre(iso.size());
            u64 run = 0;
            for (size_t i = 0; i < iso.size(); ++i) { run += g.vw[iso[i]]; pre[i] = run; }
            std::vector<int32_t> rep(static_cast<size_t>(run / C + (run % C != 0)), INT32_MAX);
            for (size_t i = 0; i < iso.size(); ++i) {
                const u64 fb = (pre[i] - g.vw[iso[i]]) / C, lb = (pre[i] - 1) / C;
                if (fb == lb) rep[fb] = std::min(rep[fb], iso[i]);
            }
            for (size_t i = 0; i < iso.size(); ++i) {
                const int32_t v = iso[i];
                const u64 fb = (pre[i] - g.vw[v]) / C, lb = (pre[i] - 1) / C;
                if (fb != lb) continue;
                const int32_t t = rep[fb];
                if (t == v) continue;
                clusters[v] = t;
                cw[v] = 0;
                cw[t] += g.vw[v];
            }
            cluster_count = count_clusters();
        }
    }
    if (static_cast<double>(cluster_count) > 0.60 * n) {  // two-hop, src/coarsen.cu:1166-1259
        form_proposals(g, clusters, cw, roles, C, seed, level, 4, false, 0, false, prop, acc, touched);
        std::vector<int32_t> fav(static_cast<size_t>(n), kInvalid);
        for (i64 v = 0; v < n; ++v)
            fav[v] = cw[clusters[v]] == static_cast<u64>(g.vw[v]) ? prop.target[v] : kInvalid;
        const auto order = admission_order(fav, prop.gain, prop.tie);
        const size_t count = order.size();
        std::vector<int32_t> flag(count, 0);
        u64 rank = 0, pairs = 0;
        for (size_t i = 0; i < count; ++i) {
            rank = (i == 0 || fav[order[i - 1]] != fav[order[i]]) ? 1 : rank + 1;
            flag[i] = (rank % 2 == 0) && i > 0 && static_cast<u64>(g.vw[order[i - 1]]) <= C - g.vw[order[i]];
            pairs += flag[i];
        }
        const u64 budget = static_cast<u64>(std::max<i64>(0, cluster_count - desired));
        if (std::min(pairs, budget) > 0) {
            u64 position = 0;
            // Decisions read clusters[] of the pair's first element, which no
            // commit of this batch changes (it has an odd rank).
            for (size_t i = 0; i < count; ++i) {
                if (!flag[i]) continue;
                const u64 pos = position++;
                if (pos >= budget) continue;
                const int32_t v = order[i], s = clusters[v], t = clusters[order[i - 1]];
                if (s == t) continue;
                cw[s] -= g.vw[v];
                cw[t] += g.vw[v];
                clusters[v] = t;
            }
        }
        cluster_count = count_clusters();
    }
    // compaction (src/coarsen.cu:1261-1298)
    std::vector<int32_t> ids(static_cast<size_t>(n));
    int32_t next = 0;
    for (i64 c = 0; c < n; ++c) { ids[c] = next; next += cw[c] > 0; }
    out.nc = next;
    out.map.resize(static_cast<size_t>(n));
    out.cvw.assign(static_cast<size_t>(next), 0);
    for (i64 v = 0; v < n; ++v) {
        out.map[v] = ids[clusters[v]];
        out.cvw[out.map[v]] += g.vw[v];  // 32-bit accumulation like the reference
    }
    out.max_w = 0;
    for (u32 w : out.cvw) out.max_w = std::max<u64>(out.max_w, w);
    ws.max_vw = out.max_w;
    if (out.max_w > C) fail(5, "SCLP coarsening exceeded cluster capacity");
    return out;
}

// contract_typed / contract_short_rows (src/coarsen.cu:1394-1673): the exact
// coarse CSR (rows sorted by neighbour, parallel edges summed, intra-cluster
// edges dropped) plus the carried row bounds and degree metadata.
Graph contract(const Graph& fine, const Aggregate& agg, Workspace& ws) {
    const i64 n = fine.n, nc = agg.nc;
    const bool count_raw = ws.positive && n >= 65536 && fine.maximum_degree <= 512;
    std::vector<u64> next(static_cast<size_t>(nc), 0), raw(static_cast<size_t>(nc), 0);
    const bool bounded = n > 0 && ws.maximum_row_weight <= UINT64_MAX / static_cast<u64>(n);
    for (i64 v = 0; v < n; ++v) {
        const int32_t c = agg.map[v];
        raw[c] += static_cast<u64>(fine.deg(v));
        const u64 a = ws.row_bounds[v];
        next[c] = bounded ? next[c] + a : (~0ULL - next[c] < a ? ~0ULL : next[c] + a);
    }
    u64 row_bound = 0, raw_bound = 0;
    for (i64 c = 0; c < nc; ++c) { row_bound = std::max(row_bound, next[c]); raw_bound = std::max(raw_bound, raw[c]); }
    if (!count_raw) raw_bound = UINT64_MAX;
    const u64 degree_bound = count_raw && fine.maximum_degree <= 128 ? raw_bound : row_bound;
    const bool short_rows = count_raw && raw_bound <= 512;
    // Members of every coarse row, then per-row accumulation.
    std::vector<int32_t> start(static_cast<size_t>(nc + 1), 0), members(static_cast<size_t>(n));
    for (i64 v = 0; v < n; ++v) ++start[agg.map[v] + 1];
    for (i64 c = 0; c < nc; ++c) start[c + 1] += start[c];
    {
        std::vector<int32_t> cursor(start.begin(), start.end() - 1);
        for (i64 v = 0; v < n; ++v) members[cursor[agg.map[v]]++] = static_cast<int32_t>(v);
    }
    Graph coarse;
    coarse.n = nc;
    coarse.off.assign(static_cast<size_t>(nc + 1), 0);
    std::vector<u64> acc(static_cast<size_t>(nc), UINT64_MAX);
    std::vector<int32_t> touched;
    for (i64 c = 0; c < nc; ++c) {
        touched.clear();
        for (int32_t i = start[c]; i < start[c + 1]; ++i) {
            const int32_t v = members[i];
            for (i64 e = fine.off[v]; e < fine.off[v + 1]; ++e) {
                const int32_t t = agg.map[fine.nbr[e]];
                if (t == c) continue;
                if (acc[t] == UINT64_MAX) { acc[t] = 0; touched.push_back(t); }
                acc[t] += fine.ew[e];
            }
        }
        std::sort(touched.begin(), touched.end());
        for (int32_t t : touched) {
            coarse.nbr.push_back(t);
            coarse.ew.push_back(static_cast<u32>(acc[t]));  // 32-bit coarse weights
            acc[t] = UINT64_MAX;
        }
        coarse.off[c + 1] = static_cast<int32_t>(coarse.nbr.size());
    }
    coarse.m = static_cast<i64>(coarse.nbr.size());
    coarse.vw = agg.cvw;
    coarse.implicit_unit = false;
    if (short_rows) {
        coarse.incident_weight_bound = row_bound;
        coarse.maximum_degree = degree_bound;
        coarse.has_heavy_rows = degree_bound >= 4096;
    } else {
        coarse.incident_weight_bound = row_bound;
        if (ws.positive) {
            coarse.maximum_degree = degree_bound;
            coarse.has_heavy_rows = degree_bound >= 4096;
        }
    }
    ws.maximum_row_weight = row_bound;
    ws.row_bounds.swap(next);
    return coarse;
}

struct Hierarchy {
    std::vector<Graph> levels;
    std::vector<std::vector<int32_t>> maps;
};

// coarsen_impl (src/coarsen.cu:1762-2060).
Hierarchy coarsen(Graph input, const Options& o) {
    Hierarchy h;
    Workspace ws;
    if (input.n > 0) level0_metadata(input, ws);
    const i64 cutoff = std::max<i64>(32, static_cast<i64>(o.cluster_size_factor) * o.parts);
    Graph current = std::move(input);
    for (int level = 0; level < o.max_levels && current.n > cutoff; ++level) {
        const u32 level_seed = o.seed + static_cast<u32>(level);
        int factor = o.cluster_size_factor;
        if (o.progressive) {
            const i64 fine = std::max(o.fine_factor, (512 + o.parts - 1) / o.parts);
            const i64 denom = static_cast<i64>(o.growth) * o.parts;
            const i64 remaining = (current.n + denom - 1) / denom;
            factor = static_cast<int>(std::max<i64>(factor, std::min<i64>(fine, remaining)));
        }
        const i64 avg = current.m / current.n;
        const bool matching = o.seed_matching && current.n >= 65536 && !current.has_heavy_rows &&
                              (avg < 8 || current.maximum_degree <= 256) && avg < o.heavy_limit &&
                              ws.sorted_unique && ws.positive;
        Aggregate agg = aggregate(current, ws, o.parts, level_seed, level, factor, o.pack_isolated, matching, o.fast_path);
        current.has_heavy_rows = agg.stats_heavy;
        current.maximum_degree = agg.stats_max_degree;
        const double ratio = static_cast<double>(agg.nc) / static_cast<double>(current.n);
        if (agg.nc >= current.n || ratio > o.stop_ratio) break;
        Graph coarse = contract(current, agg, ws);
        h.levels.push_back(std::move(current));
        h.maps.push_back(std::move(agg.map));
        current = std::move(coarse);
        ws.sorted_unique = true;
    }
    h.levels.push_back(std::move(current));
    return h;
}

// initial_partition_metis (src/initial_partition_metis.cu:86-183), production
// mode (require_feasible = false).
std::vector<int32_t> initial_partition(const Graph& g, int parts, double eps, u32 seed) {
    const i64 n = g.n;
    if (n <= 0 || parts < 2 || parts > kMaxParts || parts > n || !std::isfinite(eps) || eps < 1.0)
        fail(1, "invalid METIS initialization options");
    u64 total = 0, edge_total = 0;
    for (u32 w : g.vw) total += w;
    for (u32 w : g.ew) edge_total += w;
    const u64 capacity = partition_capacity(total, parts, eps);
    u64 vg = 0, eg = 0;
    for (u32 w : g.vw) {
        if (!w) fail(1, "METIS requires positive vertex weights");
        if (w > capacity) fail(1, "a vertex exceeds partition capacity");
        vg = std::gcd(vg, static_cast<u64>(w));
    }
    for (u32 w : g.ew) eg = std::gcd(eg, static_cast<u64>(w));
    if (!eg) eg = 1;
    const u64 limit = static_cast<u64>(INT64_MAX);
    if (total / vg > limit || edge_total / eg > limit) fail(1, "weighted coarse graph exceeds METIS signed weight range");
    std::vector<idx_t> xadj(static_cast<size_t>(n + 1), 0), adj, adjw, vwgt(static_cast<size_t>(n));
    for (i64 v = 0; v < n; ++v) {
        vwgt[v] = static_cast<idx_t>(g.vw[v] / vg);
        for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
            if (g.nbr[e] == v || !g.ew[e]) continue;
            adj.push_back(g.nbr[e]);
            adjw.push_back(static_cast<idx_t>(g.ew[e] / eg));
        }
        xadj[v + 1] = static_cast<idx_t>(adj.size());
    }
    idx_t nn = n, ncon = 1, k = parts, obj = 0;
    std::vector<idx_t> part(static_cast<size_t>(n));
    idx_t options[kMetisOptions];
    if (METIS_SetDefaultOptions(options) != kMetisOk) fail(5, "METIS_SetDefaultOptions failed");
    options[kMetisSeed] = static_cast<idx_t>(seed & 0x7fffffffU);
    options[kMetisNumbering] = 0;
    real_t upper = static_cast<real_t>(eps);
    if (upper <= 1.0f) upper = std::nextafter(1.0f, INFINITY);
    if (adj.empty()) { adj.push_back(0); adjw.push_back(0); }  // METIS reads a valid pointer
    const int status = METIS_PartGraphKway(&nn, &ncon, xadj.data(), adj.data(), vwgt.data(), nullptr,
                                           adjw.data(), &k, nullptr, &upper, options, &obj, part.data());
    if (status != kMetisOk) fail(5, "METIS_PartGraphKway failed: " + std::to_string(status));
    std::vector<int32_t> labels(static_cast<size_t>(n));
    for (i64 v = 0; v < n; ++v) {
        if (part[v] < 0 || part[v] >= parts) fail(5, "METIS returned an invalid partition label");
        labels[v] = static_cast<int32_t>(part[v]);
    }
    return labels;
}

// ---------------------------------------------------------------- refinement

u64 cut_of(const Graph& g, const std::vector<int32_t>& labels) {  // refine_cut_kernel
    u64 d = 0;
    for (i64 v = 0; v < g.n; ++v)
        for (i64 e = g.off[v]; e < g.off[v + 1]; ++e)
            if (labels[v] != labels[g.nbr[e]]) d += g.ew[e];
    if (d & 1ULL) fail(5, "refinement cut is not symmetric");
    return d / 2;
}

// Deterministic gain bucket: the smallest j with 1.5^j >= x, evaluated
// exactly in integers (balance_gain_bucket, incremental.cuh:553-557, computes
// ceil(log(x)/log(1.5)) in floating point; the two agree except where x is an
// exact power of 1.5, where floating point may land on either side).
int gain_bucket(u64 best_conn, u64 current, u64 relief) {
    if (best_conn > current) return 0;
    if (best_conn == current) return 1;
    const unsigned __int128 G = current - best_conn, R = relief;  // x = G / R
    // j in [-23, 24]: 1.5^j >= G/R  <=>  3^j R >= 2^j G  (j >= 0)
    //                               <=>  2^-j R >= 3^-j G (j < 0)
    for (int j = -23; j <= 24; ++j) {
        unsigned __int128 lhs = R, rhs = G;
        if (j >= 0) {
            for (int i = 0; i < j; ++i) { lhs *= 3; rhs *= 2; }
        } else {
            for (int i = 0; i < -j; ++i) { lhs *= 2; rhs *= 3; }
        }
        if (lhs >= rhs) return std::max(2, std::min(49, 25 + j));
    }
    return 49;
}

// Order key of the deterministic repair (bucket ranks and receiver tickets).
inline u32 repair_hash(int32_t v) { return mix32(static_cast<u32>(v) ^ 0x85ebca6bU); }

struct JointMove {  // exchange.cuh:9-13
    int vertices[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
    int size = 0, a = -1, b = -1, id = 0;
    i64 gain = 0, net = 0;
};

struct Refiner {
    const Graph& g;
    int k;
    u64 C;
    std::vector<int32_t>& labels;
    std::vector<u64> loads;
    i64 n;
    std::vector<u64> A, totals;  // dense affinity n*k and row totals
    std::vector<int32_t> targets, locks, flags;
    std::vector<i64> gains;
    std::vector<double> prices;
    bool priced = false;
    struct Sample { i64 loss = 0; u64 weight = 0; };
    std::vector<Sample> samples;
    u64 cut = 0;
    u64 revision = 0;
    orc_refine_stats stats{};  // RefineStats (include/refine.hpp:28-53)

    Refiner(const Graph& graph, int parts, std::vector<int32_t>& lab, std::vector<u64> ld, u64 capacity)
        : g(graph), k(parts), C(capacity), labels(lab), loads(std::move(ld)), n(graph.n) {}

    u64 max_load() const { return *std::max_element(loads.begin(), loads.end()); }

    // incremental_build_affinity (incremental.cuh:61-140), dense layout.
    void build() {
        A.assign(static_cast<size_t>(n * k), 0);
        totals.assign(static_cast<size_t>(n), 0);
        for (i64 v = 0; v < n; ++v)
            for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
                const int32_t u = g.nbr[e];
                if (u == v) continue;
                A[v * k + labels[u]] += g.ew[e];
                totals[v] += g.ew[e];
            }
    }
    u64 a(i64 v, int p) const { return A[static_cast<size_t>(v * k + p)]; }

    // estimated_repair_cost (incremental.cuh:156-160); slack wraps for
    // overloaded parts exactly like the reference's unsigned arithmetic.
    double cost(int p, u64 w) const {
        const u64 slack = C - loads[p];
        return w > slack ? prices[p] * static_cast<double>(w - slack) : 0.0;
    }

    // incremental_update_cache_and_cut + incremental_commit
    // (incremental.cuh:440-547) for one batch; returns the cut decrease.
    i64 apply(const std::vector<int32_t>& movers, bool lp, bool sample) {
        i64 delta = 0;
        for (int32_t v : movers) {
            const int32_t s = labels[v], t = targets[v];
            i64 gv = 0;
            for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
                const int32_t u = g.nbr[e];
                if (u == v) continue;
                const int32_t old = labels[u];
                const bool moves = flags[u] != 0;
                const int32_t nw = moves ? targets[u] : old;
                const u64 w = g.ew[e];
                A[static_cast<size_t>(u) * k + s] -= w;
                A[static_cast<size_t>(u) * k + t] += w;
                if (!moves || u > v) gv += static_cast<i64>(w) * ((s != old) - (t != nw));
            }
            delta += gv;
            if (sample) { samples[s].loss += -gv; samples[s].weight += g.vw[v]; }
        }
        for (int32_t v : movers) {
            const int32_t s = labels[v], t = targets[v];
            loads[s] -= g.vw[v];
            loads[t] += g.vw[v];
            labels[v] = t;
            if (lp) locks[v] = 1;
        }
        if (delta >= 0) {
            if (static_cast<u64>(delta) > cut) fail(5, "incremental cut underflow");
            cut -= static_cast<u64>(delta);
        } else cut += static_cast<u64>(-delta);
        return delta;
    }

    // enumerate_repair_destination (rebalance_select.cuh:9-75), dense layout,
    // with the slack CDF of initialize_receiver_slack (:79-104).
    int repair_destination(i64 v, int src, u64 w, const std::vector<u64>& cdf, u64& conn, u64& current) const {
        current = a(v, src);
        conn = 0;
        int part = -1;
        u64 best_slack = 0;
        if (current != totals[v]) {
            for (int p = 0; p < k; ++p) {
                if (p == src || loads[p] >= C || w > C - loads[p]) continue;
                const u64 value = a(v, p), slack = C - loads[p];
                if (part < 0 || value > conn || (value == conn && slack > best_slack)) { part = p; conn = value; best_slack = slack; }
            }
            if (conn) return part;
            part = -1;
            conn = 0;
        }
        const u32 hash = mix32(static_cast<u32>(v));
        if (loads[src] >= C && w <= cdf[k]) {
            const u64 total = cdf[k - 1];
            if (!total) return -1;
            const u64 ticket = static_cast<u64>(hash) % total;
            int lo = 0, hi = k;
            while (lo < hi) { const int mid = (lo + hi) / 2; if (cdf[mid] <= ticket) lo = mid + 1; else hi = mid; }
            return lo;
        }
        u64 total = 0;
        for (int p = 0; p < k; ++p)
            if (p != src && loads[p] < C && w <= C - loads[p]) { const u64 s = C - loads[p]; total = UINT64_MAX - total < s ? UINT64_MAX : total + s; }
        if (!total) return -1;
        u64 ticket = static_cast<u64>(hash) % total;
        for (int p = 0; p < k; ++p)
            if (p != src && loads[p] < C && w <= C - loads[p]) {
                const u64 s = C - loads[p];
                if (ticket < s) return p;
                ticket -= s;
            }
        return -1;
    }

    // One capacity repair (RebalanceGraph, rebalance_graph.cuh:160-280) in
    // the deterministic order: ranks within a bucket and receiver tickets
    // follow the (hash, id) repair order.  Returns feasibility.
    int repairs = 0;
    bool repair(u64* gain_sum = nullptr) {
        if (max_load() <= C) return true;
        ++repairs;
        constexpr int W = 800;
        int iterations = 0;
        std::vector<u64> counts(static_cast<size_t>(k) * W), prefix(counts.size()), slack(static_cast<size_t>(k)),
            requests(static_cast<size_t>(k)), cdf(static_cast<size_t>(k) + 1), ranks(static_cast<size_t>(n));
        std::vector<int32_t> ids(static_cast<size_t>(n));
        // Deterministic repair order: (hash, id).  Ranks inside a bucket and
        // receiver tickets follow it; a hashed order spreads donors over the
        // part the way the reference's atomic arrival order does.
        std::vector<int32_t> order(static_cast<size_t>(n));
        std::iota(order.begin(), order.end(), 0);
        std::sort(order.begin(), order.end(), [](int32_t x, int32_t y) {
            const u32 hx = repair_hash(x), hy = repair_hash(y);
            return hx != hy ? hx < hy : x < y;
        });
        while (true) {
            std::fill(flags.begin(), flags.end(), 0);
            std::fill(counts.begin(), counts.end(), 0);
            u64 carry = 0, minimum = UINT64_MAX;
            for (int p = 0; p < k; ++p) {
                slack[p] = loads[p] < C ? C - loads[p] : 0;
                requests[p] = 0;
                if (slack[p]) minimum = std::min(minimum, slack[p]);
                carry = UINT64_MAX - carry < slack[p] ? UINT64_MAX : carry + slack[p];
                cdf[p] = carry;
            }
            cdf[k] = minimum;
            std::vector<int32_t> donors;
            for (i64 oi = 0; oi < n; ++oi) {
                const i64 v = order[oi];
                const int src = labels[v];
                if (loads[src] <= C) continue;
                const u64 w = g.vw[v];
                targets[v] = -1;
                ids[v] = -1;
                u64 conn = 0, current = 0;
                const int best = repair_destination(v, src, w, cdf, conn, current);
                if (best < 0) continue;
                const u64 excess = loads[src] - C;
                const u64 relief = w < excess ? w : excess;
                const int bucket = src * W + gain_bucket(conn, current, relief) * 16 + static_cast<int>(mix32(static_cast<u32>(v)) % 16);
                targets[v] = best;
                ids[v] = bucket;
                ranks[v] = counts[bucket];
                counts[bucket] += w;
                donors.push_back(static_cast<int32_t>(v));
            }
            for (int p = 0; p < k; ++p) {  // balance_scan_buckets
                u64 run = 0;
                for (int b = 0; b < W; ++b) { prefix[p * W + b] = run; run += counts[p * W + b]; }
            }
            // reserve_receiver_prefixes (:86-156), synchronous attempts.
            std::vector<int32_t> active;
            for (int32_t v : donors) {
                const int b = ids[v];
                if (prefix[b] + ranks[v] < loads[b / W] - C) active.push_back(v);
            }
            std::vector<std::vector<uint64_t>> tried(static_cast<size_t>(active.size()), std::vector<uint64_t>(2, 0));
            std::vector<int> want(active.size(), -1);
            std::vector<char> done(active.size(), 0), dead(active.size(), 0);
            for (int attempt = 0; attempt < k; ++attempt) {
                bool any = false;
                for (size_t i = 0; i < active.size(); ++i) {
                    want[i] = -1;
                    if (done[i] || dead[i]) continue;
                    const int32_t v = active[i];
                    const u64 w = g.vw[v];
                    int target = -1;
                    if (!attempt) target = targets[v];
                    else {
                        u64 best = 0, room = 0;
                        for (int p = 0; p < k; ++p) {
                            if (p == labels[v] || (tried[i][p / 64] >> (p & 63) & 1)) continue;
                            const u64 avail = requests[p] < slack[p] ? slack[p] - requests[p] : 0;
                            if (avail < w) continue;
                            const u64 c = a(v, p);
                            if (target < 0 || c > best || (c == best && avail > room)) { target = p; best = c; room = avail; }
                        }
                    }
                    if (target < 0) { dead[i] = 1; continue; }
                    want[i] = target;
                    any = true;
                }
                if (!any) break;
                for (size_t i = 0; i < active.size(); ++i) {  // repair order
                    const int t = want[i];
                    if (t < 0) continue;
                    tried[i][t / 64] |= 1ULL << (t & 63);
                    const u64 w = g.vw[active[i]];
                    const u64 begin = requests[t];
                    requests[t] += w;
                    if (begin <= slack[t] && w <= slack[t] - begin) {
                        targets[active[i]] = t;
                        flags[active[i]] = 1;
                        done[i] = 1;
                    }
                }
            }
            std::vector<int32_t> movers;
            for (size_t i = 0; i < active.size(); ++i)
                if (done[i]) movers.push_back(active[i]);
            for (size_t i = 0; i < active.size(); ++i)
                if (!done[i]) targets[active[i]] = -1;
            i64 delta = 0;
            if (!movers.empty()) {
                delta = apply(movers, false, priced);
                ++revision;
                stats.accepted += movers.size();
                if (delta >= 0) stats.rebalance_cut_gain += static_cast<u64>(delta);
                else stats.rebalance_cut_loss += static_cast<u64>(-delta);
            }
            if (gain_sum && delta > 0) *gain_sum += static_cast<u64>(delta);
            ++iterations;
            ++stats.admission_iterations;
            for (int32_t v : movers) flags[v] = 0;
            const bool feasible = max_load() <= C;
            if (feasible || movers.empty() || iterations >= 2 * k + 4) return feasible;
        }
    }

    // LP round (incremental.cuh:166-198, 361-393 and the loop of :911-961 /
    // lp_graph.cuh:57-92).  Returns the number of movers.
    i64 lp_round(double filter) {
        for (i64 v = 0; v < n; ++v) {
            targets[v] = -1;
            gains[v] = INT64_MIN;
            flags[v] = 0;
            if (locks[v]) { locks[v] = 0; continue; }
            const int src = labels[v];
            const u64 current = a(v, src);
            if (current == totals[v]) continue;
            u64 best = 0;
            int target = -1;
            double best_score = -DBL_MAX;
            for (int p = 0; p < k; ++p) {
                const u64 conn = a(v, p);
                if (p == src || !conn) continue;
                if (priced) {
                    const double score = static_cast<double>(conn) - cost(p, g.vw[v]);
                    if (target < 0 || score > best_score) { best_score = score; best = conn; target = p; }
                } else if (target < 0 || conn > best) { best = conn; target = p; }
            }
            if (target >= 0 && (best >= current || current - best < static_cast<u64>(filter * static_cast<double>(current)))) {
                targets[v] = target;
                gains[v] = best >= current ? static_cast<i64>(best - current) : -static_cast<i64>(current - best);
            }
        }
        std::vector<int32_t> movers;
        for (i64 v = 0; v < n; ++v) {
            if (targets[v] < 0) continue;
            const int s = labels[v], t = targets[v];
            const i64 gain = gains[v];
            i64 corr = 0;
            for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
                const int32_t u = g.nbr[e];
                if (u == v || targets[u] < 0 || !(gains[u] > gain || (gains[u] == gain && u < v))) continue;
                corr += static_cast<i64>(g.ew[e]) * ((targets[u] == t) - (targets[u] == s) - (labels[u] == t) + (labels[u] == s));
            }
            bool keep;
            if (priced) {
                const u64 w = g.vw[v];
                const double adjustment = cost(s, w) - cost(t, w);
                keep = static_cast<double>(gain + corr) + adjustment >= 0;
            } else keep = gain + corr >= 0;
            if (keep) movers.push_back(static_cast<int32_t>(v));
        }
        for (int32_t v : movers) flags[v] = 1;
        stats.proposals += movers.size();
        if (!movers.empty()) {
            const i64 delta = apply(movers, true, false);
            ++revision;
            stats.accepted += movers.size();
            if (delta >= 0) stats.lp_cut_gain += static_cast<u64>(delta);
            else stats.lp_cut_loss += static_cast<u64>(-delta);
        }
        for (int32_t v : movers) flags[v] = 0;
        return static_cast<i64>(movers.size());
    }

    // capacity-complementary exchange (incremental.cuh:974-1041,
    // exchange.cuh, complementary_moves.cuh).
    void exchange(int rounds, u64& best_cut) {
        const int sw = std::min(128, std::max(32, 4096 / k));
        const int slots = k * sw * 2;
        std::vector<u64> quotient(static_cast<size_t>(k) * k, 0);
        std::vector<int> visits(static_cast<size_t>(k) * k, 0), partner(static_cast<size_t>(k));
        for (i64 v = 0; v < n; ++v) {  // joint_quotient
            const int pa = labels[v];
            for (int b = 0; b < k; ++b) if (pa < b && a(v, b)) quotient[pa * k + b] += a(v, b);
        }
        auto gap = [](i64 net, i64 lo, i64 hi) -> i64 { return net < lo ? lo - net : net > hi ? net - hi : 0; };
        int empty = 0;
        for (int pass = 0; pass < rounds; ++pass) {
            // joint_match (exchange.cuh:55-82)
            std::fill(partner.begin(), partner.end(), -1);
            for (int round = 0; round < k / 2; ++round) {
                std::vector<int> choice(static_cast<size_t>(k), -1);
                for (int p = 0; p < k; ++p) {
                    if (partner[p] >= 0) continue;
                    int best = -1;
                    double score = -1;
                    for (int q = 0; q < k; ++q) {
                        if (q == p || partner[q] >= 0) continue;
                        const int pair = std::min(p, q) * k + std::max(p, q);
                        if (!quotient[pair]) continue;
                        const double penalty = 1.0 + visits[pair];
                        const double value = static_cast<double>(quotient[pair]) / (penalty * penalty);
                        if (value > score || (value == score && q < best)) { score = value; best = q; }
                    }
                    choice[p] = best;
                }
                int progress = 0;
                std::vector<int> next = partner;
                for (int p = 0; p < k; ++p) {
                    if (partner[p] >= 0) continue;
                    const int best = choice[p];
                    if (best >= 0 && choice[best] == p) {
                        next[p] = best;
                        if (p < best) { ++visits[p * k + best]; ++progress; }
                    }
                }
                partner = next;
                if (!progress) break;
            }
            // joint_seeds (:83-93)
            std::vector<u64> seeds(static_cast<size_t>(k) * sw, UINT64_MAX);
            for (i64 v = 0; v < n; ++v) {
                const int p = labels[v], q = partner[p];
                if (q < 0 || !a(v, q)) continue;
                const u32 h = mix32(static_cast<u32>(v) ^ mix32(static_cast<u32>(pass + 17)));
                u64& slot = seeds[static_cast<size_t>(p) * sw + h % sw];
                slot = std::min(slot, (static_cast<u64>(h) << 32) | static_cast<u32>(v));
            }
            std::vector<JointMove> moves(static_cast<size_t>(slots)), archive(static_cast<size_t>(slots) * 4);
            for (int slot = 0; slot < slots; ++slot) grow(slot, sw, seeds, partner, moves[slot], &archive[static_cast<size_t>(slot) * 4], gap);
            // remove_if empty, sort by JointNetOrder, unique by canonical set
            std::vector<JointMove> frag;
            for (const auto& x : archive) if (x.size) frag.push_back(x);
            std::sort(frag.begin(), frag.end(), [](const JointMove& x, const JointMove& y) {
                if (x.a != y.a) return x.a < y.a;
                if (x.net != y.net) return x.net < y.net;
                if (x.gain != y.gain) return x.gain > y.gain;
                if (x.size != y.size) return x.size < y.size;
                for (int j = 0; j < x.size; ++j) if (x.vertices[j] != y.vertices[j]) return x.vertices[j] < y.vertices[j];
                return x.id < y.id;
            });
            {
                std::vector<JointMove> u;
                for (size_t i = 0; i < frag.size(); ++i)
                    if (i == 0 || !same(frag[i - 1], frag[i])) u.push_back(frag[i]);
                frag.swap(u);
            }
            const int fragments = static_cast<int>(frag.size());
            std::vector<JointMove> pool(moves);
            pool.resize(static_cast<size_t>(slots + 2 * fragments));
            for (int i = 0; i < fragments; ++i) combine(frag, i, slots, &pool[static_cast<size_t>(slots)], gap);
            std::vector<JointMove> act;
            for (const auto& x : pool) if (x.size) act.push_back(x);
            if (act.empty()) { if (++empty >= 2) break; continue; }
            std::sort(act.begin(), act.end(), [](const JointMove& x, const JointMove& y) {
                if (x.a != y.a) return x.a < y.a;
                if (x.gain != y.gain) return x.gain > y.gain;
                return x.id < y.id;
            });
            const int count = static_cast<int>(act.size());
            std::vector<int> owners(static_cast<size_t>(n), INT_MAX);
            for (int i = 0; i < count; ++i) for (int j = 0; j < act[i].size; ++j) owners[act[i].vertices[j]] = std::min(owners[act[i].vertices[j]], i);
            for (int i = 0; i < count; ++i) for (int j = 0; j < act[i].size; ++j) if (owners[act[i].vertices[j]] != i) { act[i].size = 0; break; }
            std::fill(owners.begin(), owners.end(), INT_MAX);
            for (int i = 0; i < count; ++i)
                for (int j = 0; j < act[i].size; ++j) {
                    const int v = act[i].vertices[j];
                    owners[v] = i;
                    targets[v] = labels[v] == act[i].a ? act[i].b : act[i].a;
                }
            std::vector<u64> events(static_cast<size_t>(count), 0);  // joint_events (:227-262)
            for (int i = 0; i < count; ++i) {
                if (!act[i].size) continue;
                for (int j = 0; j < act[i].size; ++j) {
                    const int v = act[i].vertices[j];
                    for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
                        const int u = g.nbr[e], other = owners[u];
                        if (u == v || (other != INT_MAX && v > u)) continue;
                        if (other != INT_MAX && labels[u] != act[i].a && labels[u] != act[i].b) continue;
                        const i64 w = g.ew[e];
                        const int before = labels[v] != labels[u];
                        if (other == i || other == INT_MAX) {
                            const int after = targets[v] != (other == i ? targets[u] : labels[u]);
                            events[i] += static_cast<u64>((before - after) * w);
                        } else {
                            const int middle = i < other ? targets[v] != labels[u] : labels[v] != targets[u];
                            const int after = targets[v] != targets[u];
                            const u64 first = static_cast<u64>((before - middle) * w), last = static_cast<u64>((middle - after) * w);
                            events[i] += i < other ? first : last;
                            events[other] += i < other ? last : first;
                        }
                    }
                }
            }
            std::vector<int> stops(static_cast<size_t>(k), -1);  // joint_prefix (:263-284)
            for (int pa = 0; pa < k; ++pa) {
                i64 gsum = 0, net = 0, best = 0;
                int stop = -1;
                for (int i = 0; i < count; ++i) {
                    if (act[i].a != pa || !act[i].size) continue;
                    gsum += static_cast<i64>(events[i]);
                    net += act[i].net;
                    const i64 lo = static_cast<i64>(loads[pa]) - static_cast<i64>(C);
                    const i64 hi = static_cast<i64>(C) - static_cast<i64>(loads[act[i].b]);
                    if (!gap(net, lo, hi) && gsum > best) { best = gsum; stop = i; }
                }
                stops[pa] = stop;
            }
            std::fill(flags.begin(), flags.end(), 0);
            for (int i = 0; i < count; ++i)
                if (act[i].size && i <= stops[act[i].a])
                    for (int j = 0; j < act[i].size; ++j) flags[act[i].vertices[j]] = 1;
            std::vector<int32_t> movers;
            for (i64 v = 0; v < n; ++v) if (flags[v]) movers.push_back(static_cast<int32_t>(v));
            if (movers.empty()) { if (++empty >= 2) break; continue; }
            empty = 0;
            const i64 delta = apply(movers, false, false);
            ++revision;
            for (int32_t v : movers) flags[v] = 0;
            if (delta <= 0) fail(5, "non-improving boundary group batch");
            if (max_load() > C || cut >= best_cut) fail(5, "capacity exchange violated cut/capacity");
            best_cut = cut;
            stats.group_cut_gain += static_cast<u64>(delta);
            stats.group_accepted += movers.size();
        }
    }

    static bool same(const JointMove& x, const JointMove& y) {  // joint_same_move
        if (!x.size || x.size != y.size || x.a != y.a || x.b != y.b || x.gain != y.gain || x.net != y.net) return false;
        for (int j = 0; j < x.size; ++j) {
            bool found = false;
            for (int t = 0; t < y.size; ++t) found |= x.vertices[j] == y.vertices[t];
            if (!found) return false;
        }
        return true;
    }

    // joint_grow (exchange.cuh:95-204), one slot.
    template <class Gap>
    void grow(int slot, int sw, const std::vector<u64>& seeds, const std::vector<int>& partner, JointMove& out,
              JointMove* arch, Gap gap) const {
        const int policy = slot % 2;
        JointMove best;
        best.id = slot;
        out = best;
        for (int j = 0; j < 4; ++j) arch[j] = JointMove{};
        const u64 enc = seeds[static_cast<size_t>(slot / 2)];
        if (enc == UINT64_MAX) return;
        const int root = static_cast<int>(static_cast<u32>(enc)), source = labels[root], target = partner[source];
        if (target < 0) return;
        int members[8] = {root, -1, -1, -1, -1, -1, -1, -1};
        int size = 1, counts[2] = {1, 0};
        i64 net = g.vw[root];
        const i64 lo = static_cast<i64>(loads[source]) - static_cast<i64>(C);
        const i64 hi = static_cast<i64>(C) - static_cast<i64>(loads[target]);
        i64 gain = static_cast<i64>(a(root, target)) - static_cast<i64>(a(root, source));
        for (int step = 0; step < 8; ++step) {
            if (gain > 0 && size <= 4) {
                JointMove st;
                st.size = size;
                st.a = std::min(source, target);
                st.b = std::max(source, target);
                st.gain = gain;
                st.net = source == st.a ? net : -net;
                st.id = slot * 4 + step;
                for (int j = 0; j < size; ++j) {
                    int pos = j;
                    while (pos && st.vertices[pos - 1] > members[j]) { st.vertices[pos] = st.vertices[pos - 1]; --pos; }
                    st.vertices[pos] = members[j];
                }
                arch[step] = st;
            }
            if (gain > best.gain && !gap(net, lo, hi)) {
                best.size = size;
                best.a = std::min(source, target);
                best.b = std::max(source, target);
                best.gain = gain;
                best.net = source == best.a ? net : -net;
                for (int j = 0; j < size; ++j) best.vertices[j] = members[j];
            }
            if (size == 8) break;
            const bool gap_first = policy == 0 && gap(net, lo, hi);
            i64 cg = LLONG_MIN, cgap = LLONG_MAX;
            int chosen = INT_MAX;
            for (int origin = -1; origin < size; ++origin) {
                const bool reverse = origin < 0;
                if (reverse && counts[1]) continue;
                const int m = reverse ? -1 : members[origin];
                const i64 begin = reverse ? 0 : g.off[m];
                const i64 end = reverse ? sw : std::min<i64>(g.off[m + 1], begin + 128);
                for (i64 e = begin; e < end; ++e) {
                    int u;
                    if (reverse) {
                        const u64 value = seeds[static_cast<size_t>(target) * sw + e];
                        if (value == UINT64_MAX) continue;
                        u = static_cast<int>(static_cast<u32>(value));
                    } else u = g.nbr[e];
                    const int p = labels[u];
                    if (p != source && p != target) continue;
                    const int side = p == source ? 0 : 1;
                    if (counts[side] >= 4) continue;
                    if (!reverse && p != labels[m]) continue;
                    bool dup = false;
                    for (int j = 0; j < size; ++j) dup |= u == members[j];
                    if (dup || g.deg(u) > 1024) continue;
                    const i64 cnet = net + (side ? -static_cast<i64>(g.vw[u]) : static_cast<i64>(g.vw[u]));
                    const i64 gp = gap(cnet, lo, hi);
                    if (net > hi && !side) continue;
                    if (net < lo && side) continue;
                    i64 marginal = static_cast<i64>(a(u, side ? source : target)) - static_cast<i64>(a(u, p));
                    if (!reverse) marginal += 2LL * g.ew[e];
                    const bool better = gap_first
                        ? (gp < cgap || (gp == cgap && (marginal > cg || (marginal == cg && u < chosen))))
                        : (marginal > cg || (marginal == cg && (gp < cgap || (gp == cgap && u < chosen))));
                    if (better) { chosen = u; cg = marginal; cgap = gp; }
                }
            }
            if (chosen == INT_MAX) break;
            const int side = labels[chosen] == source ? 0 : 1;
            i64 correction = 0;
            for (i64 e = g.off[chosen]; e < g.off[chosen + 1]; ++e)
                for (int j = 0; j < size; ++j)
                    if (g.nbr[e] == members[j]) correction += (labels[members[j]] == labels[chosen] ? 2LL : -2LL) * g.ew[e];
            const i64 cgain = static_cast<i64>(a(chosen, side ? source : target)) - static_cast<i64>(a(chosen, labels[chosen])) + correction;
            members[size++] = chosen;
            ++counts[side];
            gain += cgain;
            net += side ? -static_cast<i64>(g.vw[chosen]) : static_cast<i64>(g.vw[chosen]);
        }
        out = best;
    }

    // joint_combine (complementary_moves.cuh:31-75), fragment i.
    template <class Gap>
    void combine(const std::vector<JointMove>& arch, int i, int id_base, JointMove* out, Gap gap) const {
        const int count = static_cast<int>(arch.size());
        const JointMove x = arch[i];
        const i64 lo = static_cast<i64>(loads[x.a]) - static_cast<i64>(C);
        const i64 hi = static_cast<i64>(C) - static_cast<i64>(loads[x.b]);
        out[i] = x;
        out[i].id = id_base + i;
        if (gap(x.net, lo, hi)) out[i].size = 0;
        out[count + i] = JointMove{};
        auto bound = [&](i64 net, bool upper) {
            int l = 0, h = count;
            while (l < h) {
                const int mid = (l + h) / 2;
                const auto& y = arch[mid];
                if (y.a < x.a || (y.a == x.a && (y.net < net || (upper && y.net == net)))) l = mid + 1;
                else h = mid;
            }
            return l;
        };
        const int begin = bound(lo - x.net, false), end = bound(hi - x.net, true);
        i64 best_gain = 0;
        int best = -1, previous = -1;
        for (int r = 0; r < 4 && begin < end; ++r) {
            const int j = begin + static_cast<int>((static_cast<i64>(end - begin - 1) * r) / 3);
            if (j == previous) continue;
            previous = j;
            if (j == i) continue;
            const JointMove& y = arch[j];
            if (y.a != x.a || y.b != x.b || x.size + y.size > 8) continue;
            bool overlap = false;
            for (int u = 0; u < x.size; ++u) for (int v = 0; v < y.size; ++v) overlap |= x.vertices[u] == y.vertices[v];
            if (overlap) continue;
            i64 correction = 0;
            for (int u = 0; u < x.size; ++u) {
                const int v = x.vertices[u];
                for (i64 e = g.off[v]; e < g.off[v + 1]; ++e)
                    for (int t = 0; t < y.size; ++t)
                        if (g.nbr[e] == y.vertices[t]) correction += (labels[v] == labels[g.nbr[e]] ? 2LL : -2LL) * g.ew[e];
            }
            const i64 gain = x.gain + y.gain + correction;
            if (gain > best_gain || (gain == best_gain && gain > 0 && j < best)) { best_gain = gain; best = j; }
        }
        if (best >= 0) {
            JointMove r = x;
            const JointMove& y = arch[best];
            for (int j = 0; j < y.size; ++j) r.vertices[r.size++] = y.vertices[j];
            r.gain = best_gain;
            r.net += y.net;
            r.id = id_base + count + i;
            out[count + i] = r;
        }
    }
};

struct LevelResult { u64 cut = 0; bool refined = false; bool repair_failed = false; orc_refine_stats stats{}; };

// run_incremental_refinement_typed (incremental.cuh:660-1051); `rounds` and
// `exchange_rounds` are RefineOptions::max_rounds and exchange_rounds (the
// pipeline passes 32 and 2, app/partition_main.cu:111-118, refine.hpp:18).
LevelResult refine_level(const Graph& g, int k, double eps, std::vector<int32_t>& labels, std::vector<u64>& loads,
                         bool has_known, u64 known, int rounds = 32, int exchange_rounds = 2) {
    u64 total = 0;
    for (u64 w : loads) total += w;
    const u64 C = partition_capacity(total, k, eps);
    Refiner r(g, k, labels, loads, C);
    const i64 n = g.n;
    r.targets.assign(static_cast<size_t>(n), -1);
    r.locks.assign(static_cast<size_t>(n), 0);
    r.flags.assign(static_cast<size_t>(n), 0);
    r.gains.assign(static_cast<size_t>(n), INT64_MIN);
    r.prices.assign(static_cast<size_t>(k), 0.0);
    r.samples.assign(static_cast<size_t>(k), {});
    r.priced = total > static_cast<u64>(n);
    r.build();
    r.cut = has_known ? known : cut_of(g, labels);
    r.stats.initial_cut = r.cut;
    r.stats.capacity = C;
    LevelResult res;
    if (r.max_load() > C) {
        if (!r.repair()) {
            res.cut = r.cut;
            res.repair_failed = true;
            loads = r.loads;
            r.stats.final_cut = r.cut;
            r.stats.final_max_part_weight = r.max_load();
            res.stats = r.stats;
            return res;
        }
    }
    const u64 feasible_start = r.cut;
    u64 best = r.cut;
    std::vector<int32_t> saved_labels(labels);
    std::vector<u64> saved_loads(r.loads);
    u64 best_revision = r.revision;
    u32 max_edge = 0;
    for (u32 w : g.ew) max_edge = std::max(max_edge, w);
    const double filter = max_edge <= 1 ? 0.25 : 0.75;
    int stale = 0, empty = 0;
    for (int phase = 0; phase < rounds && stale < 3; ++phase) {
        r.stats.rounds = phase + 1;
        std::fill(r.samples.begin(), r.samples.end(), Refiner::Sample{});
        const i64 count = r.lp_round(filter);
        if (!count) { if (++empty >= 2) break; ++stale; continue; }
        empty = 0;
        if (!r.repair()) break;
        if (r.priced)
            for (int p = 0; p < k; ++p)
                if (r.samples[p].weight)
                    r.prices[p] = r.samples[p].loss > 0 ? static_cast<double>(r.samples[p].loss) / r.samples[p].weight : 0.0;
        ++stale;
        if (r.cut < best) {
            if (best - r.cut > best / 1000) stale = 0;
            best = r.cut;
            saved_labels = labels;
            saved_loads = r.loads;
            best_revision = r.revision;
            ++r.stats.checkpoint_updates;
        }
    }
    const bool restored = r.revision != best_revision;
    if (restored) { labels = saved_labels; r.loads = saved_loads; }
    r.cut = best;
    if (rounds > 0 && exchange_rounds > 0 && n <= 65536) {
        if (restored) r.build();
        r.exchange(exchange_rounds, best);
    }
    if (std::getenv("ORC_TRACE"))
        std::fprintf(stderr, "refine n=%lld start=%llu best=%llu final=%llu repairs=%d restored=%d\n", (long long)n,
                     (unsigned long long)feasible_start, (unsigned long long)best, (unsigned long long)r.cut, r.repairs, (int)restored);
    if (r.cut != best || r.cut > feasible_start || r.max_load() > C) fail(5, "incremental refinement postcondition failed");
    loads = r.loads;
    res.cut = r.cut;
    res.refined = true;
    r.stats.final_cut = r.cut;
    r.stats.final_max_part_weight = r.max_load();
    res.stats = r.stats;
    return res;
}

// ---------------------------------------------------------------- driver

struct State {
    Hierarchy h;
    std::vector<int32_t> initial;
    std::vector<std::vector<int32_t>> level_labels;
    std::vector<LevelResult> level_results;
};
thread_local State g_state;

// The caller's CSR as an oracle graph, with load_weighted_graph's and
// validate_weighted_shape's checks (src/graph.cpp:47-155).
Graph to_graph(const orc_csr* in) {
    Graph g;
    g.n = in->n;
    g.m = in->m;
    g.off.assign(in->offsets, in->offsets + in->n + 1);
    g.nbr.assign(in->neighbors, in->neighbors + in->m);
    if (in->edge_weights) g.ew.assign(in->edge_weights, in->edge_weights + in->m);
    else { g.ew.assign(static_cast<size_t>(in->m), 1u); g.implicit_unit = true; }
    if (in->vertex_weights) g.vw.assign(in->vertex_weights, in->vertex_weights + in->n);
    else g.vw.assign(static_cast<size_t>(in->n), 1u);
    if (g.off[0] != 0 || g.off[g.n] != g.m) fail(1, "invalid weighted CSR shape");
    for (i64 v = 0; v < g.n; ++v) if (g.off[v] > g.off[v + 1]) fail(1, "weighted CSR offsets are not monotone");
    for (i64 e = 0; e < g.m; ++e) if (g.nbr[e] < 0 || g.nbr[e] >= g.n) fail(1, "weighted CSR contains an invalid neighbor");
    for (u32 w : g.vw) if (!w) fail(1, "vertex weights must be positive");
    return g;
}

int run(const orc_csr* in, int32_t k, double eps, uint32_t seed, uint32_t flags, int32_t* labels_out, uint64_t* cut_out) {
    if (!in || in->n <= 0 || in->m < 0 || !in->offsets) fail(1, "invalid graph");
    if (k < 2 || k > kMaxParts || !std::isfinite(eps) || eps < 1.0) fail(1, "invalid partition capacity options");
    Graph g = to_graph(in);
    u64 total = 0;
    for (u32 w : g.vw) total += w;
    partition_capacity(total, k, eps);
    Options o;
    o.parts = k;
    o.seed = seed;
    o.cluster_size_factor = k <= 8 ? std::max(64, (512 + k - 1) / k) : std::max(2, (32 + k - 1) / k);
    o.pack_isolated = true;
    o.progressive = k >= 16;
    o.seed_matching = !(flags & ORC_FLAG_NO_SEED_MATCHING);
    g_state = State{};
    g_state.h = coarsen(std::move(g), o);
    auto& h = g_state.h;
    if (flags & ORC_FLAG_COARSEN_ONLY) return 0;
    const size_t L = h.levels.size();
    g_state.initial = initial_partition(h.levels.back(), k, eps, seed);
    g_state.level_labels.assign(L, {});
    g_state.level_results.assign(L, {});
    std::vector<int32_t> labels = g_state.initial;
    std::vector<u64> loads(static_cast<size_t>(k), 0);
    for (i64 v = 0; v < h.levels.back().n; ++v) loads[labels[v]] += h.levels.back().vw[v];
    // refine_hierarchy_impl (src/refine.cu:483-730)
    auto res = refine_level(h.levels.back(), k, eps, labels, loads, false, 0);
    u64 last_cut = res.cut;
    i64 last_refined = h.levels.back().n;
    g_state.level_labels[L - 1] = labels;
    g_state.level_results[L - 1] = res;
    for (size_t coarse = L - 1; coarse > 0; --coarse) {
        const size_t fine = coarse - 1;
        const Graph& fg = h.levels[fine];
        std::vector<int32_t> projected(static_cast<size_t>(fg.n));
        for (i64 v = 0; v < fg.n; ++v) projected[v] = labels[h.maps[fine][v]];
        labels.swap(projected);
        u64 t = 0;
        for (u64 w : loads) t += w;
        const u64 C = partition_capacity(t, k, eps);
        const u64 projected_max = *std::max_element(loads.begin(), loads.end());
        const bool refine = fine == 0 || projected_max > C || static_cast<double>(fg.n) >= 2.0 * static_cast<double>(last_refined);
        LevelResult lr;
        if (refine) {
            lr = refine_level(fg, k, eps, labels, loads, true, last_cut);
            if (!lr.repair_failed) last_refined = fg.n;
        } else {
            lr.cut = last_cut;
        }
        last_cut = lr.cut;
        g_state.level_labels[fine] = labels;
        g_state.level_results[fine] = lr;
    }
    u64 t = 0;
    for (u64 w : loads) t += w;
    if (*std::max_element(loads.begin(), loads.end()) > partition_capacity(t, k, eps))
        fail(5, "final original partition violates capacity");
    {  // src/refine.cu:709-716
        u64 directed = 0;
        for (u32 w : h.levels[0].ew) directed += w;
        if (directed & 1ULL) fail(5, "symmetric graph has odd directed edge weight");
    }
    if (labels_out) std::copy(labels.begin(), labels.end(), labels_out);
    if (cut_out) *cut_out = last_cut;
    return 0;
}

}  // namespace

extern "C" {

int orc_partition(const orc_csr* graph, int32_t k, double epsilon, uint32_t seed, uint32_t flags,
                  int32_t* labels_out, uint64_t* cut_out) {
    try {
        return run(graph, k, epsilon, seed, flags, labels_out, cut_out);
    } catch (const Fail& f) {
        g_error = f.what();
        return f.status;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 5;
    }
}

int orc_refine(const orc_csr* in, int32_t k, double epsilon, int32_t max_rounds, int32_t exchange_rounds,
               int32_t* labels, orc_refine_stats* stats) {
    try {
        if (!in || in->n <= 0 || in->m < 0 || !in->offsets || !labels || k < 2 || k > kMaxParts ||
            max_rounds < 0 || max_rounds > 64 || exchange_rounds < 0 || exchange_rounds > 8 ||
            !std::isfinite(epsilon) || epsilon < 1.0)
            fail(1, "invalid refinement options");
        Graph g = to_graph(in);
        std::vector<int32_t> lab(labels, labels + in->n);
        std::vector<u64> loads(static_cast<size_t>(k), 0);
        for (i64 v = 0; v < g.n; ++v) {
            if (lab[v] < 0 || lab[v] >= k) fail(1, "refinement partition has an invalid part id");
            loads[lab[v]] += g.vw[v];
        }
        const LevelResult r = refine_level(g, k, epsilon, lab, loads, false, 0, max_rounds, exchange_rounds);
        if (stats) *stats = r.stats;
        if (r.repair_failed) fail(2, "initial refinement capacity repair failed");
        std::copy(lab.begin(), lab.end(), labels);
        return 0;
    } catch (const Fail& f) {
        g_error = f.what();
        return f.status;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 5;
    }
}

const char* orc_last_error(void) { return g_error.c_str(); }

int orc_level_count(void) { return static_cast<int>(g_state.h.levels.size()); }

int orc_level_size(int32_t level, int64_t* n, int64_t* m) {
    if (level < 0 || level >= orc_level_count()) return 1;
    *n = g_state.h.levels[level].n;
    *m = g_state.h.levels[level].m;
    return 0;
}

int orc_level_copy(int32_t level, int32_t* offsets, int32_t* neighbors, uint32_t* edge_weights,
                   uint32_t* vertex_weights, int32_t* map, uint64_t* metadata) {
    if (level < 0 || level >= orc_level_count()) return 1;
    const Graph& g = g_state.h.levels[level];
    if (offsets) std::copy(g.off.begin(), g.off.end(), offsets);
    if (neighbors) std::copy(g.nbr.begin(), g.nbr.end(), neighbors);
    if (edge_weights) std::copy(g.ew.begin(), g.ew.end(), edge_weights);
    if (vertex_weights) std::copy(g.vw.begin(), g.vw.end(), vertex_weights);
    if (map && static_cast<size_t>(level) < g_state.h.maps.size())
        std::copy(g_state.h.maps[level].begin(), g_state.h.maps[level].end(), map);
    if (metadata) {
        metadata[0] = g.maximum_degree;
        metadata[1] = g.has_heavy_rows;
        metadata[2] = g.incident_weight_bound;
        metadata[3] = 0;
    }
    return 0;
}

int orc_initial_labels(int32_t* labels, int64_t capacity) {
    if (static_cast<int64_t>(g_state.initial.size()) > capacity) return 1;
    std::copy(g_state.initial.begin(), g_state.initial.end(), labels);
    return 0;
}

int orc_level_labels(int32_t level, int32_t* labels) {
    if (level < 0 || static_cast<size_t>(level) >= g_state.level_labels.size()) return 1;
    std::copy(g_state.level_labels[level].begin(), g_state.level_labels[level].end(), labels);
    return 0;
}

int orc_level_result(int32_t level, uint64_t* cut, int32_t* refined) {
    if (level < 0 || static_cast<size_t>(level) >= g_state.level_results.size()) return 1;
    *cut = g_state.level_results[level].cut;
    *refined = g_state.level_results[level].refined;
    return 0;
}

}  // extern "C"
