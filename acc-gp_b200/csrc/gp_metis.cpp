// The method's own initial-partition step: one CPU METIS k-way run on the
// coarsest graph, exactly as initial_partition_metis
// (src/initial_partition_metis.cu:86-183) does in production
// (require_feasible = false).  Links the METIS 5.1 library that ships with the
// CUDA toolkit; its ABI (64-bit idx_t, 32-bit real_t, option slots 8 = seed
// and 17 = numbering) was established by running it.
#include "gp_metis.h"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>

extern "C" {
typedef int64_t idx_t;
typedef float real_t;
int METIS_SetDefaultOptions(idx_t* options);
int METIS_PartGraphKway(idx_t* nvtxs, idx_t* ncon, idx_t* xadj, idx_t* adjncy, idx_t* vwgt, idx_t* vsize,
                        idx_t* adjwgt, idx_t* nparts, real_t* tpwgts, real_t* ubvec, idx_t* options,
                        idx_t* objval, idx_t* part);
}

namespace gp {
namespace {
constexpr int kOptions = 40, kSeed = 8, kNumbering = 17, kMetisOk = 1;
}

gp_status metis_initial_partition(const HostCsr& g, int parts, double eps, uint32_t seed, std::vector<int>& labels,
                                  std::string& error) {
    const int64_t n = g.n;
    if (n <= 0 || parts < 2 || parts > kMaxParts || parts > n || !std::isfinite(eps) || eps < 1.0) {
        error = "invalid METIS initialization options";
        return GP_INVALID_ARGUMENT;
    }
    uint64_t total = 0, edge_total = 0;
    for (uint32_t w : g.vw) total += w;
    for (uint32_t w : g.ew) edge_total += w;
    uint64_t capacity = 0;
    if (gp_status s = capacity_of(total, parts, eps, &capacity); s != GP_OK) {
        error = last_error();
        return s;
    }
    uint64_t vg = 0, eg = 0;
    for (uint32_t w : g.vw) {
        if (!w) { error = "METIS requires positive vertex weights"; return GP_INVALID_ARGUMENT; }
        if (w > capacity) { error = "a vertex exceeds partition capacity"; return GP_INVALID_ARGUMENT; }
        vg = std::gcd(vg, static_cast<uint64_t>(w));
    }
    for (uint32_t w : g.ew) eg = std::gcd(eg, static_cast<uint64_t>(w));
    if (!eg) eg = 1;
    const uint64_t limit = static_cast<uint64_t>(INT64_MAX);
    if (total / vg > limit || edge_total / eg > limit) {
        error = "weighted coarse graph exceeds METIS signed weight range";
        return GP_INVALID_ARGUMENT;
    }
    // Exact common-factor normalisation; self loops and zero edges dropped.
    std::vector<idx_t> xadj(static_cast<size_t>(n + 1), 0), adj, adjw, vwgt(static_cast<size_t>(n));
    adj.reserve(g.nbr.size());
    adjw.reserve(g.nbr.size());
    for (int64_t v = 0; v < n; ++v) {
        vwgt[v] = static_cast<idx_t>(g.vw[v] / vg);
        for (int64_t e = g.off[v]; e < g.off[v + 1]; ++e) {
            if (g.nbr[e] == v || !g.ew[e]) continue;
            adj.push_back(g.nbr[e]);
            adjw.push_back(static_cast<idx_t>(g.ew[e] / eg));
        }
        xadj[v + 1] = static_cast<idx_t>(adj.size());
    }
    if (adj.empty()) { adj.push_back(0); adjw.push_back(0); }
    idx_t nn = n, ncon = 1, k = parts, objective = 0;
    std::vector<idx_t> part(static_cast<size_t>(n));
    idx_t options[kOptions];
    if (METIS_SetDefaultOptions(options) != kMetisOk) { error = "METIS_SetDefaultOptions failed"; return GP_INTERNAL; }
    options[kSeed] = static_cast<idx_t>(seed & 0x7fffffffU);
    options[kNumbering] = 0;
    real_t upper = static_cast<real_t>(eps);
    if (upper <= 1.0f) upper = std::nextafter(1.0f, INFINITY);
    int status;
    {
        // METIS seeds one process-wide random generator per call, so calls
        // from concurrent contexts are serialised to stay reproducible.
        static std::mutex metis_mutex;
        std::lock_guard<std::mutex> lock(metis_mutex);
        status = METIS_PartGraphKway(&nn, &ncon, xadj.data(), adj.data(), vwgt.data(), nullptr, adjw.data(), &k,
                                     nullptr, &upper, options, &objective, part.data());
    }
    if (status != kMetisOk) { error = "METIS_PartGraphKway failed: " + std::to_string(status); return GP_INTERNAL; }
    labels.resize(static_cast<size_t>(n));
    for (int64_t v = 0; v < n; ++v) {
        if (part[v] < 0 || part[v] >= parts) { error = "METIS returned an invalid partition label"; return GP_INTERNAL; }
        labels[v] = static_cast<int>(part[v]);
    }
    return GP_OK;
}

}  // namespace gp
