// Internal declarations shared by the host and device translation units.
#pragma once
#include "../../include/gpart_b200.h"

#include <cstdint>
#include <string>

namespace gp {

constexpr int kMaxParts = 128;  // include/graph_types.hpp:4

void set_error(const std::string& message);
const char* last_error();
gp_status capacity_of(uint64_t total, int k, double eps, uint64_t* out);
gp_status validate_host_csr(const gp_csr* g, bool need_positive_vw);

// Worker contexts of gp_partition_batch, owned by the calling context
// (gp_batch.cpp); accessors defined in gp_partition.cu.
struct WorkerPool;
WorkerPool*& worker_pool(gp_context* ctx);
void destroy_worker_pool(WorkerPool* pool);
int context_device(const gp_context* ctx);
// Device bytes a context's arenas hold, and their release.
size_t context_reserved(const gp_context* ctx);
void context_trim(gp_context* ctx);
void copy_options(const gp_context* from, gp_context* to);

// Coarsened hierarchies of resident graphs kept on one device for later
// requests (gp_partition.cu).  A hierarchy depends on the graph, k, the
// seed and the coarsening options, not on epsilon, so requests that differ
// only in epsilon (or repeat) reuse it.  Least recently used unreferenced
// hierarchies are dropped beyond `budget_bytes`.
struct HierarchyCache;
HierarchyCache* hierarchy_cache_create(int device, uint64_t budget_bytes);
void hierarchy_cache_destroy(HierarchyCache* cache);
uint64_t hierarchy_cache_bytes(const HierarchyCache* cache);
// gp_partition_device of a resident graph (graph_key names it) through the
// cache; stats->hierarchy_reused tells whether the hierarchy came from it.
gp_status partition_resident(gp_context* ctx, HierarchyCache* cache, uint64_t graph_key, const gp_csr* device_graph,
                             int32_t k, double epsilon, uint32_t seed, uint32_t flags, int32_t* labels_device,
                             gp_stats* stats);

}  // namespace gp
