// Projection and refinement (temporary: projection only).
#include "gp_graph.h"
#include "gp_primitives.cuh"

namespace gp {
namespace {
__global__ void k_cut(i64 n, const int* off, const int* nbr, const u32* ew, const int* labels, u64* out) {
    u64 local = 0;
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int p = labels[v];
        for (int e = off[v]; e < off[v + 1]; ++e) if (labels[nbr[e]] != p) local += edge_w(ew, e);
    }
    local = warp_sum(local);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, local);
}
__global__ void k_project(i64 n, const int* map, const int* coarse, int* fine) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n) fine[v] = coarse[map[v]];
}
}  // namespace

u64 device_cut(Context& ctx, const DGraph& g, const int* labels) {
    ctx.clear_scalars(1);
    launch(k_cut, std::min(blocks_for(g.n, 256), 148 * 16), 256, 0, ctx.stream, g.n, g.off, g.nbr, g.ew, labels, ctx.dev_scalars);
    const u64 d = ctx.read_scalars(1)[0];
    if (d & 1ULL) fail(GP_INTERNAL, "refinement cut is not symmetric");
    return d / 2;
}

RefineOutcome uncoarsen(Context& ctx, Hierarchy& h, const std::vector<int>& coarse_labels, int k, double eps,
                        int* labels, bool log) {
    const size_t L = h.levels.size();
    int* cur = ctx.scratch.alloc<int>(h.levels.back().n);
    GP_CUDA(cudaMemcpyAsync(cur, coarse_labels.data(), sizeof(int) * coarse_labels.size(), cudaMemcpyHostToDevice, ctx.stream));
    for (size_t c = L - 1; c > 0; --c) {
        const DGraph& f = h.levels[c - 1];
        int* next = c - 1 == 0 ? labels : ctx.scratch.alloc<int>(f.n);
        launch(k_project, blocks_for(f.n, 256), 256, 0, ctx.stream, f.n, h.maps[c - 1], cur, next);
        cur = next;
    }
    if (L == 1) GP_CUDA(cudaMemcpyAsync(labels, cur, sizeof(int) * h.levels[0].n, cudaMemcpyDeviceToDevice, ctx.stream));
    RefineOutcome r;
    r.cut = device_cut(ctx, h.levels[0], labels);
    return r;
}
}  // namespace gp
