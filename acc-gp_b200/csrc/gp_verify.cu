// Strict invariant checks of GP_FLAG_VERIFY, the reference's --verify mode:
// the input and every coarse graph are bidirectional with equal reverse
// weights (validate_weighted_csr, src/graph.cpp:157-182), coarse graphs have
// no self loops, cluster weights and the weight cap hold and a projected
// labelling keeps its cut (verify_layer, src/coarsen.cu:1695-1758).  All
// checks run on the device and fail with the reference's messages.
#include "gp_graph.h"
#include "gp_primitives.cuh"

namespace gp {
namespace {

constexpr int kThreads = 256;

// Flags: 1 not bidirectional, 2 reverse weights differ, 4 self loop.
__global__ void k_verify_csr(i64 n, const int* off, const int* nbr, const u32* ew, bool allow_self_loops, u64* flags) {
    const int lane = threadIdx.x & 31;
    u64 bad = 0;
    for (i64 v = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < n;
         v += (static_cast<i64>(gridDim.x) * blockDim.x) >> 5) {
        for (int e = off[v] + lane; e < off[v + 1]; e += 32) {
            const int u = nbr[e];
            if (u == v && !allow_self_loops) bad |= 4;
            int lo = off[u], hi = off[u + 1];  // lower_bound of v in row u
            while (lo < hi) {
                const int mid = lo + (hi - lo) / 2;
                if (nbr[mid] < v) lo = mid + 1; else hi = mid;
            }
            if (lo == off[u + 1] || nbr[lo] != v) bad |= 1;
            else if (edge_w(ew, e) != edge_w(ew, lo)) bad |= 2;
        }
    }
    bad = __reduce_or_sync(0xffffffffu, static_cast<unsigned>(bad));
    if (lane == 0 && bad) atomicOr(flags, bad);
}

// Coarse vertex weights against the fine weights they sum, and the cap.
// Flags: 8 weight mismatch, 16 above the cap.
__global__ void k_sum_members(i64 n, const int* map, const u32* vw, u64* sums) {
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x)
        atomicAdd(sums + map[v], static_cast<u64>(vw[v]));
}
__global__ void k_check_weights(i64 nc, const u64* sums, const u32* cvw, u64 cap, u64* flags) {
    u64 bad = 0;
    for (i64 c = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; c < nc; c += static_cast<i64>(gridDim.x) * blockDim.x) {
        if (sums[c] != static_cast<u64>(cvw[c])) bad |= 8;
        if (static_cast<u64>(cvw[c]) > cap) bad |= 16;
    }
    bad = __reduce_or_sync(0xffffffffu, static_cast<unsigned>(bad));
    if ((threadIdx.x & 31) == 0 && bad) atomicOr(flags, bad);
}

// Directed cut under the labelling (x * 2654435761 + 17) mod 23 of x = v, or
// x = map[v] for the fine graph of a projection.
__device__ __forceinline__ int probe_label(const int* map, int v) {
    const u64 x = static_cast<u64>(map ? map[v] : v);
    return static_cast<int>((x * 2654435761ULL + 17) % 23);
}
__global__ void k_probe_cut(i64 n, const int* off, const int* nbr, const u32* ew, const int* map, u64* out) {
    const int lane = threadIdx.x & 31;
    u64 cut = 0;
    for (i64 v = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < n;
         v += (static_cast<i64>(gridDim.x) * blockDim.x) >> 5) {
        const int p = probe_label(map, static_cast<int>(v));
        for (int e = off[v] + lane; e < off[v + 1]; e += 32)
            if (probe_label(map, nbr[e]) != p) cut += edge_w(ew, e);
    }
    block_atomic_add(out, cut);
}

int grid(i64 items) { return static_cast<int>(std::min<i64>(blocks_for(items, kThreads), 148 * 16)); }

}  // namespace

void verify_csr(Context& ctx, const DGraph& g, bool allow_self_loops, gp_status status) {
    ctx.clear_scalars(1);
    launch(k_verify_csr, grid(g.n * 32), kThreads, 0, ctx.stream, g.n, g.off, g.nbr, g.ew, allow_self_loops,
           ctx.dev_scalars);
    const u64 flags = ctx.read_scalars(1)[0];
    if (flags & 4) fail(status, "contracted graph contains a self loop");
    if (flags & 1) fail(status, "weighted CSR is not bidirectional");
    if (flags & 2) fail(status, "weighted CSR reverse edge weights differ");
}

void verify_level(Context& ctx, const DGraph& fine, const DGraph& coarse, const int* map, u64 cluster_cap) {
    verify_csr(ctx, coarse, false, GP_INTERNAL);
    ArenaScope scope(ctx.scratch);
    u64* sums = ctx.scratch.alloc<u64>(static_cast<size_t>(coarse.n));
    GP_CUDA(cudaMemsetAsync(sums, 0, sizeof(u64) * coarse.n, ctx.stream));
    launch(k_sum_members, grid(fine.n), kThreads, 0, ctx.stream, fine.n, map, fine.vw, sums);
    ctx.clear_scalars(3);
    launch(k_check_weights, grid(coarse.n), kThreads, 0, ctx.stream, coarse.n, static_cast<const u64*>(sums), coarse.vw,
           cluster_cap, ctx.dev_scalars);
    launch(k_probe_cut, grid(fine.n * 32), kThreads, 0, ctx.stream, fine.n, fine.off, fine.nbr, fine.ew, map,
           ctx.dev_scalars + 1);
    launch(k_probe_cut, grid(coarse.n * 32), kThreads, 0, ctx.stream, coarse.n, coarse.off, coarse.nbr, coarse.ew,
           static_cast<const int*>(nullptr), ctx.dev_scalars + 2);
    const u64* sc = ctx.read_scalars(3);
    if (sc[0] & 8) fail(GP_INTERNAL, "coarsening cluster weight mismatch");
    if (sc[0] & 16) fail(GP_INTERNAL, "coarse point exceeds configured weight cap");
    if (sc[1] != sc[2]) fail(GP_INTERNAL, "cut is not conserved by coarse projection");
}

}  // namespace gp
