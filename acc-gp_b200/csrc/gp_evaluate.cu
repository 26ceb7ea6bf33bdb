// Evaluation of a labelling on a device-resident graph: the undirected cut
// and the part loads, the two quantities refine_cut_kernel and
// accumulate_part_weights_kernel (src/refine.cu:63-126) produce.  The
// reduction is deterministic: every block of a fixed grid writes its partial
// loads and partial cut to a scratch array, and one block sums the partials
// in block order.
#include "gp_graph.h"
#include "gp_primitives.cuh"

#include <mutex>

namespace gp {
namespace {

constexpr int kEvalBlocks = 148 * 4;
constexpr int kEvalThreads = 256;
// Per block: k loads, the directed cut of its rows, the count of entries it
// skipped as invalid (a label outside [0,k), a neighbour outside [0,n) or an
// offset outside [0,m]).
constexpr int kEvalStride = kMaxParts + 2;

// Pass 1: block b writes partial[b * kEvalStride + p] for p < k (loads),
// partial[b * kEvalStride + k] (directed cut of the rows it scanned) and
// partial[b * kEvalStride + k + 1] (invalid entries it skipped).  Every
// access is range-checked, so a malformed labelling or CSR cannot reach
// memory outside the caller's arrays or the block's shared table.
__global__ void __launch_bounds__(kEvalThreads) k_eval_partials(i64 n, i64 m, const int* off, const int* nbr,
                                                                const u32* ew, const u32* vw, const int* labels, int k,
                                                                u64* partial) {
    __shared__ u64 loads[kMaxParts];
    __shared__ u64 warp_cut[kEvalThreads / 32];
    __shared__ u64 warp_bad[kEvalThreads / 32];
    for (int p = threadIdx.x; p < k; p += blockDim.x) loads[p] = 0;
    __syncthreads();
    u64 bad = 0;
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int p = labels[v];
        if (static_cast<unsigned>(p) < static_cast<unsigned>(k)) atomicAdd(loads + p, static_cast<u64>(vw ? vw[v] : 1u));
        else ++bad;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u64 cut = 0;
    for (i64 v = static_cast<i64>(blockIdx.x) * (blockDim.x / 32) + warp; v < n; v += static_cast<i64>(gridDim.x) * (blockDim.x / 32)) {
        const int p = labels[v];
        const int begin = off[v], end = off[v + 1];
        if (begin < 0 || end < begin || end > m) {
            if (lane == 0) ++bad;
            continue;
        }
        for (int e = begin + lane; e < end; e += 32) {
            const int u = nbr[e];
            if (static_cast<u64>(u) >= static_cast<u64>(n)) ++bad;
            else if (labels[u] != p) cut += edge_w(ew, e);
        }
    }
    cut = warp_sum(cut);
    bad = warp_sum(bad);
    if (lane == 0) {
        warp_cut[warp] = cut;
        warp_bad[warp] = bad;
    }
    __syncthreads();
    u64* out = partial + static_cast<i64>(blockIdx.x) * kEvalStride;
    for (int p = threadIdx.x; p < k; p += blockDim.x) out[p] = loads[p];
    if (threadIdx.x == 0) {
        u64 c = 0, b = 0;
        for (int w = 0; w < kEvalThreads / 32; ++w) {
            c += warp_cut[w];
            b += warp_bad[w];
        }
        out[k] = c;
        out[k + 1] = b;
    }
}

// Pass 2: sums the partials of all blocks in block order.  With any invalid
// entry the cut output is UINT64_MAX (no real cut reaches it) and, when
// `invalid` is given, the count is stored there.
__global__ void k_eval_reduce(int blocks, int k, const u64* partial, u64* cut_out, u64* loads_out, u64* invalid) {
    __shared__ u64 sums[2];
    for (int p = threadIdx.x; p <= k + 1; p += blockDim.x) {
        u64 s = 0;
        for (int b = 0; b < blocks; ++b) s += partial[static_cast<i64>(b) * kEvalStride + p];
        if (p < k) loads_out[p] = s;
        else sums[p - k] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *cut_out = sums[1] ? ~0ULL : sums[0] / 2;
        if (invalid) *invalid = sums[1];
    }
}

void check_evaluate_args(const gp_csr* g, const int32_t* labels, int32_t k, const uint64_t* cut_out,
                         const uint64_t* loads_out) {
    if (!g || !labels || !cut_out || !loads_out || !g->offsets || (g->m > 0 && !g->neighbors))
        fail(GP_INVALID_ARGUMENT, "graph, labels and outputs must not be NULL");
    if (g->n <= 0 || g->m < 0 || g->n > 0x7fffffff || g->m > 0x7fffffff)
        fail(GP_INVALID_ARGUMENT, "graph exceeds supported 32-bit CSR limits");
    if (k < 1 || k > kMaxParts) fail(GP_INVALID_ARGUMENT, "k must be in 1..128");
}

void launch_evaluate(const gp_csr* g, const int32_t* labels, int32_t k, uint64_t* cut_out, uint64_t* loads_out,
                     u64* partial, u64* invalid, cudaStream_t s) {
    launch(k_eval_partials, kEvalBlocks, kEvalThreads, 0, s, static_cast<i64>(g->n), static_cast<i64>(g->m),
           g->offsets, g->neighbors, g->edge_weights, g->vertex_weights, labels, static_cast<int>(k), partial);
    launch(k_eval_reduce, 1, 128, 0, s, kEvalBlocks, static_cast<int>(k), static_cast<const u64*>(partial),
           reinterpret_cast<u64*>(cut_out), reinterpret_cast<u64*>(loads_out), invalid);
}

template <class F>
gp_status guarded_eval(F&& f) {
    try {
        return f();
    } catch (const Failure& e) {
        set_error(e.what());
        return e.status;
    } catch (const std::exception& e) {
        set_error(e.what());
        return GP_INTERNAL;
    }
}

}  // namespace
}  // namespace gp

// ---------------------------------------------------------------------------
// Allocation-free variant.  Some callers cannot let a library call cudaMalloc:
// a framework whose caching allocator owns the whole device-memory budget (a
// raw cudaMalloc would bypass that budget and, on a full device, fail), or a
// serving loop that must not allocate or free device memory once it runs,
// because cudaMalloc/cudaFree may synchronise the device and stall the other
// streams.  gp_evaluate_device_static needs no context and no allocation: its
// per-block partial sums live in the fixed array below, which every GPU that
// loads this library holds until the process exits.
constexpr size_t kStaticScratchWords = static_cast<size_t>(gp::kEvalBlocks) * gp::kEvalStride;  // 616 KB
static __device__ __align__(256) unsigned long long g_eval_static_scratch[kStaticScratchWords];

namespace gp {
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_mutex;
u64* g_static_address[kMaxDevices] = {};

// Device address of the static scratch on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device, with that device current, and cached.  The cache assumes
// the device's primary context (the one the runtime API uses) stays the same
// for the life of the process: after cudaDeviceReset, or under another
// context made current through the driver API, the cached address is stale.
u64* static_scratch_address() {
    int device = 0;
    GP_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= kMaxDevices) fail(GP_INVALID_ARGUMENT, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_address[device]) {
        void* address = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&address, g_eval_static_scratch);
        if (err != cudaSuccess) cudaGetLastError();  // handled here
        if (err != cudaSuccess || !address)
            fail(GP_CUDA_ERROR, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(err));
        g_static_address[device] = static_cast<u64*>(address);
    }
    return g_static_address[device];
}
}  // namespace
}  // namespace gp

using namespace gp;

extern "C" gp_status gp_evaluate_device_static(const gp_csr* graph, const int32_t* labels, int32_t k,
                                               uint64_t* cut_out, uint64_t* loads_out, void* stream) {
    return guarded_eval([&]() -> gp_status {
        check_evaluate_args(graph, labels, k, cut_out, loads_out);
        // Every partial the reduction reads is rewritten by the first pass of
        // this call, so nothing in the shared array needs clearing first.
        u64* partial = static_scratch_address();
        launch_evaluate(graph, labels, k, cut_out, loads_out, partial, nullptr, static_cast<cudaStream_t>(stream));
        return GP_OK;
    });
}

// Context accessor defined in gp_partition.cu.
namespace gp { Context& context_of(gp_context* ctx); }

extern "C" gp_status gp_evaluate_device(gp_context* ctx, const gp_csr* graph, const int32_t* labels, int32_t k,
                                        uint64_t* cut_out, uint64_t* loads_out, void* stream) {
    return guarded_eval([&]() -> gp_status {
        if (!ctx) fail(GP_INVALID_ARGUMENT, "context is NULL");
        check_evaluate_args(graph, labels, k, cut_out, loads_out);
        Context& c = context_of(ctx);
        GP_CUDA(cudaSetDevice(c.device));
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c.stream;
        ArenaScope scope(c.scratch);
        u64* partial = c.scratch.alloc<u64>(static_cast<size_t>(kEvalBlocks) * kEvalStride);
        launch_evaluate(graph, labels, k, cut_out, loads_out, partial, c.dev_scalars, s);
        // The partials live in the context arena: keep them until the
        // reduction has read them.
        GP_CUDA(cudaMemcpyAsync(c.host_scalars, c.dev_scalars, sizeof(u64), cudaMemcpyDeviceToHost, s));
        GP_CUDA(cudaStreamSynchronize(s));
        if (c.host_scalars[0])
            fail(GP_INVALID_ARGUMENT, std::to_string(c.host_scalars[0]) +
                                          " labels, neighbours or offsets out of range (labels must be in [0,k))");
        return GP_OK;
    });
}
