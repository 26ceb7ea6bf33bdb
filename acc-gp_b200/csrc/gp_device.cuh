// Device-side foundations shared by every kernel file: error handling,
// the stack arena, launch accounting and small warp/block helpers.
#pragma once
#include "gp_internal.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace gp {

using u64 = unsigned long long;
using i64 = long long;
using u32 = unsigned int;

// Errors travel as exceptions inside the library and become a gp_status at
// the C ABI (gp_partition.cu).  No exception crosses that boundary.
struct Failure : std::runtime_error {
    gp_status status;
    Failure(gp_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};
[[noreturn]] inline void fail(gp_status s, const std::string& m) { throw Failure(s, m); }

// A failed runtime call becomes a gp_status.  The failure is handled here,
// so its error is also taken off the thread's last-error slot (a no-op for
// sticky device faults, which stay set): a later launch check must not
// report it again.
#define GP_CUDA(call)                                                                          \
    do {                                                                                       \
        const cudaError_t gp_err__ = (call);                                                   \
        if (gp_err__ != cudaSuccess) {                                                         \
            cudaGetLastError();                                                                \
            ::gp::fail(gp_err__ == cudaErrorMemoryAllocation ? GP_OUT_OF_MEMORY : GP_CUDA_ERROR, \
                       std::string(#call) + ": " + cudaGetErrorString(gp_err__));             \
        }                                                                                      \
    } while (0)

// Number of kernels this library launched; every launch goes through launch().
extern thread_local u64 g_launches;

// Optional per-kernel timing: when a profiler is installed, launches of the
// kernels whose name contains its pattern are bracketed by CUDA events on
// their own stream (gp_profile_begin / gp_profile_end).
// A launch site may also report the algorithmic bytes of the launch it just
// made (account_bytes); the profiler sums them for the timed launches.
struct KernelProfiler {
    std::string pattern;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    size_t used = 0;
    bool last_timed = false;
    double bytes = 0;
    // Kernels whose work is decided on the device add their algorithmic
    // bytes here when they run (see work_counter).
    unsigned long long* device_bytes = nullptr;
    bool matches(const void* kernel);
    void before(cudaStream_t s);
    void after(cudaStream_t s);
    std::vector<std::pair<const void*, bool>> cache;
};
extern thread_local KernelProfiler* g_profiler;

inline void account_bytes(double bytes) {
    if (g_profiler && g_profiler->last_timed) g_profiler->bytes += bytes;
}
// Device counter for the algorithmic bytes of `kernel` when it is profiled,
// else nullptr; the kernel adds its bytes only if it does its work.
template <class K>
inline unsigned long long* work_counter(K kernel) {
    return g_profiler && g_profiler->device_bytes && g_profiler->matches(reinterpret_cast<const void*>(kernel))
               ? g_profiler->device_bytes : nullptr;
}

template <class... Params, class... Args>
inline void launch(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                   Args&&... args) {
    ++g_launches;
    const bool timed = g_profiler && g_profiler->matches(reinterpret_cast<const void*>(kernel));
    if (g_profiler) g_profiler->last_timed = timed;
    if (timed) g_profiler->before(stream);
    // A launch that did not start (bad configuration, missing shared-memory
    // opt-in) must fail the call, not leave its results silently unwritten.
    // This library clears the error of every failure it has handled where it
    // handles it (GP_CUDA, the server's own allocations), so what is pending
    // here belongs to this launch or to an unhandled fault.
    kernel<<<grid, block, smem, stream>>>(static_cast<Params>(args)...);
    if (const cudaError_t e = cudaGetLastError(); e != cudaSuccess)
        ::gp::fail(GP_CUDA_ERROR, std::string("kernel launch: ") + cudaGetErrorString(e));
    if (timed) g_profiler->after(stream);
}

inline int blocks_for(i64 items, int per_block) {
    const i64 b = (items + per_block - 1) / per_block;
    return static_cast<int>(b < 1 ? 1 : b);
}

// Grow-only chunked stack allocator.  Allocation is a bump inside the current
// chunk; release() pops back to a mark.  Chunks stay allocated for the next
// call, so a repeated workload performs no cudaMalloc after its first run.
class Arena {
public:
    struct Mark { size_t chunk, offset; };
    ~Arena() { reset_device(); }
    void reset_device() {
        for (auto& c : chunks_) cudaFree(c.base);
        chunks_.clear();
        current_ = 0;
    }
    Mark mark() const { return {current_, chunks_.empty() ? 0 : chunks_[current_].top}; }
    void release(Mark m) {
        if (chunks_.empty()) return;
        for (size_t c = m.chunk + 1; c < chunks_.size(); ++c) chunks_[c].top = 0;
        current_ = m.chunk;
        chunks_[current_].top = m.offset;
    }
    template <class T>
    T* alloc(size_t count) {
        return static_cast<T*>(raw(count * sizeof(T)));
    }
    void* raw(size_t bytes) {
        bytes = (bytes + 255) & ~size_t{255};
        if (bytes == 0) bytes = 256;
        while (current_ < chunks_.size()) {
            Chunk& c = chunks_[current_];
            if (c.top + bytes <= c.size) {
                void* p = c.base + c.top;
                c.top += bytes;
                note_use();
                return p;
            }
            if (current_ + 1 < chunks_.size()) { ++current_; chunks_[current_].top = 0; continue; }
            break;
        }
        Chunk c;
        c.size = bytes > chunk_bytes_ ? bytes : chunk_bytes_;
        GP_CUDA(cudaMalloc(&c.base, c.size));
        c.top = bytes;
        chunks_.push_back(c);
        current_ = chunks_.size() - 1;
        note_use();
        return c.base;
    }
    void set_chunk_bytes(size_t b) { chunk_bytes_ = b; }
    // Exchanges the whole state (chunks included) with another arena.
    void swap(Arena& o) noexcept {
        chunks_.swap(o.chunks_);
        std::swap(current_, o.current_);
        std::swap(chunk_bytes_, o.chunk_bytes_);
        std::swap(peak_, o.peak_);
    }
    size_t reserved() const { size_t s = 0; for (auto& c : chunks_) s += c.size; return s; }
    // Largest number of bytes held at once since reset_peak() (the measured
    // footprint of the work in between).
    size_t peak() const { return peak_; }
    void reset_peak() { peak_ = 0; note_use(); }

private:
    void note_use() {
        size_t used = 0;
        for (size_t i = 0; i <= current_ && i < chunks_.size(); ++i) used += chunks_[i].top;
        if (used > peak_) peak_ = used;
    }
    struct Chunk { char* base = nullptr; size_t size = 0, top = 0; };
    std::vector<Chunk> chunks_;
    size_t current_ = 0;
    size_t chunk_bytes_ = size_t{256} << 20;
    size_t peak_ = 0;
};

// Scoped release of an arena region.
struct ArenaScope {
    Arena& arena;
    Arena::Mark mark;
    explicit ArenaScope(Arena& a) : arena(a), mark(a.mark()) {}
    ~ArenaScope() { arena.release(mark); }
};

// ---------------------------------------------------------------- device helpers

// mix32 (src/coarsen.cu:173-179, seed_matching.cuh:7, refine.cu:50).
__host__ __device__ __forceinline__ u32 mix32(u32 x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    return x ^ (x >> 16);
}

// Order key of the deterministic repair (shared with the oracle).
__host__ __device__ __forceinline__ u32 repair_hash(int v) { return mix32(static_cast<u32>(v) ^ 0x85ebca6bU); }

template <class T>
__device__ __forceinline__ T warp_sum(T v, unsigned mask = 0xffffffffu) {
    for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(mask, v, d);
    return v;
}
template <class T>
__device__ __forceinline__ T warp_max(T v) {
    for (int d = 16; d; d >>= 1) { const T o = __shfl_xor_sync(0xffffffffu, v, d); v = o > v ? o : v; }
    return v;
}

__device__ __forceinline__ u32 edge_w(const u32* w, i64 e) { return w ? w[e] : 1u; }

// Block-wide reductions into one global atomic per block.  Every thread of
// the block must call them (they synchronise the block); many blocks
// updating one address would otherwise serialise on it, one atomic per warp.
template <class T>
__device__ __forceinline__ T block_sum(T v) {
    __shared__ T part[32];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    T s = 0;
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : T(0);
        s = warp_sum(s);
    }
    __syncthreads();
    return s;  // valid in thread 0
}
template <class T>
__device__ __forceinline__ T block_max(T v) {
    __shared__ T part[32];
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    T s = 0;
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : T(0);
        s = warp_max(s);
    }
    __syncthreads();
    return s;  // valid in thread 0
}
__device__ __forceinline__ void block_atomic_add(unsigned long long* out, unsigned long long v) {
    v = block_sum(v);
    if (threadIdx.x == 0 && v) atomicAdd(out, v);
}
__device__ __forceinline__ void block_atomic_add(long long* out, long long v) {
    v = block_sum(v);
    if (threadIdx.x == 0 && v) atomicAdd(reinterpret_cast<unsigned long long*>(out), static_cast<unsigned long long>(v));
}
__device__ __forceinline__ void block_atomic_max(unsigned long long* out, unsigned long long v) {
    v = block_max(v);
    if (threadIdx.x == 0 && v) atomicMax(out, v);
}

// A block's sum of one value per warp, added to a global counter without a
// barrier at the end of the kernel: warps add into shared memory as they
// finish, and the block's last warp adds the block's sum.  Warps of uneven
// work then never wait for each other.  init() must be called by every
// thread at the start of the kernel.
struct WarpSum {
    unsigned long long sum;
    unsigned arrived;
    __device__ __forceinline__ void init() {
        if (threadIdx.x == 0) { sum = 0; arrived = 0; }
        __syncthreads();
    }
    // value: the warp's total, taken from lane 0.
    __device__ __forceinline__ void finish(unsigned long long value, unsigned long long* out) {
        if ((threadIdx.x & 31) != 0) return;
        if (value) atomicAdd(&sum, value);
        __threadfence_block();
        if (atomicAdd(&arrived, 1u) == (blockDim.x >> 5) - 1) {
            const unsigned long long total = atomicAdd(&sum, 0ULL);
            if (total) atomicAdd(out, total);
        }
    }
};

// Block-aggregated append: every `active` thread writes v to its own slot of
// queue; one atomic on *count per block.  All threads of the block call it.
template <class V>
__device__ __forceinline__ void block_append(V v, bool active, V* queue, unsigned long long* count) {
    __shared__ u32 warp_base[32];
    __shared__ unsigned long long base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned mask = __ballot_sync(0xffffffffu, active);
    if (lane == 0) warp_base[warp] = __popc(mask);
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 total = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
            const u32 c = warp_base[w];
            warp_base[w] = total;
            total += c;
        }
        base = total ? atomicAdd(count, static_cast<unsigned long long>(total)) : 0ULL;
    }
    __syncthreads();
    if (active) queue[base + warp_base[warp] + __popc(mask & ((1u << lane) - 1u))] = v;
    __syncthreads();
}

}  // namespace gp
