// Projection and refinement on the B200 (Acc-GPart src/refine.cu,
// src/refinement/*.cuh): dense affinity cache, label propagation with the
// priority filter, exact cut/cache updates, capacity repair and the
// capacity-complementary exchange.  One host loop per level with one small
// read-back per LP round; every decision is a pure function of the state, so
// the result does not depend on thread scheduling.  The repair ranks donors
// and receiver tickets in the deterministic (bucket, repair hash, id) order.
#include "gp_graph.h"
#include "gp_primitives.cuh"

#include <algorithm>
#include <chrono>
#include <cfloat>
#include <climits>
#include <type_traits>
#include <cstdio>

namespace gp {
namespace {

constexpr int kBalanceWidth = 800;  // kBalanceBuckets * kBalanceSections
constexpr int kThreads = 256;

struct Sample {
    long long loss;
    u64 weight;
};

// ---------------------------------------------------------------- small kernels

__global__ void k_cut_chunks(DGraph g, const int* labels, u64* out) {
    const int c = blockIdx.x, v = g.chunk_row[c];
    const int p = labels[v];
    u64 local = 0;
    for (int e = g.chunk_begin[c] + threadIdx.x; e < chunk_end(g, c, v); e += blockDim.x)
        if (labels[g.nbr[e]] != p) local += edge_w(g.ew, e);
    block_atomic_add(out, local);
}
__global__ void k_cut(i64 n, const int* off, const int* nbr, const u32* ew, const int* labels, int heavy_min, u64* out) {
    __shared__ WarpSum cut_sum;
    cut_sum.init();
    const int lane = threadIdx.x & 31;
    u64 local = 0;
    for (i64 v = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < n;
         v += (static_cast<i64>(gridDim.x) * blockDim.x) >> 5) {
        const int p = labels[v];
        if (off[v + 1] - off[v] > heavy_min) continue;  // k_cut_chunks
        for (int e = off[v] + lane; e < off[v + 1]; e += 32)
            if (labels[nbr[e]] != p) local += edge_w(ew, e);
    }
    cut_sum.finish(warp_sum(local), out);
}

__global__ void k_project(i64 n, const int* map, const int* coarse, int* fine) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n) fine[v] = coarse[map[v]];
}

__global__ void k_loads(i64 n, int k, const int* labels, const u32* vw, u64* loads) {
    extern __shared__ u64 part[];
    for (int p = threadIdx.x; p < k; p += blockDim.x) part[p] = 0;
    __syncthreads();
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x)
        atomicAdd(part + labels[v], static_cast<u64>(vw[v]));
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x)
        if (part[p]) atomicAdd(loads + p, part[p]);
}

__global__ void k_max_load(int k, const u64* loads, u64* out) {
    u64 m = 0;
    for (int p = threadIdx.x; p < k; p += 32) m = max(m, loads[p]);
    m = warp_max(m);
    if (threadIdx.x == 0) *out = m;
}

__global__ void k_max_edge(i64 m, const u32* ew, u64* out) {
    u32 mx = 0;
    for (i64 e = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; e < m; e += static_cast<i64>(gridDim.x) * blockDim.x)
        mx = max(mx, ew[e]);
    block_atomic_max(out, static_cast<u64>(mx));
}

// publish_repair_prices (incremental.cuh:161-164).
__global__ void k_prices(int k, const Sample* samples, double* prices) {
    for (int p = threadIdx.x; p < k; p += blockDim.x)
        if (samples[p].weight)
            prices[p] = samples[p].loss > 0 ? static_cast<double>(samples[p].loss) / static_cast<double>(samples[p].weight) : 0.0;
}

// estimated_repair_cost (incremental.cuh:156-160).  Products and sums use
// explicit round-to-nearest intrinsics so no multiply-add is contracted.
__device__ __forceinline__ double repair_cost(int part, u64 weight, const u64* loads, u64 capacity, const double* prices) {
    const u64 slack = capacity - loads[part];
    return weight > slack ? __dmul_rn(prices[part], static_cast<double>(weight - slack)) : 0.0;
}

// ---------------------------------------------------------------- affinity cache

// 16-byte loads of affinity rows when a row starts on a 16-byte boundary.
template <class C> struct AffinityVec;
template <> struct AffinityVec<u32> { using V = uint4; static constexpr int N = 4; };
template <> struct AffinityVec<u64> { using V = ulonglong2; static constexpr int N = 2; };

// Adds the entries [begin, end) of row v to a shared histogram by part,
// `stride` lanes apart starting at `first`, four entries per lane at a time
// so that four neighbour and four label loads are in flight together.
template <class C>
__device__ __forceinline__ void accumulate_row(const int* nbr, const u32* ew, const int* labels, int v, int first,
                                               int end, int stride, C* hist) {
    constexpr int kUnroll = 4;
    for (int e0 = first; e0 < end; e0 += kUnroll * stride) {
        int u[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            const int e = e0 + j * stride;
            u[j] = e < end ? nbr[e] : v;
        }
        int part[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) part[j] = u[j] != v ? labels[u[j]] : -1;
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            // part >= 0 only for entries inside the row
            const C w = part[j] >= 0 ? static_cast<C>(edge_w(ew, e0 + j * stride)) : C(0);
            if (part[j] >= 0) atomicAdd(hist + part[j], w);
        }
    }
}

// incremental_build_affinity (incremental.cuh:61-140), dense layout.  A warp
// builds 32/W rows at a time, W lanes per row, each row's k-wide histogram in
// shared memory; rows longer than short_max entries are accumulated by the
// whole warp afterwards.  Heavy rows are written as zeros (k_build_chunks
// adds their sums).  Optionally sums the directed cut of the light rows,
// total - own-part affinity per row.
template <class C, int W, bool Vectorized>
__global__ void __launch_bounds__(kThreads) k_build(i64 n, const int* off, const int* nbr, const u32* ew,
                                                    const int* labels, int k, C* A, C* totals, u64* directed_cut,
                                                    const u64* gate, u64 threshold, u64* work, u64 work_bytes,
                                                    int short_max, bool long_rows_apart, int heavy_min) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ WarpSum cut_sum;
    if (gate && *gate <= threshold) return;  // incremental update chosen
    if (work && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(work, work_bytes);
    cut_sum.init();
    constexpr int N = Vectorized ? AffinityVec<C>::N : 1;
    constexpr int G = 32 / W;
    const int lane = threadIdx.x & 31, gid = lane / W, sub = lane % W;
    C* warp_hist = reinterpret_cast<C*>(smem_raw) + static_cast<size_t>(threadIdx.x >> 5) * G * k;
    C* hist = warp_hist + gid * k;
    const i64 warps = (static_cast<i64>(gridDim.x) * blockDim.x) >> 5;
    unsigned leaders = 0;
    for (int g = 0; g < G; ++g) leaders |= 1u << (g * W);
    u64 cut = 0;
    for (i64 base = ((static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * G; base < n; base += warps * G) {
        const i64 v = base + gid;
        const bool valid = v < n;
        const int begin = valid ? off[v] : 0, end = valid ? off[v + 1] : 0;
        const int deg = end - begin;
        if constexpr (Vectorized) {
            for (int p0 = sub * N; p0 < k; p0 += W * N) *reinterpret_cast<typename AffinityVec<C>::V*>(hist + p0) = {};
        } else {
            for (int p = sub; p < k; p += W) hist[p] = 0;
        }
        __syncwarp();
        if (deg <= short_max && deg <= heavy_min) {  // heavier rows belong to the chunk kernels
            accumulate_row(nbr, ew, labels, static_cast<int>(v), begin + sub, end, W, hist);
        }
        // Rows of short_max..heavy_min entries go to k_build_long when it runs.
        const bool mine = valid && !(long_rows_apart && deg > short_max && deg <= heavy_min);
        for (unsigned rest = __ballot_sync(0xffffffffu, mine && deg > short_max && deg <= heavy_min) & leaders; rest;
             rest &= rest - 1) {
            const int leader = __ffs(rest) - 1;
            const int vv = static_cast<int>(base) + leader / W;
            const int b = __shfl_sync(0xffffffffu, begin, leader), e_end = __shfl_sync(0xffffffffu, end, leader);
            C* h = warp_hist + (leader / W) * k;
            accumulate_row(nbr, ew, labels, vv, b + lane, e_end, 32, h);
        }
        __syncwarp();
        C total = 0;
        if (mine) {
            C* row = A + v * k;
            for (int p0 = sub * N; p0 < k; p0 += W * N) {
                if constexpr (Vectorized) {
                    const typename AffinityVec<C>::V x = *reinterpret_cast<const typename AffinityVec<C>::V*>(hist + p0);
                    *reinterpret_cast<typename AffinityVec<C>::V*>(row + p0) = x;
                    if constexpr (N == 4) total += x.x + x.y + x.z + x.w;
                    else total += x.x + x.y;
                } else {
                    row[p0] = hist[p0];
                    total += hist[p0];
                }
            }
        }
#pragma unroll
        for (int d = W / 2; d; d >>= 1) total += __shfl_xor_sync(0xffffffffu, total, d, W);
        if (mine && sub == 0) {
            totals[v] = total;
            if (directed_cut) cut += static_cast<u64>(total - hist[labels[v]]);
        }
        __syncwarp();
    }
    if (directed_cut) cut_sum.finish(warp_sum(cut), directed_cut);
}

// The rows of short_max..heavy_min entries (listed in `rows`), a warp per
// row: taken off a list, they spread evenly over all warps instead of
// stalling the warps of k_build that drew them.
template <class C>
__global__ void __launch_bounds__(kThreads) k_build_long(i64 count, const int* rows, const int* off, const int* nbr,
                                                         const u32* ew, const int* labels, int k, C* A, C* totals,
                                                         u64* directed_cut, const u64* gate, u64 threshold, u64* work,
                                                         u64 work_bytes) {
    extern __shared__ __align__(16) unsigned char smem_long[];
    __shared__ WarpSum cut_sum;
    if (gate && *gate <= threshold) return;
    if (work && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(work, work_bytes);
    cut_sum.init();
    const int lane = threadIdx.x & 31;
    C* hist = reinterpret_cast<C*>(smem_long) + static_cast<size_t>(threadIdx.x >> 5) * k;
    u64 cut = 0;
    for (i64 i = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; i < count;
         i += (static_cast<i64>(gridDim.x) * blockDim.x) >> 5) {
        const int v = rows[i];
        for (int p = lane; p < k; p += 32) hist[p] = 0;
        __syncwarp();
        accumulate_row(nbr, ew, labels, v, off[v] + lane, off[v + 1], 32, hist);
        __syncwarp();
        C total = 0;
        C* row = A + static_cast<i64>(v) * k;
        for (int p = lane; p < k; p += 32) {
            row[p] = hist[p];
            total += hist[p];
        }
        total = warp_sum(total);
        if (lane == 0) {
            totals[v] = total;
            if (directed_cut) cut += static_cast<u64>(total - hist[labels[v]]);
        }
        __syncwarp();
    }
    if (directed_cut) cut_sum.finish(cut, directed_cut);
}
// Sum of the row lengths of rows[0 .. *count).
__global__ void k_row_entries(const u32* count, const int* rows, const int* off, u64* out) {
    const i64 c = static_cast<i64>(*count);
    u64 sum = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < c; i += static_cast<i64>(gridDim.x) * blockDim.x)
        sum += static_cast<u64>(off[rows[i] + 1] - off[rows[i]]);
    block_atomic_add(out, sum);
}
struct IsLongRow {
    const int* off;
    int short_max, heavy_min;
    __device__ bool operator()(i64 v) const {
        const int d = off[v + 1] - off[v];
        return d > short_max && d <= heavy_min;
    }
};

// GP_FLAG_VERIFY: the incremental cache against an independent rebuild.
template <class C>
__global__ void k_compare_cache(i64 cells, const C* A, const C* B, i64 n, const C* ta, const C* tb, u64* mismatch) {
    u32 bad = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < cells; i += static_cast<i64>(gridDim.x) * blockDim.x)
        bad |= A[i] != B[i];
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x)
        bad |= ta[v] != tb[v];
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(mismatch, 1ULL);
}

// Directed cut of the heavy rows once k_build_chunks has completed them.
template <class C>
__global__ void k_heavy_cut(i64 count, const int* heavy, const int* labels, int k, const C* A, const C* totals,
                            u64* directed_cut, const u64* gate, u64 threshold) {
    if (gate && *gate <= threshold) return;
    u64 cut = 0;
    for (i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; h < count; h += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int v = heavy[h];
        cut += static_cast<u64>(totals[v] - A[static_cast<i64>(v) * k + labels[v]]);
    }
    block_atomic_add(directed_cut, cut);
}

template <class C>
__global__ void k_build_chunks(DGraph g, const int* labels, int k, C* A, C* totals, const u64* gate, u64 threshold,
                               u64* work, u64 work_bytes) {
    extern __shared__ unsigned char smem_build[];
    if (gate && *gate <= threshold) return;
    if (work && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(work, work_bytes);
    C* hist = reinterpret_cast<C*>(smem_build);
    const int c = blockIdx.x, v = g.chunk_row[c];
    for (int p = threadIdx.x; p < k; p += blockDim.x) hist[p] = 0;
    __syncthreads();
    accumulate_row(g.nbr, g.ew, labels, v, g.chunk_begin[c] + static_cast<int>(threadIdx.x), chunk_end(g, c, v),
                   static_cast<int>(blockDim.x), hist);
    __syncthreads();
    C total = 0;
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        const C x = hist[p];
        if (x) atomicAdd(A + static_cast<i64>(v) * k + p, x);
        total += x;
    }
    total = warp_sum(total);
    if ((threadIdx.x & 31) == 0 && total) atomicAdd(totals + v, total);
}

// ---------------------------------------------------------------- label propagation

struct LpParams {
    i64 n;
    int k;
    u64 capacity;
    double filter;
    const int* off;
    const int* nbr;
    const u32* ew;
    const u32* vw;
    int* labels;
    u64* loads;
    const double* prices;  // nullptr: unpriced
    int* targets;
    long long* gains;
    unsigned char* locks;
    int* flags;
    int* cand;
    int* movers;
    u64* counters;  // 0 candidates, 1 movers, 2 delta (signed), 3 max load
    int heavy_min;  // rows longer than this go through the chunk kernels
    u64* proposal;  // per vertex, the round's proposal packed for the filter (below)
};

// A vertex's proposal of the round in one word, written by the proposal
// kernels for every vertex they visit and read by the priority filter for
// each neighbour, one 8-byte gather instead of the target, gain and label
// gathers: bits 0-7 the label, 8-15 the target, bit 16 set for a proposer,
// bit 17 set when the gain does not fit the 46-bit field in bits 18-63 (the
// filter then reads the gain array).  0: not proposing.  Vertices the
// proposals do not visit (outside the frontier) keep the 0 written at the
// start of the level, as their targets stay -1.
constexpr u64 kProposer = 1ULL << 16, kGainApart = 1ULL << 17;
constexpr long long kPackedGainLimit = 1LL << 45;
__device__ __forceinline__ u64 pack_proposal(int label, int target, long long gain) {
    if (target < 0) return 0;
    const u64 head = static_cast<u64>(label & 0xff) | (static_cast<u64>(target & 0xff) << 8) | kProposer;
    if (gain < -kPackedGainLimit || gain >= kPackedGainLimit) return head | kGainApart;
    return head | (static_cast<u64>(gain) << 18);
}
__device__ __forceinline__ long long packed_gain(u64 w, const long long* gains, int u) {
    return (w & kGainApart) ? gains[u] : static_cast<long long>(w) >> 18;
}

// incremental_lp_proposal (incremental.cuh:166-198).  A warp takes 32
// consecutive vertices: each lane reads its vertex's lock, label, own-part
// affinity and row total (coalesced), and only boundary rows are scanned, by
// groups of W lanes, 32/W rows at a time.  Ties keep the lowest part id.
// Proposers are appended with one atomic per block pass (the reference
// appends per warp, append_warp, incremental.cuh:201-208; the order of the
// candidate list does not affect any result).
template <class C, int W, bool Vectorized>
__global__ void __launch_bounds__(kThreads) k_proposals(LpParams q, const C* A, const C* totals, const int* rows,
                                                        const u64* row_count) {
    using Vec = AffinityVec<C>;
    constexpr int N = Vectorized ? Vec::N : 1;
    constexpr int G = 32 / W;
    __shared__ u64 s_slack[kMaxParts];
    __shared__ double s_price[kMaxParts];
    __shared__ unsigned char s_propose[kThreads];
    const int k = q.k;
    if (q.prices)
        for (int p = threadIdx.x; p < k; p += blockDim.x) { s_slack[p] = q.capacity - q.loads[p]; s_price[p] = q.prices[p]; }
    __syncthreads();
    const int lane = threadIdx.x & 31, gid = lane / W, sub = lane % W;
    // Block-uniform passes (the append synchronises the block); warp w of the
    // block takes entries [32w, 32w + 32) of the block's 256: vertices, or
    // positions of `rows` (*row_count entries, the level's frontier) when given.
    const i64 visits = rows ? static_cast<i64>(*row_count) : q.n;
    for (i64 block_base = static_cast<i64>(blockIdx.x) * blockDim.x; block_base < visits;
         block_base += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 index = block_base + threadIdx.x;
        const i64 v = index < visits ? (rows ? rows[index] : index) : q.n;
        int src = 0;
        u64 current = 0;
        bool act = false;
        if (v < q.n) {
            if (q.locks[v]) {
                q.locks[v] = 0;
            } else {
                src = q.labels[v];
                current = A[v * k + src];
                act = current != static_cast<u64>(totals[v]);
            }
            // A gain is read only where the target is set, so only
            // proposers write one.
            if (!act) {
                q.targets[v] = -1;
                q.proposal[v] = 0;
            }
        }
        s_propose[threadIdx.x] = 0;
        __syncwarp();
        unsigned pending = __ballot_sync(0xffffffffu, act);
        while (pending) {
            unsigned mine = pending;
            for (int i = 0; i < gid; ++i) mine &= mine - 1;
            for (int i = 0; i < G; ++i) pending &= pending - 1;
            const int owner = mine ? __ffs(mine) - 1 : -1;
            const int osrc = __shfl_sync(0xffffffffu, src, owner < 0 ? 0 : owner);
            const u64 ocur = __shfl_sync(0xffffffffu, current, owner < 0 ? 0 : owner);
            const i64 vv = __shfl_sync(0xffffffffu, v, owner < 0 ? 0 : owner);
            int target = -1;
            u64 best = 0;
            double best_score = -DBL_MAX;
            if (owner >= 0) {
                const C* row = A + vv * k;
                const u64 weight = q.prices ? q.vw[vv] : 0;
                for (int p0 = sub * N; p0 < k; p0 += W * N) {
                    C val[N];
                    if constexpr (Vectorized) {
                        const typename Vec::V x = *reinterpret_cast<const typename Vec::V*>(row + p0);
                        if constexpr (N == 4) { val[0] = x.x; val[1] = x.y; val[2] = x.z; val[3] = x.w; }
                        else { val[0] = x.x; val[1] = x.y; }
                    } else {
                        val[0] = row[p0];
                    }
#pragma unroll
                    for (int e = 0; e < N; ++e) {
                        const int p = p0 + e;
                        const u64 conn = val[e];
                        if (p == osrc || !conn) continue;
                        if (q.prices) {
                            const double cost = weight > s_slack[p] ? __dmul_rn(s_price[p], static_cast<double>(weight - s_slack[p])) : 0.0;
                            const double score = __dsub_rn(static_cast<double>(conn), cost);
                            if (target < 0 || score > best_score) { target = p; best = conn; best_score = score; }
                        } else if (target < 0 || conn > best) {
                            target = p;
                            best = conn;
                        }
                    }
                }
            }
#pragma unroll
            for (int d = W / 2; d; d >>= 1) {
                const int ot = __shfl_xor_sync(0xffffffffu, target, d, W);
                const u64 ob = __shfl_xor_sync(0xffffffffu, best, d, W);
                const double os = __shfl_xor_sync(0xffffffffu, best_score, d, W);
                if (ot >= 0) {
                    const bool greater = q.prices ? os > best_score : ob > best;
                    const bool equal = q.prices ? os == best_score : ob == best;
                    if (target < 0 || greater || (equal && ot < target)) { target = ot; best = ob; best_score = os; }
                }
            }
            if (owner >= 0 && sub == 0) {
                const bool propose = target >= 0 && (best >= ocur || ocur - best < static_cast<u64>(q.filter * static_cast<double>(ocur)));
                q.targets[vv] = propose ? target : -1;
                const long long gain = best >= ocur ? static_cast<long long>(best - ocur) : -static_cast<long long>(ocur - best);
                if (propose) q.gains[vv] = gain;
                q.proposal[vv] = pack_proposal(osrc, propose ? target : -1, gain);
                s_propose[(threadIdx.x & ~31) + owner] = propose;
            }
        }
        __syncwarp();
        block_append(static_cast<int>(v), s_propose[threadIdx.x] != 0, q.cand, q.counters + 0);
    }
}

// ---------------------------------------------------------------- on-demand affinities

// Levels whose rows are short next to k (a mesh at k = 128: six neighbours
// against 128 cache words) keep no dense cache: a vertex's affinities are
// recomputed from its adjacency where they are needed, one thread per
// vertex.  The values are exactly the cache's, so every decision is the
// same; only the data read differs (the reference likewise switches to a
// sparse/on-demand affinity layout, incremental.cuh:675-741).
constexpr int kOnDemandDegree = 32;

// A row of at most D entries in registers: the part of every neighbour (-1
// for a self loop or an absent entry) and the edge weight; all loads of the
// row are issued together.
template <int D>
struct RowRegs {
    int part[D];
    u64 w[D];
    u64 total;
    __device__ __forceinline__ void load(int v, const int* off, const int* nbr, const u32* ew, const int* labels) {
        const int b = off[v], end = off[v + 1];
        int u[D];
#pragma unroll
        for (int j = 0; j < D; ++j) u[j] = b + j < end ? nbr[b + j] : v;
        total = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            const bool ok = u[j] != v;  // absent entries read as v
            part[j] = ok ? labels[u[j]] : -1;
            w[j] = ok ? edge_w(ew, b + j) : 0;
            total += w[j];
        }
    }
    // Connection to part p (0 without a neighbour in p).
    __device__ __forceinline__ u64 of(int p) const {
        u64 c = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) c += part[j] == p ? w[j] : 0;
        return c;
    }
    // Entry j holds the first occurrence of its part.
    __device__ __forceinline__ bool first(int j) const {
        if (part[j] < 0) return false;
        for (int i = 0; i < j; ++i)
            if (part[i] == part[j]) return false;
        return true;
    }
};

// k_proposals with on-demand affinities: the same target (largest
// affinity, or affinity minus repair price; lowest part on ties), filter
// and outputs.
// `rows` (*row_count entries), when given, lists the vertices to visit (the
// level's frontier); every other vertex is interior and would not propose.
template <int D>
__global__ void __launch_bounds__(kThreads) k_proposals_od(LpParams q, const int* rows, const u64* row_count) {
    __shared__ u64 s_slack[kMaxParts];
    __shared__ double s_price[kMaxParts];
    if (q.prices)
        for (int p = threadIdx.x; p < q.k; p += blockDim.x) { s_slack[p] = q.capacity - q.loads[p]; s_price[p] = q.prices[p]; }
    __syncthreads();
    const i64 visits = rows ? static_cast<i64>(*row_count) : q.n;
    for (i64 block_base = static_cast<i64>(blockIdx.x) * blockDim.x; block_base < visits;
         block_base += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 index = block_base + threadIdx.x;
        const i64 v = index < visits ? (rows ? rows[index] : index) : q.n;
        bool propose = false;
        if (v < q.n) {
            if (q.locks[v]) {
                q.locks[v] = 0;
                q.targets[v] = -1;
                q.proposal[v] = 0;
            } else {
                const int src = q.labels[v];
                RowRegs<D> r;
                r.load(static_cast<int>(v), q.off, q.nbr, q.ew, q.labels);
                const u64 current = r.of(src);
                int target = -1;
                u64 best = 0;
                if (current != r.total) {
                    const u64 weight = q.prices ? q.vw[v] : 0;
                    double best_score = -DBL_MAX;
#pragma unroll
                    for (int i = 0; i < D; ++i) {
                        const int p = r.part[i];
                        if (p == src || !r.first(i)) continue;
                        const u64 conn = r.of(p);
                        if (q.prices) {
                            const double cost = weight > s_slack[p] ? __dmul_rn(s_price[p], static_cast<double>(weight - s_slack[p])) : 0.0;
                            const double score = __dsub_rn(static_cast<double>(conn), cost);
                            if (target < 0 || score > best_score || (score == best_score && p < target)) {
                                target = p; best = conn; best_score = score;
                            }
                        } else if (target < 0 || conn > best || (conn == best && p < target)) {
                            target = p;
                            best = conn;
                        }
                    }
                }
                propose = target >= 0 &&
                          (best >= current || current - best < static_cast<u64>(q.filter * static_cast<double>(current)));
                q.targets[v] = propose ? target : -1;
                const long long gain =
                    best >= current ? static_cast<long long>(best - current) : -static_cast<long long>(current - best);
                if (propose) q.gains[v] = gain;
                q.proposal[v] = pack_proposal(src, propose ? target : -1, gain);
            }
        }
        block_append(static_cast<int>(v), propose, q.cand, q.counters + 0);
    }
}

// Correction of candidate v (part s to t, gain `gain`) from the entries
// first, first + stride, ... < end: the moves of its higher-priority
// neighbours.  Four entries per lane at a time: their neighbour ids first,
// then every neighbour's target, gain and label, all in flight together.
__device__ __forceinline__ long long filter_entries(const LpParams& q, int v, int s, int t, long long gain, int first,
                                                    int end, int stride) {
    constexpr int U = 4;
    long long corr = 0;
    for (int e0 = first; e0 < end; e0 += U * stride) {
        int u[U];
        u64 w[U];
#pragma unroll
        for (int j = 0; j < U; ++j) u[j] = e0 + j * stride < end ? q.nbr[e0 + j * stride] : v;
#pragma unroll
        for (int j = 0; j < U; ++j) w[j] = u[j] != v ? q.proposal[u[j]] : 0;
#pragma unroll
        for (int j = 0; j < U; ++j) {
            if (!(w[j] & kProposer)) continue;
            const long long gu = packed_gain(w[j], q.gains, u[j]);
            if (gu > gain || (gu == gain && u[j] < v)) {
                const int tu = static_cast<int>((w[j] >> 8) & 0xffu), lu = static_cast<int>(w[j] & 0xffu);
                corr += static_cast<long long>(edge_w(q.ew, e0 + j * stride)) *
                        ((tu == t) - (tu == s) - (lu == t) + (lu == s));
            }
        }
    }
    return corr;
}
// incremental_priority_filter (incremental.cuh:361-393): a vertex keeps its
// move when its gain corrected by the intended moves of higher-priority
// neighbours stays non-negative.  A warp takes four candidates at a time: rows of up to kFilterShort
// entries are read by eight lanes each, longer ones (up to heavy_min) by the
// whole warp after them.
constexpr int kFilterShort = 16;
__global__ void __launch_bounds__(kThreads, 6) k_filter(LpParams q) {
    constexpr int W = 8, G = 32 / W;
    const int lane = threadIdx.x & 31, gid = lane / W, sub = lane % W;
    const i64 count = static_cast<i64>(q.counters[0]);
    unsigned leaders = 0;
    for (int g = 0; g < G; ++g) leaders |= 1u << (g * W);
    const i64 warps = (static_cast<i64>(gridDim.x) * blockDim.x) >> 5;
    for (i64 base = ((static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * G; base < count;
         base += warps * G) {
        const i64 i = base + gid;
        const int v = i < count ? q.cand[i] : -1;
        const int begin = v >= 0 ? q.off[v] : 0, end = v >= 0 ? q.off[v + 1] : 0;
        const bool light = v >= 0 && end - begin <= q.heavy_min;  // heavier rows: k_filter_chunks / k_filter_finish
        const int s = light ? q.labels[v] : 0, t = light ? q.targets[v] : 0;
        const long long gain = light ? q.gains[v] : 0;
        long long corr = light && end - begin <= kFilterShort ? filter_entries(q, v, s, t, gain, begin + sub, end, W) : 0;
        for (unsigned rest = __ballot_sync(0xffffffffu, light && end - begin > kFilterShort) & leaders; rest;
             rest &= rest - 1) {
            const int leader = __ffs(rest) - 1;
            const int vv = __shfl_sync(0xffffffffu, v, leader), ss = __shfl_sync(0xffffffffu, s, leader),
                      tt = __shfl_sync(0xffffffffu, t, leader), b = __shfl_sync(0xffffffffu, begin, leader),
                      e = __shfl_sync(0xffffffffu, end, leader);
            const long long gg = __shfl_sync(0xffffffffu, gain, leader);
            const long long c = warp_sum(filter_entries(q, vv, ss, tt, gg, b + lane, e, 32));
            if (lane == leader) corr += c;
        }
#pragma unroll
        for (int d = W / 2; d; d >>= 1) corr += __shfl_xor_sync(0xffffffffu, corr, d, W);
        if (sub == 0 && light) {
            bool keep;
            if (q.prices) {
                const u64 w = q.vw[v];
                const double adj = __dsub_rn(repair_cost(s, w, q.loads, q.capacity, q.prices),
                                             repair_cost(t, w, q.loads, q.capacity, q.prices));
                keep = __dadd_rn(static_cast<double>(gain + corr), adj) >= 0;
            } else keep = gain + corr >= 0;
            q.flags[v] = keep;
        }
    }
}

// k_filter for rows of at most D entries, one thread per candidate (the
// on-demand levels: a warp per six-entry row would leave most lanes idle).
template <int D>
__global__ void __launch_bounds__(kThreads) k_filter_od(LpParams q) {
    const i64 count = static_cast<i64>(q.counters[0]);
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int v = q.cand[i];
        const int s = q.labels[v], t = q.targets[v];
        const long long gain = q.gains[v];
        const int b = q.off[v], end = q.off[v + 1];
        int u[D];
#pragma unroll
        for (int j = 0; j < D; ++j) u[j] = b + j < end ? q.nbr[b + j] : v;
        long long corr = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            if (u[j] == v) continue;
            const int tu = q.targets[u[j]];
            if (tu < 0) continue;
            const long long gu = q.gains[u[j]];
            if (!(gu > gain || (gu == gain && u[j] < v))) continue;
            const int lu = q.labels[u[j]];
            corr += static_cast<long long>(edge_w(q.ew, b + j)) * ((tu == t) - (tu == s) - (lu == t) + (lu == s));
        }
        bool keep;
        if (q.prices) {
            const u64 w = q.vw[v];
            const double adj = __dsub_rn(repair_cost(s, w, q.loads, q.capacity, q.prices),
                                         repair_cost(t, w, q.loads, q.capacity, q.prices));
            keep = __dadd_rn(static_cast<double>(gain + corr), adj) >= 0;
        } else keep = gain + corr >= 0;
        q.flags[v] = keep;
    }
}

// k_update without a cache (on-demand levels), one thread per mover: the
// exact cut change and the repair samples.
template <int D>
__global__ void __launch_bounds__(kThreads) k_update_od(i64 count, const int* movers, const u64* live_count,
                                                        const int* off, const int* nbr, const u32* ew, const u32* vw,
                                                        const int* labels, const int* targets, const int* flags,
                                                        long long* delta, Sample* samples) {
    __shared__ WarpSum delta_sum;
    delta_sum.init();
    if (live_count) count = static_cast<i64>(*live_count);
    long long total = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int v = movers[i];
        const int s = labels[v], t = targets[v];
        const int b = off[v], end = off[v + 1];
        int u[D];
#pragma unroll
        for (int j = 0; j < D; ++j) u[j] = b + j < end ? nbr[b + j] : v;
        long long gain = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            if (u[j] == v) continue;
            const int old = labels[u[j]];
            const bool moves = flags[u[j]] != 0;
            const int nw = moves ? targets[u[j]] : old;
            if (!moves || u[j] > v) gain += static_cast<long long>(edge_w(ew, b + j)) * ((s != old) - (t != nw));
        }
        total += gain;
        if (samples) {
            atomicAdd(reinterpret_cast<u64*>(&samples[s].loss), static_cast<u64>(-gain));
            atomicAdd(&samples[s].weight, static_cast<u64>(vw[v]));
        }
    }
    delta_sum.finish(static_cast<u64>(warp_sum(total)), reinterpret_cast<u64*>(delta));
}

// Conservative frontier of a level (initialize_affinity_frontier and
// AffinityView::touch, incremental.cuh:210-224, affinity.cuh:33-40): every
// vertex that was a boundary vertex at some point of the level, listed once.
// The LP proposals visit only these; a vertex outside it has every
// neighbour in its own part and would not propose.
struct Frontier {
    int* members;  // 1 when listed
    int* rows;
    u64* count;
};
__device__ __forceinline__ void touch(const Frontier& f, int v) {
    if (!f.members[v] && atomicExch(f.members + v, 1) == 0) f.rows[atomicAdd(f.count, 1ULL)] = v;
}
// After a batch of moves: the movers and their neighbours, whose boundary
// status may have changed, join the frontier; a warp per mover, the
// neighbours of heavy movers by k_touch_chunks.
__global__ void k_touch_rows(i64 count, const int* movers, const u64* live_count, const int* off, const int* nbr,
                             int heavy_min, Frontier f) {
    if (live_count) count = static_cast<i64>(*live_count);
    const int lane = threadIdx.x & 31;
    for (i64 i = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; i < count;
         i += (static_cast<i64>(gridDim.x) * blockDim.x) >> 5) {
        const int v = movers[i];
        if (lane == 0) touch(f, v);
        if (off[v + 1] - off[v] > heavy_min) continue;
        for (int e = off[v] + lane; e < off[v + 1]; e += 32) touch(f, nbr[e]);
    }
}
// The chunks of heavy rows of a list (k_heavy_chunk_list) of movers, a block
// per chunk.
__global__ void k_touch_chunks(DGraph g, const int* work, const u64* work_count, Frontier f) {
    const i64 count = static_cast<i64>(*work_count);
    for (i64 w = blockIdx.x; w < count; w += gridDim.x) {
        const int c = work[w], v = g.chunk_row[c];
        for (int e = g.chunk_begin[c] + threadIdx.x; e < chunk_end(g, c, v); e += blockDim.x) touch(f, g.nbr[e]);
    }
}

// The chunks of the heavy rows (more than heavy_min entries) among a list of
// vertices, appended to `work` (at most g.chunks entries; count at
// *work_count, cleared by the caller), so that the chunk kernels visit the
// rows that take part in a batch instead of every chunk of the level.  The
// order of the list does not matter: the chunk kernels only add exact
// integer contributions.
__global__ void k_heavy_chunk_list(i64 count, const int* list, const u64* live_count, DGraph g, int* work,
                                   u64* work_count) {
    if (live_count) count = static_cast<i64>(*live_count);
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int v = list[i];
        const int d = g.off[v + 1] - g.off[v];
        if (d <= g.heavy_min) continue;
        i64 lo = 0, hi = g.heavy_count;  // g.heavy is ascending: find v
        while (lo < hi) {
            const i64 mid = (lo + hi) >> 1;
            if (g.heavy[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        const int c0 = g.heavy_chunk0[lo], chunks = (d + kChunk - 1) / kChunk;
        const u64 base = atomicAdd(reinterpret_cast<unsigned long long*>(work_count), static_cast<unsigned long long>(chunks));
        for (int j = 0; j < chunks; ++j) work[base + static_cast<u64>(j)] = c0 + j;
    }
}
// The initial frontier of an on-demand level: rows whose connection to their
// own part is below their total weight (the proposal's boundary test).
// Every target is reset to -1, as a proposal pass over all rows leaves the
// rows that do not propose.
template <int D>
__global__ void __launch_bounds__(kThreads) k_frontier_init_od(i64 n, const int* off, const int* nbr, const u32* ew,
                                                               const int* labels, int* targets, Frontier f) {
    for (i64 block_base = static_cast<i64>(blockIdx.x) * blockDim.x; block_base < n;
         block_base += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 v = block_base + threadIdx.x;
        bool boundary = false;
        if (v < n) {
            RowRegs<D> r;
            r.load(static_cast<int>(v), off, nbr, ew, labels);
            boundary = r.of(labels[v]) != r.total;
            f.members[v] = boundary;
            targets[v] = -1;
        }
        block_append(static_cast<int>(v), boundary, f.rows, f.count);
    }
}
// The same for a level with a dense cache: own-part affinity below the total.
template <class C>
__global__ void k_frontier_init(i64 n, const C* A, const C* totals, int k, const int* labels, int* targets,
                                Frontier f) {
    for (i64 block_base = static_cast<i64>(blockIdx.x) * blockDim.x; block_base < n;
         block_base += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 v = block_base + threadIdx.x;
        bool boundary = false;
        if (v < n) {
            boundary = A[v * k + labels[v]] != totals[v];
            f.members[v] = boundary;
            targets[v] = -1;
        }
        block_append(static_cast<int>(v), boundary, f.rows, f.count);
    }
}
// Repair donors that are not in the frontier must read as non-proposers
// (target -1) in the next LP round, as after a proposal pass over all rows.
__global__ void k_reset_targets(i64 count, const u32* donors, int* targets) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) targets[donors[i]] = -1;
}

// Heavy candidates: partial corrections per chunk, then the decision
// (incremental_heavy_priority / incremental_finish_heavy_priority,
// incremental.cuh:395-438).
__global__ void k_filter_chunks(DGraph g, LpParams q, long long* corr_acc, const int* work, const u64* work_count) {
    const i64 count = static_cast<i64>(*work_count);
    for (i64 w = blockIdx.x; w < count; w += gridDim.x) {
        const int c = work[w], v = g.chunk_row[c];
        const int t = q.targets[v];
        if (t < 0) continue;
        const int s = q.labels[v];
        const long long gain = q.gains[v];
        // q.nbr and q.ew are g's arrays: four entries per thread in flight.
        long long corr = filter_entries(q, v, s, t, gain, g.chunk_begin[c] + static_cast<int>(threadIdx.x),
                                        chunk_end(g, c, v), static_cast<int>(blockDim.x));
        corr = warp_sum(corr);
        if ((threadIdx.x & 31) == 0 && corr)
            atomicAdd(reinterpret_cast<u64*>(corr_acc + g.chunk_hidx[c]), static_cast<u64>(corr));
    }
}
__global__ void k_filter_finish(i64 count, const int* heavy, const long long* corr_acc, LpParams q) {
    const i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (h >= count) return;
    const int v = heavy[h];
    const int t = q.targets[v];
    if (t < 0) return;
    const int s = q.labels[v];
    const long long total = q.gains[v] + corr_acc[h];
    bool keep;
    if (q.prices) {
        const u64 w = q.vw[v];
        const double adj = __dsub_rn(repair_cost(s, w, q.loads, q.capacity, q.prices),
                                     repair_cost(t, w, q.loads, q.capacity, q.prices));
        keep = __dadd_rn(static_cast<double>(total), adj) >= 0;
    } else keep = total >= 0;
    q.flags[v] = keep;
}

// Packed per-vertex state read by the cache update: bits 0-7 the label,
// bits 8-15 the target and bit 16 set while the vertex is in the batch being
// applied.  One 4-byte gather per neighbour replaces the label, flag and
// target gathers.  k_state_init writes the labels, k_mark_movers adds the
// batch's targets and bits, k_commit leaves each mover's new label.
constexpr u32 kMovingBit = 1u << 16;
__device__ __forceinline__ int state_label(u32 st) { return static_cast<int>(st & 0xffu); }
__device__ __forceinline__ int state_next(u32 st) {  // the label after this batch
    return static_cast<int>((st & kMovingBit) ? (st >> 8) & 0xffu : st & 0xffu);
}

__global__ void k_state_init(i64 n, const int* labels, u32* state) {
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x)
        state[v] = static_cast<u32>(labels[v]);
}

// Cut change and cache updates of the entries first, first + stride, ... <
// end of mover v (part s to part t); four entries per lane at a time, their
// neighbour, weight and state loads all issued before any is used.  An edge
// whose both ends move is counted by its larger endpoint's partner rule.
template <class C>
__device__ __forceinline__ long long update_entries(int v, int s, int t, int first, int end, int stride, const int* nbr,
                                                    const u32* ew, const u32* state, int k, C* A) {
    constexpr int U = 4;
    long long gain = 0;
    for (int e0 = first; e0 < end; e0 += U * stride) {
        int u[U];
        u32 w[U], st[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const int e = e0 + j * stride;
            u[j] = e < end ? nbr[e] : v;
            w[j] = e < end ? edge_w(ew, e) : 0u;
        }
#pragma unroll
        for (int j = 0; j < U; ++j) st[j] = u[j] != v ? state[u[j]] : 0u;
#pragma unroll
        for (int j = 0; j < U; ++j) {
            if (u[j] == v) continue;  // past the row's end, or a self loop
            if (A) {  // no cache with on-demand affinities
                atomicAdd(A + static_cast<i64>(u[j]) * k + s, static_cast<C>(0) - static_cast<C>(w[j]));
                atomicAdd(A + static_cast<i64>(u[j]) * k + t, static_cast<C>(w[j]));
            }
            const bool moves = (st[j] & kMovingBit) != 0;
            if (!moves || u[j] > v)
                gain += static_cast<long long>(w[j]) * ((s != state_label(st[j])) - (t != state_next(st[j])));
        }
    }
    return gain;
}

// Compulsory DRAM bytes of updating one moved row of `entries` entries: the
// mover id, its two offsets, its own label and target, per entry the
// neighbour id (and edge weight) and the read and write of the two cache
// counters it changes.  The neighbours' label, flag and target gathers are
// not counted: those three n-word arrays stay resident in L2.
template <class C>
__device__ __forceinline__ u64 update_row_bytes(int entries, bool weighted, bool cached) {
    return 20ULL + static_cast<u64>(entries) * (4ULL + (weighted ? 4ULL : 0ULL) + (cached ? 4ULL * sizeof(C) : 0ULL));
}

// incremental_update_cache_and_cut (incremental.cuh:440-506): exact cut delta
// and dense cache updates; optional repair samples per source part.  A warp
// takes four movers at a time: rows of up to kUpdateShort entries are done by
// eight lanes each, longer ones (up to heavy_min) by the whole warp after
// them, so a warp's memory chains cover four short rows at once.  With
// `work`, the compulsory bytes of the rows it updated are added there.
constexpr int kUpdateShort = 16;
template <class C>
__global__ void __launch_bounds__(kThreads, 6) k_update(i64 count, const int* movers, const u64* live_count, const int* off, const int* nbr,
                         const u32* ew, const u32* vw, const u32* state, int k, C* A, long long* delta,
                         Sample* samples, const u64* gate, u64 threshold, int heavy_min, u64* work) {
    constexpr int W = 8, G = 32 / W;
    __shared__ WarpSum delta_sum;
    const int lane = threadIdx.x & 31, gid = lane / W, sub = lane % W;
    if (gate && *gate > threshold) return;  // rebuild chosen
    delta_sum.init();
    if (live_count) count = static_cast<i64>(*live_count);
    unsigned leaders = 0;
    for (int g = 0; g < G; ++g) leaders |= 1u << (g * W);
    const i64 warps = (static_cast<i64>(gridDim.x) * blockDim.x) >> 5;
    long long total = 0;
    u64 bytes = 0;
    for (i64 base = ((static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * G; base < count;
         base += warps * G) {
        const i64 i = base + gid;
        const int v = i < count ? movers[i] : -1;
        const int begin = v >= 0 ? off[v] : 0, end = v >= 0 ? off[v + 1] : 0;
        const bool light = v >= 0 && end - begin <= heavy_min;  // heavier rows: k_update_chunks
        if (work && sub == 0 && light) bytes += update_row_bytes<C>(end - begin, ew != nullptr, A != nullptr);
        const u32 sv = light ? state[v] : 0u;
        const int s = state_label(sv), t = static_cast<int>((sv >> 8) & 0xffu);
        long long gain = light && end - begin <= kUpdateShort
                             ? update_entries(v, s, t, begin + sub, end, W, nbr, ew, state, k, A)
                             : 0;
        for (unsigned rest = __ballot_sync(0xffffffffu, light && end - begin > kUpdateShort) & leaders; rest;
             rest &= rest - 1) {
            const int leader = __ffs(rest) - 1;
            const int vv = __shfl_sync(0xffffffffu, v, leader), ss = __shfl_sync(0xffffffffu, s, leader),
                      tt = __shfl_sync(0xffffffffu, t, leader), b = __shfl_sync(0xffffffffu, begin, leader),
                      e = __shfl_sync(0xffffffffu, end, leader);
            const long long g = warp_sum(update_entries(vv, ss, tt, b + lane, e, 32, nbr, ew, state, k, A));
            if (lane == leader) gain += g;
        }
#pragma unroll
        for (int d = W / 2; d; d >>= 1) gain += __shfl_xor_sync(0xffffffffu, gain, d, W);
        if (sub == 0 && light) {
            total += gain;
            if (samples) {
                atomicAdd(reinterpret_cast<u64*>(&samples[s].loss), static_cast<u64>(-gain));
                atomicAdd(&samples[s].weight, static_cast<u64>(vw[v]));
            }
        }
    }
    delta_sum.finish(static_cast<u64>(warp_sum(total)), reinterpret_cast<u64*>(delta));
    if (work) {
        bytes = warp_sum(bytes);
        if (lane == 0 && bytes) atomicAdd(reinterpret_cast<unsigned long long*>(work), bytes);
    }
}

// Heavy movers, chunk-parallel (incremental_heavy_update_cache_and_cut,
// incremental.cuh:508-530): the chunks listed by k_heavy_chunk_list for the
// batch, a block per chunk, each thread with four entries' loads in flight.
template <class C>
__global__ void k_update_chunks(DGraph g, const int* chunk_list, const u64* chunk_count, const u32* state, int k, C* A,
                                long long* delta, Sample* samples, const u64* gate, u64 threshold, u64* work) {
    if (gate && *gate > threshold) return;
    const i64 count = static_cast<i64>(*chunk_count);
    for (i64 w = blockIdx.x; w < count; w += gridDim.x) {
        const int c = chunk_list[w], v = g.chunk_row[c];
        const u32 sv = state[v];
        if (work && threadIdx.x == 0)  // the chunk's entries, its row, begin and row id (no per-row mover id)
            atomicAdd(reinterpret_cast<unsigned long long*>(work),
                      update_row_bytes<C>(chunk_end(g, c, v) - g.chunk_begin[c], g.ew != nullptr, true) - 8ULL);
        const int s = state_label(sv), t = static_cast<int>((sv >> 8) & 0xffu);
        long long gain = update_entries(v, s, t, g.chunk_begin[c] + static_cast<int>(threadIdx.x), chunk_end(g, c, v),
                                        static_cast<int>(blockDim.x), g.nbr, g.ew, state, k, A);
        gain = block_sum(gain);
        if (threadIdx.x == 0 && gain) {
            atomicAdd(reinterpret_cast<u64*>(delta), static_cast<u64>(gain));
            if (samples) atomicAdd(reinterpret_cast<u64*>(&samples[s].loss), static_cast<u64>(-gain));
        }
        if (samples && threadIdx.x == 0 && g.chunk_begin[c] == g.off[v])
            atomicAdd(&samples[s].weight, static_cast<u64>(g.vw[v]));
    }
}

// Entries of the rows of a mover list: decides between updating the cache
// entry by entry and rebuilding it after the commit.
// Also marks the batch in the packed state (target and batch bit).
__global__ void k_mark_movers(i64 count, const int* movers, const u64* live_count, const int* off, const int* targets,
                              u32* state, u64* out) {
    if (live_count) count = static_cast<i64>(*live_count);
    u64 entries = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int v = movers[i];
        if (state) state[v] = (state[v] & 0xffu) | (static_cast<u32>(targets[v] & 0xff) << 8) | kMovingBit;
        if (out) entries += static_cast<u64>(off[v + 1] - off[v]);
    }
    if (out) block_atomic_add(out, entries);
}

// Candidates with a kept move -> mover list (incremental_compact_candidates).
// With `state`, also what k_mark_movers does for the list: marks each mover
// in the packed state and adds its row's entries to *entries (the rebuild
// gate), so the batch needs no separate marking launch.
__global__ void k_compact_movers(LpParams q, u32* state, u64* entries) {
    const i64 count = static_cast<i64>(q.counters[0]);
    u64 mine = 0;
    for (i64 base = static_cast<i64>(blockIdx.x) * blockDim.x; base < count; base += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 i = base + threadIdx.x;
        const int v = i < count ? q.cand[i] : 0;
        const bool keep = i < count && q.flags[v];
        if (keep && state) {
            state[v] = (state[v] & 0xffu) | (static_cast<u32>(q.targets[v] & 0xff) << 8) | kMovingBit;
            mine += static_cast<u64>(q.off[v + 1] - q.off[v]);
        }
        block_append(v, keep, q.movers, q.counters + 1);
    }
    if (entries) block_atomic_add(entries, mine);
}

// incremental_commit (incremental.cuh:532-547) with per-block aggregation of
// the part-load changes.
// Also keeps rlabels (the labels in repair order, rposition[v] the place of
// v) current and clears each mover's flag.  The last block to finish (a
// counter that every block increments once after its load changes; that
// block resets it for the next launch) writes the largest part load to
// *max_load, so no separate launch reads the loads back.
__global__ void k_commit(i64 count, const int* movers, const u64* live_count, int* labels, const int* targets,
                         const u32* vw, int k, u64* loads, unsigned char* locks, int* flags, const u32* rposition,
                         int* rlabels, u32* state, u64* max_load, unsigned int* blocks_done) {
    extern __shared__ long long diff[];
    __shared__ bool last;
    if (live_count) count = static_cast<i64>(*live_count);
    for (int p = threadIdx.x; p < k; p += blockDim.x) diff[p] = 0;
    __syncthreads();
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int v = movers[i];
        const int s = labels[v], t = targets[v];
        const long long w = vw[v];
        atomicAdd(reinterpret_cast<u64*>(diff + s), static_cast<u64>(-w));
        atomicAdd(reinterpret_cast<u64*>(diff + t), static_cast<u64>(w));
        labels[v] = t;
        rlabels[rposition[v]] = t;
        if (state) state[v] = static_cast<u32>(t);
        if (locks) locks[v] = 1;
        flags[v] = 0;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x)
        if (diff[p]) atomicAdd(loads + p, static_cast<u64>(diff[p]));
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(blocks_done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last || threadIdx.x >= 32) return;
    __threadfence();
    u64 m = 0;
    for (int p = threadIdx.x; p < k; p += 32) m = max(m, __ldcg(loads + p));
    m = warp_max(m);
    if (threadIdx.x == 0) {
        *max_load = m;
        *blocks_done = 0;
    }
}

// ---------------------------------------------------------------- repair

// Deterministic gain bucket: smallest j with 1.5^j >= (current-best)/relief,
// evaluated exactly (balance_gain_bucket, incremental.cuh:553-557, computes
// the same ceil(log(x)/log(1.5)) in floating point).  1.5^j >= G/R is
// 3^j R >= 2^j G for j >= 0 and 2^-j R >= 3^-j G for j < 0; a binary search
// over j in [-23, 24] with 128-bit products settles it.
__constant__ u64 c_pow3[25] = {1ULL, 3ULL, 9ULL, 27ULL, 81ULL, 243ULL, 729ULL, 2187ULL, 6561ULL, 19683ULL,
                               59049ULL, 177147ULL, 531441ULL, 1594323ULL, 4782969ULL, 14348907ULL, 43046721ULL,
                               129140163ULL, 387420489ULL, 1162261467ULL, 3486784401ULL, 10460353203ULL,
                               31381059609ULL, 94143178827ULL, 282429536481ULL};
__device__ __forceinline__ bool bucket_reaches(int j, u64 G, u64 R) {
    const int a = j < 0 ? -j : j;
    const unsigned __int128 p3 = c_pow3[a], p2 = static_cast<unsigned __int128>(1) << a;
    return j >= 0 ? static_cast<unsigned __int128>(R) * p3 >= static_cast<unsigned __int128>(G) * p2
                  : static_cast<unsigned __int128>(R) * p2 >= static_cast<unsigned __int128>(G) * p3;
}
__device__ int gain_bucket(u64 best, u64 current, u64 relief) {
    if (best > current) return 0;
    if (best == current) return 1;
    const u64 G = current - best, R = relief;
    if (!bucket_reaches(24, G, R)) return 49;
    int lo = -23, hi = 24;  // smallest j in [lo, hi] that reaches
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (bucket_reaches(mid, G, R)) hi = mid; else lo = mid + 1;
    }
    return max(2, min(49, 25 + lo));
}

// initialize_receiver_slack (rebalance_select.cuh:79-104) by one thread.
// One thread per part; the CDF is a saturating prefix sum over the parts.
__device__ __forceinline__ u64 saturating_add(u64 a, u64 b) { return ~0ULL - a < b ? ~0ULL : a + b; }
__global__ void __launch_bounds__(kMaxParts) k_slack(int k, const u64* loads, u64 capacity, u64* slack, u64* requests,
                                                     u64* cdf) {
    __shared__ u64 warp_total[kMaxParts / 32], warp_min[kMaxParts / 32];
    const int p = threadIdx.x, lane = p & 31, warp = p >> 5;
    const u64 room = p < k ? (loads[p] < capacity ? capacity - loads[p] : 0) : 0;
    u64 inc = room, least = room ? room : ~0ULL;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const u64 o = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc = saturating_add(inc, o);
        const u64 m = __shfl_xor_sync(0xffffffffu, least, d);
        least = m < least ? m : least;
    }
    if (lane == 31) warp_total[warp] = inc;
    if (lane == 0) warp_min[warp] = least;
    __syncthreads();
    u64 before = 0;
    for (int w = 0; w < warp; ++w) before = saturating_add(before, warp_total[w]);
    if (p < k) {
        slack[p] = room;
        requests[p] = 0;
        cdf[p] = saturating_add(before, inc);
    }
    if (p == 0) {
        u64 m = ~0ULL;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = warp_min[w] < m ? warp_min[w] : m;
        cdf[k] = m;
    }
}

// Position i of the repair order is a donor when its vertex's part is
// overloaded; rlabels holds the labels in repair order, so this reads
// sequentially.
struct IsDonor {
    const int* rlabels;
    const u64* loads;
    u64 capacity;
    __device__ bool operator()(i64 i) const { return loads[rlabels[i]] > capacity; }
};
// Labels in repair order, and each vertex's position in that order.
__global__ void k_repair_positions(i64 n, const u32* order, const int* labels, u32* position, int* rlabels) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 v = order[i];
    position[v] = static_cast<u32>(i);
    rlabels[i] = labels[v];
}
struct WriteOrdered {
    const u32* order;
    u32* out;
    __device__ void operator()(u32 slot, i64 i) const { out[slot] = order[i]; }
};

// Loads N consecutive affinities of a row (one 16-byte load when N > 1).
template <class C, int N>
__device__ __forceinline__ void load_affinities(const C* p, C (&val)[N]) {
    if constexpr (N == 1) {
        val[0] = *p;
    } else {
        const typename AffinityVec<C>::V x = *reinterpret_cast<const typename AffinityVec<C>::V*>(p);
        if constexpr (N == 4) { val[0] = x.x; val[1] = x.y; val[2] = x.z; val[3] = x.w; }
        else { val[0] = x.x; val[1] = x.y; }
    }
}

// enumerate_repair_destination (rebalance_select.cuh:9-75), dense layout, plus
// the bucket of incremental_rebalance_proposals (incremental.cuh:559-622).
// W lanes per donor; the parts' free room is staged per block.  A part p is a
// feasible destination for weight w when w <= room[p] (room = C - load for
// parts under capacity, else 0; vertex weights are positive).
template <class C, int W, bool Vectorized>
__global__ void __launch_bounds__(kThreads) k_repair_dest(i64 count, const u32* donors, const C* A, const C* totals,
                                                          const int* labels, const u32* vw, int k, const u64* loads,
                                                          u64 capacity, const u64* cdf, int* targets, u64* bucket_keys) {
    constexpr int N = Vectorized ? AffinityVec<C>::N : 1;
    constexpr int G = 32 / W;
    __shared__ u64 s_room[kMaxParts];
    for (int p = threadIdx.x; p < k; p += blockDim.x) s_room[p] = loads[p] < capacity ? capacity - loads[p] : 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, gid = lane / W, sub = lane % W;
    const i64 warps = (static_cast<i64>(gridDim.x) * blockDim.x) >> 5;
    const int span = (k + W - 1) / W;  // contiguous parts per lane for the fallback ticket
    for (i64 i0 = ((static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * G; i0 < count; i0 += warps * G) {
        const i64 i = i0 + gid;
        const bool valid = i < count;
        const int v = valid ? static_cast<int>(donors[i]) : 0;
        const int src = valid ? labels[v] : 0;
        const u64 w = valid ? vw[v] : 0;
        const u64 current = valid ? static_cast<u64>(A[static_cast<i64>(v) * k + src]) : 0;
        const bool scan = valid && current != static_cast<u64>(totals[v]);
        int part = -1;
        u64 conn = 0, best_room = 0;
        if (scan) {
            const C* row = A + static_cast<i64>(v) * k;
            for (int p0 = sub * N; p0 < k; p0 += W * N) {
                C val[N];
                load_affinities<C, N>(row + p0, val);
#pragma unroll
                for (int e = 0; e < N; ++e) {
                    const int p = p0 + e;
                    const u64 room = s_room[p];
                    if (p == src || w > room) continue;
                    const u64 value = val[e];
                    if (part < 0 || value > conn || (value == conn && room > best_room)) { part = p; conn = value; best_room = room; }
                }
            }
        }
#pragma unroll
        for (int d = W / 2; d; d >>= 1) {
            const int op = __shfl_xor_sync(0xffffffffu, part, d, W);
            const u64 oc = __shfl_xor_sync(0xffffffffu, conn, d, W);
            const u64 orm = __shfl_xor_sync(0xffffffffu, best_room, d, W);
            if (op >= 0 && (part < 0 || oc > conn || (oc == conn && (orm > best_room || (orm == best_room && op < part))))) {
                part = op; conn = oc; best_room = orm;
            }
        }
        if (!conn) part = -1;
        // Fallback ticket over the parts' room when no connected destination
        // fits: from the slack CDF when the source is at capacity, else over
        // the parts that fit w, in part order (saturating sums).
        const bool ticket = valid && part < 0 && !(loads[src] >= capacity && w <= cdf[k]);
        const u32 hash = mix32(static_cast<u32>(v));
        if (__any_sync(0xffffffffu, ticket)) {
            const int lo = sub * span, hi = min(k, lo + span);
            u64 mine = 0;
            if (ticket)
                for (int p = lo; p < hi; ++p)
                    if (p != src && w <= s_room[p]) mine = ~0ULL - mine < s_room[p] ? ~0ULL : mine + s_room[p];
            u64 upto = mine;  // inclusive scan over the group, saturating
#pragma unroll
            for (int d = 1; d < W; d <<= 1) {
                const u64 o = __shfl_up_sync(0xffffffffu, upto, d, W);
                if (sub >= d) upto = ~0ULL - upto < o ? ~0ULL : upto + o;
            }
            const u64 total = __shfl_sync(0xffffffffu, upto, W - 1, W);
            // Exclusive prefix, saturated: exact for the lane holding the
            // ticket (ticket < total), above the ticket for every later lane.
            const u64 prev = __shfl_up_sync(0xffffffffu, upto, 1, W);
            const u64 before = sub == 0 ? 0 : prev;
            int found = -1;
            if (ticket && total) {
                u64 t = static_cast<u64>(hash) % total;
                if (t >= before && (t - before) < mine) {
                    t -= before;
                    for (int p = lo; p < hi; ++p)
                        if (p != src && w <= s_room[p]) {
                            if (t < s_room[p]) { found = p; break; }
                            t -= s_room[p];
                        }
                }
            }
#pragma unroll
            for (int d = W / 2; d; d >>= 1) found = max(found, __shfl_xor_sync(0xffffffffu, found, d, W));
            if (ticket) part = found;
        }
        if (valid && sub == 0) {
            if (part < 0 && !ticket) {
                conn = 0;
                if (loads[src] >= capacity && w <= cdf[k]) {
                    const u64 sum = cdf[k - 1];
                    if (sum) {
                        const u64 t = static_cast<u64>(hash) % sum;
                        int lo = 0, hi = k;
                        while (lo < hi) { const int mid = (lo + hi) / 2; if (cdf[mid] <= t) lo = mid + 1; else hi = mid; }
                        part = lo;
                    }
                }
            }
            if (ticket) conn = 0;
            targets[v] = part;
            u64 key = ~0ULL;
            if (part >= 0) {
                const u64 excess = loads[src] - capacity;
                const u64 relief = w < excess ? w : excess;
                key = static_cast<u64>(src) * kBalanceWidth + gain_bucket(conn, current, relief) * 16 +
                      mix32(static_cast<u32>(v)) % 16;
            }
            bucket_keys[i] = key;
        }
    }
}

// k_repair_dest with on-demand affinities, one thread per donor: the best
// connected destination with room (largest affinity, then room, then lowest
// part), else the same fallback tickets.
template <int D>
__global__ void __launch_bounds__(kThreads) k_repair_dest_od(i64 count, const u32* donors, const int* off,
                                                             const int* nbr, const u32* ew, const int* labels,
                                                             const u32* vw, int k, const u64* loads, u64 capacity,
                                                             const u64* cdf, int* targets, u64* bucket_keys) {
    __shared__ u64 s_room[kMaxParts];
    for (int p = threadIdx.x; p < k; p += blockDim.x) s_room[p] = loads[p] < capacity ? capacity - loads[p] : 0;
    __syncthreads();
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int v = static_cast<int>(donors[i]);
        const int src = labels[v];
        const u64 w = vw[v];
        RowRegs<D> r;
        r.load(v, off, nbr, ew, labels);
        const u64 current = r.of(src);
        int part = -1;
        u64 conn = 0, best_room = 0;
        if (current != r.total)
#pragma unroll
            for (int j = 0; j < D; ++j) {
                const int p = r.part[j];
                if (p < 0 || p == src || !r.first(j)) continue;
                const u64 room = s_room[p];
                if (w > room) continue;
                const u64 value = r.of(p);
                if (part < 0 || value > conn || (value == conn && (room > best_room || (room == best_room && p < part)))) {
                    part = p; conn = value; best_room = room;
                }
            }
        if (!conn) part = -1;
        if (part < 0) {
            conn = 0;
            const u32 hash = mix32(static_cast<u32>(v));
            if (loads[src] >= capacity && w <= cdf[k]) {
                const u64 sum = cdf[k - 1];
                if (sum) {
                    const u64 t = static_cast<u64>(hash) % sum;
                    int lo = 0, hi = k;
                    while (lo < hi) { const int mid = (lo + hi) / 2; if (cdf[mid] <= t) lo = mid + 1; else hi = mid; }
                    part = lo;
                }
            } else {
                u64 total = 0;
                for (int p = 0; p < k; ++p)
                    if (p != src && w <= s_room[p]) total = ~0ULL - total < s_room[p] ? ~0ULL : total + s_room[p];
                if (total) {
                    u64 t = static_cast<u64>(hash) % total;
                    for (int p = 0; p < k; ++p)
                        if (p != src && w <= s_room[p]) {
                            if (t < s_room[p]) { part = p; break; }
                            t -= s_room[p];
                        }
                }
            }
        }
        targets[v] = part;
        u64 key = ~0ULL;
        if (part >= 0) {
            const u64 excess = loads[src] - capacity;
            const u64 relief = w < excess ? w : excess;
            key = static_cast<u64>(src) * kBalanceWidth + gain_bucket(conn, current, relief) * 16 + mix32(static_cast<u32>(v)) % 16;
        }
        bucket_keys[i] = key;
    }
}

// Receiver choice of one donor with on-demand affinities (k_choose, attempt
// > 0): among parts other than its own, not yet tried, whose remaining room
// holds it, the largest affinity, then the largest room, then the lowest
// part.  Parts without a neighbour have affinity 0.
template <int D>
__device__ __forceinline__ int choose_od(int v, const int* off, const int* nbr, const u32* ew, const int* labels,
                                         int k, u64 w, u64 t0, u64 t1, const u64* avail) {
    RowRegs<D> r;
    r.load(v, off, nbr, ew, labels);
    const int src = labels[v];
    int target = -1;
    u64 best = 0, room = 0;
    for (int p = 0; p < k; ++p) {
        if (p == src || (((p < 64 ? t0 : t1) >> (p & 63)) & 1)) continue;
        const u64 a = avail[p];
        if (a < w) continue;
        const u64 c = r.of(p);
        if (target < 0 || c > best || (c == best && a > room)) { target = p; best = c; room = a; }
    }
    return target;
}

template <int D>
__global__ void __launch_bounds__(kThreads) k_choose_od(i64 count, const u32* active, int attempt, const int* off,
                                                        const int* nbr, const u32* ew, const int* labels,
                                                        const u32* vw, int k, const int* proposal, const u64* slack,
                                                        const u64* requests, const u64* tried, unsigned char* state,
                                                        int* want, u64* requesters) {
    __shared__ u64 s_avail[kMaxParts];
    for (int p = threadIdx.x; p < k; p += blockDim.x) s_avail[p] = requests[p] < slack[p] ? slack[p] - requests[p] : 0;
    __syncthreads();
    u64 asked = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        if (state[i]) {
            want[i] = -1;
            continue;
        }
        const int v = static_cast<int>(active[i]);
        const int target = attempt == 0 ? proposal[v]
                                        : choose_od<D>(v, off, nbr, ew, labels, k, vw[v], tried[2 * i], tried[2 * i + 1], s_avail);
        want[i] = target;
        if (target < 0) state[i] = 2;
        else ++asked;
    }
    block_atomic_add(requesters, asked);
}

constexpr u64 kNoBucket = 0xffffffULL;  // donors without a destination sort last

__global__ void k_clamp_keys(i64 count, u64* keys) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count && keys[i] > kNoBucket) keys[i] = kNoBucket;
}
__global__ void k_repair_keys(i64 n, u64* keys, u32* order) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    keys[v] = repair_hash(static_cast<int>(v));
    order[v] = static_cast<u32>(v);
}

struct SortedWeight {
    const u32* items;
    const u32* vw;
    __device__ u64 operator()(i64 i) const { return vw[items[i]]; }
};

// Segment base per source part over the bucket-sorted donors.
__global__ void k_part_heads(i64 count, const u64* keys, const u64* prefix, u64* part_base) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count || keys[i] == kNoBucket) return;
    const u64 part = keys[i] / kBalanceWidth;
    if (i == 0 || keys[i - 1] / kBalanceWidth != part) part_base[part] = prefix[i];
}
// reserve_receiver_prefixes' donor test (rebalance_graph.cuh:104-107).
__global__ void k_donor_test(i64 count, const u64* keys, const u32* items, const u64* prefix, const u64* part_base,
                             const u64* loads, u64 capacity, unsigned char* active) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int v = static_cast<int>(items[i]);
    if (keys[i] == kNoBucket) { active[v] = 0; return; }
    const u64 part = keys[i] / kBalanceWidth;
    active[v] = prefix[i] - part_base[part] < loads[part] - capacity;
}
struct IsActive {
    const u32* donors;
    const unsigned char* active;
    __device__ bool operator()(i64 i) const { return active[donors[i]] != 0; }
};
struct WriteFrom {
    const u32* src;
    u32* out;
    __device__ void operator()(u32 slot, i64 i) const { out[slot] = src[i]; }
};

// One attempt of the receiver reservation: choose a part for every active,
// unplaced donor (attempt 0: its proposal; later: best affinity among parts
// not yet tried whose remaining virtual room holds it).  W lanes per donor;
// the parts' remaining room is staged per block.
template <class C, int W, bool Vectorized>
__global__ void __launch_bounds__(kThreads) k_choose(i64 count, const u32* active, int attempt, const C* A,
                                                     const int* labels, const u32* vw, int k, const int* proposal,
                                                     const u64* slack, const u64* requests, u64* tried,
                                                     unsigned char* state, int* want, u64* requesters) {
    constexpr int N = Vectorized ? AffinityVec<C>::N : 1;
    constexpr int G = 32 / W;
    __shared__ u64 s_avail[kMaxParts];
    for (int p = threadIdx.x; p < k; p += blockDim.x) s_avail[p] = requests[p] < slack[p] ? slack[p] - requests[p] : 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, gid = lane / W, sub = lane % W;
    const i64 warps = (static_cast<i64>(gridDim.x) * blockDim.x) >> 5;
    u64 asked = 0;
    for (i64 i0 = ((static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * G; i0 < count; i0 += warps * G) {
        const i64 i = i0 + gid;
        const bool valid = i < count;
        const unsigned char st = valid ? state[i] : 1;  // placed or out of options
        const bool open = valid && !st;
        const int v = open ? static_cast<int>(active[i]) : 0;
        int target = -1;
        if (attempt == 0) {
            if (open) target = proposal[v];
        } else {
            u64 best = 0, room = 0;
            if (open) {
                const u64 w = vw[v];
                const int src = labels[v];
                const u64 t0 = tried[2 * i], t1 = tried[2 * i + 1];
                const C* row = A + static_cast<i64>(v) * k;
                for (int p0 = sub * N; p0 < k; p0 += W * N) {
                    C val[N];
                    load_affinities<C, N>(row + p0, val);
#pragma unroll
                    for (int e = 0; e < N; ++e) {
                        const int p = p0 + e;
                        if (p == src || (((p < 64 ? t0 : t1) >> (p & 63)) & 1)) continue;
                        const u64 avail = s_avail[p];
                        if (avail < w) continue;
                        const u64 c = val[e];
                        if (target < 0 || c > best || (c == best && avail > room)) { target = p; best = c; room = avail; }
                    }
                }
            }
#pragma unroll
            for (int d = W / 2; d; d >>= 1) {
                const int ot = __shfl_xor_sync(0xffffffffu, target, d, W);
                const u64 ob = __shfl_xor_sync(0xffffffffu, best, d, W);
                const u64 orr = __shfl_xor_sync(0xffffffffu, room, d, W);
                if (ot >= 0 && (target < 0 || ob > best || (ob == best && (orr > room || (orr == room && ot < target))))) {
                    target = ot; best = ob; room = orr;
                }
            }
        }
        if (valid && sub == 0) {
            if (!open) {
                want[i] = -1;
            } else {
                want[i] = target;
                if (target < 0) state[i] = 2;
                else ++asked;
            }
        }
    }
    block_atomic_add(requesters, asked);
}

struct WriteIdx {
    u32* out;
    __device__ void operator()(u32 slot, i64 i) const { out[slot] = static_cast<u32>(i); }
};
// reserve_receiver_prefixes' ticket rule (rebalance_graph.cuh:127-153): a
// donor asking for part t is admitted when its weighted range [begin,
// begin + w) lies inside the part's immutable room, begin being the weight
// already requested for t plus the weight asked for t by the donors before
// it in repair order (the active donors' order).  Every asked weight is
// added to the part's requests, admitted or not.  Without sorting the
// requests by part: each tile of kAdmitTile donors sums the weight asked per
// part (k_part_requests), an exclusive scan over the part-major array of
// tile sums gives every tile its start per part, and k_admit_tiles finishes
// the order inside the tile (earlier warps, then earlier lanes).
constexpr int kAdmitTile = kThreads;
__global__ void k_part_requests(i64 count, const int* want, const u32* active, const u32* vw, int k, int tiles,
                                u64* tile_sums) {
    __shared__ u64 s_sum[kMaxParts];
    for (int p = threadIdx.x; p < k; p += blockDim.x) s_sum[p] = 0;
    __syncthreads();
    const i64 i = static_cast<i64>(blockIdx.x) * kAdmitTile + threadIdx.x;
    const int t = i < count ? want[i] : -1;
    const u64 w = t >= 0 ? vw[active[i]] : 0;
    const unsigned peers = __match_any_sync(0xffffffffu, t);
    u64 sum = 0;
    for (unsigned rest = peers; rest; rest &= rest - 1) sum += __shfl_sync(peers, w, __ffs(rest) - 1);
    if (t >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(reinterpret_cast<unsigned long long*>(s_sum + t), sum);
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x)
        tile_sums[static_cast<i64>(p) * tiles + blockIdx.x] = s_sum[p];
}
// `offsets`: the exclusive scan of tile_sums (part-major), so the weight
// asked for part t by the tiles before this one is offsets[t * tiles + tile]
// - offsets[t * tiles].
// The last block to finish (a finished-block counter, zero between
// launches) then adds every weight asked this attempt to its part's
// requests: per part, the scan's span over that part's tiles (the last part
// ends at the scan total).
__global__ void k_admit_tiles(i64 count, const int* want, const u32* active, const u32* vw, const u64* offsets,
                              const u64* total, int tiles, const u64* slack, u64* requests, u64* tried,
                              unsigned char* state, int* targets, int* flags, int k, unsigned int* blocks_done) {
    __shared__ bool last;
    constexpr int kWarps = kAdmitTile / 32;
    __shared__ u64 s_warp[kMaxParts][kWarps];  // per part, the weight each warp asks (then its start)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int x = threadIdx.x; x < k * kWarps; x += blockDim.x) s_warp[x / kWarps][x % kWarps] = 0;
    __syncthreads();
    const i64 i = static_cast<i64>(blockIdx.x) * kAdmitTile + threadIdx.x;
    const int t = i < count ? want[i] : -1;
    const int v = t >= 0 ? static_cast<int>(active[i]) : 0;
    const u64 w = t >= 0 ? vw[v] : 0;
    const unsigned peers = __match_any_sync(0xffffffffu, t);
    u64 before = 0, sum = 0;
    for (unsigned rest = peers; rest; rest &= rest - 1) {
        const int l = __ffs(rest) - 1;
        const u64 o = __shfl_sync(peers, w, l);
        sum += o;
        if (l < lane) before += o;
    }
    if (t >= 0 && lane == __ffs(peers) - 1) s_warp[t][warp] = sum;
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        u64 run = offsets[static_cast<i64>(p) * tiles + blockIdx.x] - offsets[static_cast<i64>(p) * tiles];
        for (int w2 = 0; w2 < kWarps; ++w2) {
            const u64 x = s_warp[p][w2];
            s_warp[p][w2] = run;
            run += x;
        }
    }
    __syncthreads();
    if (t >= 0) {
        tried[2 * i + (t >> 6)] |= 1ULL << (t & 63);
        const u64 begin = requests[t] + s_warp[t][warp] + before;
        if (begin <= slack[t] && w <= slack[t] - begin) {
            targets[v] = t;
            flags[v] = 1;
            state[i] = 1;
        }
    }
    __syncthreads();  // every read of `requests` in this block is done
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(blocks_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        const u64 first = offsets[static_cast<i64>(p) * tiles];
        const u64 end = p + 1 < k ? offsets[static_cast<i64>(p + 1) * tiles] : *total;
        requests[p] += end - first;
    }
    if (threadIdx.x == 0) *blocks_done = 0;
}
// The remaining attempts of a receiver reservation by one block, for a small
// set of open donors: the choice of k_choose and the ticket rule of k_admit,
// attempt after attempt, without a round trip to the host.  open[j] (j <
// *count, ascending) indexes the active donors, so the requests of one target
// are admitted in repair order exactly as the device-wide path does.
//
// Everything an attempt reads about a donor (vertex, weight, part, state,
// tried parts) sits in dynamic shared memory for the whole launch; state and
// tried go back to global memory at the end.  A donor's choice is the
// eligible part (not its own, not tried, room for its weight) of largest
// (affinity, room, -part).  Parts only leave eligibility during a launch
// (tried parts stay tried, rooms only shrink), so a full scan of the
// donor's affinity row also keeps a shortlist: the four eligible parts of
// largest (affinity, -part) and the largest affinity among the other
// eligible parts.  A later attempt whose best listed part, still eligible,
// has an affinity above that bound takes it without reading the row again
// (no unlisted part can reach or tie it).  When the bound is 0 and no
// eligible listed part has more, every eligible part has affinity 0 and the
// choice is the eligible part of most room: the first one in the attempt's
// order of parts by (room desc, part asc).  Otherwise the row is scanned
// anew.  Admission turns the per-warp request sums of a chunk into per-part
// prefixes once (a thread per part), so a request reads its start directly.
constexpr int kAttemptThreads = 1024;
constexpr int kAttemptCap = 2048;  // open donors handled by one block
constexpr int kShortlist = 4;
constexpr unsigned char kNoPart = 0xff;
// Dynamic shared memory of k_attempts for `count` donors (cache type C).
template <class C>
constexpr size_t attempt_smem(int count) {
    return static_cast<size_t>(count) * (2 * sizeof(u64) + (kShortlist + 1) * sizeof(C) + 2 * sizeof(u32) +
                                         4 + kShortlist);
}
template <class C, int D>
__global__ void __launch_bounds__(kAttemptThreads) k_attempts(const u32* open, const u32* count_ptr, int first_attempt,
                                                              const u32* active, const C* A, const int* off,
                                                              const int* nbr, const u32* ew, const int* labels,
                                                              const u32* vw, int k, const int* proposal,
                                                              const u64* slack, u64* requests, u64* tried,
                                                              unsigned char* state, int* targets, int* flags) {
    constexpr int kWarps = kAttemptThreads / 32;
    __shared__ u64 s_slack[kMaxParts], s_requests[kMaxParts], s_base[kMaxParts], s_avail[kMaxParts];
    __shared__ u64 s_warp[kMaxParts][kWarps];  // per part, the weight each warp requests
    __shared__ int s_want[kAttemptCap];
    __shared__ unsigned char s_order[kMaxParts];  // parts by (room desc, part asc), per attempt
    __shared__ int s_any;
    extern __shared__ __align__(16) unsigned char attempt_smem_raw[];
    const int count = static_cast<int>(*count_ptr);
    // Per-donor arrays (j < count), widest first.
    u64* d_tried = reinterpret_cast<u64*>(attempt_smem_raw);          // 2 per donor
    C* d_list_c = reinterpret_cast<C*>(d_tried + 2 * count);           // kShortlist per donor
    C* d_bound = d_list_c + kShortlist * count;                         // largest unlisted affinity
    u32* d_v = reinterpret_cast<u32*>(d_bound + count);
    u32* d_w = d_v + count;
    unsigned char* d_src = reinterpret_cast<unsigned char*>(d_w + count);
    unsigned char* d_state = d_src + count;
    unsigned char* d_list_n = d_state + count;  // listed parts; kNoPart: no shortlist yet
    unsigned char* d_bounded = d_list_n + count;  // 1 when some eligible part is unlisted
    unsigned char* d_list_p = d_bounded + count;  // kShortlist per donor
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int p = threadIdx.x; p < k; p += blockDim.x) { s_slack[p] = slack[p]; s_requests[p] = requests[p]; }
    for (int j = threadIdx.x; j < count; j += blockDim.x) {
        const u32 i = open[j];
        const u32 v = active[i];
        d_v[j] = v;
        d_w[j] = vw[v];
        d_src[j] = static_cast<unsigned char>(labels[v]);
        d_state[j] = state[i];
        d_tried[2 * j] = tried[2 * i];
        d_tried[2 * j + 1] = tried[2 * i + 1];
        d_list_n[j] = kNoPart;
    }
    __syncthreads();
    for (int attempt = first_attempt; attempt < k; ++attempt) {
        if (threadIdx.x == 0) s_any = 0;
        for (int p = threadIdx.x; p < k; p += blockDim.x)
            s_avail[p] = s_requests[p] < s_slack[p] ? s_slack[p] - s_requests[p] : 0;
        __syncthreads();
        if (attempt > 0 && A) {
            // Rank of part p: the parts before it, counted by 8 lanes.
            const int p = threadIdx.x >> 3, sub = threadIdx.x & 7;
            int rank = 0;
            if (p < k) {
                const u64 a = s_avail[p];
                for (int q = sub; q < k; q += 8) rank += s_avail[q] > a || (s_avail[q] == a && q < p);
            }
            rank += __shfl_xor_sync(0xffffffffu, rank, 1);
            rank += __shfl_xor_sync(0xffffffffu, rank, 2);
            rank += __shfl_xor_sync(0xffffffffu, rank, 4);
            if (p < k && sub == 0) s_order[rank] = static_cast<unsigned char>(p);
            __syncthreads();
        }
        // Choice (k_choose).
        for (int j = threadIdx.x; j < count; j += blockDim.x) {
            int target = -1;
            if (!d_state[j]) {
                const int v = static_cast<int>(d_v[j]);
                const u64 w = d_w[j];
                const u64 t0 = d_tried[2 * j], t1 = d_tried[2 * j + 1];
                auto eligible = [&](int p) {
                    return !(((p < 64 ? t0 : t1) >> (p & 63)) & 1) && s_avail[p] >= w;
                };
                if (attempt == 0) {
                    target = proposal[v];
                } else if (!A) {  // on-demand affinities
                    target = choose_od<D>(v, off, nbr, ew, labels, k, w, t0, t1, s_avail);
                } else {
                    bool decided = false;
                    const int listed = d_list_n[j];
                    if (listed != kNoPart) {
                        C best = 0;
                        u64 room = 0;
                        for (int q = 0; q < listed; ++q) {
                            const int p = d_list_p[kShortlist * j + q];
                            if (!eligible(p)) continue;
                            const C c = d_list_c[kShortlist * j + q];
                            const u64 avail = s_avail[p];
                            if (target < 0 || c > best || (c == best && (avail > room || (avail == room && p < target)))) {
                                target = p;
                                best = c;
                                room = avail;
                            }
                        }
                        // Every eligible part listed: the best listed one
                        // (or none) is the choice.  Otherwise the best must
                        // beat every unlisted affinity.
                        decided = !d_bounded[j] || (target >= 0 && best > d_bound[j]);
                        if (!decided && d_bound[j] == 0 && (target < 0 || best == 0)) {
                            // Every eligible part has affinity 0 (the unlisted
                            // ones at most the bound, the listed ones at most
                            // the best): the one with the most room, the
                            // lowest part on equal room.
                            const int src = d_src[j];
                            target = -1;
                            for (int r = 0; r < k; ++r) {
                                const int p = s_order[r];
                                if (s_avail[p] < w) break;  // the rest have less room
                                if (p == src || (((p < 64 ? t0 : t1) >> (p & 63)) & 1)) continue;
                                target = p;
                                break;
                            }
                            decided = true;
                        }
                    }
                    if (!decided) {
                        // Full scan of the row: the choice and a new shortlist.
                        const int src = d_src[j];
                        const C* row = A + static_cast<i64>(v) * k;
                        target = -1;
                        C best = 0, bound = 0;
                        u64 room = 0;
                        int n_list = 0;
                        bool bounded = false;
                        int lp[kShortlist];
                        C lc[kShortlist];
                        // A slice of affinities loaded together (one round
                        // trip for 64 bytes of the row), then scanned in part
                        // order.
                        constexpr int kSlice = 64 / static_cast<int>(sizeof(C));
                        for (int p0 = 0; p0 < k; p0 += kSlice) {
                            C slice[kSlice];
#pragma unroll
                            for (int q = 0; q < kSlice; ++q) slice[q] = p0 + q < k ? row[p0 + q] : C(0);
#pragma unroll
                            for (int q = 0; q < kSlice; ++q) {
                                const int p = p0 + q;
                                if (p >= k) break;
                                if (p == src || !eligible(p)) continue;
                                const C c = slice[q];
                                const u64 avail = s_avail[p];
                                if (target < 0 || c > best || (c == best && avail > room)) { target = p; best = c; room = avail; }
                                // Shortlist by (affinity desc, part asc): parts
                                // arrive in ascending order, so a part enters
                                // only past a strictly smaller affinity.
                                if (n_list == kShortlist && !(c > lc[kShortlist - 1])) {
                                    bound = bounded ? (c > bound ? c : bound) : c;
                                    bounded = true;
                                    continue;
                                }
                                if (n_list == kShortlist) {
                                    const C out = lc[kShortlist - 1];
                                    bound = bounded ? (out > bound ? out : bound) : out;
                                    bounded = true;
                                } else {
                                    ++n_list;
                                }
                                int at = n_list - 1;
#pragma unroll
                                for (int q2 = kShortlist - 1; q2 > 0; --q2)
                                    if (q2 <= at && lc[q2 - 1] < c) { lc[q2] = lc[q2 - 1]; lp[q2] = lp[q2 - 1]; at = q2 - 1; }
#pragma unroll
                                for (int q2 = 0; q2 < kShortlist; ++q2)
                                    if (q2 == at) { lc[q2] = c; lp[q2] = p; }
                            }
                        }
#pragma unroll
                        for (int q = 0; q < kShortlist; ++q)
                            if (q < n_list) {
                                d_list_p[kShortlist * j + q] = static_cast<unsigned char>(lp[q]);
                                d_list_c[kShortlist * j + q] = lc[q];
                            }
                        d_list_n[j] = static_cast<unsigned char>(n_list);
                        d_bounded[j] = bounded;
                        d_bound[j] = bound;
                    }
                }
                if (target < 0) d_state[j] = 2;
                else s_any = 1;
            }
            s_want[j] = target;
        }
        __syncthreads();
        if (!s_any) break;
        // Admission in chunks of one request per thread, in j order: each
        // request starts after the weight requested for its part by earlier
        // requests (earlier chunks, earlier warps, earlier lanes).
        for (int p = threadIdx.x; p < k; p += blockDim.x) s_base[p] = s_requests[p];
        for (int chunk = 0; chunk < count; chunk += blockDim.x) {
            for (int x = threadIdx.x; x < kWarps * k; x += blockDim.x) s_warp[x / kWarps][x % kWarps] = 0;
            __syncthreads();
            const int j = chunk + threadIdx.x;
            const int t = j < count ? s_want[j] : -1;
            const u64 w = t >= 0 ? d_w[j] : 0;
            const unsigned peers = __match_any_sync(0xffffffffu, t);
            u64 before = 0, sum = 0;
            for (unsigned rest = peers; rest; rest &= rest - 1) {
                const int l = __ffs(rest) - 1;
                const u64 o = __shfl_sync(peers, w, l);
                sum += o;
                if (l < lane) before += o;
            }
            if (t >= 0 && lane == __ffs(peers) - 1) s_warp[t][warp] = sum;
            __syncthreads();
            // Per part, the weight requested before each warp (from the
            // running base), and the base for the next chunk: warp `warp`
            // scans the parts warp, warp + 32, ... across its lanes (lane l
            // holds warp l's sum).
            static_assert(kWarps == 32, "one lane per warp of the block");
            for (int p = warp; p < k; p += kWarps) {
                const u64 x = s_warp[p][lane], base = s_base[p];
                u64 inc = x;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const u64 o = __shfl_up_sync(0xffffffffu, inc, d);
                    if (lane >= d) inc += o;
                }
                s_warp[p][lane] = base + inc - x;
                __syncwarp();
                if (lane == 31) s_base[p] = base + inc;
            }
            __syncthreads();
            if (t >= 0) {
                const u64 begin = s_warp[t][warp] + before;
                d_tried[2 * j + (t >> 6)] |= 1ULL << (t & 63);
                if (begin <= s_slack[t] && w <= s_slack[t] - begin) {
                    targets[d_v[j]] = t;
                    flags[d_v[j]] = 1;
                    d_state[j] = 1;
                }
            }
            __syncthreads();
        }
        for (int p = threadIdx.x; p < k; p += blockDim.x) s_requests[p] = s_base[p];
        __syncthreads();
    }
    for (int p = threadIdx.x; p < k; p += blockDim.x) requests[p] = s_requests[p];
    for (int j = threadIdx.x; j < count; j += blockDim.x) {
        const u32 i = open[j];
        state[i] = d_state[j];
        tried[2 * i] = d_tried[2 * j];
        tried[2 * i + 1] = d_tried[2 * j + 1];
    }
}
struct IsOpen {
    const unsigned char* state;
    __device__ bool operator()(i64 i) const { return state[i] == 0; }
};

struct IsPlaced {
    const unsigned char* state;
    __device__ bool operator()(i64 i) const { return state[i] == 1; }
};
struct WriteActiveVertex {
    const u32* active;
    int* out;
    __device__ void operator()(u32 slot, i64 i) const { out[slot] = static_cast<int>(active[i]); }
};

// ---------------------------------------------------------------- exchange

constexpr int kJointSeeds = 128, kJointSide = 4, kJointArchive = 4;

struct JointMove {  // exchange.cuh:9-13
    int vertices[2 * kJointSide];
    int size, a, b, id;
    long long gain, net;
};

__host__ __device__ inline JointMove empty_move() {
    JointMove m;
    for (int j = 0; j < 8; ++j) m.vertices[j] = -1;
    m.size = 0; m.a = -1; m.b = -1; m.id = 0; m.gain = 0; m.net = 0;
    return m;
}
__device__ __forceinline__ long long joint_gap(long long net, long long lo, long long hi) {
    return net < lo ? lo - net : net > hi ? net - hi : 0;
}
__device__ bool joint_same(const JointMove& x, const JointMove& y) {  // joint_same_move
    if (!x.size || x.size != y.size || x.a != y.a || x.b != y.b || x.gain != y.gain || x.net != y.net) return false;
    for (int j = 0; j < x.size; ++j) {
        bool found = false;
        for (int t = 0; t < y.size; ++t) found |= x.vertices[j] == y.vertices[t];
        if (!found) return false;
    }
    return true;
}
// Sort keys of a joint move.  (k1, k2, k3, k4), compared as unsigned words
// in that order, is a monotone projection of the comparator's leading
// fields: unequal keys decide a comparison the same way the comparator does,
// and only equal keys need the comparator itself.  A signed field enters as
// its value clamped to [-2^53, 2^53) with one value for each side beyond, 55
// bits; the words after a clamped field are zero.
struct MoveKey {
    u64 k1, k2, k3, k4;
};
constexpr long long kKeyLimit = 1LL << 53;
__device__ __forceinline__ u64 field_key(long long v, bool descending, bool& clamped) {
    clamped = v < -kKeyLimit || v >= kKeyLimit;
    const long long c = v < -kKeyLimit ? -kKeyLimit - 1 : v >= kKeyLimit ? kKeyLimit : v;
    const u64 u = static_cast<u64>(c + kKeyLimit + 1);  // 0 .. 2^54
    return descending ? (1ULL << 54) - u : u;
}
struct NetOrder {  // JointNetOrder (complementary_moves.cuh:5-14)
    __device__ bool operator()(const JointMove& x, const JointMove& y) const {
        if (x.a != y.a) return x.a < y.a;
        if (x.net != y.net) return x.net < y.net;
        if (x.gain != y.gain) return x.gain > y.gain;
        if (x.size != y.size) return x.size < y.size;
        for (int j = 0; j < x.size; ++j) if (x.vertices[j] != y.vertices[j]) return x.vertices[j] < y.vertices[j];
        return x.id < y.id;
    }
    // k1 = (a + 1, net ascending), k2 = (gain descending, size), then the
    // 32-bit fields vertex 0 + 1, ..., vertex size-1 + 1, id + 2^31, the
    // first four of them in k3 and k4 (zero-padded): a move of up to three
    // vertices is then fully keyed.
    __device__ static MoveKey key(const JointMove& x) {
        bool net_clamped, gain_clamped;
        const u64 net = field_key(x.net, false, net_clamped);
        const u64 gain = field_key(x.gain, true, gain_clamped);
        MoveKey r;
        r.k1 = (static_cast<u64>(x.a + 1) << 55) | net;
        r.k2 = net_clamped ? 0 : (gain << 8) | (gain_clamped ? 0 : static_cast<u64>(x.size));
        u64 f[4] = {0, 0, 0, 0};
        if (!net_clamped && !gain_clamped) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                f[j] = j < x.size ? static_cast<u64>(static_cast<u32>(x.vertices[j] + 1))
                     : j == x.size ? static_cast<u64>(static_cast<u32>(x.id) ^ 0x80000000u)
                                   : 0;
        }
        r.k3 = (f[0] << 32) | f[1];
        r.k4 = (f[2] << 32) | f[3];
        return r;
    }
};
struct MoveOrder {  // JointOrder (exchange.cuh:29-36)
    __device__ bool operator()(const JointMove& x, const JointMove& y) const {
        if ((x.size != 0) != (y.size != 0)) return x.size != 0;
        if (x.a != y.a) return x.a < y.a;
        if (x.gain != y.gain) return x.gain > y.gain;
        return x.id < y.id;
    }
    // k1 = (empty, a + 1, gain descending), k2 = id.
    __device__ static MoveKey key(const JointMove& x) {
        bool gain_clamped;
        const u64 gain = field_key(x.gain, true, gain_clamped);
        MoveKey r;
        r.k1 = (static_cast<u64>(x.size == 0) << 63) | (static_cast<u64>(x.a + 1) << 55) | gain;
        r.k2 = gain_clamped ? 0 : static_cast<u64>(static_cast<long long>(x.id) + 2147483649LL);
        r.k3 = 0;
        r.k4 = 0;
        return r;
    }
};
template <class Cmp>
__global__ void k_move_keys(int count, const JointMove* moves, MoveKey* keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) keys[i] = Cmp::key(moves[i]);
}
// Whether move b sorts before move a (both real entries).
template <class Cmp>
__device__ __forceinline__ bool move_before(const MoveKey& kb, const MoveKey& ka, const JointMove* moves, int b, int a,
                                            Cmp cmp) {
    if (kb.k1 != ka.k1) return kb.k1 < ka.k1;
    if (kb.k2 != ka.k2) return kb.k2 < ka.k2;
    if (kb.k3 != ka.k3) return kb.k3 < ka.k3;
    if (kb.k4 != ka.k4) return kb.k4 < ka.k4;
    return cmp(moves[b], moves[a]);
}

// One bitonic stage over an index permutation padded to a power of two.
template <class Cmp>
__global__ void k_bitonic(int size, int count, const JointMove* moves, const MoveKey* keys, int* idx, int kk, int jj,
                          Cmp cmp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= size) return;
    const int x = i ^ jj;
    if (x <= i) return;
    const int a = idx[i], b = idx[x];
    // Padding (index >= count) sorts after every real entry.
    bool greater;
    if (a >= count) greater = b < count;
    else if (b >= count) greater = false;
    else greater = move_before(keys[b], keys[a], moves, b, a, cmp);
    const bool up = (i & kk) == 0;
    if (greater == up) { idx[i] = b; idx[x] = a; }
}
// One compare-exchange step (partner distance jj, direction block kk) over
// the shared-memory segment that starts at permutation position `base`.
template <class Cmp>
__device__ __forceinline__ void bitonic_step_smem(int seg, int base, int count, int kk, int jj, const JointMove* moves,
                                                  MoveKey* s_key, int* s_idx, Cmp cmp) {
    for (int p = threadIdx.x; p < seg / 2; p += blockDim.x) {
        const int i = (p / jj) * 2 * jj + p % jj;
        const int x = i + jj;
        const int a = s_idx[i], b = s_idx[x];
        bool greater;
        if (a >= count) greater = b < count;
        else if (b >= count) greater = false;
        else greater = move_before(s_key[x], s_key[i], moves, b, a, cmp);
        const bool up = ((base + i) & kk) == 0;
        if (greater == up) {
            s_idx[i] = b;
            s_idx[x] = a;
            const MoveKey t = s_key[i];
            s_key[i] = s_key[x];
            s_key[x] = t;
        }
    }
    __syncthreads();
}
// Bitonic stages on segments of kBitonicSegment indices held in shared
// memory with their keys: for kk from kk_first to kk_last, every jj below the
// segment size (the first kk starts at jj_first).  Same compare-exchange as
// k_bitonic.
constexpr int kBitonicSegment = 4096;
constexpr size_t kBitonicEntryBytes = sizeof(MoveKey) + sizeof(int);
template <class Cmp>
__global__ void __launch_bounds__(1024) k_bitonic_local(int size, int count, const JointMove* moves, const MoveKey* keys,
                                                       int* idx, int kk_first, int kk_last, int jj_first, Cmp cmp) {
    extern __shared__ __align__(16) unsigned char bitonic_smem[];
    MoveKey* s_key = reinterpret_cast<MoveKey*>(bitonic_smem);
    int* s_idx = reinterpret_cast<int*>(s_key + kBitonicSegment);
    const int base = blockIdx.x * kBitonicSegment;
    const int seg = min(kBitonicSegment, size - base);
    for (int i = threadIdx.x; i < seg; i += blockDim.x) {
        const int a = idx[base + i];
        s_idx[i] = a;
        if (a < count) s_key[i] = keys[a];
    }
    __syncthreads();
    for (int kk = kk_first; kk <= kk_last; kk <<= 1)
        for (int jj = kk == kk_first ? jj_first : kk >> 1; jj; jj >>= 1)
            bitonic_step_smem(seg, base, count, kk, jj, moves, s_key, s_idx, cmp);
    for (int i = threadIdx.x; i < seg; i += blockDim.x) idx[base + i] = s_idx[i];
}
// A whole sort of up to kBitonicSegment moves in one block: the full network
// over indices in shared memory (the same compare-exchange steps as
// k_bitonic_local over one segment) and the gather of the sorted moves.
// The keys stay in place, indexed by move, so an exchange writes two
// indices and no keys.
template <class Cmp>
__global__ void __launch_bounds__(1024) k_sort_moves_block(int size, int count, const JointMove* in, JointMove* out,
                                                          Cmp cmp) {
    extern __shared__ __align__(16) unsigned char bitonic_smem[];
    MoveKey* s_key = reinterpret_cast<MoveKey*>(bitonic_smem);  // by move
    int* s_idx = reinterpret_cast<int*>(s_key + size);
    for (int i = threadIdx.x; i < size; i += blockDim.x) {
        s_idx[i] = i;
        if (i < count) s_key[i] = Cmp::key(in[i]);
    }
    __syncthreads();
    for (int kk = 2; kk <= size; kk <<= 1)
        for (int jj = kk >> 1; jj; jj >>= 1) {
            for (int p = threadIdx.x; p < size / 2; p += blockDim.x) {
                const int i = (p / jj) * 2 * jj + p % jj;
                const int x = i + jj;
                const int a = s_idx[i], b = s_idx[x];
                bool greater;
                if (a >= count) greater = b < count;
                else if (b >= count) greater = false;
                else greater = move_before(s_key[b], s_key[a], in, b, a, cmp);
                if (greater == ((i & kk) == 0)) {
                    s_idx[i] = b;
                    s_idx[x] = a;
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < count; i += blockDim.x) out[i] = in[s_idx[i]];
}
__global__ void k_iota(int n, int* idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) idx[i] = i;
}
__global__ void k_gather_moves(int count, const int* idx, const JointMove* in, JointMove* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = in[idx[i]];
}

// joint_quotient (exchange.cuh:41-54).
template <class C>
__global__ void k_quotient(i64 n, const int* labels, const C* A, int k, u64* quotient) {
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int a = labels[v];
        for (int b = a + 1; b < k; ++b) {
            const C w = A[v * k + b];
            if (w) atomicAdd(quotient + a * k + b, static_cast<u64>(w));
        }
    }
}
// joint_match (exchange.cuh:55-82): rounds of mutual best choices.  The
// pair scores quotient / (1 + visits)^2 are computed once into shared memory
// (a pair's visits change only when it is matched, after which neither part
// takes part in later rounds); each round a warp per part picks its best
// unmatched partner, the highest score and on ties the lowest part.
constexpr int kMatchThreads = 1024;
__global__ void __launch_bounds__(kMatchThreads) k_match_parts(int k, const u64* quotient, int* partner, int* visits) {
    extern __shared__ double s_score[];  // k * k, pair (a, b) with a < b at a * k + b; -1 = no edge
    __shared__ int s_partner[kMaxParts], s_choice[kMaxParts], s_progress;
    for (int x = threadIdx.x; x < k * k; x += blockDim.x) {
        const int a = x / k, b = x % k;
        double score = -1;
        if (a < b && quotient[x]) {
            const double penalty = 1.0 + visits[x];
            score = __ddiv_rn(static_cast<double>(quotient[x]), __dmul_rn(penalty, penalty));
        }
        s_score[x] = score;
    }
    for (int p = threadIdx.x; p < k; p += blockDim.x) s_partner[p] = -1;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    for (int round = 0; round < k / 2; ++round) {
        if (threadIdx.x == 0) s_progress = 0;
        for (int p = warp; p < k; p += warps) {
            double score = -1;
            int best = -1;
            if (s_partner[p] < 0) {
                for (int q = lane; q < k; q += 32) {
                    if (q == p || s_partner[q] >= 0) continue;
                    const double value = s_score[min(p, q) * k + max(p, q)];
                    if (value > score) { score = value; best = q; }
                }
            }
#pragma unroll
            for (int d = 16; d; d >>= 1) {
                const double other = __shfl_xor_sync(0xffffffffu, score, d);
                const int other_best = __shfl_xor_sync(0xffffffffu, best, d);
                if (other > score || (other == score && other_best >= 0 && (best < 0 || other_best < best))) {
                    score = other;
                    best = other_best;
                }
            }
            if (lane == 0) s_choice[p] = best;
        }
        __syncthreads();
        if (threadIdx.x < k) {
            const int p = threadIdx.x, best = s_choice[p];
            if (best >= 0 && s_choice[best] == p) {
                s_partner[p] = best;
                if (p < best) { ++visits[p * k + best]; atomicAdd(&s_progress, 1); }
            }
        }
        __syncthreads();
        const int gained = s_progress;
        __syncthreads();
        if (!gained) break;
    }
    for (int p = threadIdx.x; p < k; p += blockDim.x) partner[p] = s_partner[p];
}
// joint_seeds (exchange.cuh:83-93).
template <class C>
__global__ void k_seeds(i64 n, const int* labels, const C* A, int k, const int* partner, u64* seeds, int sw, int pass) {
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x) {
        const int p = labels[v], q = partner[p];
        if (q < 0 || !A[v * k + q]) continue;
        const u32 h = mix32(static_cast<u32>(v) ^ mix32(static_cast<u32>(pass + 17)));
        atomicMin(seeds + static_cast<i64>(p) * sw + (h % sw), (static_cast<u64>(h) << 32) | static_cast<u32>(v));
    }
}

// joint_grow (exchange.cuh:95-204): one warp per (seed, policy) slot.
template <class C>
__global__ void k_grow(int slots, int sw, const u64* seeds, const int* partner, const int* off, const int* nbr,
                       const u32* ew, const u32* masses, const int* labels, const C* A, int k, const u64* loads,
                       u64 capacity, JointMove* moves, JointMove* archive) {
    const int lane = threadIdx.x & 31;
    const int slot = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (slot >= slots) return;
    const int policy = slot % 2;
    JointMove best = empty_move();
    best.id = slot;
    if (!lane) {
        moves[slot] = best;
        for (int j = 0; j < kJointArchive; ++j) archive[slot * kJointArchive + j] = empty_move();
    }
    const u64 enc = seeds[slot / 2];
    if (enc == ~0ULL) return;
    const int root = static_cast<int>(static_cast<u32>(enc)), source = labels[root], target = partner[source];
    if (target < 0) return;
    auto aff = [&](int u, int p) -> long long { return static_cast<long long>(A[static_cast<i64>(u) * k + p]); };
    int members[8] = {root, -1, -1, -1, -1, -1, -1, -1};
    int size = 1, counts[2] = {1, 0};
    long long net = masses[root];
    const long long lo = static_cast<long long>(loads[source]) - static_cast<long long>(capacity);
    const long long hi = static_cast<long long>(capacity) - static_cast<long long>(loads[target]);
    long long gain = aff(root, target) - aff(root, source);
    for (int step = 0; step < 8; ++step) {
        if (!lane && gain > 0 && size <= kJointArchive) {
            JointMove st = empty_move();
            st.size = size; st.a = min(source, target); st.b = max(source, target);
            st.gain = gain; st.net = source == st.a ? net : -net; st.id = slot * kJointArchive + step;
            for (int j = 0; j < size; ++j) {
                int pos = j;
                while (pos && st.vertices[pos - 1] > members[j]) { st.vertices[pos] = st.vertices[pos - 1]; --pos; }
                st.vertices[pos] = members[j];
            }
            archive[slot * kJointArchive + step] = st;
        }
        if (gain > best.gain && !joint_gap(net, lo, hi)) {
            best.size = size; best.a = min(source, target); best.b = max(source, target);
            best.gain = gain; best.net = source == best.a ? net : -net;
            for (int j = 0; j < size; ++j) best.vertices[j] = members[j];
        }
        if (size == 8) break;
        const bool gap_first = policy == 0 && joint_gap(net, lo, hi);
        long long cg = LLONG_MIN, cgap = LLONG_MAX;
        int chosen = INT_MAX;
        for (int origin = -1; origin < size; ++origin) {
            const bool reverse = origin < 0;
            if (reverse && counts[1]) continue;
            const int m = reverse ? -1 : members[origin];
            const int begin = reverse ? 0 : off[m];
            const int end = reverse ? sw : min(off[m + 1], begin + 128);
            for (int e = begin + lane; e < end; e += 32) {
                int u;
                if (reverse) {
                    const u64 value = seeds[static_cast<i64>(target) * sw + e];
                    if (value == ~0ULL) continue;
                    u = static_cast<int>(static_cast<u32>(value));
                } else u = nbr[e];
                const int p = labels[u];
                if (p != source && p != target) continue;
                const int side = p == source ? 0 : 1;
                if (counts[side] >= kJointSide) continue;
                if (!reverse && p != labels[m]) continue;
                bool dup = false;
                for (int j = 0; j < size; ++j) dup |= u == members[j];
                if (dup || off[u + 1] - off[u] > 1024) continue;
                const long long cnet = net + (side ? -static_cast<long long>(masses[u]) : static_cast<long long>(masses[u]));
                const long long gp = joint_gap(cnet, lo, hi);
                if (net > hi && !side) continue;
                if (net < lo && side) continue;
                long long marginal = aff(u, side ? source : target) - aff(u, p);
                if (!reverse) marginal += 2LL * edge_w(ew, e);
                const bool better = gap_first
                    ? (gp < cgap || (gp == cgap && (marginal > cg || (marginal == cg && u < chosen))))
                    : (marginal > cg || (marginal == cg && (gp < cgap || (gp == cgap && u < chosen))));
                if (better) { chosen = u; cg = marginal; cgap = gp; }
            }
        }
        for (int d = 16; d; d >>= 1) {
            const int u = __shfl_down_sync(0xffffffffu, chosen, d);
            const long long g = __shfl_down_sync(0xffffffffu, cg, d);
            const long long gp = __shfl_down_sync(0xffffffffu, cgap, d);
            const bool better = gap_first ? (gp < cgap || (gp == cgap && (g > cg || (g == cg && u < chosen))))
                                          : (g > cg || (g == cg && (gp < cgap || (gp == cgap && u < chosen))));
            if (lane + d < 32 && better) { chosen = u; cg = g; cgap = gp; }
        }
        chosen = __shfl_sync(0xffffffffu, chosen, 0);
        if (chosen == INT_MAX) break;
        const int side = labels[chosen] == source ? 0 : 1;
        long long correction = 0;
        for (int e = off[chosen] + lane; e < off[chosen + 1]; e += 32)
            for (int j = 0; j < size; ++j)
                if (nbr[e] == members[j]) correction += (labels[members[j]] == labels[chosen] ? 2LL : -2LL) * edge_w(ew, e);
        correction = warp_sum(correction);
        const long long cgain = aff(chosen, side ? source : target) - aff(chosen, labels[chosen]) + correction;
        members[size++] = chosen;
        ++counts[side];
        gain += cgain;
        net += side ? -static_cast<long long>(masses[chosen]) : static_cast<long long>(masses[chosen]);
    }
    if (!lane) moves[slot] = best;
}

struct NonEmptyMove {
    const JointMove* moves;
    __device__ bool operator()(i64 i) const { return moves[i].size != 0; }
};
struct CopyMove {
    const JointMove* in;
    JointMove* out;
    __device__ void operator()(u32 slot, i64 i) const { out[slot] = in[i]; }
};
struct UniqueHead {
    const JointMove* moves;
    __device__ bool operator()(i64 i) const { return i == 0 || !joint_same(moves[i - 1], moves[i]); }
};

// joint_combine (complementary_moves.cuh:31-75): one warp per fragment.
__global__ void k_combine(int count, const JointMove* archive, const int* off, const int* nbr, const u32* ew,
                          const int* labels, const u64* loads, u64 capacity, int id_base, JointMove* out) {
    const int lane = threadIdx.x & 31, i = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (i >= count) return;
    const JointMove x = archive[i];
    const long long lo = static_cast<long long>(loads[x.a]) - static_cast<long long>(capacity);
    const long long hi = static_cast<long long>(capacity) - static_cast<long long>(loads[x.b]);
    if (!lane) {
        JointMove y = x;
        y.id = id_base + i;
        if (joint_gap(x.net, lo, hi)) y.size = 0;
        out[i] = y;
        out[count + i] = empty_move();
    }
    // First position whose move does not come before (x.a, net) (after it,
    // with upper).  The warp probes 32 evenly spaced positions at once, so
    // each round trip narrows the range 32-fold; the answer is the binary
    // search's (the predicate holds on a prefix of the sorted fragments).
    auto bound = [&](long long net, bool upper) {
        int l = 0, h = count;  // the answer lies in [l, h]
        while (l < h) {
            const int p = l + static_cast<int>((static_cast<long long>(h - l) * lane) / 32);
            bool before = false;
            if (p < h) {
                const JointMove& y = archive[p];
                before = y.a < x.a || (y.a == x.a && (y.net < net || (upper && y.net == net)));
            }
            const unsigned yes = __ballot_sync(0xffffffffu, before);
            if (!yes) return l;  // position l already does not come before
            const int last = 31 - __clz(yes);
            const int lp = __shfl_sync(0xffffffffu, p, last);
            const int np = last < 31 ? __shfl_sync(0xffffffffu, p, last + 1) : h;
            l = lp + 1;
            h = np > l ? np : l;
        }
        return l;
    };
    const int begin = bound(lo - x.net, false), end = bound(hi - x.net, true);
    // The (up to four) partner candidates, in the reference's probe order.
    int cand[4];
    int ncand = 0, previous = -1;
    for (int r = 0; r < 4 && begin < end; ++r) {
        const int j = begin + static_cast<int>((static_cast<long long>(end - begin - 1) * r) / 3);
        if (j == previous) continue;
        previous = j;
        if (j == i) continue;
        const JointMove& y = archive[j];
        if (y.a != x.a || y.b != x.b || x.size + y.size > 8) continue;
        bool overlap = false;
        for (int u = 0; u < x.size; ++u) for (int w = 0; w < y.size; ++w) overlap |= x.vertices[u] == y.vertices[w];
        if (!overlap) cand[ncand++] = j;
    }
    // One pass over x's rows corrects every candidate at once (each row is
    // read once, not once per candidate).  The candidates' vertices sit in
    // 32 fixed register slots (slot 8c + t: vertex t of candidate c, -1 when
    // absent), so a neighbour is tested against all of them without local
    // memory; a move's vertices are distinct, so a neighbour meets each
    // candidate at most once.
    long long correction[4] = {0, 0, 0, 0};
    if (ncand) {
        int yv[32];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const JointMove* y = c < ncand ? archive + cand[c] : nullptr;
            const int size = y ? y->size : 0;
#pragma unroll
            for (int t = 0; t < 8; ++t) yv[8 * c + t] = t < size ? y->vertices[t] : -1;
        }
        for (int u = 0; u < x.size; ++u) {
            const int v = x.vertices[u];
            const int lv = labels[v];
            const int end = off[v + 1];
            // Four entries per lane in flight.
            for (int e0 = off[v] + lane; e0 < end; e0 += 4 * 32) {
                int w4[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) w4[j] = e0 + 32 * j < end ? nbr[e0 + 32 * j] : -1;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int w = w4[j];
                    if (w < 0) continue;
                    unsigned hit = 0;
#pragma unroll
                    for (int q = 0; q < 32; ++q) hit |= w == yv[q] ? 1u << (q >> 3) : 0u;
                    if (!hit) continue;
                    const long long contrib = (lv == labels[w] ? 2LL : -2LL) * edge_w(ew, e0 + 32 * j);
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (hit & (1u << c)) correction[c] += contrib;
                }
            }
        }
    }
    long long best_gain = 0;
    int best = -1;
    for (int c = 0; c < ncand; ++c) {
        const int j = cand[c];
        const long long gain = x.gain + archive[j].gain + warp_sum(correction[c]);
        if (gain > best_gain || (gain == best_gain && gain > 0 && j < best)) { best_gain = gain; best = j; }
    }
    if (!lane && best >= 0) {
        JointMove r = x;
        const JointMove y = archive[best];
        for (int j = 0; j < y.size; ++j) r.vertices[r.size++] = y.vertices[j];
        r.gain = best_gain;
        r.net += y.net;
        r.id = id_base + count + i;
        out[count + i] = r;
    }
}
__global__ void k_claim(int count, const JointMove* moves, int* owners) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count && moves[i].size)
        for (int j = 0; j < moves[i].size; ++j) atomicMin(owners + moves[i].vertices[j], i);
}
__global__ void k_resolve(int count, JointMove* moves, const int* owners) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    for (int j = 0; j < moves[i].size; ++j)
        if (owners[moves[i].vertices[j]] != i) { moves[i].size = 0; break; }
}
__global__ void k_mark(int count, const JointMove* moves, const int* labels, int* owners, int* targets) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count)
        for (int j = 0; j < moves[i].size; ++j) {
            const int v = moves[i].vertices[j];
            owners[v] = i;
            targets[v] = labels[v] == moves[i].a ? moves[i].b : moves[i].a;
        }
}
// joint_events (exchange.cuh:227-262).  The rows of the moves' vertices
// are cut into chunks of kEventChunk entries, a warp per chunk, so that a
// hub among a move's vertices does not leave one warp with the whole row.
// chunk_off[x] (x = move * 8 + vertex slot) is the exclusive prefix of the
// chunk counts (EventChunks) and *total_chunks their sum.
constexpr int kEventChunk = 256;
struct EventChunks {
    const JointMove* moves;
    const int* off;
    __device__ u32 operator()(i64 x) const {
        const JointMove& m = moves[x >> 3];
        const int j = static_cast<int>(x & 7);
        if (j >= m.size) return 0;
        const int v = m.vertices[j];
        return static_cast<u32>((off[v + 1] - off[v] + kEventChunk - 1) / kEventChunk);
    }
};
__global__ void k_events(int count, const JointMove* moves, const u32* chunk_off, const u32* total_chunks,
                         const int* owners, const int* targets, const int* labels, const int* off, const int* nbr,
                         const u32* ew, u64* events) {
    const int lane = threadIdx.x & 31;
    const u32 total = *total_chunks;
    const int items = count * 8;
    for (u32 w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total; w += (gridDim.x * blockDim.x) >> 5) {
        int lo = 0, hi = items - 1;  // the last item whose chunks start at or before w
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (chunk_off[mid] <= w) lo = mid; else hi = mid - 1;
        }
        const int i = lo >> 3;
        const int ma = moves[i].a, mb = moves[i].b, v = moves[i].vertices[lo & 7];
        const int begin = off[v] + static_cast<int>(w - chunk_off[lo]) * kEventChunk;
        const int end = min(off[v + 1], begin + kEventChunk);
        u64 own = 0;
        for (int e = begin + lane; e < end; e += 32) {
            const int u = nbr[e], other = owners[u];
            if (u == v || (other != INT_MAX && v > u)) continue;
            if (other != INT_MAX && labels[u] != ma && labels[u] != mb) continue;
            const long long wt = edge_w(ew, e);
            const int before = labels[v] != labels[u];
            if (other == i || other == INT_MAX) {
                const int after = targets[v] != (other == i ? targets[u] : labels[u]);
                own += static_cast<u64>((before - after) * wt);
            } else {
                const int middle = i < other ? targets[v] != labels[u] : labels[v] != targets[u];
                const int after = targets[v] != targets[u];
                const u64 first = static_cast<u64>((before - middle) * wt), last = static_cast<u64>((middle - after) * wt);
                own += i < other ? first : last;
                atomicAdd(events + other, i < other ? last : first);
            }
        }
        own = warp_sum(own);
        if (!lane && own) atomicAdd(events + i, own);
    }
}
// joint_prefix (exchange.cuh:263-284), a block per part a: the running gain
// and net of a's moves (in order, empty moves adding nothing) are block
// scans, and the stop is the first feasible move whose running gain is the
// largest one above zero, the move at which the serial scan last improved.
constexpr int kPrefixThreads = kScanThreads;
__global__ void __launch_bounds__(kPrefixThreads) k_prefix(int count, int k, const JointMove* moves, const u64* events,
                                                           const u64* loads, u64 capacity, int* stops) {
    __shared__ long long s_scan[9];
    __shared__ int s_range[2];
    __shared__ long long s_best_gain[kPrefixThreads / 32];
    __shared__ int s_best_index[kPrefixThreads / 32];
    const int a = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < 2) {
        const int key = a + static_cast<int>(threadIdx.x);  // first move of part a, first after it
        int low = 0, high = count;
        while (low < high) { const int mid = (low + high) / 2; if (moves[mid].a < key) low = mid + 1; else high = mid; }
        s_range[threadIdx.x] = low;
    }
    __syncthreads();
    const int first = s_range[0], last = s_range[1];
    const long long lo = static_cast<long long>(loads[a]) - static_cast<long long>(capacity);
    long long gain_carry = 0, net_carry = 0, best = 0;
    int stop = -1;
    for (int base = first; base < last; base += kPrefixThreads) {
        const int i = base + static_cast<int>(threadIdx.x);
        const bool valid = i < last && moves[i].size;
        const long long g = valid ? static_cast<long long>(events[i]) : 0;
        const long long d = valid ? moves[i].net : 0;
        long long g_total, d_total;
        const long long gain = gain_carry + block_exclusive_scan(g, g_total, s_scan) + g;
        const long long net = net_carry + block_exclusive_scan(d, d_total, s_scan) + d;
        gain_carry += g_total;
        net_carry += d_total;
        if (valid) {
            const long long hi = static_cast<long long>(capacity) - static_cast<long long>(loads[moves[i].b]);
            if (!joint_gap(net, lo, hi) && gain > best) { best = gain; stop = i; }
        }
    }
    // Largest gain, earliest move on ties.
#pragma unroll
    for (int d = 16; d; d >>= 1) {
        const long long og = __shfl_xor_sync(0xffffffffu, best, d);
        const int oi = __shfl_xor_sync(0xffffffffu, stop, d);
        if (og > best || (og == best && oi >= 0 && (stop < 0 || oi < stop))) { best = og; stop = oi; }
    }
    if (!lane) { s_best_gain[warp] = best; s_best_index[warp] = stop; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kPrefixThreads / 32; ++w)
            if (s_best_gain[w] > best || (s_best_gain[w] == best && s_best_index[w] >= 0 && (stop < 0 || s_best_index[w] < stop))) {
                best = s_best_gain[w];
                stop = s_best_index[w];
            }
        stops[a] = stop;
    }
}
__global__ void k_accept(int count, const JointMove* moves, const int* stops, int* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count && moves[i].size && i <= stops[moves[i].a])
        for (int j = 0; j < moves[i].size; ++j) flags[moves[i].vertices[j]] = 1;
}
struct Flagged {
    const int* flags;
    __device__ bool operator()(i64 v) const { return flags[v] != 0; }
};

// ---------------------------------------------------------------- host side


struct LevelResult {
    u64 cut = 0;
    bool refined = false, repair_failed = false;
};

template <class T>
class LevelRefiner {
public:
    LevelRefiner(Context& c, const DGraph& g, int k, double eps, int* labels, u64* loads, u64 total, bool log,
                 bool verify, const Mapping& mapping, const RefineBudget& budget = RefineBudget{})
        : ctx(c), g(g), k(k), eps(eps), labels(labels), loads(loads), total(total), log(log), verify(verify),
          mapping(mapping), budget(budget) {}

    LevelResult run(bool has_known, u64 known);
    LevelStats stats;

private:
    Context& ctx;
    DGraph g;  // the level; small levels get their own chunk list (run())
    int k;
    double eps;
    int* labels;
    u64* loads;
    u64 total;
    bool log;
    bool verify;
    const Mapping& mapping;
    RefineBudget budget;
    T* check_A = nullptr;       // verify: independent rebuild of the cache
    T* check_totals = nullptr;

    u64 C = 0;
    i64 n = 0;
    T* A = nullptr;
    T* totals = nullptr;
    int* targets = nullptr;
    long long* gains = nullptr;
    u64* proposal = nullptr;  // packed proposals for the filter (pack_proposal)
    unsigned char* locks = nullptr;
    int* flags = nullptr;
    int* cand = nullptr;
    int* movers = nullptr;
    double* prices = nullptr;
    Sample* samples = nullptr;
    u32* rorder = nullptr;
    u32* rposition = nullptr;  // place of each vertex in the repair order
    int* rlabels = nullptr;    // labels in repair order
    u32* state = nullptr;      // packed label / target / batch bit per vertex (dense-cache levels)
    int* chunk_work = nullptr;      // chunks of the heavy rows taking part in a batch (k_heavy_chunk_list)
    u64* chunk_work_count = nullptr;
    u64* counters = nullptr;  // device: 0 cand, 1 movers, 2 delta, 3 max load, 4.. scratch
    long long* corr_acc = nullptr;  // per heavy row: priority-filter correction
    u64 cut = 0, revision = 0;
    u64 rebuild_entries = ~0ULL;  // mover entries above which apply() rebuilds the cache
    i64 repair_iterations = 0, repair_donors = 0;  // for the per-level log line
    bool on_demand = false;  // no dense cache: affinities recomputed from the rows
    Frontier frontier{};         // levels above 65,536 vertices: the rows the LP proposals visit
    bool frontier_on = false;
    int* long_rows = nullptr;  // rows built by k_build_long (large levels)
    i64 long_count = 0, long_entries = 0;
    u64 max_load_host = 0;

    cudaStream_t s() const { return ctx.stream; }
    int grid_for(i64 items, int per_block) const { return static_cast<int>(std::min<i64>(blocks_for(items, per_block), 148 * 32)); }
    // Blocks of the list-driven chunk kernels: enough to fill the GPU, never
    // more than there are chunks.
    int chunk_grid() const { return static_cast<int>(std::min<i64>(g.chunks, 148 * 16)); }
    // The chunks of the heavy rows among `list` (count at `live`, or
    // host_count) into chunk_work.
    void list_heavy_chunks(const int* list, const u64* live, i64 host_count) {
        GP_CUDA(cudaMemsetAsync(chunk_work_count, 0, sizeof(u64), s()));
        launch(k_heavy_chunk_list, grid_for(host_count, kThreads), kThreads, 0, s(), host_count, list, live, g,
               chunk_work, chunk_work_count);
    }

    // Rebuilds the cache and row totals from the labels; with directed_cut
    // also sums the directed cut (device counter, cleared by the caller).
    void build(u64* directed_cut = nullptr, const u64* gate = nullptr, u64 threshold = 0) {
        if (on_demand) return;
        build_into(A, totals, directed_cut, gate, threshold);
    }
    void build_into(T* A, T* totals, u64* directed_cut, const u64* gate, u64 threshold) {
        constexpr int W = 8;
        const bool vec = (static_cast<size_t>(k) * sizeof(T)) % 16 == 0;
        const size_t smem = static_cast<size_t>(kThreads / 32) * (32 / W) * k * sizeof(T);
        const int grid = grid_for(n * W, kThreads);
        // Algorithmic bytes of each kernel: the CSR entries it reads (each
        // neighbour, its weight and its label gather), the offsets, the
        // cache rows and totals it writes and each written row's own label.
        // k_build writes the rows of every vertex but the long ones (heavy
        // rows as zeros, their sums added by k_build_chunks).
        const u64 entry = 8ULL + (g.ew ? 4ULL : 0ULL), row = (static_cast<u64>(k) + 1) * sizeof(T) + 4ULL;
        const u64 short_entries = static_cast<u64>(g.m - g.heavy_entries - long_entries);
        const u64 bytes = 4ULL * (n + 1) + short_entries * entry + static_cast<u64>(n - long_count) * row;
        const u64 long_bytes = static_cast<u64>(long_count) * (12ULL + row) + static_cast<u64>(long_entries) * entry;
        const u64 chunk_bytes = 12ULL * static_cast<u64>(g.chunks) + static_cast<u64>(g.heavy_entries) * entry;
        const bool apart = long_count > 0;
        if (vec)
            launch(k_build<T, W, true>, grid, kThreads, smem, s(), n, g.off, g.nbr, g.ew, static_cast<const int*>(labels),
                   k, A, totals, directed_cut, gate, threshold, work_counter(k_build<T, W, true>), bytes,
                   mapping.build_short, apart, g.heavy_min);
        else
            launch(k_build<T, W, false>, grid, kThreads, smem, s(), n, g.off, g.nbr, g.ew, static_cast<const int*>(labels),
                   k, A, totals, directed_cut, gate, threshold, work_counter(k_build<T, W, false>), bytes,
                   mapping.build_short, apart, g.heavy_min);
        if (apart)
            launch(k_build_long<T>, grid_for(long_count * 32, kThreads), kThreads, (kThreads / 32) * k * sizeof(T), s(),
                   long_count, static_cast<const int*>(long_rows), g.off, g.nbr, g.ew, static_cast<const int*>(labels), k,
                   A, totals, directed_cut, gate, threshold, work_counter(k_build_long<T>), long_bytes);
        if (g.chunks) {
            launch(k_build_chunks<T>, static_cast<int>(g.chunks), 256, sizeof(T) * k, s(), g,
                   static_cast<const int*>(labels), k, A, totals, gate, threshold, work_counter(k_build_chunks<T>),
                   chunk_bytes);
            if (directed_cut)
                launch(k_heavy_cut<T>, blocks_for(g.heavy_count, kThreads), kThreads, 0, s(), g.heavy_count,
                       static_cast<const int*>(g.heavy), static_cast<const int*>(labels), k, static_cast<const T*>(A),
                       static_cast<const T*>(totals), directed_cut, gate, threshold);
        }
    }
    // Applies the movers listed in `list` (count on device at `live`):
    // cache/cut update, commit, flag reset.  Without repair samples, a batch
    // whose rows hold more entries than rebuild_entries rebuilds the cache
    // after the commit instead (identical values: the cache is an exact sum);
    // settle() then takes the new cut from the rebuild.  counters: 2 delta,
    // 3 max load, 6 mover entries, 7 directed cut of a rebuild.
    // `marked`: the list's producer has zeroed counters[2..7] and done what
    // k_mark_movers does (k_compact_movers for a label-propagation batch).
    void apply(const int* list, const u64* live, i64 host_count, bool lp, bool sample, bool marked = false) {
        // counters[2..7]: cut change, largest load, (free), rebuild gate
        // entries and rebuild decision; [4] and [5] hold nothing across it.
        if (!marked) GP_CUDA(cudaMemsetAsync(counters + 2, 0, 6 * sizeof(u64), s()));
        const u64* gate = sample || on_demand ? nullptr : counters + 6;
        const u64 threshold = gate ? rebuild_entries : ~0ULL;
        if ((gate || state) && !marked)
            launch(k_mark_movers, grid_for(host_count, kThreads), kThreads, 0, s(), host_count, list, live, g.off,
                   static_cast<const int*>(targets), state, gate ? counters + 6 : static_cast<u64*>(nullptr));
        if (on_demand)
            with_row_size([&](auto d) {
                launch(k_update_od<decltype(d)::value>, grid_for(host_count, kThreads), kThreads, 0, s(), host_count, list,
                       live, static_cast<const int*>(g.off), static_cast<const int*>(g.nbr), static_cast<const u32*>(g.ew),
                       static_cast<const u32*>(g.vw), static_cast<const int*>(labels), static_cast<const int*>(targets),
                       static_cast<const int*>(flags), reinterpret_cast<long long*>(counters + 2),
                       sample ? samples : static_cast<Sample*>(nullptr));
            });
        else
            launch(k_update<T>, grid_for(host_count * 8, kThreads), kThreads, 0, s(), host_count, list, live, g.off, g.nbr,
                   g.ew, g.vw, static_cast<const u32*>(state), k, A, reinterpret_cast<long long*>(counters + 2),
                   sample ? samples : static_cast<Sample*>(nullptr), gate, threshold, g.heavy_min,
                   work_counter(k_update<T>));
        if (g.chunks) {
            list_heavy_chunks(list, live, host_count);
            launch(k_update_chunks<T>, chunk_grid(), 256, 0, s(), g, static_cast<const int*>(chunk_work),
                   static_cast<const u64*>(chunk_work_count), static_cast<const u32*>(state), k, A,
                   reinterpret_cast<long long*>(counters + 2), sample ? samples : static_cast<Sample*>(nullptr), gate,
                   threshold, work_counter(k_update_chunks<T>));
        }
        // At most four blocks per SM: each block also aggregates its load
        // changes and reports to the finished-block counter, so a grid sized
        // by an upper bound of the movers would mostly pay that.
        launch(k_commit, std::min(grid_for(host_count, kThreads), 148 * 4), kThreads, sizeof(long long) * k, s(),
               host_count, list, live,
               labels, targets, g.vw, k, loads, lp ? locks : static_cast<unsigned char*>(nullptr), flags,
               static_cast<const u32*>(rposition), rlabels, state, counters + 3,
               reinterpret_cast<unsigned int*>(counters + 8));
        if (frontier_on) {
            launch(k_touch_rows, grid_for(host_count * 32, kThreads), kThreads, 0, s(), host_count, list, live, g.off,
                   g.nbr, g.heavy_min, frontier);
            if (g.chunks)  // the heavy movers' chunks listed for the update above
                launch(k_touch_chunks, chunk_grid(), 256, 0, s(), g, static_cast<const int*>(chunk_work),
                       static_cast<const u64*>(chunk_work_count), frontier);
        }
        if (gate) build(counters + 7, gate, threshold);
    }
    // Cut decrease of the last apply from host copies of counters[2..7].
    long long settled_delta(const u64* h) const {
        if (h[4] <= rebuild_entries) return static_cast<long long>(h[0]);
        if (h[5] & 1ULL) fail(GP_INTERNAL, "refinement cut is not symmetric");
        return static_cast<long long>(cut) - static_cast<long long>(h[5] / 2);
    }
    // Lanes per row of the affinity cache: about four 16-byte loads (or four
    // scalars) per lane.  f(width, vectorized) launches the instantiation.
    template <class F>
    void with_groups(F&& f) const {
        const bool vec = (static_cast<size_t>(k) * sizeof(T)) % 16 == 0;
        const int per_lane = vec ? 4 * AffinityVec<T>::N : 4;
        const int W = k <= 2 * per_lane ? 2 : k <= 4 * per_lane ? 4 : k <= 8 * per_lane ? 8 : 16;
        auto go = [&](auto width) {
            if (vec) f(width, std::true_type{});
            else f(width, std::false_type{});
        };
        if (W == 2) go(std::integral_constant<int, 2>{});
        else if (W == 4) go(std::integral_constant<int, 4>{});
        else if (W == 8) go(std::integral_constant<int, 8>{});
        else go(std::integral_constant<int, 16>{});
    }
    // Row-register size of the on-demand kernels for this level.
    template <class F>
    void with_row_size(F&& f) const {
        if (g.maximum_degree <= 8) f(std::integral_constant<int, 8>{});
        else if (g.maximum_degree <= 16) f(std::integral_constant<int, 16>{});
        else f(std::integral_constant<int, kOnDemandDegree>{});
    }
    void proposals(const LpParams& q) {
        const int grid = grid_for(n, kThreads);
        if (on_demand) {
            const int* rows = frontier_on ? frontier.rows : nullptr;
            const u64* count = frontier_on ? frontier.count : nullptr;
            with_row_size([&](auto d) {
                launch(k_proposals_od<decltype(d)::value>, grid, kThreads, 0, s(), q, rows, count);
            });
            return;
        }
        const T* a = A;
        const T* t = totals;
        const int* rows = frontier_on ? frontier.rows : nullptr;
        const u64* count = frontier_on ? frontier.count : nullptr;
        with_groups([&](auto width, auto vec) {
            launch(k_proposals<T, decltype(width)::value, decltype(vec)::value>, grid, kThreads, 0, s(), q, a, t, rows,
                   count);
        });
    }
    // GP_FLAG_VERIFY after every batch (incremental.cuh:846-853, 870-877):
    // the incremental cut equals a CSR scan and the cache equals an
    // independent rebuild.
    void check_state(const char* cut_message) {
        if (!verify) return;
        if (device_cut(ctx, g, labels) != cut) fail(GP_INTERNAL, cut_message);
        if (on_demand) return;  // no cache to compare
        if (!check_A) {
            check_A = ctx.persist.alloc<T>(static_cast<size_t>(n) * k);
            check_totals = ctx.persist.alloc<T>(n);
        }
        build_into(check_A, check_totals, nullptr, nullptr, 0);
        ctx.clear_scalars(1);
        launch(k_compare_cache<T>, grid_for(n * k, kThreads), kThreads, 0, s(), static_cast<i64>(n) * k,
               static_cast<const T*>(A), static_cast<const T*>(check_A), n, static_cast<const T*>(totals),
               static_cast<const T*>(check_totals), ctx.dev_scalars);
        if (ctx.read_scalars(1)[0]) fail(GP_INTERNAL, "affinity cache differs from independent CSR rebuild");
    }
    void account(long long delta) {
        if (delta >= 0) {
            if (static_cast<u64>(delta) > cut) fail(GP_INTERNAL, "incremental cut underflow");
            cut -= static_cast<u64>(delta);
        } else cut += static_cast<u64>(-delta);
    }
    void enqueue_lp_round(double filter);
    i64 lp_round(double filter);
    bool repair();
    void exchange(u64& best);
};

// The device work of one label-propagation round, up to the read-back of its
// counters (every launch is sized by the level, not by a count read back).
template <class T>
void LevelRefiner<T>::enqueue_lp_round(double filter) {
    GP_CUDA(cudaMemsetAsync(counters, 0, 8 * sizeof(u64), s()));  // [0..1] here, [2..7] for apply
    LpParams q{n,     k,      C,     filter, g.off, g.nbr, g.ew,   g.vw,     labels,     loads,
               prices, targets, gains, locks, flags, cand,  movers, counters, g.heavy_min, proposal};
    proposals(q);
    if (on_demand)
        with_row_size([&](auto d) { launch(k_filter_od<decltype(d)::value>, grid_for(n, kThreads), kThreads, 0, s(), q); });
    else
        launch(k_filter, grid_for(n * 8, kThreads), kThreads, 0, s(), q);
    if (g.chunks) {
        GP_CUDA(cudaMemsetAsync(corr_acc, 0, sizeof(long long) * g.heavy_count, s()));
        list_heavy_chunks(cand, counters, n);
        launch(k_filter_chunks, chunk_grid(), 256, 0, s(), g, q, corr_acc, static_cast<const int*>(chunk_work),
               static_cast<const u64*>(chunk_work_count));
        launch(k_filter_finish, blocks_for(g.heavy_count, kThreads), kThreads, 0, s(), g.heavy_count,
               static_cast<const int*>(g.heavy), static_cast<const long long*>(corr_acc), q);
    }
    launch(k_compact_movers, grid_for(n, kThreads), kThreads, 0, s(), q, state,
           on_demand ? static_cast<u64*>(nullptr) : counters + 6);
    apply(movers, counters + 1, n, true, false, true);
}

template <class T>
i64 LevelRefiner<T>::lp_round(double filter) {
    enqueue_lp_round(filter);
    GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, counters, 8 * sizeof(u64), cudaMemcpyDeviceToHost, s()));
    GP_CUDA(cudaStreamSynchronize(s()));
    const i64 count = static_cast<i64>(ctx.host_scalars[1]);
    const long long delta = settled_delta(ctx.host_scalars + 2);
    max_load_host = ctx.host_scalars[3];
    stats.proposals += static_cast<u64>(count);
    if (count) {
        stats.accepted += static_cast<u64>(count);
        if (delta >= 0) stats.lp_gain += static_cast<u64>(delta);
        else stats.lp_loss += static_cast<u64>(-delta);
        account(delta);
        ++revision;
        check_state("incremental cut differs from CSR scan");
    }
    return count;
}

// One capacity repair (RebalanceGraph, rebalance_graph.cuh:160-280) in the
// deterministic order.  Returns feasibility.
template <class T>
bool LevelRefiner<T>::repair() {
    if (max_load_host <= C) return true;
    Arena& A_ = ctx.scratch;
    ArenaScope scope(A_);
    u64* slack = A_.alloc<u64>(k);
    u64* requests = A_.alloc<u64>(k);
    u64* cdf = A_.alloc<u64>(k + 1);
    u64* part_base = A_.alloc<u64>(k);
    u32* donors = A_.alloc<u32>(n);
    u32* donor_count = reinterpret_cast<u32*>(counters + 4);
    unsigned char* active_flag = A_.alloc<unsigned char>(n);
    int iterations = 0;
    while (true) {
        ArenaScope it(A_);
        launch(k_slack, 1, kMaxParts, 0, s(), k, loads, C, slack, requests, cdf);
        select_if(A_, s(), n, IsDonor{rlabels, loads, C}, WriteOrdered{rorder, donors}, donor_count);
        GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, counters + 4, sizeof(u64), cudaMemcpyDeviceToHost, s()));
        GP_CUDA(cudaStreamSynchronize(s()));
        const i64 dcount = static_cast<i64>(ctx.host_scalars[0] & 0xffffffffULL);
        ++repair_iterations;
        repair_donors += dcount;
        i64 placed = 0;
        long long delta = 0;
        if (dcount > 0) {
            u64* keys = A_.alloc<u64>(dcount);
            u64* keys_alt = A_.alloc<u64>(dcount);
            u32* items = A_.alloc<u32>(dcount);
            u32* items_alt = A_.alloc<u32>(dcount);
            if (on_demand)
                with_row_size([&](auto d) {
                    launch(k_repair_dest_od<decltype(d)::value>, grid_for(dcount, kThreads), kThreads, 0, s(), dcount,
                           static_cast<const u32*>(donors), static_cast<const int*>(g.off), static_cast<const int*>(g.nbr),
                           static_cast<const u32*>(g.ew), static_cast<const int*>(labels), static_cast<const u32*>(g.vw),
                           k, static_cast<const u64*>(loads), C, static_cast<const u64*>(cdf), targets, keys);
                });
            else
                with_groups([&](auto width, auto vec) {
                    constexpr int W = decltype(width)::value;
                    launch(k_repair_dest<T, W, decltype(vec)::value>, grid_for(dcount * W, kThreads), kThreads, 0, s(),
                           dcount, donors, static_cast<const T*>(A), static_cast<const T*>(totals), labels, g.vw, k, loads,
                           C, cdf, targets, keys);
                });
            GP_CUDA(cudaMemcpyAsync(items, donors, sizeof(u32) * dcount, cudaMemcpyDeviceToDevice, s()));
            // Stable sort by bucket keeps the repair order inside a bucket;
            // bucket keys are below k*800 < 2^17, the sentinel sorts last.
            launch(k_clamp_keys, blocks_for(dcount, kThreads), kThreads, 0, s(), dcount, keys);
            radix_sort_pairs(A_, s(), dcount, keys, items, keys_alt, items_alt, 0, 24);
            u64* prefix = A_.alloc<u64>(dcount);
            exclusive_scan<u64>(A_, s(), dcount, SortedWeight{items, g.vw}, prefix, static_cast<u64*>(nullptr));
            launch(k_part_heads, blocks_for(dcount, kThreads), kThreads, 0, s(), dcount, keys, prefix, part_base);
            launch(k_donor_test, blocks_for(dcount, kThreads), kThreads, 0, s(), dcount, keys, items, prefix, part_base,
                   loads, C, active_flag);
            // Active donors, back in repair order.
            u32* active = A_.alloc<u32>(dcount);
            select_if(A_, s(), dcount, IsActive{donors, active_flag}, WriteFrom{donors, active}, donor_count);
            GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, counters + 4, sizeof(u64), cudaMemcpyDeviceToHost, s()));
            GP_CUDA(cudaStreamSynchronize(s()));
            const i64 acount = static_cast<i64>(ctx.host_scalars[0] & 0xffffffffULL);
            if (acount > 0) {
                u64* tried = A_.alloc<u64>(2 * acount);
                unsigned char* state = A_.alloc<unsigned char>(acount);
                int* want = A_.alloc<int>(acount);
                GP_CUDA(cudaMemsetAsync(tried, 0, sizeof(u64) * 2 * acount, s()));
                GP_CUDA(cudaMemsetAsync(state, 0, acount, s()));
                const int tiles = blocks_for(acount, kAdmitTile);
                u64* tile_sums = A_.alloc<u64>(static_cast<size_t>(k) * tiles);
                u64* tile_offsets = A_.alloc<u64>(static_cast<size_t>(k) * tiles);
                u64* tile_total = A_.alloc<u64>(1);
                u32* open = A_.alloc<u32>(acount);
                u32* open_count = reinterpret_cast<u32*>(counters + 5);
                // Small sets of open donors finish all their attempts in one block.
                auto finish_in_block = [&](int first_attempt) {
                    auto go = [&](auto d) {
                        // Sized for kAttemptCap donors (the count is on the
                        // device); the limit is set on every call, as it
                        // belongs to the kernel on whichever device is current.
                        constexpr size_t smem = attempt_smem<T>(kAttemptCap);
                        GP_CUDA(cudaFuncSetAttribute(k_attempts<T, decltype(d)::value>,
                                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     static_cast<int>(smem)));
                        launch(k_attempts<T, decltype(d)::value>, 1, kAttemptThreads, smem, s(), static_cast<const u32*>(open),
                               static_cast<const u32*>(open_count), first_attempt, static_cast<const u32*>(active),
                               static_cast<const T*>(A), static_cast<const int*>(g.off), static_cast<const int*>(g.nbr),
                               static_cast<const u32*>(g.ew), static_cast<const int*>(labels), g.vw, k,
                               static_cast<const int*>(targets), static_cast<const u64*>(slack), requests, tried, state,
                               targets, flags);
                    };
                    // The row size matters only for on-demand affinities; a
                    // dense level takes the smallest instantiation (fewest
                    // registers: one block of 1024 threads has 64 each).
                    if (on_demand) with_row_size(go);
                    else go(std::integral_constant<int, 8>{});
                };
                if (acount <= kAttemptCap) {
                    select_if(A_, s(), acount, IsOpen{state}, WriteIdx{open}, open_count);
                    finish_in_block(0);
                }
                for (int attempt = 0; attempt < k && acount > kAttemptCap; ++attempt) {
                    GP_CUDA(cudaMemsetAsync(counters + 5, 0, sizeof(u64), s()));
                    if (on_demand)
                        with_row_size([&](auto d) {
                            launch(k_choose_od<decltype(d)::value>, grid_for(acount, kThreads), kThreads, 0, s(), acount,
                                   static_cast<const u32*>(active), attempt, static_cast<const int*>(g.off),
                                   static_cast<const int*>(g.nbr), static_cast<const u32*>(g.ew),
                                   static_cast<const int*>(labels), static_cast<const u32*>(g.vw), k,
                                   static_cast<const int*>(targets), static_cast<const u64*>(slack),
                                   static_cast<const u64*>(requests), static_cast<const u64*>(tried), state, want,
                                   counters + 5);
                        });
                    else
                        with_groups([&](auto width, auto vec) {
                            constexpr int W = decltype(width)::value;
                            launch(k_choose<T, W, decltype(vec)::value>, grid_for(acount * W, kThreads), kThreads, 0, s(),
                                   acount, active, attempt, static_cast<const T*>(A), labels, g.vw, k, targets, slack,
                                   requests, tried, state, want, counters + 5);
                        });
                    // Admission of this attempt's requests (a no-op when none
                    // asked), then one read-back of the number that asked.
                    launch(k_part_requests, tiles, kAdmitTile, 0, s(), acount, static_cast<const int*>(want),
                           static_cast<const u32*>(active), static_cast<const u32*>(g.vw), k, tiles, tile_sums);
                    exclusive_scan<u64>(A_, s(), static_cast<i64>(k) * tiles, LoadOf<u64>{tile_sums}, tile_offsets,
                                        tile_total);
                    launch(k_admit_tiles, tiles, kAdmitTile, 0, s(), acount, static_cast<const int*>(want),
                           static_cast<const u32*>(active), static_cast<const u32*>(g.vw),
                           static_cast<const u64*>(tile_offsets), static_cast<const u64*>(tile_total), tiles,
                           static_cast<const u64*>(slack), requests, tried, state, targets, flags, k,
                           reinterpret_cast<unsigned int*>(counters + 8));
                    GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, counters + 5, sizeof(u64), cudaMemcpyDeviceToHost, s()));
                    GP_CUDA(cudaStreamSynchronize(s()));
                    const i64 rcount = static_cast<i64>(ctx.host_scalars[0]);
                    if (!rcount) break;
                    // At most rcount donors remain open.
                    if (rcount <= kAttemptCap && attempt + 1 < k) {
                        select_if(A_, s(), acount, IsOpen{state}, WriteIdx{open}, open_count);
                        finish_in_block(attempt + 1);
                        break;
                    }
                }
                // Movers = placed donors, in repair order, applied with their
                // count left on the device (counters[9], whose upper half
                // stays zero): one read-back brings the count and the
                // batch's counters together.  An empty batch changes nothing
                // on the device.
                select_if(A_, s(), acount, IsPlaced{state}, WriteActiveVertex{active, movers},
                          reinterpret_cast<u32*>(counters + 9));
                apply(movers, counters + 9, acount, false, samples != nullptr);
                GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, counters + 2, 8 * sizeof(u64), cudaMemcpyDeviceToHost, s()));
                GP_CUDA(cudaStreamSynchronize(s()));
                placed = static_cast<i64>(ctx.host_scalars[7] & 0xffffffffULL);
                if (placed) {
                    delta = settled_delta(ctx.host_scalars);
                    max_load_host = ctx.host_scalars[1];
                    stats.accepted += static_cast<u64>(placed);
                    if (delta >= 0) stats.rebalance_gain += static_cast<u64>(delta);
                    else stats.rebalance_loss += static_cast<u64>(-delta);
                    account(delta);
                    ++revision;
                    check_state("GPU rebalance cut mismatch");
                }
            }
        }
        if (frontier_on && dcount > 0)
            launch(k_reset_targets, blocks_for(dcount, kThreads), kThreads, 0, s(), dcount,
                   static_cast<const u32*>(donors), targets);
        ++iterations;
        ++stats.admission_iterations;
        const bool feasible = max_load_host <= C;
        if (feasible || placed == 0 || iterations >= 2 * k + 4) return feasible;
    }
}

template <class T>
void LevelRefiner<T>::exchange(u64& best_cut) {
    Arena& A_ = ctx.scratch;
    ArenaScope scope(A_);
    const int sw = std::min(kJointSeeds, std::max(32, 4096 / k));
    const int slots = k * sw * 2;
    u64* quotient = A_.alloc<u64>(static_cast<size_t>(k) * k);
    int* visits = A_.alloc<int>(static_cast<size_t>(k) * k);
    int* partner = A_.alloc<int>(k);
    u64* seeds = A_.alloc<u64>(static_cast<size_t>(k) * sw);
    JointMove* moves = A_.alloc<JointMove>(slots);
    JointMove* archive = A_.alloc<JointMove>(static_cast<size_t>(slots) * kJointArchive);
    JointMove* frag = A_.alloc<JointMove>(static_cast<size_t>(slots) * kJointArchive);
    JointMove* frag_sorted = A_.alloc<JointMove>(static_cast<size_t>(slots) * kJointArchive);
    const size_t pool_cap = static_cast<size_t>(slots) + 2 * static_cast<size_t>(slots) * kJointArchive;
    JointMove* pool = A_.alloc<JointMove>(pool_cap);
    JointMove* act = A_.alloc<JointMove>(pool_cap);
    JointMove* act_sorted = A_.alloc<JointMove>(pool_cap);
    int* idx = A_.alloc<int>(2 * pool_cap);
    MoveKey* move_keys = A_.alloc<MoveKey>(pool_cap);
    int* owners = A_.alloc<int>(n);
    u64* events = A_.alloc<u64>(pool_cap);
    int* stops = A_.alloc<int>(k);
    u32* cnt = reinterpret_cast<u32*>(counters + 4);
    GP_CUDA(cudaMemsetAsync(quotient, 0, sizeof(u64) * k * k, s()));
    GP_CUDA(cudaMemsetAsync(visits, 0, sizeof(int) * k * k, s()));
    launch(k_quotient<T>, grid_for(n, kThreads), kThreads, 0, s(), n, labels, static_cast<const T*>(A), k, quotient);
    auto read_count = [&]() -> i64 {
        GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, counters + 4, sizeof(u64), cudaMemcpyDeviceToHost, s()));
        GP_CUDA(cudaStreamSynchronize(s()));
        return static_cast<i64>(ctx.host_scalars[0] & 0xffffffffULL);
    };
    auto sort_moves = [&](JointMove* in, JointMove* out, int count, auto cmp) {
        using Cmp = decltype(cmp);
        int size = 1;
        while (size < count) size <<= 1;
        // (Shared-memory limits are set to one value for every size, on every
        // call that needs more than the default: the limit belongs to the
        // kernel for the whole process, on whichever device is current, and
        // concurrent worker contexts must not lower it under each other's
        // launches.)
        if (size <= kBitonicSegment) {
            const size_t smem = kBitonicEntryBytes * size;
            if (smem > 48 * 1024)
                GP_CUDA(cudaFuncSetAttribute(k_sort_moves_block<Cmp>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(kBitonicEntryBytes * kBitonicSegment)));
            launch(k_sort_moves_block<Cmp>, 1, 1024, smem, s(), size, count, static_cast<const JointMove*>(in), out,
                   cmp);
            return;
        }
        launch(k_iota, blocks_for(size, kThreads), kThreads, 0, s(), size, idx);
        launch(k_move_keys<Cmp>, blocks_for(count, kThreads), kThreads, 0, s(), count,
               static_cast<const JointMove*>(in), move_keys);
        // Stages whose partner distance stays inside a segment run in shared
        // memory, the rest one launch per stage.
        const size_t smem = kBitonicEntryBytes * kBitonicSegment;
        GP_CUDA(cudaFuncSetAttribute(k_bitonic_local<Cmp>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
        const int segments = size / kBitonicSegment;
        const JointMove* m = in;
        const MoveKey* mk = move_keys;
        launch(k_bitonic_local<Cmp>, segments, 1024, smem, s(), size, count, m, mk, idx, 2, kBitonicSegment, 1, cmp);
        for (int kk = 2 * kBitonicSegment; kk <= size; kk <<= 1) {
            for (int jj = kk >> 1; jj >= kBitonicSegment; jj >>= 1)
                launch(k_bitonic<Cmp>, blocks_for(size, kThreads), kThreads, 0, s(), size, count, m, mk, idx, kk, jj,
                       cmp);
            launch(k_bitonic_local<Cmp>, segments, 1024, smem, s(), size, count, m, mk, idx, kk, kk,
                   kBitonicSegment / 2, cmp);
        }
        launch(k_gather_moves, blocks_for(count, kThreads), kThreads, 0, s(), count, static_cast<const int*>(idx),
               static_cast<const JointMove*>(in), out);
    };
    int empty = 0;
    for (int pass = 0; pass < budget.exchange_rounds; ++pass) {
        const size_t match_smem = sizeof(double) * k * k;
        // One value for every k: the limit belongs to the kernel for the whole
        // process, and concurrent worker contexts must not lower it under
        // each other's launches.
        GP_CUDA(cudaFuncSetAttribute(k_match_parts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(sizeof(double) * kMaxParts * kMaxParts)));
        launch(k_match_parts, 1, kMatchThreads, match_smem, s(), k, quotient, partner, visits);
        GP_CUDA(cudaMemsetAsync(seeds, 0xff, sizeof(u64) * k * sw, s()));
        launch(k_seeds<T>, grid_for(n, kThreads), kThreads, 0, s(), n, labels, static_cast<const T*>(A), k, partner,
               seeds, sw, pass);
        launch(k_grow<T>, blocks_for(slots, 8), kThreads, 0, s(), slots, sw, seeds, partner, g.off, g.nbr, g.ew, g.vw,
               labels, static_cast<const T*>(A), k, loads, C, moves, archive);
        select_if(A_, s(), static_cast<i64>(slots) * kJointArchive, NonEmptyMove{archive}, CopyMove{archive, frag}, cnt);
        int fragments = static_cast<int>(read_count());
        if (fragments) {
            sort_moves(frag, frag_sorted, fragments, NetOrder{});
            select_if(A_, s(), fragments, UniqueHead{frag_sorted}, CopyMove{frag_sorted, frag}, cnt);
            fragments = static_cast<int>(read_count());
        }
        const int pool_size = slots + 2 * fragments;
        GP_CUDA(cudaMemcpyAsync(pool, moves, sizeof(JointMove) * slots, cudaMemcpyDeviceToDevice, s()));
        if (fragments)
            launch(k_combine, blocks_for(fragments, 8), kThreads, 0, s(), fragments, static_cast<const JointMove*>(frag),
                   g.off, g.nbr, g.ew, labels, loads, C, slots, pool + slots);
        select_if(A_, s(), pool_size, NonEmptyMove{pool}, CopyMove{pool, act}, cnt);
        const int active = static_cast<int>(read_count());
        if (!active) { if (++empty >= 2) break; continue; }
        sort_moves(act, act_sorted, active, MoveOrder{});
        fill<int>(s(), owners, n, INT_MAX);
        launch(k_claim, blocks_for(active, kThreads), kThreads, 0, s(), active, static_cast<const JointMove*>(act_sorted), owners);
        launch(k_resolve, blocks_for(active, kThreads), kThreads, 0, s(), active, act_sorted, static_cast<const int*>(owners));
        fill<int>(s(), owners, n, INT_MAX);
        launch(k_mark, blocks_for(active, kThreads), kThreads, 0, s(), active, static_cast<const JointMove*>(act_sorted),
               static_cast<const int*>(labels), owners, targets);
        GP_CUDA(cudaMemsetAsync(events, 0, sizeof(u64) * active, s()));
        {
            ArenaScope es(A_);
            u32* chunk_off = A_.alloc<u32>(static_cast<size_t>(active) * 8);
            u32* total_chunks = A_.alloc<u32>(1);
            exclusive_scan<u32>(A_, s(), static_cast<i64>(active) * 8,
                                EventChunks{static_cast<const JointMove*>(act_sorted), g.off}, chunk_off, total_chunks);
            launch(k_events, 148 * 8, kThreads, 0, s(), active, static_cast<const JointMove*>(act_sorted),
                   static_cast<const u32*>(chunk_off), static_cast<const u32*>(total_chunks),
                   static_cast<const int*>(owners), static_cast<const int*>(targets), static_cast<const int*>(labels),
                   g.off, g.nbr, g.ew, events);
        }
        launch(k_prefix, k, kPrefixThreads, 0, s(), active, k, static_cast<const JointMove*>(act_sorted),
               static_cast<const u64*>(events), static_cast<const u64*>(loads), C, stops);
        launch(k_accept, blocks_for(active, kThreads), kThreads, 0, s(), active, static_cast<const JointMove*>(act_sorted),
               static_cast<const int*>(stops), flags);
        // The accepted moves applied with their count left on the device
        // (as the repair does): one read-back for the count and the
        // batch's counters; an empty batch changes nothing.
        select_if(A_, s(), n, Flagged{flags}, WriteIndex{movers}, reinterpret_cast<u32*>(counters + 9));
        apply(movers, counters + 9, n, false, false);
        GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, counters + 2, 8 * sizeof(u64), cudaMemcpyDeviceToHost, s()));
        GP_CUDA(cudaStreamSynchronize(s()));
        const i64 count = static_cast<i64>(ctx.host_scalars[7] & 0xffffffffULL);
        if (!count) { if (++empty >= 2) break; continue; }
        empty = 0;
        const long long delta = settled_delta(ctx.host_scalars);
        max_load_host = ctx.host_scalars[1];
        account(delta);
        ++revision;
        check_state("incremental cut differs from CSR scan");
        if (delta <= 0) fail(GP_INTERNAL, "non-improving boundary group batch");
        stats.group_gain += static_cast<u64>(delta);
        stats.group_accepted += static_cast<u64>(count);
        if (max_load_host > C || cut >= best_cut) fail(GP_INTERNAL, "capacity exchange violated cut/capacity");
        best_cut = cut;
    }
}

// run_incremental_refinement_typed (incremental.cuh:660-1051).
template <class T>
LevelResult LevelRefiner<T>::run(bool has_known, u64 known) {
    Arena& A_ = ctx.scratch;
    ArenaScope scope(A_);
    n = g.n;
    // Smaller levels: rows above a lower threshold (coarse hubs) go through
    // the block-per-chunk kernels instead of one warp each, which otherwise
    // set the time of every row-parallel pass of the level.
    const int heavy_min = n <= 65536 ? mapping.refine_heavy_small
                          : n <= (1 << 20) ? mapping.refine_heavy_mid : mapping.refine_heavy_large;
    if (heavy_min != g.heavy_min && (g.maximum_degree > static_cast<u64>(std::min(heavy_min, g.heavy_min)) || g.heavy_count))
        build_chunks(ctx, g, heavy_min, &A_);
    uint64_t cap = 0;
    if (gp_status st = capacity_of(total, k, eps, &cap); st != GP_OK) fail(st, last_error());
    C = cap;
    const bool priced = total > static_cast<u64>(n);
    // Short rows next to k (levels large enough to skip the exchange step,
    // which reads the cache): recompute affinities on demand.
    on_demand = n > 65536 && g.maximum_degree <= static_cast<u64>(std::min(mapping.on_demand_degree, kOnDemandDegree)) &&
                3 * g.maximum_degree < static_cast<u64>(k);
    if (!on_demand) {
        A = A_.alloc<T>(static_cast<size_t>(n) * k);
        totals = A_.alloc<T>(n);
        if (n > 65536) {  // long rows of the level and their entries, for k_build_long
            long_rows = A_.alloc<int>(n);
            ctx.clear_scalars(2);
            u32* count_dev = reinterpret_cast<u32*>(ctx.dev_scalars);
            select_if(A_, s(), n, IsLongRow{g.off, mapping.build_short, g.heavy_min}, WriteIndex{long_rows}, count_dev);
            launch(k_row_entries, grid_for(n, kThreads), kThreads, 0, s(), static_cast<const u32*>(count_dev),
                   static_cast<const int*>(long_rows), g.off, ctx.dev_scalars + 1);
            const u64* sc = ctx.read_scalars(2);
            long_count = static_cast<i64>(static_cast<u32>(sc[0] & 0xffffffffULL));
            long_entries = static_cast<i64>(sc[1]);
        }
    }
    targets = A_.alloc<int>(n);
    gains = A_.alloc<long long>(n);
    proposal = A_.alloc<u64>(n);
    GP_CUDA(cudaMemsetAsync(proposal, 0, sizeof(u64) * n, s()));
    locks = A_.alloc<unsigned char>(n);
    flags = A_.alloc<int>(n);
    cand = A_.alloc<int>(n);
    movers = A_.alloc<int>(n);
    // [8]: k_commit's finished-block count, zero between launches; [9]: the
    // repair's placed-donor count (a 32-bit count in a zeroed word).
    counters = A_.alloc<u64>(10);
    GP_CUDA(cudaMemsetAsync(counters + 8, 0, 2 * sizeof(u64), s()));
    corr_acc = A_.alloc<long long>(g.heavy_count + 1);
    if (g.chunks) {
        chunk_work = A_.alloc<int>(g.chunks);
        chunk_work_count = A_.alloc<u64>(1);
    }
    int* saved_labels = A_.alloc<int>(n);
    u64* saved_loads = A_.alloc<u64>(k);
    GP_CUDA(cudaMemsetAsync(locks, 0, n, s()));
    GP_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * n, s()));
    fill<int>(s(), targets, n, -1);
    if (priced) {
        prices = A_.alloc<double>(k);
        samples = A_.alloc<Sample>(k);
        GP_CUDA(cudaMemsetAsync(prices, 0, sizeof(double) * k, s()));
        GP_CUDA(cudaMemsetAsync(samples, 0, sizeof(Sample) * k, s()));
    }
    {  // repair order: ascending (repair hash, id)
        rorder = A_.alloc<u32>(n);
        u32* rorder_alt = A_.alloc<u32>(n);
        u64* keys = A_.alloc<u64>(n);
        u64* keys_alt = A_.alloc<u64>(n);
        launch(k_repair_keys, blocks_for(n, kThreads), kThreads, 0, s(), n, keys, rorder);
        radix_sort_pairs(A_, s(), n, keys, rorder, keys_alt, rorder_alt, 0, 32);
        rposition = A_.alloc<u32>(n);
        rlabels = A_.alloc<int>(n);
        launch(k_repair_positions, blocks_for(n, kThreads), kThreads, 0, s(), n, static_cast<const u32*>(rorder),
               static_cast<const int*>(labels), rposition, rlabels);
    }
    // An entry-by-entry update touches two random cache counters per entry
    // (about 128 bytes of DRAM traffic); a rebuild writes the whole cache and
    // reads the CSR once.
    rebuild_entries = (static_cast<u64>(n) * k * sizeof(T) + 8ULL * static_cast<u64>(g.m)) /
                      static_cast<u64>(std::max(1, mapping.rebuild_divisor));
    GP_CUDA(cudaMemsetAsync(counters + 7, 0, sizeof(u64), s()));
    if (!on_demand) {
        state = A_.alloc<u32>(n);
        launch(k_state_init, grid_for(n, kThreads), kThreads, 0, s(), n, static_cast<const int*>(labels), state);
    }
    build(has_known ? nullptr : counters + 7);
    launch(k_max_load, 1, 32, 0, s(), k, loads, counters + 3);
    GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, counters + 3, 5 * sizeof(u64), cudaMemcpyDeviceToHost, s()));
    GP_CUDA(cudaStreamSynchronize(s()));
    max_load_host = ctx.host_scalars[0];
    if (has_known) {
        cut = known;
    } else if (on_demand) {
        cut = device_cut(ctx, g, labels);
    } else {
        if (ctx.host_scalars[4] & 1ULL) fail(GP_INTERNAL, "refinement cut is not symmetric");
        cut = ctx.host_scalars[4] / 2;
    }
    LevelResult res;
    stats.initial_cut = cut;
    if (max_load_host > C) {
        if (!repair()) {
            res.cut = cut;
            res.repair_failed = true;
            stats.repair_failed = true;
            stats.final_cut = cut;
            stats.final_max_load = max_load_host;
            return res;
        }
    }
    // Levels above 65,536 vertices (no exchange step): the LP proposals visit
    // a conservative frontier when it starts with at most a quarter of the
    // rows (the reference's rule, incremental.cuh:783-797).
    if (n > 65536) {
        frontier.members = A_.alloc<int>(n);
        frontier.rows = A_.alloc<int>(n);
        frontier.count = A_.alloc<u64>(1);
        GP_CUDA(cudaMemsetAsync(frontier.count, 0, sizeof(u64), s()));
        if (on_demand)
            with_row_size([&](auto d) {
                launch(k_frontier_init_od<decltype(d)::value>, grid_for(n, kThreads), kThreads, 0, s(), n,
                       static_cast<const int*>(g.off), static_cast<const int*>(g.nbr), static_cast<const u32*>(g.ew),
                       static_cast<const int*>(labels), targets, frontier);
            });
        else
            launch(k_frontier_init<T>, grid_for(n, kThreads), kThreads, 0, s(), n, static_cast<const T*>(A),
                   static_cast<const T*>(totals), k, static_cast<const int*>(labels), targets, frontier);
        GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, frontier.count, sizeof(u64), cudaMemcpyDeviceToHost, s()));
        GP_CUDA(cudaStreamSynchronize(s()));
        frontier_on = ctx.host_scalars[0] <= static_cast<u64>(n) / 4;
    }
    const u64 feasible_start = cut;
    u64 best = cut;
    GP_CUDA(cudaMemcpyAsync(saved_labels, labels, sizeof(int) * n, cudaMemcpyDeviceToDevice, s()));
    GP_CUDA(cudaMemcpyAsync(saved_loads, loads, sizeof(u64) * k, cudaMemcpyDeviceToDevice, s()));
    u64 best_revision = revision;
    double filter = 0.25;
    if (g.ew) {
        ctx.clear_scalars(1);
        launch(k_max_edge, std::min(blocks_for(g.m, kThreads), 148 * 8), kThreads, 0, s(), g.m, g.ew, ctx.dev_scalars);
        filter = ctx.read_scalars(1)[0] <= 1 ? 0.25 : 0.75;
    }
    int stale = 0, empty = 0, rounds = 0;
    for (int phase = 0; phase < budget.rounds && stale < 3; ++phase) {
        ++rounds;
        if (samples) GP_CUDA(cudaMemsetAsync(samples, 0, sizeof(Sample) * k, s()));
        const i64 count = lp_round(filter);
        if (!count) { if (++empty >= 2) break; ++stale; continue; }
        empty = 0;
        if (!repair()) break;
        if (prices) launch(k_prices, 1, 128, 0, s(), k, static_cast<const Sample*>(samples), prices);
        ++stale;
        if (cut < best) {
            if (best - cut > best / 1000) stale = 0;
            best = cut;
            GP_CUDA(cudaMemcpyAsync(saved_labels, labels, sizeof(int) * n, cudaMemcpyDeviceToDevice, s()));
            GP_CUDA(cudaMemcpyAsync(saved_loads, loads, sizeof(u64) * k, cudaMemcpyDeviceToDevice, s()));
            best_revision = revision;
            ++stats.checkpoint_updates;
        }
    }
    const bool restored = revision != best_revision;
    if (restored) {
        GP_CUDA(cudaMemcpyAsync(labels, saved_labels, sizeof(int) * n, cudaMemcpyDeviceToDevice, s()));
        if (state)
            launch(k_state_init, grid_for(n, kThreads), kThreads, 0, s(), n, static_cast<const int*>(labels), state);
        launch(k_repair_positions, blocks_for(n, kThreads), kThreads, 0, s(), n, static_cast<const u32*>(rorder),
               static_cast<const int*>(labels), rposition, rlabels);
        GP_CUDA(cudaMemcpyAsync(loads, saved_loads, sizeof(u64) * k, cudaMemcpyDeviceToDevice, s()));
        launch(k_max_load, 1, 32, 0, s(), k, loads, counters + 3);
        GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, counters + 3, sizeof(u64), cudaMemcpyDeviceToHost, s()));
        GP_CUDA(cudaStreamSynchronize(s()));
        max_load_host = ctx.host_scalars[0];
    }
    cut = best;
    if (budget.rounds > 0 && budget.exchange_rounds > 0 && n <= 65536) {
        if (restored) build();
        exchange(best);
    }
    if (cut != best || cut > feasible_start || max_load_host > C) fail(GP_INTERNAL, "incremental refinement postcondition failed");
    if (log)
        std::printf("refine_level vertices=%lld initial_cut=%llu final_cut=%llu rounds=%d repair_iterations=%lld "
                    "repair_donors=%lld maximum_degree=%llu affinities=%s\n", static_cast<long long>(n),
                    static_cast<unsigned long long>(feasible_start), static_cast<unsigned long long>(cut), rounds,
                    static_cast<long long>(repair_iterations), static_cast<long long>(repair_donors),
                    static_cast<unsigned long long>(g.maximum_degree), on_demand ? "on_demand" : "dense");
    stats.rounds = rounds;
    stats.final_cut = cut;
    stats.final_max_load = max_load_host;
    res.cut = cut;
    res.refined = true;
    return res;
}

}  // namespace

u64 device_cut(Context& ctx, const DGraph& g, const int* labels) {
    ctx.clear_scalars(1);
    launch(k_cut, std::min(blocks_for(g.n * 32, 256), 148 * 32), 256, 0, ctx.stream, g.n, g.off, g.nbr, g.ew, labels,
           g.heavy_min, ctx.dev_scalars);
    if (g.chunks) launch(k_cut_chunks, static_cast<int>(g.chunks), 256, 0, ctx.stream, g, labels, ctx.dev_scalars);
    const u64 d = ctx.read_scalars(1)[0];
    if (d & 1ULL) fail(GP_INTERNAL, "refinement cut is not symmetric");
    return d / 2;
}

// refine_hierarchy_impl (src/refine.cu:483-730).
RefineOutcome uncoarsen(Context& ctx, Hierarchy& h, const std::vector<int>& coarse_labels, int k, double eps,
                        int* labels, bool log, bool verify, const Mapping& mapping) {
    cudaStream_t s = ctx.stream;
    const size_t L = h.levels.size();
    std::vector<int*> level_labels(L);
    level_labels[0] = labels;
    for (size_t i = 1; i < L; ++i) level_labels[i] = ctx.persist.alloc<int>(h.levels[i].n);
    u64* loads = ctx.persist.alloc<u64>(k);
    const DGraph& coarsest = h.levels.back();
    GP_CUDA(cudaMemcpyAsync(level_labels[L - 1], coarse_labels.data(), sizeof(int) * coarsest.n, cudaMemcpyHostToDevice, s));
    GP_CUDA(cudaMemsetAsync(loads, 0, sizeof(u64) * k, s));
    launch(k_loads, std::min(blocks_for(coarsest.n, 256), 148 * 4), 256, sizeof(u64) * k, s, coarsest.n, k,
           level_labels[L - 1], coarsest.vw, loads);
    GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, loads, sizeof(u64) * k, cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    u64 total = 0, maxload = 0;
    for (int p = 0; p < k; ++p) { total += ctx.host_scalars[p]; maxload = std::max<u64>(maxload, ctx.host_scalars[p]); }
    auto refine = [&](const DGraph& g, int* lab, bool has_known, u64 known) {
        const auto t_begin = std::chrono::steady_clock::now();
        const LevelResult r =
            g.incident_bound <= 0xffffffffULL
                ? LevelRefiner<u32>(ctx, g, k, eps, lab, loads, total, log, verify, mapping).run(has_known, known)
                : LevelRefiner<u64>(ctx, g, k, eps, lab, loads, total, log, verify, mapping).run(has_known, known);
        if (log) {  // host time of the level; the stream is drained first
            GP_CUDA(cudaStreamSynchronize(s));
            std::printf("refine_level_time vertices=%lld ms=%.3f\n", static_cast<long long>(g.n),
                        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count());
        }
        return r;
    };
    LevelResult res = refine(coarsest, level_labels[L - 1], false, 0);
    u64 last_cut = res.cut;
    i64 last_refined = coarsest.n;
    RefineOutcome out;
    out.levels_refined = res.refined;
    uint64_t cap = 0;
    if (gp_status st = capacity_of(total, k, eps, &cap); st != GP_OK) fail(st, last_error());
    for (size_t c = L - 1; c > 0; --c) {
        const size_t f = c - 1;
        const DGraph& fg = h.levels[f];
        launch(k_project, blocks_for(fg.n, 256), 256, 0, s, fg.n, h.maps[f], level_labels[c], level_labels[f]);
        if (verify) {  // projection keeps the cut and the part weights (src/refine.cu:636-656)
            ArenaScope vs(ctx.scratch);
            u64* fine_loads = ctx.scratch.alloc<u64>(k);
            GP_CUDA(cudaMemsetAsync(fine_loads, 0, sizeof(u64) * k, s));
            launch(k_loads, std::min(blocks_for(fg.n, 256), 148 * 4), 256, sizeof(u64) * k, s, fg.n, k,
                   static_cast<const int*>(level_labels[f]), fg.vw, fine_loads);
            const u64 fine_cut = device_cut(ctx, fg, level_labels[f]);
            const u64 coarse_cut = device_cut(ctx, h.levels[c], level_labels[c]);
            std::vector<u64> a(k), b(k);
            GP_CUDA(cudaMemcpyAsync(a.data(), fine_loads, sizeof(u64) * k, cudaMemcpyDeviceToHost, s));
            GP_CUDA(cudaMemcpyAsync(b.data(), loads, sizeof(u64) * k, cudaMemcpyDeviceToHost, s));
            GP_CUDA(cudaStreamSynchronize(s));
            if (fine_cut != coarse_cut || fine_cut != last_cut || a != b)
                fail(GP_INTERNAL, "GPU projection failed cut or part-weight preservation");
        }
        GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, loads, sizeof(u64) * k, cudaMemcpyDeviceToHost, s));
        GP_CUDA(cudaStreamSynchronize(s));
        maxload = 0;
        for (int p = 0; p < k; ++p) maxload = std::max<u64>(maxload, ctx.host_scalars[p]);
        const bool refine_here = f == 0 || maxload > cap || static_cast<double>(fg.n) >= 2.0 * static_cast<double>(last_refined);
        LevelResult lr;
        if (refine_here) {
            lr = refine(fg, level_labels[f], true, last_cut);
            if (!lr.repair_failed) last_refined = fg.n;
            out.levels_refined += lr.refined;
        } else {
            lr.cut = last_cut;
        }
        last_cut = lr.cut;
    }
    GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, loads, sizeof(u64) * k, cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    maxload = 0;
    for (int p = 0; p < k; ++p) maxload = std::max<u64>(maxload, ctx.host_scalars[p]);
    if (maxload > cap) fail(GP_INTERNAL, "final original partition violates capacity");
    if (verify && device_cut(ctx, h.levels[0], labels) != last_cut) fail(GP_INTERNAL, "final cut differs from CSR scan");
    out.cut = last_cut;
    out.max_load = maxload;
    return out;
}

// refine_partition (src/refine.cu:470-481): one graph, its labels measured,
// one run_incremental_refinement with the caller's round budgets.
LevelStats refine_single(Context& ctx, const DGraph& g, int* labels, int k, double eps, const RefineBudget& budget,
                         bool log, bool verify, const Mapping& mapping) {
    cudaStream_t s = ctx.stream;
    u64* loads = ctx.persist.alloc<u64>(k);
    GP_CUDA(cudaMemsetAsync(loads, 0, sizeof(u64) * k, s));
    launch(k_loads, std::min(blocks_for(g.n, 256), 148 * 4), 256, sizeof(u64) * k, s, g.n, k,
           static_cast<const int*>(labels), g.vw, loads);
    GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, loads, sizeof(u64) * k, cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    u64 total = 0;
    for (int p = 0; p < k; ++p) total += ctx.host_scalars[p];
    if (g.incident_bound <= 0xffffffffULL) {
        LevelRefiner<u32> r(ctx, g, k, eps, labels, loads, total, log, verify, mapping, budget);
        r.run(false, 0);
        return r.stats;
    }
    LevelRefiner<u64> r(ctx, g, k, eps, labels, loads, total, log, verify, mapping, budget);
    r.run(false, 0);
    return r.stats;
}

}  // namespace gp
