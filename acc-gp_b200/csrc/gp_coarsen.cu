// Coarsening on the B200: stable-receiver aggregation and exact coarse-CSR
// contraction (Acc-GPart src/coarsen.cu, src/coarsening/*.cuh).
//
// Per level (aggregate_typed, src/coarsen.cu:467-1380):
//   seed matching -> <=4 rounds of {frozen roles, exact per-cluster
//   affinities, admission, commit} -> isolated packing -> two-hop pairing ->
//   compaction; then contraction (src/coarsen.cu:1394-1673).
// Every rule reproduces the reference exactly; the kernels differ: affinity
// and proposal decoding are fused per degree class, admission sorts only the
// requests of targets whose total demand overflows, and the coarse CSR is
// built row-locally with one global radix sort reserved for the few huge rows.
#include "gp_graph.h"
#include "gp_primitives.cuh"

#include <algorithm>
#include <chrono>
#include <cstdio>

namespace gp {

thread_local u64 g_launches = 0;

namespace {

constexpr int kLowDegree = 8;       // SCLP_LOW_DEGREE
constexpr int kMediumDegree = 256;  // SCLP_MEDIUM_DEGREE
constexpr int kLargeDegree = kHeavyRow;   // rows above use a chunked global table
constexpr int kMediumHash = 512;          // SCLP_MEDIUM_HASH_SIZE
constexpr int kLargeHash = 2 * kHeavyRow; // shared-memory table of the large class
constexpr int kSegment = 4096;            // table slots summarised per block
constexpr int kBlockSortRow = 4096;       // contraction: one block sorts rows up to this in shared memory
constexpr int kBigSortRow = 8192;         // one 1024-thread block (dynamic shared memory) up to this
constexpr int kBigSortThreads = 1024;
constexpr int kMediumWarps = 4;

// ---------------------------------------------------------------- metadata

// record_bound_kernel (src/coarsen.cu:51-99) plus the weight invariants of
// aggregate_typed (:483-493).  Scalars: 0 max row bound, 1 unsorted,
// 2 zero weight, 3 non-unit weight, 4 max raw degree, 5 total vertex
// weight, 6 max vertex weight.
template <int W>
__global__ void __launch_bounds__(256) k_level0_meta(i64 n, const int* off, const int* nbr, const u32* ew,
                                                     const u32* vw, u64* bounds, u64* sc) {
    const int lane = threadIdx.x & (W - 1);
    constexpr int kGroups = 32 / W;  // rows per warp and pass
    const i64 warps = (static_cast<i64>(gridDim.x) * blockDim.x) >> 5;
    u64 d_max = 0, raw_max = 0, total = 0, v_max = 0;
    u32 flags = 0;
    // Warp-uniform pass count, so the group shuffles see the whole warp.
    for (i64 base = ((static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * kGroups; base < n;
         base += warps * kGroups) {
        const i64 v = base + (threadIdx.x & 31) / W;
        const bool valid = v < n;
        const i64 begin = valid ? off[v] : 0, end = valid ? off[v + 1] : 0;
        const bool heavy = end - begin > kHeavyRow;  // summed by k_level0_meta_chunks
        u64 d = 0;
        for (i64 e = begin + lane; !heavy && e < end; e += W) {
            const u64 w = edge_w(ew, e);
            d = ~0ULL - d < w ? ~0ULL : d + w;
            if (e > begin && nbr[e] <= nbr[e - 1]) flags |= 1u;
            if (!w) flags |= 2u;
            if (w != 1) flags |= 4u;
        }
#pragma unroll
        for (int s = W / 2; s; s >>= 1) {
            const u64 o = __shfl_xor_sync(0xffffffffu, d, s, W);
            d = ~0ULL - d < o ? ~0ULL : d + o;
        }
        if (valid && lane == 0) {
            bounds[v] = d;
            d_max = d > d_max ? d : d_max;
            raw_max = static_cast<u64>(end - begin) > raw_max ? static_cast<u64>(end - begin) : raw_max;
            total += vw[v];
            v_max = vw[v] > v_max ? vw[v] : v_max;
        }
    }
    block_atomic_max(sc + 0, d_max);
    if (__syncthreads_or(flags & 1u) && threadIdx.x == 0) atomicOr(sc + 1, 1ULL);
    if (__syncthreads_or(flags & 2u) && threadIdx.x == 0) atomicOr(sc + 2, 1ULL);
    if (__syncthreads_or(flags & 4u) && threadIdx.x == 0) atomicOr(sc + 3, 1ULL);
    block_atomic_max(sc + 4, raw_max);
    block_atomic_add(sc + 5, total);
    block_atomic_max(sc + 6, v_max);
}

// Heavy rows of record_bound_kernel, one block per chunk.
__global__ void k_level0_meta_chunks(DGraph g, u64* bounds, u64* sc) {
    const int c = blockIdx.x, v = g.chunk_row[c];
    const int begin = g.off[v];
    u64 d = 0;
    u32 flags = 0;
    for (int e = g.chunk_begin[c] + threadIdx.x; e < chunk_end(g, c, v); e += blockDim.x) {
        const u64 w = edge_w(g.ew, e);
        d += w;
        if (e > begin && g.nbr[e] <= g.nbr[e - 1]) flags |= 1u;
        if (!w) flags |= 2u;
        if (w != 1) flags |= 4u;
    }
    d = warp_sum(d);
    flags = __reduce_or_sync(0xffffffffu, flags);
    if ((threadIdx.x & 31) == 0) {
        if (d) atomicAdd(bounds + v, d);
        if (flags & 1u) atomicOr(sc + 1, 1ULL);
        if (flags & 2u) atomicOr(sc + 2, 1ULL);
        if (flags & 4u) atomicOr(sc + 3, 1ULL);
    }
}
__global__ void k_heavy_bound_max(i64 count, const int* heavy, const u64* bounds, u64* sc) {
    const i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (h < count) atomicMax(sc + 0, bounds[heavy[h]]);
}

// Directed edge-weight sum (packed-weight decision, src/coarsen.cu:1839-1848).
__global__ void k_weight_sum(i64 m, const u32* ew, u64* out) {
    u64 s = 0;
    for (i64 e = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; e < m; e += static_cast<i64>(gridDim.x) * blockDim.x)
        s += ew[e];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

// Degree classes (sclp_compact_degree_classes, aggregation.cuh:5-71): exact
// max degree, heavy flag and class lists, the medium class ending at
// medium_degree (at most kMediumDegree).  The reference's large class is
// split at large_narrow so that its shorter rows run with a smaller shared
// table.  Scalars: 0 max degree, 1 heavy, 2..5 list sizes (low, medium,
// large up to large_narrow, heavy), 6 heavy hash slots, 7 isolated vertices,
// 8 list size of the large rows above large_narrow.
__global__ void __launch_bounds__(256) k_degree_classes(i64 n, const int* off, int* low, int* medium, int* large,
                                                        int* heavy, int* large_wide, int medium_degree,
                                                        int large_narrow, u64* sc) {
    u64 d_max = 0, isolated = 0;
    int big = 0;
    // Block-uniform passes: the appends synchronise the block.
    for (i64 base = static_cast<i64>(blockIdx.x) * blockDim.x; base < n; base += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 v = base + threadIdx.x;
        const bool valid = v < n;
        const i64 deg = valid ? off[v + 1] - off[v] : 0;
        d_max = static_cast<u64>(deg) > d_max ? static_cast<u64>(deg) : d_max;
        big |= valid && deg >= 4096;
        isolated += valid && deg == 0;
        const int cls = !valid                ? -1
                        : deg <= kLowDegree    ? 0
                        : deg <= medium_degree ? 1
                        : deg <= large_narrow  ? 2
                        : deg <= kLargeDegree  ? 4
                                               : 3;
        block_append(static_cast<int>(v), cls == 0, low, sc + 2);
        block_append(static_cast<int>(v), cls == 1, medium, sc + 3);
        block_append(static_cast<int>(v), cls == 2, large, sc + 4);
        block_append(static_cast<int>(v), cls == 3, heavy, sc + 5);
        block_append(static_cast<int>(v), cls == 4, large_wide, sc + 8);
    }
    block_atomic_max(sc + 0, d_max);
    if (__syncthreads_or(big) && threadIdx.x == 0) atomicOr(sc + 1, 1ULL);
    block_atomic_add(sc + 7, isolated);
}

__host__ __device__ inline u64 heavy_slots(i64 deg) {
    u64 s = kLargeHash;
    while (s < 2 * static_cast<u64>(deg)) s <<= 1;
    return s;
}

struct HeavySlots {
    const int* rows;
    const int* off;
    __device__ u64 operator()(i64 i) const { return heavy_slots(off[rows[i] + 1] - off[rows[i]]); }
};

// ---------------------------------------------------------------- seed matching

// matching_choose (seed_matching.cuh:12-71): heaviest capacity-feasible
// neighbour; ties by the symmetric hash, then the larger id.
template <int W>
__global__ void k_match_choose(i64 n, const int* off, const int* nbr, const u32* ew, const u32* vw, u64 capacity,
                               u32 salt, int* choice) {
    const i64 v = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) / W;
    const int lane = threadIdx.x & (W - 1);
    const bool valid = v < n;
    int best = -1;
    u32 bw = 0, bh = 0;
    if (valid && off[v + 1] - off[v] <= 1024) {
        const u64 weight = vw[v];
        for (i64 e = off[v] + lane; e < off[v + 1]; e += W) {
            const int u = nbr[e];
            if (u == v || weight > capacity || static_cast<u64>(vw[u]) > capacity - weight) continue;
            const int lo = min(static_cast<int>(v), u), hi = max(static_cast<int>(v), u);
            const u32 h = mix32(static_cast<u32>(lo) ^ mix32(static_cast<u32>(hi) ^ salt));
            const u32 w = edge_w(ew, e);
            if (best < 0 || w > bw || (w == bw && (h > bh || (h == bh && u > best)))) { best = u; bw = w; bh = h; }
        }
    }
#pragma unroll
    for (int d = W / 2; d; d >>= 1) {
        const int ob = __shfl_xor_sync(0xffffffffu, best, d, W);
        const u32 ow = __shfl_xor_sync(0xffffffffu, bw, d, W);
        const u32 oh = __shfl_xor_sync(0xffffffffu, bh, d, W);
        if (ob >= 0 && (best < 0 || ow > bw || (ow == bw && (oh > bh || (oh == bh && ob > best))))) { best = ob; bw = ow; bh = oh; }
    }
    if (valid && lane == 0) choice[v] = best;
}

// matching_commit + matching_roots + residual_seed_weights.
__global__ void k_match_roots(i64 n, const int* choice, int* clusters) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int u = choice[v];
    int root = static_cast<int>(v);
    if (u >= 0 && choice[u] == v) root = min(static_cast<int>(v), u);
    clusters[v] = root;
}

__global__ void k_cluster_weights(i64 n, const int* clusters, const u32* vw, u64* cw) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n) atomicAdd(cw + clusters[v], static_cast<u64>(vw[v]));
}

__global__ void k_count_nonzero(i64 n, const u64* values, u64* out) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    block_atomic_add(out, i < n && values[i] != 0 ? 1ULL : 0ULL);
}

// ---------------------------------------------------------------- rounds

struct RoundParams {
    const int* off;
    const int* nbr;
    const u32* ew;
    const u32* vw;
    const int* clusters;
    const u64* cw;
    const unsigned char* roles;
    const u64* recv;  // per cluster: its weight, or all ones when its role excludes it (k_roles)
    u64 capacity;
    u32 tie_salt;
    bool filter_roles;  // receivers only, with admissibility
    bool second_on;     // regret needed
    int* proposals;
    u64* gains;
    u64* regret;
    u32* ties;
};

// residual_freeze_roles (singleton_growth.cuh:27-40); also resets proposals.
// Also writes recv[v], the cluster weight with the role folded in (all ones
// for a mover, which no capacity admits), so that considering a neighbour
// cluster is one gather instead of the role and weight gathers.
__global__ void k_roles(i64 n, const int* clusters, const u32* vw, const u64* cw, u32 salt, u32 threshold,
                        bool all_singletons, unsigned char* roles, u64* recv, int* proposals) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const u64 weight = cw[v];
    const bool role = clusters[v] == v && weight == static_cast<u64>(vw[v]) &&
                      (all_singletons || mix32(static_cast<u32>(v) ^ salt) < threshold);
    roles[v] = role;
    recv[v] = role ? ~0ULL : weight;
    proposals[v] = kInvalid;
}

// Candidate summary of one row: best (value, tie) with the reference's
// zero-value rule, the runner-up value and the connection to the own cluster.
struct Summary {
    u64 current, best, tie, second;
};

__device__ __forceinline__ bool better(u64 a, u64 ta, u64 b, u64 tb) {  // sclp_better_candidate
    return a > b || (a == b && a != 0 && ta > tb);
}
__device__ __forceinline__ void add_candidate(Summary& s, u64 value, u64 tie) {  // sclp_update_two
    if (better(value, tie, s.best, s.tie)) {
        s.second = max(s.second, s.best);
        s.best = value;
        s.tie = tie;
    } else s.second = max(s.second, value);
}
__device__ __forceinline__ void merge(Summary& s, const Summary& o) {
    s.current = max(s.current, o.current);
    if (better(o.best, o.tie, s.best, s.tie)) {
        s.second = max(max(s.second, o.second), s.best);
        s.best = o.best;
        s.tie = o.tie;
    } else s.second = max(max(s.second, o.second), o.best);
}
template <int W>
__device__ __forceinline__ void reduce_summary(Summary& s) {
#pragma unroll
    for (int d = W / 2; d; d >>= 1) {
        Summary o;
        o.current = __shfl_xor_sync(0xffffffffu, s.current, d, W);
        o.best = __shfl_xor_sync(0xffffffffu, s.best, d, W);
        o.tie = __shfl_xor_sync(0xffffffffu, s.tie, d, W);
        o.second = __shfl_xor_sync(0xffffffffu, s.second, d, W);
        merge(s, o);
    }
}

// One distinct neighbour cluster `c` with connection `conn`.
__device__ __forceinline__ void consider(const RoundParams& p, Summary& s, int v, int src, int c, u64 conn) {
    if (c == src) { s.current = conn; return; }
    if (p.filter_roles) {
        const u64 base = p.recv[c];  // all ones (above any capacity) for a mover cluster
        if (!(base != 0 && base <= p.capacity && p.cw[src] <= p.capacity - base)) return;
    }
    const u64 tie = (static_cast<u64>(mix32(static_cast<u32>(v) ^ mix32(static_cast<u32>(c)) ^ p.tie_salt)) << 32) |
                    (0xffffffffULL - static_cast<u32>(c));
    add_candidate(s, conn, tie);
}

// consider() split in two so that callers can issue the receiver gathers of
// several clusters before using any of them.
__device__ __forceinline__ void gather_cluster(const RoundParams& p, int src, int c, u64& base) {
    const bool other = p.filter_roles && c >= 0 && c != src;
    base = other ? p.recv[c] : 0;
}
__device__ __forceinline__ void consider_gathered(const RoundParams& p, Summary& s, int v, int src, u64 own, int c,
                                                  u64 conn, u64 base) {
    if (c < 0) return;
    if (c == src) { s.current = conn; return; }
    if (p.filter_roles && !(base != 0 && base <= p.capacity && own <= p.capacity - base)) return;
    const u64 tie = (static_cast<u64>(mix32(static_cast<u32>(v) ^ mix32(static_cast<u32>(c)) ^ p.tie_salt)) << 32) |
                    (0xffffffffULL - static_cast<u32>(c));
    add_candidate(s, conn, tie);
}

// sclp_decode_gain_kernel (aggregation.cuh:513-557) for a mover row.
__device__ __forceinline__ void decode(const RoundParams& p, int v, int src, const Summary& s) {
    const u64 gain = s.best > s.current ? s.best - s.current : 0;
    if (!gain) return;
    const int target = static_cast<int>(0xffffffffULL - (s.tie & 0xffffffffULL));
    if (target < 0 || target == src) return;
    p.proposals[v] = target;
    p.gains[v] = gain;
    if (p.second_on) p.regret[v] = s.best - s.second;
    p.ties[v] = static_cast<u32>(s.tie >> 32);
}

__device__ __forceinline__ bool is_mover(const RoundParams& p, int v, int& src) {
    src = p.clusters[v];
    return p.roles[src] != 0;
}

// Open-addressing tables of (cluster, connection) for the medium, large and
// heavy affinity classes, linear probing.  SplitTable: int keys (-1 = empty)
// and u64 connections, two atomics per entry.  PackedTable: one u64 per slot,
// the cluster in the high 32 bits (all ones = empty) and the connection in the
// low 32; used when every row's weight sum is below 2^32, so a slot's sum
// never carries into its key: the CAS that claims a slot deposits the first
// weight, one atomic per entry, 8 bytes per slot instead of 12.
struct SplitTable {
    int* keys;
    u64* vals;
    static constexpr bool kClaimCarriesWeight = false;
    static constexpr size_t kSlotBytes = sizeof(int) + sizeof(u64);
    __device__ __forceinline__ void clear(u64 sl) const { keys[sl] = -1; vals[sl] = 0; }
    // Previous key of the slot (-1: it was empty and now holds c).
    __device__ __forceinline__ int claim(u64 sl, int c, u32) const { return atomicCAS(keys + sl, -1, c); }
    __device__ __forceinline__ void add(u64 sl, u32 w) const { atomicAdd(vals + sl, static_cast<u64>(w)); }
    __device__ __forceinline__ void read(u64 sl, int& c, u64& conn) const {
        c = keys[sl];
        conn = c >= 0 ? vals[sl] : 0;
    }
};
constexpr u64 kEmptySlot = 0xffffffff00000000ULL;
struct PackedTable {
    int* keys;  // unused
    u64* vals;  // the packed slots
    static constexpr bool kClaimCarriesWeight = true;
    static constexpr size_t kSlotBytes = sizeof(u64);
    __device__ __forceinline__ void clear(u64 sl) const { vals[sl] = kEmptySlot; }
    __device__ __forceinline__ int claim(u64 sl, int c, u32 w) const {
        const u64 prev = atomicCAS(vals + sl, kEmptySlot, (static_cast<u64>(static_cast<u32>(c)) << 32) | w);
        return static_cast<int>(prev >> 32);
    }
    __device__ __forceinline__ void add(u64 sl, u32 w) const { atomicAdd(vals + sl, static_cast<u64>(w)); }
    __device__ __forceinline__ void read(u64 sl, int& c, u64& conn) const {
        const u64 x = vals[sl];
        c = static_cast<int>(x >> 32);
        conn = x & 0xffffffffULL;
    }
};

// Adds the entries first, first + stride, ... < end of row v into table T
// of mask + 1 slots.  Four entries per thread go through together, so that
// their neighbour and cluster gathers and their claims are in flight at once.
template <class Table, class Index>
__device__ __forceinline__ void hash_row(const RoundParams& p, int v, Index first, Index end, int stride, const Table& T,
                                         u64 mask) {
    constexpr int kUnroll = 4;
    for (Index e0 = first; e0 < end; e0 += kUnroll * stride) {
        int u[kUnroll], c[kUnroll];
        u32 w[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            const Index e = e0 + j * stride;
            u[j] = e < end ? p.nbr[e] : v;
        }
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            c[j] = u[j] != v ? p.clusters[u[j]] : -1;
            w[j] = u[j] != v ? edge_w(p.ew, e0 + j * stride) : 0;
        }
        u64 sl[kUnroll];
        int prev[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            sl[j] = mix32(static_cast<u32>(c[j])) & mask;
            prev[j] = c[j] >= 0 ? T.claim(sl[j], c[j], w[j]) : -1;
        }
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            if (c[j] < 0) continue;
            while (prev[j] != -1 && prev[j] != c[j]) {
                sl[j] = (sl[j] + 1) & mask;
                prev[j] = T.claim(sl[j], c[j], w[j]);
            }
            if (prev[j] == c[j] || !Table::kClaimCarriesWeight) T.add(sl[j], w[j]);
        }
    }
}

// consider() for the table slots first, first + stride, ... < size, four
// slots per step with their gathers in flight together.
template <class Table, class Slot>
__device__ __forceinline__ void consider_slots(const RoundParams& p, Summary& s, int v, int src, const Table& T,
                                               Slot first, Slot size, int stride) {
    const u64 own = p.filter_roles ? p.cw[src] : 0;
    for (Slot s0 = first; s0 < size; s0 += 4 * stride) {
        int c[4];
        u64 conn[4], base[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const Slot sl = s0 + j * stride;
            c[j] = -1;
            conn[j] = 0;
            if (sl < size) T.read(sl, c[j], conn[j]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) gather_cluster(p, src, c[j], base[j]);
#pragma unroll
        for (int j = 0; j < 4; ++j) consider_gathered(p, s, v, src, own, c[j], conn[j], base[j]);
    }
}

// Rows of degree <= 8: one 8-lane group per row; equal clusters are grouped
// with match_any (sclp_affinity_low_match_kernel, aggregation.cuh:268-341).
__global__ void k_affinity_low(i64 count, const int* rows, RoundParams p) {
    const int lane = threadIdx.x & 31, sub = lane & 7;
    const i64 index = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 3;
    int v = -1, src = -1;
    bool row = index < count;
    if (row) {
        v = rows ? rows[index] : static_cast<int>(index);
        row = is_mover(p, v, src);
    }
    bool valid = false;
    int c = kInvalid;
    u64 w = 0;
    if (row) {
        const i64 begin = p.off[v], deg = p.off[v + 1] - begin;
        if (sub < deg) {
            const int u = p.nbr[begin + sub];
            if (u != v) { valid = true; c = p.clusters[u]; w = edge_w(p.ew, begin + sub); }
        }
    }
    // Group equal clusters only among this row's 8 lanes.
    const unsigned active = __ballot_sync(0xffffffffu, valid) & (0xffu << (lane & 24));
    Summary s{0, 0, 0, 0};
    if (valid) {
        const unsigned peers = __match_any_sync(active, c);
        u64 conn = 0;
        for (unsigned rem = peers; rem; rem &= rem - 1) conn += __shfl_sync(peers, w, __ffs(rem) - 1);
        if (lane == __ffs(peers) - 1) consider(p, s, v, src, c, conn);
    }
    reduce_summary<8>(s);
    if (row && sub == 0) decode(p, v, src, s);
}

// Rows of degree 9..256: one warp per row; up to 32 entries one per lane
// with match_any, longer rows through a 512-slot shared hash
// (sclp_affinity_medium_hash_kernel, aggregation.cuh:343-422).
template <class Table>
__global__ void __launch_bounds__(kMediumWarps * 32) k_affinity_medium(i64 count, const int* rows, RoundParams p) {
    __shared__ __align__(16) unsigned char raw[kMediumWarps * kMediumHash * Table::kSlotBytes];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    u64* vals = reinterpret_cast<u64*>(raw);
    const Table T{reinterpret_cast<int*>(vals + kMediumWarps * kMediumHash) + wib * kMediumHash, vals + wib * kMediumHash};
    for (i64 index = static_cast<i64>(blockIdx.x) * kMediumWarps + wib; index < count;
         index += static_cast<i64>(gridDim.x) * kMediumWarps) {
        const int v = rows[index];
        int src;
        if (!is_mover(p, v, src)) continue;
        const i64 begin = p.off[v], end = p.off[v + 1];
        if (end - begin <= 32) {
            // One entry per lane: equal clusters are grouped with match_any,
            // no table needed (as k_affinity_low does for 8 lanes).
            const i64 e = begin + lane;
            const int u = e < end ? p.nbr[e] : v;
            const bool valid = u != v;
            const int c = valid ? p.clusters[u] : kInvalid;
            const u64 w = valid ? edge_w(p.ew, e) : 0;
            const unsigned active = __ballot_sync(0xffffffffu, valid);
            Summary s{0, 0, 0, 0};
            if (valid) {
                const unsigned peers = __match_any_sync(active, c);
                u64 conn = 0;
                for (unsigned rem = peers; rem; rem &= rem - 1) conn += __shfl_sync(peers, w, __ffs(rem) - 1);
                if (lane == __ffs(peers) - 1) consider(p, s, v, src, c, conn);
            }
            reduce_summary<32>(s);
            if (lane == 0) decode(p, v, src, s);
            continue;
        }
        int size = 32;
        while (size < 2 * (end - begin)) size <<= 1;
        for (int sl = lane; sl < size; sl += 32) T.clear(sl);
        __syncwarp();
        hash_row(p, v, begin + lane, end, 32, T, static_cast<u64>(size - 1));
        __syncwarp();
        Summary s{0, 0, 0, 0};
        consider_slots(p, s, v, src, T, lane, size, 32);
        reduce_summary<32>(s);
        if (lane == 0) decode(p, v, src, s);
        __syncwarp();
    }
}

// Rows of degree 257..kLargeDegree: a 256-thread block per row with an
// open-addressing table in shared memory of at least twice the row's
// entries (values first, then keys).
template <class Table>
__global__ void __launch_bounds__(256, 5) k_affinity_large(i64 count, const int* rows, RoundParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Summary warp_sum_s[8];
    const int v = rows[blockIdx.x];
    int src;
    if (!is_mover(p, v, src)) return;
    const i64 begin = p.off[v], end = p.off[v + 1];
    u64 size = 32;
    while (size < 2 * static_cast<u64>(end - begin)) size <<= 1;
    u64* vals = reinterpret_cast<u64*>(smem_raw);
    const Table T{reinterpret_cast<int*>(vals + size), vals};
    for (u64 sl = threadIdx.x; sl < size; sl += blockDim.x) T.clear(sl);
    __syncthreads();
    hash_row(p, v, begin + static_cast<i64>(threadIdx.x), end, static_cast<int>(blockDim.x), T, size - 1);
    __syncthreads();
    Summary s{0, 0, 0, 0};
    consider_slots(p, s, v, src, T, static_cast<u64>(threadIdx.x), size, static_cast<int>(blockDim.x));
    reduce_summary<32>(s);
    if ((threadIdx.x & 31) == 0) warp_sum_s[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < 8 ? warp_sum_s[threadIdx.x] : Summary{0, 0, 0, 0};
        reduce_summary<32>(s);
        if (threadIdx.x == 0) decode(p, v, src, s);
    }
}

// Rows above kHeavyRow: every chunk inserts its entries into the row's
// global open-addressing table; segments of the table are then summarised
// block-wise and the partial summaries merged per row.
template <class Table>
__global__ void __launch_bounds__(256) k_affinity_heavy_insert(DGraph g, const u64* table_off, int* keys, u64* vals,
                                                                RoundParams p) {
    const int c = blockIdx.x, v = g.chunk_row[c];
    int src;
    if (!is_mover(p, v, src)) return;
    const int h = g.chunk_hidx[c];
    const u64 size = heavy_slots(g.off[v + 1] - g.off[v]);
    hash_row(p, v, g.chunk_begin[c] + static_cast<int>(threadIdx.x), chunk_end(g, c, v), static_cast<int>(blockDim.x),
             Table{keys + table_off[h], vals + table_off[h]}, size - 1);
}
// Also empties the slots it read, so the tables start the next round clean
// without clearing them all.  Each thread holds 16 slots of the segment,
// 256 apart, all loaded before any is used.
template <class Table>
__global__ void __launch_bounds__(256) k_affinity_heavy_summary(const int* heavy, const int* seg_hidx,
                                                                 const int* seg_index, const u64* table_off, int* keys,
                                                                 u64* vals, RoundParams p, Summary* partial) {
    constexpr int kPerThread = kSegment / 256;
    __shared__ Summary warp_part[8];
    const int sg = blockIdx.x, h = seg_hidx[sg], v = heavy[h];
    int src;
    if (!is_mover(p, v, src)) return;
    const u64 base = table_off[h] + static_cast<u64>(seg_index[sg]) * kSegment + threadIdx.x;
    const Table T{keys + base, vals + base};
    int c[kPerThread];
    u64 conn[kPerThread];
#pragma unroll
    for (int j = 0; j < kPerThread; ++j) T.read(static_cast<u64>(j) * 256, c[j], conn[j]);
    Summary sm{0, 0, 0, 0};
    const u64 own = p.filter_roles ? p.cw[src] : 0;
#pragma unroll
    for (int j0 = 0; j0 < kPerThread; j0 += 4) {
        u64 cwt[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) gather_cluster(p, src, c[j0 + q], cwt[q]);
#pragma unroll
        for (int q = 0; q < 4; ++q) consider_gathered(p, sm, v, src, own, c[j0 + q], conn[j0 + q], cwt[q]);
    }
#pragma unroll
    for (int j = 0; j < kPerThread; ++j)
        if (c[j] >= 0) T.clear(static_cast<u64>(j) * 256);
    reduce_summary<32>(sm);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = sm;
    __syncthreads();
    if (threadIdx.x < 32) {
        sm = threadIdx.x < 8 ? warp_part[threadIdx.x] : Summary{0, 0, 0, 0};
        reduce_summary<32>(sm);
        if (threadIdx.x == 0) partial[sg] = sm;
    }
}
__global__ void k_affinity_heavy_finish(i64 count, const int* heavy, const int* seg_off, const Summary* partial,
                                        RoundParams p) {
    const int lane = threadIdx.x & 31;
    const i64 h = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (h >= count) return;
    const int v = heavy[h];
    int src;
    if (!is_mover(p, v, src)) return;
    Summary sm{0, 0, 0, 0};
    for (int i = seg_off[h] + lane; i < seg_off[h + 1]; i += 32) merge(sm, partial[i]);
    reduce_summary<32>(sm);
    if (lane == 0) decode(p, v, src, sm);
}
struct HeavySegments {
    const int* rows;
    const int* off;
    i64 count;
    __device__ int operator()(i64 i) const {
        return i >= count ? 0 : static_cast<int>(heavy_slots(off[rows[i] + 1] - off[rows[i]]) / kSegment);
    }
};
__global__ void k_emit_segments(i64 count, const int* heavy, const int* off, const int* seg_off, int* seg_hidx,
                                int* seg_index) {
    const i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (h >= count) return;
    const int segs = static_cast<int>(heavy_slots(off[heavy[h] + 1] - off[heavy[h]]) / kSegment);
    for (int i = 0; i < segs; ++i) {
        seg_hidx[seg_off[h] + i] = static_cast<int>(h);
        seg_index[seg_off[h] + i] = i;
    }
}

// Admission (src/coarsen.cu:1015-1075).  Total demand per target first;
// requests to a target whose whole demand fits are accepted without any
// ordering, the rest are ordered by (target, regret desc, tie desc, vertex).
__global__ void k_requests(i64 n, const int* proposals, const u32* vw, u64* demand) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n && proposals[v] != kInvalid) atomicAdd(demand + proposals[v], static_cast<u64>(vw[v]));
}

// accept: 0 reject, 1 accept, 2 needs the ordered prefix test.
__global__ void k_classify(i64 n, const int* proposals, const u64* cw, const u64* demand, u64 capacity,
                           unsigned char* accept) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int t = proposals[v];
    if (t == kInvalid) { accept[v] = 0; return; }
    const u64 base = cw[t];
    accept[v] = base > capacity ? 0 : demand[t] <= capacity - base ? 1 : 2;
}

struct NeedsOrder {
    const unsigned char* accept;
    __device__ bool operator()(i64 v) const { return accept[v] == 2; }
};
struct HasValue {
    const int* values;
    __device__ bool operator()(i64 v) const { return values[v] != kInvalid; }
};

// Keys for the LSD passes over an ordered list of vertices.
__global__ void k_key_tie(i64 count, const u32* items, const u32* ties, u64* keys) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) keys[i] = static_cast<u64>(~ties[items[i]]);
}
__global__ void k_key_gain(i64 count, const u32* items, const u64* gains, u64 mask, u64* keys) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) keys[i] = mask - (gains[items[i]] & mask);
}
__global__ void k_key_target(i64 count, const u32* items, const int* targets, u64* keys) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) keys[i] = static_cast<u64>(targets[items[i]]);
}

// order_by_target for at most one sort tile of items, in one block: each of
// the three stable stages builds its keys from the current order and sorts
// them in shared memory, the same passes the separate launches make.
__global__ void __launch_bounds__(kSortThreads) k_order_small(int count, u32* items, const u32* ties,
                                                             const u64* key_values, u64 mask, int key_bits,
                                                             const int* targets, int target_bits) {
    __shared__ SortTileSmem sm;
    u64 k[kSortItems];
    u32 v[kSortItems];
    bool valid[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const i64 i = sort_index(0, j);
        valid[j] = i < count;
        v[j] = valid[j] ? items[i] : 0u;
    }
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) k[j] = valid[j] ? static_cast<u64>(~ties[v[j]]) : 0;
    tile_sort_passes<true>(sm, k, v, valid, 0, 32);
    if (key_bits > 0) {
#pragma unroll
        for (int j = 0; j < kSortItems; ++j) k[j] = valid[j] ? mask - (key_values[v[j]] & mask) : 0;
        tile_sort_passes<true>(sm, k, v, valid, 0, key_bits);
    }
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) k[j] = valid[j] ? static_cast<u64>(targets[v[j]]) : 0;
    tile_sort_passes<true>(sm, k, v, valid, 0, target_bits);
#pragma unroll
    for (int j = 0; j < kSortItems; ++j)
        if (valid[j]) items[sort_index(0, j)] = v[j];
}

// Segment heads of an ordered list grouped by target.
__global__ void k_segment_heads(i64 count, const u32* items, const int* targets, const u64* prefix, u64* segment_base,
                                int* segment_first) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int t = targets[items[i]];
    if (i == 0 || targets[items[i - 1]] != t) {
        if (segment_base) segment_base[t] = prefix[i];
        if (segment_first) segment_first[t] = static_cast<int>(i);
    }
}

struct OrderedWeight {
    const u32* items;
    const u32* vw;
    __device__ u64 operator()(i64 i) const { return vw[items[i]]; }
};

// sclp_commit_kernel's test (aggregation.cuh:641): base <= C and the
// inclusive weight prefix within the target fits in C - base.
__global__ void k_ordered_accept(i64 count, const u32* items, const int* targets, const u32* vw, const u64* prefix,
                                 const u64* segment_base, const u64* cw, u64 capacity, unsigned char* accept) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int v = static_cast<int>(items[i]);
    const int t = targets[v];
    const u64 base = cw[t];
    const u64 inclusive = prefix[i] + vw[v] - segment_base[t];
    accept[v] = base <= capacity && inclusive <= capacity - base;
}

__global__ void k_commit(i64 n, const int* proposals, const unsigned char* accept, const u32* vw, int* clusters,
                         u64* cw) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int t = proposals[v];
    if (t == kInvalid || (accept && accept[v] != 1)) return;
    const u64 w = vw[v];
    atomicAdd(cw + clusters[v], 0ULL - w);
    atomicAdd(cw + t, w);
    clusters[v] = t;
}

// ---------------------------------------------------------------- isolated, two-hop

struct IsolatedWeight {
    const int* list;
    const u32* vw;
    __device__ u64 operator()(i64 i) const { return vw[list[i]]; }
};
struct IsIsolated {
    const int* off;
    __device__ bool operator()(i64 v) const { return off[v] == off[v + 1]; }
};

// isolated_representative_kernel / isolated_commit_kernel (aggregation.cuh:713-745);
// `prefix` is exclusive here.
__global__ void k_isolated_rep(i64 count, const int* list, const u64* prefix, const u32* vw, u64 capacity, int* reps) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int v = list[i];
    const u64 incl = prefix[i] + vw[v];
    const u64 fb = prefix[i] / capacity, lb = (incl - 1) / capacity;
    if (fb == lb) atomicMin(reps + fb, v);
}
__global__ void k_isolated_commit(i64 count, const int* list, const u64* prefix, const u32* vw, u64 capacity,
                                  const int* reps, int* clusters, u64* cw) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int v = list[i];
    const u64 incl = prefix[i] + vw[v];
    const u64 fb = prefix[i] / capacity, lb = (incl - 1) / capacity;
    if (fb != lb) return;
    const int t = reps[fb];
    if (t == v) return;
    clusters[v] = t;
    cw[v] = 0;
    atomicAdd(cw + t, static_cast<u64>(vw[v]));
}

// sclp_singleton_favorite_kernel (aggregation.cuh:654-664).
__global__ void k_favorites(i64 n, const u32* vw, const u64* cw, const int* clusters, int* proposals) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n && cw[clusters[v]] != static_cast<u64>(vw[v])) proposals[v] = kInvalid;
}

// sclp_pair_flags_kernel (aggregation.cuh:666-676): even 1-based ranks inside
// a favourite's group pair with their predecessor when both fit.
__global__ void k_pair_flags(i64 count, const u32* items, const int* favorites, const int* segment_first,
                             const u32* vw, u64 capacity, u32* flags) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int v = static_cast<int>(items[i]);
    const i64 rank = i - segment_first[favorites[v]] + 1;
    flags[i] = (rank % 2 == 0) && i > 0 && static_cast<u64>(vw[items[i - 1]]) <= capacity - vw[v];
}
struct LoadU32 {
    const u32* p;
    __device__ u32 operator()(i64 i) const { return p[i]; }
};
// sclp_two_hop_pair_commit_kernel (aggregation.cuh:678-696).
__global__ void k_pair_commit(i64 count, const u32* items, const u32* flags, const u32* positions, u64 budget,
                              const u32* vw, int* clusters, u64* cw) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count || !flags[i] || positions[i] >= budget) return;
    const int v = static_cast<int>(items[i]);
    const int s = clusters[v], t = clusters[items[i - 1]];
    if (s == t) return;
    const u64 w = vw[v];
    atomicAdd(cw + s, 0ULL - w);
    atomicAdd(cw + t, w);
    clusters[v] = t;
}

// ---------------------------------------------------------------- compaction

struct NonEmptyInt {
    const u64* cw;
    __device__ int operator()(i64 i) const { return cw[i] > 0 ? 1 : 0; }
};
__global__ void k_iota_clusters(i64 n, const u32* vw, int* clusters, u64* cw) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    clusters[v] = static_cast<int>(v);
    cw[v] = vw[v];
}
__global__ void k_count_isolated(i64 n, const int* off, u64* out) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    block_atomic_add(out, v < n && off[v] == off[v + 1] ? 1ULL : 0ULL);
}
__global__ void k_map(i64 n, const int* clusters, const int* ids, const u32* vw, int* map, u32* cvw) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int c = ids[clusters[v]];
    map[v] = c;
    atomicAdd(cvw + c, vw[v]);
}
__global__ void k_max_u32(i64 n, const u32* values, u64* out) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    block_atomic_max(out, i < n ? static_cast<u64>(values[i]) : 0ULL);
}

// ---------------------------------------------------------------- contraction

// contract_record_bounds (src/coarsen.cu:101-120) plus raw row sizes and
// member counts.
__global__ void k_contract_bounds(i64 n, const int* map, const int* off, const u64* fine_bounds, u64* coarse_bounds,
                                  int* raw, bool bounded) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int c = map[v];
    atomicAdd(raw + c, off[v + 1] - off[v]);
    const u64 a = fine_bounds[v];
    if (bounded) { atomicAdd(coarse_bounds + c, a); return; }
    u64 prev = atomicCAS(coarse_bounds + c, 0ULL, 0ULL);
    while (true) {
        const u64 sum = ~0ULL - prev < a ? ~0ULL : prev + a;
        const u64 seen = atomicCAS(coarse_bounds + c, prev, sum);
        if (seen == prev) break;
        prev = seen;
    }
}
__global__ void k_max_pair(i64 n, const u64* a, const int* b, u64* out) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    block_atomic_max(out, i < n ? a[i] : 0ULL);
    block_atomic_max(out + 1, i < n ? static_cast<u64>(b[i]) : 0ULL);
}

struct LoadInt {
    const int* p;
    __device__ int operator()(i64 i) const { return p[i]; }
};

// contraction_row_scatter (contraction_rows.cuh:18-38): every fine row is
// copied into its coarse row's raw segment; intra-cluster entries -> INT_MAX.
// The row's slot in the segment is reserved first (one atomic per row), then
// light rows are copied by 8 lanes and heavy rows chunk-parallel.
__global__ void k_row_base(i64 n, const int* off, const int* map, int* cursor, int* base) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n) base[v] = atomicAdd(cursor + map[v], off[v + 1] - off[v]);
}
// W lanes per fine row (8 for short rows, 32 when rows are long, so that a
// level of few dense rows still has enough memory requests in flight), four
// entries per lane at a time.
template <int W>
__global__ void k_scatter(i64 n, const int* off, const int* nbr, const u32* ew, const int* map, const int* base,
                          int* raw_t, u32* raw_w) {
    constexpr int U = 4;
    const i64 v = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) / W;
    const int lane = threadIdx.x % W;
    if (v >= n) return;
    const int begin = off[v], end = off[v + 1];
    if (end - begin > kHeavyRow) return;
    const int c = map[v];
    const int out = base[v] - begin;
    for (int e0 = begin + lane; e0 < end; e0 += U * W) {
        int u[U], t[U];
        u32 w[U];
#pragma unroll
        for (int j = 0; j < U; ++j) u[j] = e0 + j * W < end ? nbr[e0 + j * W] : 0;
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const bool in = e0 + j * W < end;
            t[j] = in ? map[u[j]] : 0;
            w[j] = in ? edge_w(ew, e0 + j * W) : 0u;
        }
#pragma unroll
        for (int j = 0; j < U; ++j)
            if (e0 + j * W < end) {
                raw_t[out + e0 + j * W] = t[j] == c ? INT_MAX : t[j];
                raw_w[out + e0 + j * W] = w[j];
            }
    }
}
// A block per chunk; every thread's entries (kChunk / blockDim of them) have
// their neighbour and map gathers in flight together.
__global__ void k_scatter_chunks(DGraph g, const int* map, const int* base, int* raw_t, u32* raw_w) {
    constexpr int U = 8;
    const int ch = blockIdx.x, v = g.chunk_row[ch];
    const int c = map[v];
    const int out = base[v] - g.off[v];
    const int end = chunk_end(g, ch, v), stride = static_cast<int>(blockDim.x);
    for (int e0 = g.chunk_begin[ch] + static_cast<int>(threadIdx.x); e0 < end; e0 += U * stride) {
        int u[U], t[U];
#pragma unroll
        for (int j = 0; j < U; ++j) u[j] = e0 + j * stride < end ? g.nbr[e0 + j * stride] : 0;
#pragma unroll
        for (int j = 0; j < U; ++j) t[j] = e0 + j * stride < end ? map[u[j]] : 0;
#pragma unroll
        for (int j = 0; j < U; ++j)
            if (e0 + j * stride < end) {
                raw_t[out + e0 + j * stride] = t[j] == c ? INT_MAX : t[j];
                raw_w[out + e0 + j * stride] = edge_w(g.ew, e0 + j * stride);
            }
    }
}

// Row classes by raw size: 0 <= 128 entries, 1 <= 512, 2 <= 1024, 3 <= 2048,
// 4 <= 4096, 5 <= 8192, 6 larger; sc[kRowClasses] counts the records of class 6.
constexpr int kRowClasses = 7;
__global__ void k_row_classes(i64 nc, const int* raw, int* lists, i64 stride, u64* sc) {
    const i64 c = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int r = c < nc ? raw[c] : 0;
    const int cls = c >= nc                  ? -1
                    : r <= 128               ? 0
                    : r <= 512               ? 1
                    : r <= 1024              ? 2
                    : r <= 2048              ? 3
                    : r <= kBlockSortRow     ? 4
                    : r <= kBigSortRow       ? 5
                                             : 6;
#pragma unroll
    for (int k = 0; k < kRowClasses; ++k) block_append(static_cast<int>(c), cls == k, lists + k * stride, sc + k);
    block_atomic_add(sc + kRowClasses, cls == kRowClasses - 1 ? static_cast<u64>(r) : 0ULL);
}

// contraction_warp_sort / contraction_sort_row (contraction_rows.cuh:40-116):
// striped bitonic network over Items*32 keys, then a segmented warp scan
// that sums equal keys; writes the unique sorted run back at `begin`.
// Writes the unique keys of a sorted warp row (striped: item it of lane l is
// position it*32 + l; INT_MAX marks dropped or absent entries) back at
// `begin`, summing the weights of equal keys.
template <int Items>
__device__ __forceinline__ void warp_emit_row(const int (&keys)[Items], const u32 (&vals)[Items], int begin,
                                              int* keys_io, u32* w_io, int lane, int* count_out) {
    int count = 0;
    int carry_key = INT_MAX;
    u32 carry_sum = 0;
#pragma unroll
    for (int it = 0; it < Items; ++it) {
        const int key = keys[it];
        u32 sum = vals[it];
        if (!lane && key == carry_key) sum += carry_sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int ok = __shfl_up_sync(0xffffffffu, key, d);
            const u32 os = __shfl_up_sync(0xffffffffu, sum, d);
            if (lane >= d && key == ok) sum += os;
        }
        const int next_stripe = it + 1 < Items ? keys[it + 1] : INT_MAX;
        const int following = __shfl_down_sync(0xffffffffu, key, 1);
        const int following_stripe = __shfl_sync(0xffffffffu, next_stripe, 0);
        const int next_key = lane < 31 ? following : following_stripe;
        const bool emit = key != INT_MAX && key != next_key;
        const unsigned mask = __ballot_sync(0xffffffffu, emit);
        if (emit) {
            const int out = begin + count + __popc(mask & ((1u << lane) - 1u));
            keys_io[out] = key;
            w_io[out] = sum;
        }
        count += __popc(mask);
        carry_key = __shfl_sync(0xffffffffu, key, 31);
        carry_sum = __shfl_sync(0xffffffffu, sum, 31);
    }
    *count_out = count;
}


template <int Items>
__device__ void warp_sort_row(int begin, int degree, int* keys_io, u32* w_io, int lane, int* count_out) {
    int keys[Items];
    u32 vals[Items];
#pragma unroll
    for (int it = 0; it < Items; ++it) {
        const int pos = lane + 32 * it;
        keys[it] = pos < degree ? keys_io[begin + pos] : INT_MAX;
        vals[it] = pos < degree ? w_io[begin + pos] : 0u;
    }
    for (int size = 2; size <= 32 * Items; size <<= 1) {
        for (int dist = size >> 1; dist; dist >>= 1) {
            int nk[Items];
            u32 nv[Items];
#pragma unroll
            for (int it = 0; it < Items; ++it) {
                const int index = it * 32 + lane;
                int ok;
                u32 ov;
                if (dist >= 32) {
                    ok = keys[it ^ (dist / 32)];
                    ov = vals[it ^ (dist / 32)];
                } else {
                    ok = __shfl_xor_sync(0xffffffffu, keys[it], dist);
                    ov = __shfl_xor_sync(0xffffffffu, vals[it], dist);
                }
                const bool lower = ((index & dist) == 0) == ((index & size) == 0);
                const bool take = lower ? ok < keys[it] : ok > keys[it];
                nk[it] = take ? ok : keys[it];
                nv[it] = take ? ov : vals[it];
            }
#pragma unroll
            for (int it = 0; it < Items; ++it) { keys[it] = nk[it]; vals[it] = nv[it]; }
        }
    }
    warp_emit_row<Items>(keys, vals, begin, keys_io, w_io, lane, count_out);
}

// Rows of 129..512 raw entries: stable LSD radix sort of the warp's row in
// its shared-memory slice (8-bit digits over `bits` bits; dropped entries
// carry the key nc), then the same run reduction as the network sort.
template <int Items>
__device__ void warp_radix_row(int begin, int degree, int* keys_io, u32* w_io, int lane, int* count_out, int nc,
                               int bits, int* skeys, u32* svals, u32* counts) {
    int k[Items];
    u32 v[Items];
#pragma unroll
    for (int j = 0; j < Items; ++j) {
        const int pos = j * 32 + lane;
        const int t = pos < degree ? keys_io[begin + pos] : INT_MAX;
        k[j] = t == INT_MAX ? nc : t;
        v[j] = pos < degree ? w_io[begin + pos] : 0u;
    }
    for (int shift = 0; shift < bits; shift += kRadixBits) {
        for (int d = lane; d < kRadix; d += 32) counts[d] = 0;
        __syncwarp();
        u32 rank[Items];
#pragma unroll
        for (int j = 0; j < Items; ++j) {
            const bool valid = j * 32 + lane < degree;
            const int digit = (k[j] >> shift) & (kRadix - 1);
            const unsigned active = __ballot_sync(0xffffffffu, valid);
            if (valid) {
                const unsigned peers = __match_any_sync(active, digit);
                const unsigned below = peers & ((1u << lane) - 1u);
                rank[j] = counts[digit] + __popc(below);
                __syncwarp(active);
                if (below == 0) counts[digit] += __popc(peers);
            }
            __syncwarp();
        }
        // Exclusive scan of the digit counts, eight consecutive digits a lane.
        u32 c8[kRadix / 32], sum = 0;
#pragma unroll
        for (int q = 0; q < kRadix / 32; ++q) { c8[q] = counts[lane * (kRadix / 32) + q]; sum += c8[q]; }
        u32 incl = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const u32 o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += o;
        }
        u32 run = incl - sum;
        __syncwarp();
#pragma unroll
        for (int q = 0; q < kRadix / 32; ++q) { counts[lane * (kRadix / 32) + q] = run; run += c8[q]; }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < Items; ++j)
            if (j * 32 + lane < degree) {
                const u32 p = counts[(k[j] >> shift) & (kRadix - 1)] + rank[j];
                skeys[p] = k[j];
                svals[p] = v[j];
            }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < Items; ++j)
            if (j * 32 + lane < degree) { k[j] = skeys[j * 32 + lane]; v[j] = svals[j * 32 + lane]; }
        __syncwarp();
    }
#pragma unroll
    for (int j = 0; j < Items; ++j)
        if (k[j] == nc) k[j] = INT_MAX;
    warp_emit_row<Items>(k, v, begin, keys_io, w_io, lane, count_out);
}

template <bool Long>
__global__ void __launch_bounds__(256) k_sort_rows_warp(i64 count, const int* rows, const int* raw_off, int* raw_t,
                                                        u32* raw_w, int* ucount, int nc, int bits) {
    __shared__ int skeys[Long ? 8 : 1][512];
    __shared__ u32 svals[Long ? 8 : 1][512];
    __shared__ u32 counts[Long ? 8 : 1][kRadix];
    const i64 index = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (index >= count) return;
    const int c = rows[index];
    const int begin = raw_off[c], degree = raw_off[c + 1] - begin;
    int out = 0;
    if (Long) {
        const int w = Long ? (threadIdx.x >> 5) : 0;
        if (degree <= 256)
            warp_radix_row<8>(begin, degree, raw_t, raw_w, lane, &out, nc, bits, skeys[w], svals[w], counts[w]);
        else
            warp_radix_row<16>(begin, degree, raw_t, raw_w, lane, &out, nc, bits, skeys[w], svals[w], counts[w]);
    } else {
        if (degree <= 32) warp_sort_row<1>(begin, degree, raw_t, raw_w, lane, &out);
        else if (degree <= 64) warp_sort_row<2>(begin, degree, raw_t, raw_w, lane, &out);
        else warp_sort_row<4>(begin, degree, raw_t, raw_w, lane, &out);
    }
    if (lane == 0) ucount[c] = out;
}

// Stable LSD passes over one row of `degree` raw entries, Items per thread;
// leaves the sorted keys/values in shared memory.
template <int Items>
__device__ __forceinline__ void sort_row_in_smem(int* keys, u32* vals, u32 (*warp_count)[kRadix], u32* local_base,
                                                 u32* scan_u, const int* raw_t, const u32* raw_w, int begin, int degree,
                                                 int nc, int bits) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int k[Items];
    u32 v[Items];
    bool valid[Items];
#pragma unroll
    for (int j = 0; j < Items; ++j) {
        const int i = warp * (32 * Items) + j * 32 + lane;
        valid[j] = i < degree;
        const int t = valid[j] ? raw_t[begin + i] : 0;
        k[j] = t == INT_MAX ? nc : t;
        v[j] = valid[j] ? raw_w[begin + i] : 0u;
    }
    for (int shift = 0; shift < bits; shift += kRadixBits) {
        u32 pos[Items];
        rank_tile<Items, int>(warp_count, local_base, scan_u, k, valid, shift, pos);
#pragma unroll
        for (int j = 0; j < Items; ++j)
            if (valid[j]) { keys[pos[j]] = k[j]; vals[pos[j]] = v[j]; }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < Items; ++j) {
            const int i = warp * (32 * Items) + j * 32 + lane;
            if (valid[j]) { k[j] = keys[i]; v[j] = vals[i]; }
        }
        __syncthreads();
    }
}

// Rows of 513..2048 raw entries: stable LSD radix sort by target in shared
// memory (8-bit digits over the bits of nc; dropped intra-cluster entries
// take the key nc and sort last), then one thread per run of equal keys sums
// it and writes the unique run back at the row's start.  One instantiation
// per row class (Items = 4 or 8 per thread: rows up to 1024 or 2048), each
// launched on its own list, so the shorter class runs with its own register
// count and shared memory and more blocks fit on an SM.
template <int Items>
__global__ void __launch_bounds__(256) k_sort_rows_block(const int* rows, const int* raw_off, int* raw_t, u32* raw_w,
                                                         int* ucount, int nc, int bits) {
    static_assert(Items * 256 <= 2048, "row class of the 256-thread block sort");
    __shared__ int keys[Items * 256];
    __shared__ u32 vals[Items * 256];
    __shared__ u32 warp_count[8][kRadix];
    __shared__ u32 local_base[kRadix];
    __shared__ u32 scan_u[33];
    __shared__ int scan_smem[33];
    const int c = rows[blockIdx.x];
    const int begin = raw_off[c], degree = raw_off[c + 1] - begin;
    sort_row_in_smem<Items>(keys, vals, warp_count, local_base, scan_u, raw_t, raw_w, begin, degree, nc, bits);
    // keys/vals hold the sorted row; heads of runs and their exclusive scan.
    const int per = (degree + blockDim.x - 1) / blockDim.x;
    int local = 0;
    for (int q = 0; q < per; ++q) {
        const int i = threadIdx.x * per + q;
        if (i < degree) local += keys[i] != nc && (i == 0 || keys[i] != keys[i - 1]);
    }
    int total;
    int run = block_exclusive_scan<int>(local, total, scan_smem);
    for (int q = 0; q < per; ++q) {
        const int i = threadIdx.x * per + q;
        if (i < degree && keys[i] != nc && (i == 0 || keys[i] != keys[i - 1])) {
            u64 sum = 0;
            for (int j = i; j < degree && keys[j] == keys[i]; ++j) sum += vals[j];
            raw_t[begin + run] = keys[i];
            raw_w[begin + run] = static_cast<u32>(sum);
            ++run;
        }
    }
    if (threadIdx.x == 0) ucount[c] = total;
}

// Rows of 2049..4096 (Threads 512) and 4097..8192 (Threads 1024) raw
// entries: the same in-place sort by one block of Threads threads, 8 items
// each, in dynamic shared memory.  Eight items per thread keep the register
// count at 64, so two 512-thread blocks fit on an SM where the 256-thread,
// 16-item block needed 128 registers and fit two of 256.
template <int Threads>
constexpr size_t big_sort_smem() {
    return sizeof(int) * Threads * 8 * 2 + sizeof(u32) * (Threads / 32) * kRadix + sizeof(u32) * (kRadix + 33) +
           sizeof(int) * 33;
}
template <int Threads>
__global__ void __launch_bounds__(Threads, 1024 / Threads) k_sort_rows_big(const int* rows, const int* raw_off,
                                                                          int* raw_t, u32* raw_w, int* ucount, int nc,
                                                                          int bits) {
    constexpr int kRow = Threads * 8;
    extern __shared__ __align__(16) unsigned char big_smem[];
    int* keys = reinterpret_cast<int*>(big_smem);
    u32* vals = reinterpret_cast<u32*>(keys + kRow);
    u32 (*warp_count)[kRadix] = reinterpret_cast<u32 (*)[kRadix]>(vals + kRow);
    u32* local_base = reinterpret_cast<u32*>(warp_count + Threads / 32);
    u32* scan_u = local_base + kRadix;
    int* scan_i = reinterpret_cast<int*>(scan_u + 33);
    const int c = rows[blockIdx.x];
    const int begin = raw_off[c], degree = raw_off[c + 1] - begin;
    sort_row_in_smem<8>(keys, vals, warp_count, local_base, scan_u, raw_t, raw_w, begin, degree, nc, bits);
    const int per = (degree + blockDim.x - 1) / blockDim.x;
    int local = 0;
    for (int q = 0; q < per; ++q) {
        const int i = threadIdx.x * per + q;
        if (i < degree) local += keys[i] != nc && (i == 0 || keys[i] != keys[i - 1]);
    }
    int total;
    int run = block_exclusive_scan_wide<int>(local, total, scan_i);
    for (int q = 0; q < per; ++q) {
        const int i = threadIdx.x * per + q;
        if (i < degree && keys[i] != nc && (i == 0 || keys[i] != keys[i - 1])) {
            u64 sum = 0;
            for (int j = i; j < degree && keys[j] == keys[i]; ++j) sum += vals[j];
            raw_t[begin + run] = keys[i];
            raw_w[begin + run] = static_cast<u32>(sum);
            ++run;
        }
    }
    if (threadIdx.x == 0) ucount[c] = total;
}

// Rows above 8192 raw entries: records (row rank, target) -> global radix
// sort.  Flat over records; the row of a record is found by binary search.
// With vals == nullptr the record's weight rides in the low 32 bits of its
// key word (key << 32 | weight), so the sort moves one 8-byte word per record.
// Every large row has more records than a block has threads, so the records
// of one block pass span at most two rows: one thread finds the row of the
// pass's first record by binary search and the others step past at most
// one boundary.
__global__ void k_large_records(i64 records, i64 count, const int* rows, const int* raw_off, const int* rec_off,
                                const int* raw_t, const u32* raw_w, int tbits, u64* keys, u32* vals) {
    __shared__ int s_row;
    const u64 sentinel = (1ULL << tbits) - 1;
    for (i64 base = static_cast<i64>(blockIdx.x) * blockDim.x; base < records;
         base += static_cast<i64>(gridDim.x) * blockDim.x) {
        if (threadIdx.x == 0) {
            int lo = 0, hi = static_cast<int>(count);  // last j with rec_off[j] <= base
            while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (rec_off[mid] <= base) lo = mid; else hi = mid; }
            s_row = lo;
        }
        __syncthreads();
        const i64 r = base + threadIdx.x;
        int j = s_row;
        __syncthreads();  // s_row is rewritten by the next pass
        if (r >= records) continue;
        if (j + 1 < count && rec_off[j + 1] <= r) ++j;
        const int pos = raw_off[rows[j]] + static_cast<int>(r - rec_off[j]);
        const int t = raw_t[pos];
        const u64 key = (static_cast<u64>(j) << tbits) | (t == INT_MAX ? sentinel : static_cast<u64>(t));
        if (vals) {
            keys[r] = key;
            vals[r] = raw_w[pos];
        } else {
            keys[r] = (key << 32) | raw_w[pos];
        }
    }
}
struct LargeRowSize {
    const int* rows;
    const int* raw_off;
    __device__ int operator()(i64 i) const { return raw_off[rows[i] + 1] - raw_off[rows[i]]; }
};
struct UniqueCount {
    const int* ucount;
    i64 nc;
    __device__ int operator()(i64 i) const { return i < nc ? ucount[i] : 0; }
};
// Records are (key, weight) pairs, or packed key << 32 | weight words when
// shift is 32 (vals unused).
struct RecordHead {
    const u64* keys;
    u64 sentinel_mask;
    int shift;
    __device__ u32 operator()(i64 i) const {
        const u64 k = keys[i] >> shift;
        if ((k & sentinel_mask) == sentinel_mask) return 0;
        return (i == 0 || (keys[i - 1] >> shift) != k) ? 1u : 0u;
    }
};
__global__ void k_large_write(i64 records, const u64* keys, const u32* vals, int shift, const u32* hpos, int tbits,
                              const int* rows, const int* rec_off, const int* raw_off, int* raw_t, u32* raw_w) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= records) return;
    const u64 k = keys[i] >> shift;
    const u64 tmask = (1ULL << tbits) - 1;
    if ((k & tmask) == tmask || (i > 0 && (keys[i - 1] >> shift) == k)) return;
    const int j = static_cast<int>(k >> tbits);
    u64 sum = 0;
    for (i64 r = i; r < records && (keys[r] >> shift) == k; ++r)
        sum += shift ? (keys[r] & 0xffffffffULL) : vals[r];
    const int c = rows[j];
    const int pos = raw_off[c] + static_cast<int>(hpos[i] - hpos[rec_off[j]]);
    raw_t[pos] = static_cast<int>(k & tmask);
    raw_w[pos] = static_cast<u32>(sum);
}
__global__ void k_large_counts(i64 count, const int* rows, const int* rec_off, const u32* hpos, const u32* total,
                               i64 records, int* ucount) {
    const i64 j = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const u32 first = hpos[rec_off[j]];
    const u32 last = j + 1 < count ? hpos[rec_off[j + 1]] : *total;
    ucount[rows[j]] = static_cast<int>(last - first);
}

// contraction_copy_rows (contraction_rows.cuh:140-154); heavy coarse rows by
// chunks.  W lanes per row as in k_scatter.
template <int W>
__global__ void k_copy_rows(i64 nc, const int* raw_off, const int* raw_t, const u32* raw_w, const int* off, int* nbr,
                            u32* ew) {
    constexpr int U = 4;
    const i64 c = (static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x) / W;
    const int lane = threadIdx.x % W;
    if (c >= nc) return;
    const int begin = off[c], end = off[c + 1], raw = raw_off[c];
    if (end - begin > kHeavyRow) return;
    for (int e0 = begin + lane; e0 < end; e0 += U * W) {
        int t[U];
        u32 w[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const bool in = e0 + j * W < end;
            t[j] = in ? raw_t[raw + e0 + j * W - begin] : 0;
            w[j] = in ? raw_w[raw + e0 + j * W - begin] : 0u;
        }
#pragma unroll
        for (int j = 0; j < U; ++j)
            if (e0 + j * W < end) {
                nbr[e0 + j * W] = t[j];
                ew[e0 + j * W] = w[j];
            }
    }
}
__global__ void k_copy_chunks(DGraph g, const int* raw_off, const int* raw_t, const u32* raw_w) {
    constexpr int U = 8;
    const int ch = blockIdx.x, c = g.chunk_row[ch];
    const int shift = raw_off[c] - g.off[c];
    const int end = chunk_end(g, ch, c), stride = static_cast<int>(blockDim.x);
    for (int e0 = g.chunk_begin[ch] + static_cast<int>(threadIdx.x); e0 < end; e0 += U * stride) {
        int t[U];
        u32 w[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const bool in = e0 + j * stride < end;
            t[j] = in ? raw_t[shift + e0 + j * stride] : 0;
            w[j] = in ? raw_w[shift + e0 + j * stride] : 0u;
        }
#pragma unroll
        for (int j = 0; j < U; ++j)
            if (e0 + j * stride < end) {
                g.nbr[e0 + j * stride] = t[j];
                g.ew[e0 + j * stride] = w[j];
            }
    }
}

// ---------------------------------------------------------------- chunk lists

__global__ void k_heavy_counts(i64 n, const int* off, int heavy_min, u64* sc) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    u64 rows = 0, chunks = 0, entries = 0;
    if (v < n) {
        const int d = off[v + 1] - off[v];
        if (d > heavy_min) { rows = 1; chunks = (d + kChunk - 1) / kChunk; entries = d; }
    }
    block_atomic_add(sc, rows);
    block_atomic_add(sc + 1, chunks);
    block_atomic_add(sc + 2, entries);
}
struct IsHeavyRow {
    const int* off;
    int heavy_min;
    __device__ bool operator()(i64 v) const { return off[v + 1] - off[v] > heavy_min; }
};
struct ChunkCount {
    const int* heavy;
    const int* off;
    __device__ int operator()(i64 h) const { return (off[heavy[h] + 1] - off[heavy[h]] + kChunk - 1) / kChunk; }
};
__global__ void k_emit_chunks(i64 count, const int* heavy, const int* off, const int* chunk_off, int* chunk_row,
                              int* chunk_hidx, int* chunk_begin) {
    const i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (h >= count) return;
    const int v = heavy[h], d = off[v + 1] - off[v];
    const int chunks = (d + kChunk - 1) / kChunk;
    for (int i = 0; i < chunks; ++i) {
        chunk_row[chunk_off[h] + i] = v;
        chunk_hidx[chunk_off[h] + i] = static_cast<int>(h);
        chunk_begin[chunk_off[h] + i] = off[v] + i * kChunk;
    }
}

// ---------------------------------------------------------------- host orchestration

struct Workspace {  // SclpWorkspace::Impl state (src/coarsen.cu:299-396)
    bool positive = false, unit = false, sorted_unique = false, invariants_known = false;
    bool packed_weights = false;
    i64 original_vertices = 0;
    u64 maximum_row_weight = 0, total_vw = 0, max_vw = 0;
    u64* row_bounds = nullptr;  // device, current level
};

struct AggregateOut {
    int* map = nullptr;
    u32* cvw = nullptr;
    i64 nc = 0;
    u64 max_w = 0, capacity = 0, stats_max_degree = 0;
    bool stats_heavy = false;
};

constexpr int kThreads = 256;

// Orders `items` (vertex ids, `count` of them, ascending on entry) by
// (target asc, key desc, tie desc): three stable LSD stages (one block for at
// most one sort tile).
void order_by_target(Context& ctx, i64 count, u32*& items, u32*& items_alt, const int* targets, const u64* key_values,
                     int key_bits, const u32* ties, int target_bits) {
    if (count <= kSortTile) {
        const u64 mask = key_bits >= 64 ? ~0ULL : ((1ULL << key_bits) - 1);
        launch(k_order_small, 1, kSortThreads, 0, ctx.stream, static_cast<int>(count), items, ties, key_values, mask,
               key_bits, targets, target_bits);
        return;
    }
    Arena& A = ctx.scratch;
    ArenaScope scope(A);
    u64* keys = A.alloc<u64>(static_cast<size_t>(count));
    u64* keys_alt = A.alloc<u64>(static_cast<size_t>(count));
    const int blocks = blocks_for(count, kThreads);
    launch(k_key_tie, blocks, kThreads, 0, ctx.stream, count, items, ties, keys);
    radix_sort_pairs(A, ctx.stream, count, keys, items, keys_alt, items_alt, 0, 32);
    if (key_bits > 0) {
        const u64 mask = key_bits >= 64 ? ~0ULL : ((1ULL << key_bits) - 1);
        launch(k_key_gain, blocks, kThreads, 0, ctx.stream, count, items, key_values, mask, keys);
        radix_sort_pairs(A, ctx.stream, count, keys, items, keys_alt, items_alt, 0, key_bits);
    }
    launch(k_key_target, blocks, kThreads, 0, ctx.stream, count, items, targets, keys);
    radix_sort_pairs(A, ctx.stream, count, keys, items, keys_alt, items_alt, 0, target_bits);
}

struct WriteU32Index {
    u32* dst;
    __device__ void operator()(u32 slot, i64 i) const { dst[slot] = static_cast<u32>(i); }
};

class Aggregator {
public:
    Aggregator(Context& c, const DGraph& g, Workspace& ws, const CoarsenOptions& o, int level, int factor, u32 seed,
               bool matching)
        : ctx(c), g(g), ws(ws), o(o), level(level), factor(factor), seed(seed), matching(matching) {}

    AggregateOut run();

private:
    Context& ctx;
    const DGraph& g;
    Workspace& ws;
    const CoarsenOptions& o;
    int level, factor;
    u32 seed;
    bool matching;

    int* clusters = nullptr;
    u64* cw = nullptr;
    unsigned char* roles = nullptr;
    u64* recv = nullptr;  // receiver weights (k_roles)
    int* proposals = nullptr;
    u64* gains = nullptr;
    u64* regret = nullptr;
    u32* ties = nullptr;
    int* lists[5] = {};
    i64 list_size[5] = {};
    // Global tables of the heavy rows (see k_affinity_heavy_*).
    u64* table_off = nullptr;
    int* table_keys = nullptr;  // SplitTable keys (unused when packed)
    u64* table_vals = nullptr;  // SplitTable connections, or PackedTable slots
    bool packed = false;        // every row's weight sum below 2^32: PackedTable
    u64 table_slots = 0;
    int* seg_off = nullptr;
    int* seg_hidx = nullptr;
    int* seg_index = nullptr;
    Summary* partial = nullptr;
    i64 segments = 0;
    int gain_bits = 64, target_bits = 32;

    u64 count_clusters() {
        ctx.clear_scalars(1);
        launch(k_count_nonzero, blocks_for(g.n, kThreads), kThreads, 0, ctx.stream, g.n, cw, ctx.dev_scalars);
        return ctx.read_scalars(1)[0];
    }
    void form_proposals(u64 capacity, int round, bool filter_roles, u32 threshold, bool need_regret);
    // Table-based classes: medium, large (two table sizes) and heavy rows.
    template <class Table>
    void launch_tables(const RoundParams& p) {
        if (list_size[1]) {
            const int blocks = static_cast<int>(std::min<i64>(blocks_for(list_size[1], kMediumWarps), 148 * 64));
            launch(k_affinity_medium<Table>, blocks, kMediumWarps * 32, 0, ctx.stream, list_size[1], lists[1], p);
        }
        // Shared tables of at least twice the longest row of the class.
        for (int c : {2, 4}) {
            if (!list_size[c]) continue;
            size_t slots = 32;
            while (slots < 2 * static_cast<size_t>(c == 2 ? std::min(o.mapping.large_narrow, kLargeDegree) : kLargeDegree))
                slots <<= 1;
            const size_t smem = slots * Table::kSlotBytes;
            // The limit belongs to the kernel for the whole process, and
            // worker contexts launch it from several threads: every call sets
            // the same value, the largest table (2 x kLargeDegree slots).
            GP_CUDA(cudaFuncSetAttribute(k_affinity_large<Table>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(2 * kLargeDegree * Table::kSlotBytes)));
            launch(k_affinity_large<Table>, static_cast<int>(list_size[c]), 256, smem, ctx.stream, list_size[c], lists[c], p);
        }
        if (g.heavy_count) {
            launch(k_affinity_heavy_insert<Table>, static_cast<int>(g.chunks), 256, 0, ctx.stream, g, table_off,
                   table_keys, table_vals, p);
            launch(k_affinity_heavy_summary<Table>, static_cast<int>(segments), 256, 0, ctx.stream, g.heavy, seg_hidx,
                   seg_index, table_off, table_keys, table_vals, p, partial);
        }
    }
};

void Aggregator::form_proposals(u64 capacity, int round, bool filter_roles, u32 threshold, bool need_regret) {
    const u32 role_salt = seed ^ (static_cast<u32>(level) * 0x9e3779b9U) ^ (static_cast<u32>(round) * 0x85ebca6bU) ^ 0x27d4eb2dU;
    const u32 tie_salt = seed ^ (static_cast<u32>(level) * 0xc2b2ae35U) ^ (static_cast<u32>(round) * 0x165667b1U) ^ 0xd3a2646cU;
    const i64 n = g.n;
    launch(k_roles, blocks_for(n, kThreads), kThreads, 0, ctx.stream, n, clusters, g.vw, cw, role_salt, threshold,
           !filter_roles, roles, recv, proposals);
    RoundParams p{g.off, g.nbr, g.ew, g.vw, clusters, cw, roles, recv, capacity, tie_salt, filter_roles,
                  filter_roles && need_regret, proposals, gains, regret, ties};
    if (list_size[0])
        launch(k_affinity_low, blocks_for(list_size[0] * 8, kThreads), kThreads, 0, ctx.stream, list_size[0], lists[0], p);
    if (packed) launch_tables<PackedTable>(p);
    else launch_tables<SplitTable>(p);
    if (g.heavy_count) {
        launch(k_affinity_heavy_finish, blocks_for(g.heavy_count * 32, kThreads), kThreads, 0, ctx.stream,
               g.heavy_count, g.heavy, seg_off, partial, p);
    }
}

AggregateOut Aggregator::run() {
    Arena& A = ctx.scratch;
    cudaStream_t s = ctx.stream;
    const i64 n = g.n;
    const int vb = blocks_for(n, kThreads);
    AggregateOut out;
    const u64 total = ws.total_vw, maxv = ws.max_vw;
    const u64 denom = static_cast<u64>(factor) * static_cast<u64>(o.parts);
    out.capacity = std::max(maxv, total / denom + (total % denom != 0));
    const u64 C = out.capacity;

    clusters = A.alloc<int>(n);
    cw = A.alloc<u64>(n);
    roles = A.alloc<unsigned char>(n);
    recv = A.alloc<u64>(n);
    proposals = A.alloc<int>(n);
    gains = A.alloc<u64>(n);
    regret = A.alloc<u64>(n);
    ties = A.alloc<u32>(n);
    i64 cluster_count = n;
    if (matching) {  // src/coarsen.cu:505-535
        int* choice = proposals;
        const u32 salt = seed ^ (static_cast<u32>(level) * 0x9e3779b9U);
        if (g.m / n < 8)
            launch(k_match_choose<1>, vb, kThreads, 0, s, n, g.off, g.nbr, g.ew, g.vw, C, salt, choice);
        else
            launch(k_match_choose<32>, blocks_for(n * 32, kThreads), kThreads, 0, s, n, g.off, g.nbr, g.ew, g.vw, C, salt, choice);
        launch(k_match_roots, vb, kThreads, 0, s, n, choice, clusters);
        GP_CUDA(cudaMemsetAsync(cw, 0, sizeof(u64) * n, s));
        launch(k_cluster_weights, vb, kThreads, 0, s, n, clusters, g.vw, cw);
        cluster_count = static_cast<i64>(count_clusters());
    } else {
        launch(k_iota_clusters, vb, kThreads, 0, s, n, g.vw, clusters, cw);
    }
    // A slot's connection is at most its row's weight sum.
    packed = ws.maximum_row_weight < 0xffffffffULL;
    // Degree classes, once per level.
    i64 isolated = 0;
    {
        for (int c = 0; c < 5; ++c) lists[c] = nullptr;
        if (g.maximum_degree <= kLowDegree) {
            out.stats_max_degree = g.maximum_degree;
            out.stats_heavy = false;
            list_size[0] = n;
            list_size[1] = list_size[2] = list_size[3] = list_size[4] = 0;
            ctx.clear_scalars(1);
            launch(k_count_isolated, vb, kThreads, 0, s, n, g.off, ctx.dev_scalars);
            isolated = static_cast<i64>(ctx.read_scalars(1)[0]);
        } else {
            int* storage = A.alloc<int>(static_cast<size_t>(n) * 5);
            for (int c = 0; c < 5; ++c) lists[c] = storage + static_cast<size_t>(n) * c;
            ctx.clear_scalars(9);
            launch(k_degree_classes, static_cast<int>(std::min<i64>(vb, 148 * 8)), kThreads, 0, s, n, g.off, lists[0],
                   lists[1], lists[2], lists[3], lists[4], std::min(o.mapping.medium_degree, kMediumDegree),
                   std::min(o.mapping.large_narrow, kLargeDegree), ctx.dev_scalars);
            const u64* sc = ctx.read_scalars(9);
            out.stats_max_degree = sc[0];
            out.stats_heavy = sc[1] != 0;
            for (int c = 0; c < 4; ++c) list_size[c] = static_cast<i64>(sc[2 + c]);
            list_size[4] = static_cast<i64>(sc[8]);
            isolated = static_cast<i64>(sc[7]);
            if (g.heavy_count) {
                const i64 hc = g.heavy_count;
                table_off = A.alloc<u64>(hc);
                seg_off = A.alloc<int>(hc + 1);
                exclusive_scan<u64>(A, s, hc, HeavySlots{g.heavy, g.off}, table_off, ctx.dev_scalars);
                exclusive_scan<int>(A, s, hc + 1, HeavySegments{g.heavy, g.off, hc}, seg_off,
                                    reinterpret_cast<int*>(ctx.dev_scalars + 1));
                const u64* hs = ctx.read_scalars(2);
                table_slots = hs[0];
                segments = static_cast<i64>(hs[1] & 0xffffffffULL);
                table_vals = A.alloc<u64>(table_slots);
                table_keys = packed ? nullptr : A.alloc<int>(table_slots);
                // Cleared once; every round's summary empties what it used.
                if (packed) {
                    fill<u64>(s, table_vals, static_cast<i64>(table_slots), kEmptySlot);
                } else {
                    GP_CUDA(cudaMemsetAsync(table_keys, 0xff, sizeof(int) * table_slots, s));
                    GP_CUDA(cudaMemsetAsync(table_vals, 0, sizeof(u64) * table_slots, s));
                }
                seg_hidx = A.alloc<int>(segments);
                seg_index = A.alloc<int>(segments);
                partial = A.alloc<Summary>(segments);
                launch(k_emit_segments, blocks_for(hc, kThreads), kThreads, 0, s, hc, g.heavy, g.off, seg_off, seg_hidx,
                       seg_index);
            }
        }
    }
    // row_gain_bits (src/coarsen.cu:649-656) and target_bits.
    target_bits = std::max(1, bit_length(static_cast<u64>(n - 1)));
    gain_bits = std::max(1, std::min(ws.packed_weights ? 32 : 64, bit_length(ws.maximum_row_weight)));

    const i64 desired = (n + 1) / 2;
    u64 bound = matching ? (maxv > C / 2 ? C : 2 * maxv) : maxv;
    unsigned char* accept = A.alloc<unsigned char>(n);
    u64* demand = A.alloc<u64>(n);
    for (int round = 0; round < 4; ++round) {  // src/coarsen.cu:982-1128
        if (static_cast<double>(cluster_count) <= 0.60 * n) break;
        const i64 removable = std::max<i64>(0, cluster_count - desired);
        const double fraction = std::min(0.50, static_cast<double>(removable) / static_cast<double>(cluster_count));
        const auto threshold = static_cast<u32>(fraction * 4294967296.0);
        const u64 room = C - bound;
        const u64 degree = out.stats_max_degree;
        const bool all_fit = o.fast_path && (degree == 0 || bound <= room / maxv / degree);
        const u64 next_bound = all_fit ? bound + bound * degree * maxv : C;
        form_proposals(C, round, true, threshold, !all_fit);
        if (all_fit) {
            launch(k_commit, vb, kThreads, 0, s, n, proposals, static_cast<const unsigned char*>(nullptr), g.vw, clusters, cw);
        } else {
            GP_CUDA(cudaMemsetAsync(demand, 0, sizeof(u64) * n, s));
            launch(k_requests, vb, kThreads, 0, s, n, proposals, g.vw, demand);
            launch(k_classify, vb, kThreads, 0, s, n, proposals, cw, demand, C, accept);
            ArenaScope rs(A);
            u32* items = A.alloc<u32>(n);
            u32* count_dev = reinterpret_cast<u32*>(ctx.dev_scalars);
            select_if(A, s, n, NeedsOrder{accept}, WriteU32Index{items}, count_dev);
            const i64 count = static_cast<i64>(static_cast<u32>(ctx.read_scalars(1)[0] & 0xffffffffULL));
            if (count > 0) {
                u32* items_alt = A.alloc<u32>(count);
                order_by_target(ctx, count, items, items_alt, proposals, regret, gain_bits, ties, target_bits);
                u64* prefix = A.alloc<u64>(count);
                exclusive_scan<u64>(A, s, count, OrderedWeight{items, g.vw}, prefix, static_cast<u64*>(nullptr));
                const int cb = blocks_for(count, kThreads);
                launch(k_segment_heads, cb, kThreads, 0, s, count, items, proposals, prefix, demand, static_cast<int*>(nullptr));
                launch(k_ordered_accept, cb, kThreads, 0, s, count, items, proposals, g.vw, prefix, demand, cw, C, accept);
            }
            launch(k_commit, vb, kThreads, 0, s, n, proposals, accept, g.vw, clusters, cw);
        }
        const i64 before = cluster_count;
        cluster_count = static_cast<i64>(count_clusters());
        if (cluster_count > before) fail(GP_INTERNAL, "residual singleton merge accounting failed");
        bound = next_bound;
        if (o.log)
            std::printf("ml_residual_round level=%d round=%d regret_elided=%d clusters=%lld\n", level, round,
                        all_fit ? 1 : 0, static_cast<long long>(cluster_count));
        if (static_cast<double>(cluster_count) <= 0.60 * n) break;
    }
    if (o.pack_isolated && isolated > 1) {  // src/coarsen.cu:1130-1161
        ArenaScope is(A);
        int* list = A.alloc<int>(isolated);
        u64* prefix = A.alloc<u64>(isolated);
        select_if(A, s, n, IsIsolated{g.off}, WriteIndex{list}, static_cast<u32*>(nullptr));
        u64* total_dev = ctx.dev_scalars;
        exclusive_scan<u64>(A, s, isolated, IsolatedWeight{list, g.vw}, prefix, total_dev);
        const u64 iso_total = ctx.read_scalars(1)[0];
        const i64 bins = static_cast<i64>(iso_total / C + (iso_total % C != 0));
        int* reps = A.alloc<int>(bins);
        fill<int>(s, reps, bins, INT_MAX);
        const int ib = blocks_for(isolated, kThreads);
        launch(k_isolated_rep, ib, kThreads, 0, s, isolated, list, prefix, g.vw, C, reps);
        launch(k_isolated_commit, ib, kThreads, 0, s, isolated, list, prefix, g.vw, C, reps, clusters, cw);
        cluster_count = static_cast<i64>(count_clusters());
    }
    if (static_cast<double>(cluster_count) > 0.60 * n) {  // two-hop, src/coarsen.cu:1166-1259
        form_proposals(C, 4, false, 0, false);
        launch(k_favorites, vb, kThreads, 0, s, n, g.vw, cw, clusters, proposals);
        ArenaScope ts(A);
        u32* items = A.alloc<u32>(n);
        select_if(A, s, n, HasValue{proposals}, WriteU32Index{items}, reinterpret_cast<u32*>(ctx.dev_scalars));
        const i64 count = static_cast<i64>(static_cast<u32>(ctx.read_scalars(1)[0] & 0xffffffffULL));
        const u64 budget = static_cast<u64>(std::max<i64>(0, cluster_count - desired));
        if (count > 0 && budget > 0) {
            u32* items_alt = A.alloc<u32>(count);
            order_by_target(ctx, count, items, items_alt, proposals, gains, gain_bits, ties, target_bits);
            int* first = A.alloc<int>(n);  // first position of every favourite's group
            const int cb = blocks_for(count, kThreads);
            launch(k_segment_heads, cb, kThreads, 0, s, count, items, proposals, static_cast<const u64*>(nullptr),
                                                            static_cast<u64*>(nullptr), first);
            u32* flags = A.alloc<u32>(count);
            u32* positions = A.alloc<u32>(count);
            launch(k_pair_flags, cb, kThreads, 0, s, count, items, proposals, first, g.vw, C, flags);
            exclusive_scan<u32>(A, s, count, LoadU32{flags}, positions, static_cast<u32*>(nullptr));
            launch(k_pair_commit, cb, kThreads, 0, s, count, items, flags, positions, budget, g.vw, clusters, cw);
        }
        cluster_count = static_cast<i64>(count_clusters());
    }
    // Compaction (src/coarsen.cu:1261-1298).
    {
        ArenaScope cs(A);
        int* ids = A.alloc<int>(n);
        u64* nc_dev = ctx.dev_scalars;
        GP_CUDA(cudaMemsetAsync(nc_dev, 0, sizeof(u64), s));
        exclusive_scan<int>(A, s, n, NonEmptyInt{cw}, ids, reinterpret_cast<int*>(nc_dev));
        out.nc = static_cast<i64>(static_cast<int>(ctx.read_scalars(1)[0] & 0xffffffffULL));
        out.map = ctx.persist.alloc<int>(n);
        out.cvw = ctx.persist.alloc<u32>(out.nc);
        GP_CUDA(cudaMemsetAsync(out.cvw, 0, sizeof(u32) * out.nc, s));
        launch(k_map, vb, kThreads, 0, s, n, clusters, ids, g.vw, out.map, out.cvw);
        ctx.clear_scalars(1);
        launch(k_max_u32, blocks_for(out.nc, kThreads), kThreads, 0, s, out.nc, out.cvw, ctx.dev_scalars);
        out.max_w = ctx.read_scalars(1)[0];
    }
    ws.max_vw = out.max_w;
    if (out.max_w > C) fail(GP_INTERNAL, "SCLP coarsening exceeded cluster capacity");
    return out;
}


// contract_typed / contract_short_rows (src/coarsen.cu:1394-1673): the exact
// coarse CSR plus the carried row bounds and degree metadata.
DGraph contract(Context& ctx, const DGraph& fine, AggregateOut& agg, Workspace& ws) {
    Arena& A = ctx.scratch;
    cudaStream_t s = ctx.stream;
    const i64 n = fine.n, nc = agg.nc;
    const int vb = blocks_for(n, kThreads);
    u64* next_bounds = ctx.persist.alloc<u64>(nc);
    ArenaScope scope(A);
    int* raw = A.alloc<int>(nc + 1);
    GP_CUDA(cudaMemsetAsync(next_bounds, 0, sizeof(u64) * nc, s));
    GP_CUDA(cudaMemsetAsync(raw, 0, sizeof(int) * (nc + 1), s));
    const bool bounded = n > 0 && ws.maximum_row_weight <= ~0ULL / static_cast<u64>(n);
    launch(k_contract_bounds, vb, kThreads, 0, s, n, agg.map, fine.off, ws.row_bounds, next_bounds, raw, bounded);
    ctx.clear_scalars(2);
    launch(k_max_pair, blocks_for(nc, kThreads), kThreads, 0, s, nc, next_bounds, raw, ctx.dev_scalars);
    const u64* sc = ctx.read_scalars(2);
    const u64 row_bound = sc[0], raw_max = sc[1];
    const bool count_raw = ws.positive && n >= 65536 && fine.maximum_degree <= 512;
    const u64 raw_bound = count_raw ? raw_max : ~0ULL;
    const u64 degree_bound = count_raw && fine.maximum_degree <= 128 ? raw_bound : row_bound;
    const bool short_rows = count_raw && raw_bound <= 512;

    // Raw segments of every coarse row, filled by one scatter of the fine CSR.
    int* raw_off = A.alloc<int>(nc + 1);
    exclusive_scan<int>(A, s, nc + 1, LoadInt{raw}, raw_off, static_cast<int*>(nullptr));
    int* cursor = A.alloc<int>(nc);
    GP_CUDA(cudaMemcpyAsync(cursor, raw_off, sizeof(int) * nc, cudaMemcpyDeviceToDevice, s));
    int* raw_t = A.alloc<int>(fine.m);
    u32* raw_w = A.alloc<u32>(fine.m);
    {
        ArenaScope bs(A);
        int* base = A.alloc<int>(n);
        launch(k_row_base, vb, kThreads, 0, s, n, fine.off, agg.map, cursor, base);
        // A warp per row when the light rows (at most kHeavyRow entries; the
        // heavier ones go by chunks) average more than 64 entries.
        if (fine.m - fine.heavy_entries > 64 * (n - fine.heavy_count))
            launch(k_scatter<32>, blocks_for(n * 32, kThreads), kThreads, 0, s, n, fine.off, fine.nbr, fine.ew, agg.map,
                   static_cast<const int*>(base), raw_t, raw_w);
        else
            launch(k_scatter<8>, blocks_for(n * 8, kThreads), kThreads, 0, s, n, fine.off, fine.nbr, fine.ew, agg.map,
                   static_cast<const int*>(base), raw_t, raw_w);
        if (fine.chunks)
            launch(k_scatter_chunks, static_cast<int>(fine.chunks), 256, 0, s, fine, agg.map,
                   static_cast<const int*>(base), raw_t, raw_w);
    }
    // Row classes by raw size.
    int* lists = A.alloc<int>(static_cast<size_t>(nc) * kRowClasses);
    ctx.clear_scalars(kRowClasses + 1);
    launch(k_row_classes, blocks_for(nc, kThreads), kThreads, 0, s, nc, raw, lists, nc, ctx.dev_scalars);
    const u64* cls = ctx.read_scalars(kRowClasses + 1);
    i64 count[kRowClasses];
    for (int c = 0; c < kRowClasses; ++c) count[c] = static_cast<i64>(cls[c]);
    const i64 large_records = static_cast<i64>(cls[kRowClasses]);
    int* ucount = raw;  // raw sizes are no longer needed once the classes exist
    if (count[0])
        launch(k_sort_rows_warp<false>, blocks_for(count[0] * 32, kThreads), kThreads, 0, s, count[0], lists, raw_off,
               raw_t, raw_w, ucount, static_cast<int>(nc), bit_length(static_cast<u64>(nc)));
    if (count[1])
        launch(k_sort_rows_warp<true>, blocks_for(count[1] * 32, kThreads), kThreads, 0, s, count[1], lists + nc,
               raw_off, raw_t, raw_w, ucount, static_cast<int>(nc), bit_length(static_cast<u64>(nc)));
    auto sort_block = [&](auto items, int cls) {
        constexpr int I = decltype(items)::value;
        launch(k_sort_rows_block<I>, static_cast<int>(count[cls]), 256, 0, s, lists + cls * nc, raw_off, raw_t, raw_w,
               ucount, static_cast<int>(nc), bit_length(static_cast<u64>(nc)));
    };
    if (count[2]) sort_block(std::integral_constant<int, 4>{}, 2);
    if (count[3]) sort_block(std::integral_constant<int, 8>{}, 3);
    auto sort_big = [&](auto threads, int cls) {
        constexpr int T = decltype(threads)::value;
        constexpr size_t smem = big_sort_smem<T>();
        // Set on every call (one fixed value per instantiation): the
        // attribute belongs to the kernel, on whichever device is current.
        GP_CUDA(cudaFuncSetAttribute(k_sort_rows_big<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
        launch(k_sort_rows_big<T>, static_cast<int>(count[cls]), T, smem, s, lists + cls * nc, raw_off, raw_t, raw_w,
               ucount, static_cast<int>(nc), bit_length(static_cast<u64>(nc)));
    };
    if (count[4]) sort_big(std::integral_constant<int, 512>{}, 4);
    if (count[5]) sort_big(std::integral_constant<int, kBigSortThreads>{}, 5);
    if (count[6]) {
        ArenaScope ls(A);
        const int* large = lists + 6 * nc;
        int* rec_off = A.alloc<int>(count[6]);
        exclusive_scan<int>(A, s, count[6], LargeRowSize{large, raw_off}, rec_off,
                            static_cast<int*>(nullptr));
        const int tbits = bit_length(static_cast<u64>(nc));
        const int jbits = std::max(1, bit_length(static_cast<u64>(count[6] - 1)));
        // (row, target) keys of up to 32 bits carry the weight in the same
        // word: the sort then moves 8 bytes per record and pass, not 12.
        const bool packed = tbits + jbits <= 32;
        const int shift = packed ? 32 : 0;
        u64* keys = A.alloc<u64>(large_records);
        u64* keys_alt = A.alloc<u64>(large_records);
        u32* vals = packed ? nullptr : A.alloc<u32>(large_records);
        u32* vals_alt = packed ? nullptr : A.alloc<u32>(large_records);
        launch(k_large_records, std::min(blocks_for(large_records, kThreads), 148 * 16), kThreads, 0, s,
               large_records, count[6], large, raw_off, static_cast<const int*>(rec_off), raw_t, raw_w, tbits, keys,
               vals);
        radix_sort_pairs(A, s, large_records, keys, vals, keys_alt, vals_alt, shift, shift + tbits + jbits);
        u32* hpos = A.alloc<u32>(large_records);
        u32* heads_total = reinterpret_cast<u32*>(ctx.dev_scalars);
        exclusive_scan<u32>(A, s, large_records, RecordHead{keys, (1ULL << tbits) - 1, shift}, hpos, heads_total);
        launch(k_large_write, blocks_for(large_records, kThreads), kThreads, 0, s, large_records,
               static_cast<const u64*>(keys), static_cast<const u32*>(vals), shift, static_cast<const u32*>(hpos),
               tbits, large, rec_off, raw_off, raw_t, raw_w);
        launch(k_large_counts, blocks_for(count[6], kThreads), kThreads, 0, s, count[6], large, rec_off, hpos,
                                                                                 heads_total, large_records, ucount);
    }
    // Final offsets, then the compact copy into the level's own storage.
    DGraph coarse;
    coarse.n = nc;
    coarse.off = ctx.persist.alloc<int>(nc + 1);
    u64* m_dev = ctx.dev_scalars + 8;
    GP_CUDA(cudaMemsetAsync(m_dev, 0, sizeof(u64), s));
    exclusive_scan<int>(A, s, nc + 1, UniqueCount{ucount, nc}, coarse.off, static_cast<int*>(nullptr));
    GP_CUDA(cudaMemcpyAsync(ctx.host_scalars, coarse.off + nc, sizeof(int), cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    coarse.m = *reinterpret_cast<const int*>(ctx.host_scalars);
    coarse.nbr = ctx.persist.alloc<int>(coarse.m);
    coarse.ew = ctx.persist.alloc<u32>(coarse.m);
    build_chunks(ctx, coarse);
    if (coarse.m - coarse.heavy_entries > 64 * (nc - coarse.heavy_count))
        launch(k_copy_rows<32>, blocks_for(nc * 32, kThreads), kThreads, 0, s, nc, raw_off, raw_t, raw_w, coarse.off,
               coarse.nbr, coarse.ew);
    else
        launch(k_copy_rows<8>, blocks_for(nc * 8, kThreads), kThreads, 0, s, nc, raw_off, raw_t, raw_w, coarse.off,
               coarse.nbr, coarse.ew);
    if (coarse.chunks)
        launch(k_copy_chunks, static_cast<int>(coarse.chunks), 256, 0, s, coarse, static_cast<const int*>(raw_off),
               static_cast<const int*>(raw_t), static_cast<const u32*>(raw_w));
    coarse.vw = agg.cvw;
    coarse.implicit_unit = false;
    coarse.incident_bound = row_bound;
    if (short_rows || ws.positive) {
        coarse.maximum_degree = degree_bound;
        coarse.has_heavy_rows = degree_bound >= 4096;
    }
    ws.maximum_row_weight = row_bound;
    ws.row_bounds = next_bounds;
    return coarse;
}

}  // namespace

// Heavy-row list and chunk list of a level, in the hierarchy's storage.
void build_chunks(Context& ctx, DGraph& g, int heavy_min, Arena* storage) {
    cudaStream_t s = ctx.stream;
    Arena& out = storage ? *storage : ctx.persist;
    g.heavy_min = heavy_min;
    g.heavy = nullptr;
    g.heavy_chunk0 = nullptr;
    g.heavy_count = 0;
    g.chunks = 0;
    g.heavy_entries = 0;
    if (g.n <= 0) return;
    ctx.clear_scalars(3);
    launch(k_heavy_counts, blocks_for(g.n, kThreads), kThreads, 0, s, g.n, g.off, heavy_min, ctx.dev_scalars);
    const u64* sc = ctx.read_scalars(3);
    g.heavy_count = static_cast<i64>(sc[0]);
    g.chunks = static_cast<i64>(sc[1]);
    g.heavy_entries = static_cast<i64>(sc[2]);
    if (!g.heavy_count) return;
    g.heavy = out.alloc<int>(g.heavy_count);
    g.chunk_row = out.alloc<int>(g.chunks);
    g.chunk_hidx = out.alloc<int>(g.chunks);
    g.chunk_begin = out.alloc<int>(g.chunks);
    g.heavy_chunk0 = out.alloc<int>(g.heavy_count);
    int* chunk_off = g.heavy_chunk0;
    ArenaScope scope(ctx.scratch);
    select_if(ctx.scratch, s, g.n, IsHeavyRow{g.off, heavy_min}, WriteIndex{g.heavy}, static_cast<u32*>(nullptr));
    exclusive_scan<int>(ctx.scratch, s, g.heavy_count, ChunkCount{g.heavy, g.off}, chunk_off, static_cast<int*>(nullptr));
    launch(k_emit_chunks, blocks_for(g.heavy_count, kThreads), kThreads, 0, s, g.heavy_count, g.heavy, g.off,
           static_cast<const int*>(chunk_off), g.chunk_row, g.chunk_hidx, g.chunk_begin);
}

// coarsen_impl (src/coarsen.cu:1762-2060).
Hierarchy coarsen(Context& ctx, const DGraph& input, const CoarsenOptions& o) {
    cudaStream_t s = ctx.stream;
    Hierarchy h;
    Workspace ws;
    DGraph current = input;
    if (current.n > 0) {
        build_chunks(ctx, current);
        ws.row_bounds = ctx.persist.alloc<u64>(current.n);
        ctx.clear_scalars(7);
        const int meta_grid = static_cast<int>(std::min<i64>(blocks_for(current.n * 8, kThreads), 148 * 16));
        // 8 lanes per row unless the light rows (the heavier ones go by
        // chunks) average more than 64 entries.
        if (current.m - current.heavy_entries <= 64 * (current.n - current.heavy_count))
            launch(k_level0_meta<8>, meta_grid, kThreads, 0, s, current.n, current.off, current.nbr, current.ew,
                   current.vw, ws.row_bounds, ctx.dev_scalars);
        else
            launch(k_level0_meta<32>, meta_grid, kThreads, 0, s, current.n, current.off, current.nbr, current.ew,
                   current.vw, ws.row_bounds, ctx.dev_scalars);
        if (current.chunks) {
            // The row pass wrote 0 for heavy rows; their chunks add the sums.
            launch(k_level0_meta_chunks, static_cast<int>(current.chunks), 256, 0, s, current, ws.row_bounds,
                   ctx.dev_scalars);
            launch(k_heavy_bound_max, blocks_for(current.heavy_count, kThreads), kThreads, 0, s, current.heavy_count,
                   static_cast<const int*>(current.heavy), static_cast<const u64*>(ws.row_bounds), ctx.dev_scalars);
        }
        const u64* sc = ctx.read_scalars(7);
        ws.original_vertices = current.n;
        ws.maximum_row_weight = sc[0];
        current.incident_bound = sc[0];
        ws.sorted_unique = sc[1] == 0;
        ws.positive = sc[2] == 0;
        ws.unit = sc[3] == 0;
        current.maximum_degree = sc[4];
        current.has_heavy_rows = sc[4] >= 4096;
        ws.total_vw = sc[5];
        ws.max_vw = sc[6];
        ws.invariants_known = true;
        if (ws.unit) {
            ws.packed_weights = static_cast<u64>(current.m) <= 0xffffffffULL;
        } else {
            ctx.clear_scalars(1);
            launch(k_weight_sum, std::min(blocks_for(current.m, kThreads), 148 * 8), kThreads, 0, s, 
                current.m, current.ew, ctx.dev_scalars);
            ws.packed_weights = ctx.read_scalars(1)[0] <= 0xffffffffULL;
        }
    }
    const i64 cutoff = std::max<i64>(32, static_cast<i64>(o.cluster_size_factor) * o.parts);
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
                              (avg < 8 || current.maximum_degree <= 256) && avg < o.heavy_limit && ws.sorted_unique &&
                              ws.positive;
        const Arena::Mark mark = ctx.scratch.mark();
        const auto t_begin = std::chrono::steady_clock::now();
        Aggregator aggregator(ctx, current, ws, o, level, factor, level_seed, matching);
        AggregateOut agg = aggregator.run();
        const auto t_aggregated = std::chrono::steady_clock::now();
        current.has_heavy_rows = agg.stats_heavy;
        current.maximum_degree = agg.stats_max_degree;
        const double ratio = static_cast<double>(agg.nc) / static_cast<double>(current.n);
        if (o.log)
            std::printf("ml_coarsen_map level=%d vertices=%lld coarse_vertices=%lld ratio=%g capacity=%llu\n", level,
                        static_cast<long long>(current.n), static_cast<long long>(agg.nc), ratio,
                        static_cast<unsigned long long>(agg.capacity));
        ctx.scratch.release(mark);
        if (agg.nc >= current.n || ratio > o.stop_ratio) {
            if (o.log) std::printf("ml_coarsen_stop reason=insufficient_contraction\n");
            break;
        }
        DGraph coarse = contract(ctx, current, agg, ws);
        ctx.scratch.release(mark);
        if (o.log) {  // host time per stage; the stream is drained first
            GP_CUDA(cudaStreamSynchronize(s));
            const auto t_contracted = std::chrono::steady_clock::now();
            std::printf("ml_level_time level=%d aggregate_ms=%.3f contract_ms=%.3f\n", level,
                        std::chrono::duration<double, std::milli>(t_aggregated - t_begin).count(),
                        std::chrono::duration<double, std::milli>(t_contracted - t_aggregated).count());
        }
        if (o.verify) {
            verify_level(ctx, current, coarse, agg.map, agg.capacity);
            if (o.log) std::printf("ml_layer_verify level=%d map=ok weights=ok csr=ok projection_cut=ok\n", level);
        }
        h.levels.push_back(current);
        h.maps.push_back(agg.map);
        current = coarse;
        ws.sorted_unique = true;
    }
    h.levels.push_back(current);
    return h;
}

void keep_levels(Context& ctx, const Hierarchy& h) {
    ctx.kept.clear();
    for (size_t i = 0; i < h.levels.size(); ++i) {
        const DGraph& g = h.levels[i];
        Context::HostLevel lv;
        lv.n = g.n;
        lv.m = g.m;
        lv.off.resize(g.n + 1);
        lv.nbr.resize(g.m);
        lv.ew.resize(g.m);
        lv.vw.resize(g.n);
        GP_CUDA(cudaMemcpy(lv.off.data(), g.off, sizeof(int) * (g.n + 1), cudaMemcpyDeviceToHost));
        if (g.m) GP_CUDA(cudaMemcpy(lv.nbr.data(), g.nbr, sizeof(int) * g.m, cudaMemcpyDeviceToHost));
        if (g.ew) { if (g.m) GP_CUDA(cudaMemcpy(lv.ew.data(), g.ew, sizeof(u32) * g.m, cudaMemcpyDeviceToHost)); }
        else std::fill(lv.ew.begin(), lv.ew.end(), 1u);
        GP_CUDA(cudaMemcpy(lv.vw.data(), g.vw, sizeof(u32) * g.n, cudaMemcpyDeviceToHost));
        if (i < h.maps.size()) {
            lv.map.resize(g.n);
            GP_CUDA(cudaMemcpy(lv.map.data(), h.maps[i], sizeof(int) * g.n, cudaMemcpyDeviceToHost));
        }
        lv.meta[0] = g.maximum_degree;
        lv.meta[1] = g.has_heavy_rows;
        lv.meta[2] = g.incident_bound;
        ctx.kept.push_back(std::move(lv));
    }
}

}  // namespace gp
