// Device-wide scan, stable selection and LSD radix sort, written for this
// library (no CUB/Thrust on the hot path).  All run on one stream and use the
// arena for temporaries.  Tiles are 256 threads x 8 items.
#pragma once
#include "gp_device.cuh"

namespace gp {
namespace {  // kernels are private to each translation unit

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one value per thread (256 threads).
template <class T>
__device__ __forceinline__ T block_exclusive_scan(T value, T& total, T* smem /* >= 8 */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = value;
    for (int d = 1; d < 32; d <<= 1) {
        const T o = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += o;
    }
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T s = lane < (kScanThreads / 32) ? smem[lane] : T(0);
        T si = s;
        for (int d = 1; d < 8; d <<= 1) {
            const T o = __shfl_up_sync(0xffffffffu, si, d);
            if (lane >= d) si += o;
        }
        if (lane < (kScanThreads / 32)) smem[lane] = si - s;
        if (lane == (kScanThreads / 32) - 1) smem[8] = si;
    }
    __syncthreads();
    const T result = smem[warp] + inc - value;
    total = smem[8];
    __syncthreads();
    return result;
}

// Block-wide exclusive scan for any block of up to 1024 threads (a multiple
// of 32); smem holds at least 33 values.
template <class T>
__device__ __forceinline__ T block_exclusive_scan_wide(T value, T& total, T* smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    T inc = value;
    for (int d = 1; d < 32; d <<= 1) {
        const T o = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += o;
    }
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const T s = lane < warps ? smem[lane] : T(0);
        T si = s;
        for (int d = 1; d < 32; d <<= 1) {
            const T o = __shfl_up_sync(0xffffffffu, si, d);
            if (lane >= d) si += o;
        }
        if (lane < warps) smem[lane] = si - s;
        if (lane == 31) smem[32] = si;
    }
    __syncthreads();
    const T result = smem[warp] + inc - value;
    total = smem[32];
    __syncthreads();
    return result;
}

template <class T, class In>
__global__ void k_tile_sums(i64 n, In in, T* sums) {
    __shared__ T smem[9];
    const i64 base = static_cast<i64>(blockIdx.x) * kScanTile;
    T local = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const i64 i = base + static_cast<i64>(j) * kScanThreads + threadIdx.x;
        if (i < n) local += in(i);
    }
    T total;
    block_exclusive_scan<T>(local, total, smem);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Exclusive scan of `count` values in place, by one block; optional total.
template <class T>
__global__ void k_scan_small(i64 count, T* values, T* total) {
    __shared__ T smem[9];
    T carry = 0;
    for (i64 base = 0; base < count; base += kScanTile) {
        T v[kScanItems];
        T local = 0;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            const i64 i = base + static_cast<i64>(threadIdx.x) * kScanItems + j;
            v[j] = i < count ? values[i] : T(0);
            local += v[j];
        }
        T tile_total;
        T run = block_exclusive_scan<T>(local, tile_total, smem) + carry;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            const i64 i = base + static_cast<i64>(threadIdx.x) * kScanItems + j;
            if (i < count) values[i] = run;
            run += v[j];
        }
        carry += tile_total;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

// Up to this many tiles (4 Mi items), the writing pass of a scan or
// selection takes each tile's start from the raw tile sums (every block adds
// up the sums before it, at most eight per thread) instead of a separate
// launch that scans them.
constexpr int kDirectScanTiles = 2048;

// sums[0] + ... + sums[tiles - 1], by the whole block; every thread gets it.
template <class T>
__device__ __forceinline__ T sum_before(const T* sums, int tiles, T* smem /* >= 9 */) {
    T local = 0;
    for (int t = threadIdx.x; t < tiles; t += kScanThreads) local += sums[t];
    T total;
    block_exclusive_scan<T>(local, total, smem);
    return total;
}

// Direct: `offsets` holds the tile sums, not their exclusive scan.
template <class T, class In, bool Direct = false>
__global__ void k_scan_tiles(i64 n, In in, const T* offsets, T* out, T* total) {
    __shared__ T smem[9];
    const i64 base = static_cast<i64>(blockIdx.x) * kScanTile;
    T v[kScanItems];
    T local = 0;
    // Thread t owns the contiguous items [t*8, t*8+8) of the tile.
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const i64 i = base + static_cast<i64>(threadIdx.x) * kScanItems + j;
        v[j] = i < n ? in(i) : T(0);
        local += v[j];
    }
    T start = T(0);
    if (offsets) start = Direct ? sum_before(offsets, static_cast<int>(blockIdx.x), smem) : offsets[blockIdx.x];
    T tile_total;
    T run = block_exclusive_scan<T>(local, tile_total, smem) + start;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const i64 i = base + static_cast<i64>(threadIdx.x) * kScanItems + j;
        if (i < n) out[i] = run;
        run += v[j];
    }
    if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *total = run;
}

template <class T>
struct LoadOf {
    const T* p;
    __device__ __forceinline__ T operator()(i64 i) const { return p[i]; }
};

// out[i] = sum_{j<i} in(j); *total (device) = sum of all, when non-null.
// `out` may alias the array `in` reads from.
template <class T, class In>
void exclusive_scan(Arena& arena, cudaStream_t s, i64 n, In in, T* out, T* total) {
    if (n <= 0) {
        if (total) GP_CUDA(cudaMemsetAsync(total, 0, sizeof(T), s));
        return;
    }
    const int tiles = blocks_for(n, kScanTile);
    if (tiles == 1) {
        launch(k_scan_tiles<T, In>, 1, kScanThreads, 0, s, n, in, static_cast<const T*>(nullptr), out, total);
        return;
    }
    ArenaScope scope(arena);
    T* sums = arena.alloc<T>(static_cast<size_t>(tiles));
    launch(k_tile_sums<T, In>, tiles, kScanThreads, 0, s, n, in, sums);
    if (tiles <= kDirectScanTiles) {
        launch(k_scan_tiles<T, In, true>, tiles, kScanThreads, 0, s, n, in, static_cast<const T*>(sums), out, total);
        return;
    }
    launch(k_scan_small<T>, 1, kScanThreads, 0, s, tiles, sums, static_cast<T*>(nullptr));
    launch(k_scan_tiles<T, In>, tiles, kScanThreads, 0, s, n, in, sums, out, total);
}

// ---------------------------------------------------------------- selection

template <class Pred>
__global__ void k_select_count(i64 n, Pred pred, u32* counts) {
    __shared__ u32 smem[9];
    const i64 base = static_cast<i64>(blockIdx.x) * kScanTile;
    u32 local = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const i64 i = base + static_cast<i64>(threadIdx.x) * kScanItems + j;
        local += (i < n && pred(i)) ? 1u : 0u;
    }
    u32 total;
    block_exclusive_scan<u32>(local, total, smem);
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

template <class Pred, class Out, bool Direct = false>
__global__ void k_select_write(i64 n, Pred pred, const u32* offsets, Out out, u32* count) {
    __shared__ u32 smem[9];
    const i64 base = static_cast<i64>(blockIdx.x) * kScanTile;
    bool f[kScanItems];
    u32 local = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const i64 i = base + static_cast<i64>(threadIdx.x) * kScanItems + j;
        f[j] = i < n && pred(i);
        local += f[j];
    }
    u32 start = 0;
    if (offsets) start = Direct ? sum_before(offsets, static_cast<int>(blockIdx.x), smem) : offsets[blockIdx.x];
    u32 total;
    u32 run = block_exclusive_scan<u32>(local, total, smem) + start;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const i64 i = base + static_cast<i64>(threadIdx.x) * kScanItems + j;
        if (f[j]) out(run++, i);
    }
    if (count && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *count = run;
}

struct WriteIndex {
    int* dst;
    __device__ __forceinline__ void operator()(u32 slot, i64 i) const { dst[slot] = static_cast<int>(i); }
};

// Stable compaction: calls out(slot, i) for every i with pred(i), slots in
// ascending i; *count (device) receives the number selected.
template <class Pred, class Out>
void select_if(Arena& arena, cudaStream_t s, i64 n, Pred pred, Out out, u32* count) {
    if (n <= 0) {
        if (count) GP_CUDA(cudaMemsetAsync(count, 0, sizeof(u32), s));
        return;
    }
    const int tiles = blocks_for(n, kScanTile);
    if (tiles == 1) {
        launch(k_select_write<Pred, Out>, 1, kScanThreads, 0, s, n, pred, static_cast<const u32*>(nullptr), out, count);
        return;
    }
    ArenaScope scope(arena);
    u32* counts = arena.alloc<u32>(static_cast<size_t>(tiles));
    launch(k_select_count<Pred>, tiles, kScanThreads, 0, s, n, pred, counts);
    if (tiles <= kDirectScanTiles) {
        launch(k_select_write<Pred, Out, true>, tiles, kScanThreads, 0, s, n, pred, static_cast<const u32*>(counts), out,
               count);
        return;
    }
    launch(k_scan_small<u32>, 1, kScanThreads, 0, s, tiles, counts, static_cast<u32*>(nullptr));
    launch(k_select_write<Pred, Out>, tiles, kScanThreads, 0, s, n, pred, counts, out, count);
}

// ---------------------------------------------------------------- radix sort

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kDirectTiles = 64;  // up to this many tiles, downsweeps read the raw histogram

// Item i of a tile lives in warp i/256, register slot (i%256)/32, lane i%32,
// so the order (warp, slot, lane) is the input order and ranks stay stable.
__device__ __forceinline__ i64 sort_index(i64 base, int j) {
    return base + (threadIdx.x >> 5) * (32 * kSortItems) + j * 32 + (threadIdx.x & 31);
}

__global__ void k_radix_upsweep(i64 count, const u64* keys, int shift, u32* hist) {
    __shared__ u32 local[kRadix];
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) local[d] = 0;
    __syncthreads();
    const i64 base = static_cast<i64>(blockIdx.x) * kSortTile;
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const i64 i = sort_index(base, j);
        if (i < count) atomicAdd(&local[(keys[i] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) hist[static_cast<i64>(d) * gridDim.x + blockIdx.x] = local[d];
}

// Shared state of one sort tile: per-warp digit counts (turned into per-warp
// prefixes), the tile's digit prefix, the global base of each digit for this
// tile, and the tile's items in digit order.
struct SortTileSmem {
    u32 warp_count[kSortThreads / 32][kRadix];
    u32 local_base[kRadix];
    u32 digit_base[kRadix];
    u32 scan[9];
    u64 keys[kSortTile];
    u32 vals[kSortTile];
};
static_assert(kSortThreads == kRadix, "one digit per thread in the tile prefix");

// Position of every valid item of the tile in the tile's stable digit order:
// local_base[d] (items of smaller digits) + items of digit d in earlier warps
// + items of digit d earlier in this warp.  Returns the digit (-1: invalid).
__device__ __forceinline__ void tile_positions(SortTileSmem& sm, const u64 (&k)[kSortItems], const bool (&valid)[kSortItems],
                                               int shift, u32 (&pos)[kSortItems], int (&digit)[kSortItems]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = lane; d < kRadix; d += 32) sm.warp_count[warp][d] = 0;
    __syncwarp();
    u32 rank[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        digit[j] = valid[j] ? static_cast<int>((k[j] >> shift) & (kRadix - 1)) : -1;
        const unsigned active = __ballot_sync(0xffffffffu, valid[j]);
        if (valid[j]) {
            const unsigned peers = __match_any_sync(active, digit[j]);
            const unsigned below = peers & ((1u << lane) - 1u);
            rank[j] = sm.warp_count[warp][digit[j]] + __popc(below);
            __syncwarp(active);
            if (below == 0) sm.warp_count[warp][digit[j]] += __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    const int d = threadIdx.x;
    u32 run = 0;
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) {
        const u32 c = sm.warp_count[w][d];
        sm.warp_count[w][d] = run;
        run += c;
    }
    u32 total;
    sm.local_base[d] = block_exclusive_scan<u32>(run, total, sm.scan);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; ++j)
        if (valid[j]) pos[j] = sm.local_base[digit[j]] + sm.warp_count[warp][digit[j]] + rank[j];
}

// The same ranking for a tile of Items items per thread held in registers in
// the warp-striped layout (item j of lane l of warp w is tile index
// w*32*Items + j*32 + l), keys of any integer type.  warp_count is
// [blockDim/32][kRadix], local_base [kRadix], scan >= 33 values; blockDim.x
// is a multiple of 32 from kRadix to 1024.
template <int Items, class K>
__device__ __forceinline__ void rank_tile(u32 (*warp_count)[kRadix], u32* local_base, u32* scan, const K (&k)[Items],
                                          const bool (&valid)[Items], int shift, u32 (&pos)[Items]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = lane; d < kRadix; d += 32) warp_count[warp][d] = 0;
    __syncwarp();
    u32 rank[Items];
#pragma unroll
    for (int j = 0; j < Items; ++j) {
        const int digit = static_cast<int>((static_cast<u64>(k[j]) >> shift) & (kRadix - 1));
        const unsigned active = __ballot_sync(0xffffffffu, valid[j]);
        if (valid[j]) {
            const unsigned peers = __match_any_sync(active, digit);
            const unsigned below = peers & ((1u << lane) - 1u);
            rank[j] = warp_count[warp][digit] + __popc(below);
            __syncwarp(active);
            if (below == 0) warp_count[warp][digit] += __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    const int d = threadIdx.x;  // threads below kRadix own one digit each
    u32 run = 0;
    if (d < kRadix)
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
            const u32 c = warp_count[w][d];
            warp_count[w][d] = run;
            run += c;
        }
    u32 total;
    const u32 base = block_exclusive_scan_wide<u32>(run, total, scan);
    if (d < kRadix) local_base[d] = base;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < Items; ++j) {
        const int digit = static_cast<int>((static_cast<u64>(k[j]) >> shift) & (kRadix - 1));
        if (valid[j]) pos[j] = local_base[digit] + warp_count[warp][digit] + rank[j];
    }
}

// One pass of a multi-tile sort.  The tile is ordered by digit in shared
// memory first, so the scatter writes runs of equal digits to consecutive
// addresses instead of one isolated element per thread.
// Direct: `offsets` is the raw digit-major tile histogram and every block
// derives its own digit bases from it (for few tiles, instead of a scan).
template <bool WithValues, bool Direct>
__global__ void __launch_bounds__(kSortThreads) k_radix_downsweep(i64 count, const u64* keys, const u32* vals, int shift,
                                                                  const u32* offsets, u64* keys_out, u32* vals_out) {
    __shared__ SortTileSmem sm;
    const i64 base = static_cast<i64>(blockIdx.x) * kSortTile;
    const int tile_items = static_cast<int>(count - base < kSortTile ? count - base : kSortTile);
    if constexpr (Direct) {
        const u32* row = offsets + static_cast<i64>(threadIdx.x) * gridDim.x;
        u32 total = 0, before = 0;
        for (int t = 0; t < static_cast<int>(gridDim.x); ++t) {
            const u32 c = row[t];
            total += c;
            before += t < static_cast<int>(blockIdx.x) ? c : 0u;
        }
        u32 all;
        sm.digit_base[threadIdx.x] = block_exclusive_scan<u32>(total, all, sm.scan) + before;
    } else {
        sm.digit_base[threadIdx.x] = offsets[static_cast<i64>(threadIdx.x) * gridDim.x + blockIdx.x];
    }
    u64 k[kSortItems];
    u32 v[kSortItems];
    bool valid[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const i64 i = sort_index(base, j);
        valid[j] = i < count;
        k[j] = valid[j] ? keys[i] : 0;
        if (WithValues) v[j] = valid[j] ? vals[i] : 0;
    }
    u32 pos[kSortItems];
    int digit[kSortItems];
    tile_positions(sm, k, valid, shift, pos, digit);
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        if (!valid[j]) continue;
        sm.keys[pos[j]] = k[j];
        if (WithValues) sm.vals[pos[j]] = v[j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tile_items; i += kSortThreads) {
        const u64 key = sm.keys[i];
        const int d = static_cast<int>((key >> shift) & (kRadix - 1));
        const u32 out = sm.digit_base[d] + static_cast<u32>(i) - sm.local_base[d];
        keys_out[out] = key;
        if (WithValues) vals_out[out] = sm.vals[i];
    }
}

// The LSD passes over bits [begin_bit, end_bit) of one tile held in
// registers in the sort_index layout: every pass reorders the items through
// shared memory.
template <bool WithValues>
__device__ __forceinline__ void tile_sort_passes(SortTileSmem& sm, u64 (&k)[kSortItems], u32 (&v)[kSortItems],
                                                 const bool (&valid)[kSortItems], int begin_bit, int end_bit) {
    for (int shift = begin_bit; shift < end_bit; shift += kRadixBits) {
        u32 pos[kSortItems];
        int digit[kSortItems];
        tile_positions(sm, k, valid, shift, pos, digit);
#pragma unroll
        for (int j = 0; j < kSortItems; ++j) {
            if (!valid[j]) continue;
            sm.keys[pos[j]] = k[j];
            if (WithValues) sm.vals[pos[j]] = v[j];
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSortItems; ++j) {
            if (!valid[j]) continue;
            const i64 i = sort_index(0, j);
            k[j] = sm.keys[i];
            if (WithValues) v[j] = sm.vals[i];
        }
        __syncthreads();
    }
}

// Whole sort of at most one tile by one block; the result is written back in
// place.
template <bool WithValues>
__global__ void __launch_bounds__(kSortThreads) k_radix_tile_sort(int count, u64* keys, u32* vals, int begin_bit, int end_bit) {
    __shared__ SortTileSmem sm;
    u64 k[kSortItems];
    u32 v[kSortItems];
    bool valid[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const i64 i = sort_index(0, j);
        valid[j] = i < count;
        k[j] = valid[j] ? keys[i] : 0;
        if (WithValues) v[j] = valid[j] ? vals[i] : 0;
    }
    tile_sort_passes<WithValues>(sm, k, v, valid, begin_bit, end_bit);
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        if (!valid[j]) continue;
        const i64 i = sort_index(0, j);
        keys[i] = k[j];
        if (WithValues) vals[i] = v[j];
    }
}

// Stable LSD sort of (keys, vals) by bits [begin_bit, end_bit).  keys/vals are
// swapped with keys_alt/vals_alt as needed so that on return keys/vals hold
// the sorted sequence.  vals may be null.
inline void radix_sort_pairs(Arena& arena, cudaStream_t s, i64 count, u64*& keys, u32*& vals, u64*& keys_alt,
                             u32*& vals_alt, int begin_bit, int end_bit) {
    if (count <= 1 || end_bit <= begin_bit) return;
    if (count <= kSortTile) {
        if (vals)
            launch(k_radix_tile_sort<true>, 1, kSortThreads, 0, s, static_cast<int>(count), keys, vals, begin_bit, end_bit);
        else
            launch(k_radix_tile_sort<false>, 1, kSortThreads, 0, s, static_cast<int>(count), keys, vals, begin_bit, end_bit);
        return;
    }
    ArenaScope scope(arena);
    const int tiles = blocks_for(count, kSortTile);
    u32* hist = arena.alloc<u32>(static_cast<size_t>(tiles) * kRadix);
    const bool direct = tiles <= kDirectTiles;
    for (int shift = begin_bit; shift < end_bit; shift += kRadixBits) {
        launch(k_radix_upsweep, tiles, kSortThreads, 0, s, count, keys, shift, hist);
        if (!direct)
            exclusive_scan<u32>(arena, s, static_cast<i64>(tiles) * kRadix, LoadOf<u32>{hist}, hist, static_cast<u32*>(nullptr));
        if (vals && direct)
            launch(k_radix_downsweep<true, true>, tiles, kSortThreads, 0, s, count, keys, vals, shift, hist, keys_alt, vals_alt);
        else if (vals)
            launch(k_radix_downsweep<true, false>, tiles, kSortThreads, 0, s, count, keys, vals, shift, hist, keys_alt, vals_alt);
        else if (direct)
            launch(k_radix_downsweep<false, true>, tiles, kSortThreads, 0, s, count, keys, vals, shift, hist, keys_alt, vals_alt);
        else
            launch(k_radix_downsweep<false, false>, tiles, kSortThreads, 0, s, count, keys, vals, shift, hist, keys_alt, vals_alt);
        account_bytes(static_cast<double>(count) * (vals ? 24.0 : 16.0) + static_cast<double>(tiles) * kRadix * 4.0);
        std::swap(keys, keys_alt);
        if (vals) std::swap(vals, vals_alt);
    }
}

inline int bit_length(u64 x) {
    int b = 0;
    while (x) { ++b; x >>= 1; }
    return b;
}

// ---------------------------------------------------------------- misc kernels

template <class T>
__global__ void k_fill(i64 n, T* p, T value) {
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<i64>(gridDim.x) * blockDim.x)
        p[i] = value;
}
template <class T>
inline void fill(cudaStream_t s, T* p, i64 n, T value) {
    if (n <= 0) return;
    const int blocks = static_cast<int>(std::min<i64>(blocks_for(n, 256), 148 * 16));
    launch(k_fill<T>, blocks, 256, 0, s, n, p, value);
}

}  // namespace
}  // namespace gp
