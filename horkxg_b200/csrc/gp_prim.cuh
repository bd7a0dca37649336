// Hand-written device primitives used by every stage: block/device scans,
// stable LSD radix sorts (device-wide and one-block-per-segment) and warp
// bitonic sorts.  They replace the reference's Thrust/CUB call sites
// (src/coarsen.cu:898-1803, src/initial_partition_gpu.cu:230-238,
// src/refine_incremental.cuh:190-277).
#pragma once

#include <cstring>

#include "gp_common.cuh"

namespace gp {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// ---------------------------------------------------------------------------
// Warp and block scans (sum)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_inclusive_sum(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Warp-cooperative walk over the edges of up to 32 rows, one row per lane
// (first edge `begin`, `deg` edges, 0 for no row).  The rows' edges are laid
// back to back in a virtual position space and visited 32 at a time, so short
// rows leave no lane idle.  f(valid, owner, edge) is called by every lane in
// every step (valid is false past the last edge, so f may use warp
// collectives); owner is the lane whose row the edge belongs to and is
// non-decreasing across the lanes of a step.
template <typename F>
__device__ __forceinline__ void warp_edge_walk(i64 begin, i64 deg, F&& f) {
    const int lane = threadIdx.x & 31;
    const i64 inc = warp_inclusive_sum(deg);
    const i64 pre = inc - deg;
    const i64 total = __shfl_sync(0xffffffffu, inc, 31);
    for (i64 base = 0; base < total; base += 32) {
        const i64 q = base + lane;
        int lo = 0;
#pragma unroll
        for (int step = 16; step; step >>= 1) {
            const i64 probe = __shfl_sync(0xffffffffu, pre, lo + step);
            if (probe <= q) lo += step;
        }
        const i64 my_pre = __shfl_sync(0xffffffffu, pre, lo);
        const i64 my_begin = __shfl_sync(0xffffffffu, begin, lo);
        f(q < total, lo, my_begin + (q - my_pre));
    }
}

// Appends the lanes whose `pred` holds to a list of length *counter with one
// atomic per warp; returns each appending lane's slot.  All 32 lanes call it.
__device__ __forceinline__ u64 warp_append(bool pred, u64* counter) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (!m) return 0;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader)
        base = atomicAdd(reinterpret_cast<unsigned long long*>(counter), static_cast<unsigned long long>(__popc(m)));
    base = __shfl_sync(0xffffffffu, base, leader);
    return static_cast<u64>(base) + __popc(m & lanemask_lt());
}

// Rows a warp takes at once in a warp_edge_walk loop over `count` rows: up to
// 32 when there are many, down to one per warp when there are few (a walk
// over fewer rows than warps would leave most warps idle).
__device__ __forceinline__ int rows_per_warp(i64 count, i64 warps) {
    const i64 g = count / (warps > 0 ? warps : 1);
    return static_cast<int>(g < 1 ? 1 : (g > 32 ? 32 : g));
}

// Inclusive sum over runs of equal, non-decreasing `key` across the warp.
template <typename T, typename K>
__device__ __forceinline__ T warp_run_sum(T v, K key) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T o = __shfl_up_sync(0xffffffffu, v, d);
        const K ok = __shfl_up_sync(0xffffffffu, key, d);
        if (lane >= d && ok == key) v += o;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int d = 16; d; d >>= 1) {
        const T o = __shfl_xor_sync(0xffffffffu, v, d);
        v = o > v ? o : v;
    }
    return v;
}

// Exclusive block-wide sum for blockDim.x == kThreads; `total` gets the sum.
// `shared` needs kWarps + 1 entries.  Contains __syncthreads.
template <typename T>
__device__ __forceinline__ T block_exclusive_sum(T v, T* shared, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const T inc = warp_inclusive_sum(v);
    if (lane == 31) shared[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T s = lane < kWarps ? shared[lane] : T(0);
        const T si = warp_inclusive_sum(s);
        if (lane < kWarps) shared[lane] = si - s;
        if (lane == kWarps - 1) shared[kWarps] = si;
    }
    __syncthreads();
    const T out = shared[warp] + inc - v;
    if (total) *total = shared[kWarps];
    __syncthreads();
    return out;
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* shared) {
    T total;
    block_exclusive_sum(v, shared, &total);
    return total;
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan, reduce-then-scan over tiles of 2048 elements.
// F maps an index to the value scanned (lets callers scan predicates without
// materialising them).
// ---------------------------------------------------------------------------
constexpr int kScanItems = 8;
constexpr int kScanTile = kThreads * kScanItems;

template <typename T>
struct ArrayInput {
    const T* a;
    __device__ T operator()(i64 i) const { return a[i]; }
};

template <typename T, typename F>
__global__ void __launch_bounds__(kThreads) scan_tile_sums_kernel(F f, i64 n, T* sums) {
    __shared__ T shared[kWarps + 1];
    const i64 base = static_cast<i64>(blockIdx.x) * kScanTile;
    T local = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const i64 i = base + j * kThreads + threadIdx.x;
        if (i < n) local += f(i);
    }
    const T total = block_sum(local, shared);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename T, typename F>
__global__ void __launch_bounds__(kThreads) scan_tiles_kernel(F f, i64 n, T* out, const T* offsets, T* total_out) {
    __shared__ T shared[kWarps + 1];
    const i64 base = static_cast<i64>(blockIdx.x) * kScanTile + static_cast<i64>(threadIdx.x) * kScanItems;
    T vals[kScanItems];
    T local = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const i64 i = base + j;
        vals[j] = i < n ? f(i) : T(0);
        local += vals[j];
    }
    T block_total;
    T run = block_exclusive_sum(local, shared, &block_total);
    run += offsets ? offsets[blockIdx.x] : T(0);
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const i64 i = base + j;
        if (i < n) out[i] = run;
        run += vals[j];
    }
    if (total_out && blockIdx.x == gridDim.x - 1 && threadIdx.x == kThreads - 1) *total_out = run;
}

// out[i] = sum_{j<i} f(j); *total_dev (device, optional) = sum of all.
// out may alias the array f reads (each element is read before it is written
// by the same thread).
template <typename T, typename F>
void exclusive_scan(Device& d, F f, T* out, i64 n, T* total_dev = nullptr) {
    if (n <= 0) {
        if (total_dev) GP_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(T), d.stream));
        return;
    }
    const i64 tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        launch(d, "scan_tiles_kernel", scan_tiles_kernel<T, F>, 1, kThreads, 0, f, n, out, nullptr, total_dev);
        GP_LAUNCH();
        return;
    }
    Buf<T> sums(d, static_cast<size_t>(tiles));
    launch(d, "scan_tile_sums_kernel", scan_tile_sums_kernel<T, F>, static_cast<int>(tiles), kThreads, 0, f, n, sums.get());
    GP_LAUNCH();
    exclusive_scan<T>(d, ArrayInput<T>{sums.get()}, sums.get(), tiles, nullptr);
    launch(d, "scan_tiles_kernel", scan_tiles_kernel<T, F>, static_cast<int>(tiles), kThreads, 0, f, n, out, sums.get(), total_dev);
    GP_LAUNCH();
}

template <typename T>
void exclusive_scan_array(Device& d, const T* in, T* out, i64 n, T* total_dev = nullptr) {
    exclusive_scan<T>(d, ArrayInput<T>{in}, out, n, total_dev);
}

// ---------------------------------------------------------------------------
// Stable tile ranking for LSD radix sorting (8-bit digits).
// A tile of kThreads * kSortItems keys is split into one contiguous chunk per
// warp; inside a chunk element j*32+lane is visited in increasing order, so
// ranks preserve input order (stability).
// ---------------------------------------------------------------------------
constexpr int kSortItems = 8;
constexpr int kSortTile = kThreads * kSortItems;
constexpr int kRadix = 256;

struct RankShared {
    u32 warp_count[kWarps][kRadix];
    u32 tile_count[kRadix];
    i64 digit_base[kRadix];
    i64 scan_tmp[kWarps + 1];
};

template <typename K>
__device__ __forceinline__ u32 digit_of(K key, int shift) {
    return static_cast<u32>((key >> shift) & K(kRadix - 1));
}

// Scatters one tile [tile_begin, tile_end) of (keys, vals) into
// (out_keys, out_vals) at positions sh.digit_base[d] + stable rank, then
// advances sh.digit_base.  All threads of the block must call it.
template <typename K, typename V>
__device__ void scatter_tile(const K* keys, const V* vals, K* out_keys, V* out_vals,
                             i64 tile_begin, i64 tile_end, int shift, RankShared& sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 chunk = tile_begin + static_cast<i64>(warp) * 32 * kSortItems;
    K k[kSortItems];
    V v[kSortItems];
    u32 dg[kSortItems];
    u32 rank[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const i64 i = chunk + j * 32 + lane;
        const bool ok = i < tile_end;
        dg[j] = kRadix;
        if (ok) {
            k[j] = keys[i];
            if (vals) v[j] = vals[i];
            dg[j] = digit_of(k[j], shift);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, dg[j]);
        const int leader = __ffs(peers) - 1;
        u32 old = 0;
        if (ok && lane == leader) {
            old = sh.warp_count[warp][dg[j]];
            sh.warp_count[warp][dg[j]] = old + __popc(peers);
        }
        old = __shfl_sync(0xffffffffu, old, leader);
        rank[j] = old + __popc(peers & lanemask_lt());
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kThreads) {
        u32 run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const u32 c = sh.warp_count[w][d];
            sh.warp_count[w][d] = run;
            run += c;
        }
        sh.tile_count[d] = run;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        if (dg[j] < kRadix) {
            const i64 pos = sh.digit_base[dg[j]] + sh.warp_count[warp][dg[j]] + rank[j];
            out_keys[pos] = k[j];
            if (vals) out_vals[pos] = v[j];
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kThreads) {
        sh.digit_base[d] += sh.tile_count[d];
#pragma unroll
        for (int w = 0; w < kWarps; ++w) sh.warp_count[w][d] = 0;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Device-wide stable LSD radix sort of (K, V) pairs: a fixed grid of blocks,
// each owning a contiguous range; per 8-bit pass an upsweep histogram, a scan
// of the digit-major histogram, and an ordered downsweep scatter.
// ---------------------------------------------------------------------------
template <typename K>
__global__ void __launch_bounds__(kThreads) radix_hist_kernel(const K* keys, i64 n, int shift, u32* hist) {
    __shared__ u32 h[kRadix];
    for (int d = threadIdx.x; d < kRadix; d += kThreads) h[d] = 0;
    __syncthreads();
    const i64 lo = n * blockIdx.x / gridDim.x, hi = n * (blockIdx.x + 1) / gridDim.x;
    for (i64 i = lo + threadIdx.x; i < hi; i += kThreads) atomicAdd(&h[digit_of(keys[i], shift)], 1u);
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kThreads) hist[static_cast<i64>(d) * gridDim.x + blockIdx.x] = h[d];
}

template <typename K, typename V>
__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(const K* keys, const V* vals, K* out_keys,
                                                                 V* out_vals, i64 n, int shift,
                                                                 const i64* offsets) {
    __shared__ RankShared sh;
    for (int d = threadIdx.x; d < kRadix; d += kThreads) {
        sh.digit_base[d] = offsets[static_cast<i64>(d) * gridDim.x + blockIdx.x];
        for (int w = 0; w < kWarps; ++w) sh.warp_count[w][d] = 0;
    }
    __syncthreads();
    const i64 lo = n * blockIdx.x / gridDim.x, hi = n * (blockIdx.x + 1) / gridDim.x;
    for (i64 t = lo; t < hi; t += kSortTile)
        scatter_tile(keys, vals, out_keys, out_vals, t, t + kSortTile < hi ? t + kSortTile : hi, shift, sh);
}

struct U32ToI64 {
    const u32* a;
    __device__ i64 operator()(i64 i) const { return static_cast<i64>(a[i]); }
};

template <typename K, typename V>
__device__ void block_radix_sort_segment(K* keys, V* vals, K* keys_alt, V* vals_alt, i64 count, int begin_bit,
                                         int end_bit, RankShared& sh);

// Whole sort of a small array by one block (all passes in one launch).
template <typename K, typename V>
__global__ void __launch_bounds__(kThreads) small_radix_sort_kernel(K* keys, V* vals, K* keys_alt, V* vals_alt, i64 n,
                                                                    int begin_bit, int end_bit) {
    __shared__ RankShared sh;
    block_radix_sort_segment(keys, vals, keys_alt, vals_alt, n, begin_bit, end_bit, sh);
}

constexpr i64 kSmallSort = 8192;   // one-block sort up to this many keys

// Sorts bits [begin_bit, end_bit) of the keys.  On return the sorted data is
// in (keys, vals) (the routine copies back after an odd number of passes).
// Small arrays are sorted by one block in one launch: on small graphs the
// multi-launch passes cost more in launch latency than in work.
template <typename K, typename V>
void radix_sort(Device& d, K* keys, V* vals, K* keys_alt, V* vals_alt, i64 n, int begin_bit, int end_bit) {
    if (n <= 1 || begin_bit >= end_bit) return;
    if (n <= kSmallSort) {
        launch(d, "small_radix_sort_kernel", small_radix_sort_kernel<K, V>, 1, kThreads, 0, keys, vals, keys_alt,
               vals_alt, n, begin_bit, end_bit);
        GP_LAUNCH();
        return;
    }
    const int grid = static_cast<int>(std::min<i64>(std::max<i64>(1, (n + kSortTile - 1) / kSortTile),
                                                    static_cast<i64>(d.grid_limit(4))));
    Buf<u32> hist(d, static_cast<size_t>(kRadix) * grid);
    Buf<i64> offs(d, static_cast<size_t>(kRadix) * grid);
    K* src_k = keys;
    V* src_v = vals;
    K* dst_k = keys_alt;
    V* dst_v = vals_alt;
    int passes = 0;
    for (int shift = begin_bit; shift < end_bit; shift += 8, ++passes) {
        launch(d, "radix_hist_kernel", radix_hist_kernel<K>, grid, kThreads, 0, src_k, n, shift, hist.get());
        GP_LAUNCH();
        exclusive_scan<i64>(d, U32ToI64{hist.get()}, offs.get(), static_cast<i64>(kRadix) * grid);
        launch(d, "radix_scatter_kernel", radix_scatter_kernel<K, V>, grid, kThreads, 0, src_k, src_v, dst_k, dst_v, n, shift,
                                                                    offs.get());
        GP_LAUNCH();
        std::swap(src_k, dst_k);
        std::swap(src_v, dst_v);
    }
    if (passes & 1) {
        GP_CUDA(cudaMemcpyAsync(keys, keys_alt, n * sizeof(K), cudaMemcpyDeviceToDevice, d.stream));
        if (vals) GP_CUDA(cudaMemcpyAsync(vals, vals_alt, n * sizeof(V), cudaMemcpyDeviceToDevice, d.stream));
    }
}

// ---------------------------------------------------------------------------
// One block sorts one segment [seg_begin, seg_end) completely (all passes),
// ping-ponging between the primary and alternate buffers and leaving the
// result in the primary buffer.  Generic pointers: the buffers may be global
// or shared memory.
// ---------------------------------------------------------------------------
template <typename K, typename V>
__device__ void block_radix_sort_segment(K* keys, V* vals, K* keys_alt, V* vals_alt, i64 count,
                                         int begin_bit, int end_bit, RankShared& sh) {
    K* sk = keys;
    V* sv = vals;
    K* dk = keys_alt;
    V* dv = vals_alt;
    int passes = 0;
    for (int shift = begin_bit; shift < end_bit; shift += 8, ++passes) {
        for (int dgt = threadIdx.x; dgt < kRadix; dgt += kThreads) sh.tile_count[dgt] = 0;
        __syncthreads();
        for (i64 i = threadIdx.x; i < count; i += kThreads) atomicAdd(&sh.tile_count[digit_of(sk[i], shift)], 1u);
        __syncthreads();
        // Exclusive scan of the 256 digit counts (one per thread).
        i64 c = threadIdx.x < kRadix ? static_cast<i64>(sh.tile_count[threadIdx.x]) : 0;
        const i64 ex = block_exclusive_sum<i64>(c, sh.scan_tmp, nullptr);
        for (int dgt = threadIdx.x; dgt < kRadix; dgt += kThreads) {
            sh.digit_base[dgt] = ex;
            for (int w = 0; w < kWarps; ++w) sh.warp_count[w][dgt] = 0;
        }
        __syncthreads();
        for (i64 t = 0; t < count; t += kSortTile)
            scatter_tile(sk, sv, dk, dv, t, t + kSortTile < count ? t + kSortTile : count, shift, sh);
        K* tk = sk; sk = dk; dk = tk;
        V* tv = sv; sv = dv; dv = tv;
    }
    if (passes & 1) {
        for (i64 i = threadIdx.x; i < count; i += kThreads) {
            keys[i] = keys_alt[i];
            if (vals) vals[i] = vals_alt[i];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Warp bitonic sort of 32 (key, value) pairs, ascending by key.
// ---------------------------------------------------------------------------
template <typename K, typename V>
__device__ __forceinline__ void warp_bitonic_sort(K& key, V& val) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const K ok = __shfl_xor_sync(0xffffffffu, key, stride);
            const V ov = __shfl_xor_sync(0xffffffffu, val, stride);
            const bool up = (lane & size) == 0;
            const bool lower = (lane & stride) == 0;
            // lower lane keeps min when ascending
            const bool take_other = (lower == up) ? (ok < key) : (ok > key);
            if (take_other) { key = ok; val = ov; }
        }
    }
}

// Number of significant bits of x (0 for x == 0).
inline int bit_width_u64(u64 x) {
    int b = 0;
    while (x) { ++b; x >>= 1; }
    return b;
}

}  // namespace gp
