// CSR contraction (src/coarsen.cu:1674-1814), restated as a segmented
// problem instead of one global sort of all m edge records:
//
// 1. every coarse row c gets a segment of the size of its members' fine
//    degrees; a warp-batched pass scatters each fine row's (map[u], w) pairs
//    into its coarse row's segment (internal edges become a sentinel);
// 2. every segment is sorted by target and its runs of equal targets summed:
//    a warp bitonic sort in registers for segments of <= 32 entries, a warp
//    radix sort in the warp's shared memory for <= 256, a block radix sort in
//    shared memory sized to the segment class for <= 4096, and, for larger
//    segments, a block that ranks the targets through a shared-memory bitmap
//    of the coarse id range instead of sorting;
// 3. row lengths are scanned into the coarse offsets and the unique entries
//    copied out.
//
// Output rows are sorted by target with parallel edges summed, exactly as
// the reference's sort + reduce_by_key + write_coarse_csr_kernel produce them.
#pragma once

#include "gp_prim.cuh"
#include "gp_sclp.cuh"

namespace gp {

// Largest segment sorted in shared memory: two key and two value buffers
// (plus the ranking scratch) stay under the 227 KB a block may use.
template <typename W>
__host__ __device__ constexpr int seg_smem_capacity() { return 4096; }
constexpr int kWarpSegCap = 256;    // warp radix sort
constexpr int kMidSegCap = 1024;    // block radix sort with a 1024-entry buffer

constexpr i64 kGiantSeg = 1 << 16;  // above: rows spread over many blocks

// Row-size classes: 0 empty, 1 <= 32, 2 <= kWarpSegCap, 3 <= kMidSegCap,
// 4 <= seg_smem_capacity, 5 <= kGiantSeg, 6 larger.
constexpr int kRowClasses = 7;

// Fine-degree sum per coarse row.
template <typename O>
__global__ void row_fine_degree_kernel(i64 n, const O* off, const i32* map, i64* fdeg) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const i64 d = static_cast<i64>(off[v + 1]) - off[v];
    if (d) atomicAdd(reinterpret_cast<unsigned long long*>(&fdeg[map[v]]), static_cast<unsigned long long>(d));
}

// Warp handles 32 consecutive fine rows: reserves each row's slot range in
// its coarse segment, then walks the rows' edges 32 at a time in a virtual
// position space (exclusive prefix of the rows' degrees); a lane finds its
// row by a 5-step shuffle binary search.  Hub rows (degree > kHubDegree) are
// reserved and scattered by the chunked hub kernels instead.
template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) scatter_edges_kernel(
    i64 n, const O* __restrict__ off, const i32* __restrict__ nbr, const W* __restrict__ ew,
    const i32* __restrict__ map, const i64* __restrict__ temp_off, i64* cursor, u32 sentinel,
    u32* __restrict__ tgt, W* __restrict__ wt) {
    const int lane = threadIdx.x & 31;
    const i64 v0 = ((static_cast<i64>(blockIdx.x) * kThreads + threadIdx.x) >> 5) * 32;
    if (v0 >= n) return;
    const i64 v = v0 + lane;
    const bool has = v < n;
    const i64 rs = has ? static_cast<i64>(off[v]) : 0;
    i64 deg = has ? static_cast<i64>(off[v + 1]) - rs : 0;
    if (deg > kHubDegree) deg = 0;
    const i32 c = has ? map[v] : 0;
    i64 dst = 0;
    if (deg > 0)
        dst = temp_off[c] + static_cast<i64>(atomicAdd(reinterpret_cast<unsigned long long*>(&cursor[c]),
                                                        static_cast<unsigned long long>(deg)));
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
        // lanes past the last non-empty row have pre == total > q, so `lo`
        // is the last row starting at or before q, which is non-empty
        const i64 my_pre = __shfl_sync(0xffffffffu, pre, lo);
        const i64 my_rs = __shfl_sync(0xffffffffu, rs, lo);
        const i64 my_dst = __shfl_sync(0xffffffffu, dst, lo);
        const i32 my_c = __shfl_sync(0xffffffffu, c, lo);
        if (q < total) {
            const i64 e = my_rs + (q - my_pre);
            const i32 t = map[nbr[e]];
            const i64 out = my_dst + (q - my_pre);
            tgt[out] = t == my_c ? sentinel : static_cast<u32>(t);
            wt[out] = weight_at(ew, e);
        }
    }
}

// Segment reservation of hub rows (hub_dst[h]).
template <typename O>
__global__ void hub_reserve_kernel(i64 hubs, const i32* __restrict__ hub_list, const O* __restrict__ off,
                                   const i32* __restrict__ map, const i64* __restrict__ temp_off, i64* cursor,
                                   i64* hub_dst) {
    const i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (h >= hubs) return;
    const i32 v = hub_list[h];
    const i32 c = map[v];
    const i64 deg = static_cast<i64>(off[v + 1]) - static_cast<i64>(off[v]);
    hub_dst[h] = temp_off[c] + static_cast<i64>(atomicAdd(reinterpret_cast<unsigned long long*>(&cursor[c]),
                                                           static_cast<unsigned long long>(deg)));
}

// Sum runs of equal keys of a sorted segment (keys, vals)[0, count); the
// unique non-sentinel (key, sum) pairs are written to (out_k, out_v) in
// order.  Block-cooperative; returns the unique count in every thread.
template <typename W>
struct RunShared {
    i64 scan_tmp[kWarps + 1];
    u64 wscan_tmp[kWarps + 1];
};

template <typename W>
__device__ i64 block_reduce_runs(const u32* keys, const W* vals, i64 count, u32 sentinel, u32* out_k, W* out_v,
                                 RunShared<W>& sh) {
    i64 unique_carry = 0;   // unique runs emitted before this tile
    W w_carry = 0;          // running weight sum before this tile
    constexpr int kItems = 8;
    for (i64 t0 = 0; t0 < count; t0 += static_cast<i64>(kThreads) * kItems) {
        const i64 base = t0 + static_cast<i64>(threadIdx.x) * kItems;
        u32 k[kItems];
        W w[kItems];
        i64 heads = 0;
        W wsum = 0;
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            const i64 i = base + j;
            k[j] = i < count ? keys[i] : sentinel;
            w[j] = i < count ? vals[i] : W(0);
            const bool head = i < count && k[j] != sentinel && (i == 0 || keys[i - 1] != k[j]);
            heads += head ? 1 : 0;
            wsum += w[j];
        }
        i64 heads_total;
        const i64 head_ex = block_exclusive_sum<i64>(heads, sh.scan_tmp, &heads_total);
        u64 wtotal;
        const u64 w_ex = block_exclusive_sum<u64>(static_cast<u64>(wsum), sh.wscan_tmp, &wtotal);
        // Pass 1: heads record their exclusive weight prefix in out_v.
        i64 u = unique_carry + head_ex;
        W run = w_carry + static_cast<W>(w_ex);
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            const i64 i = base + j;
            const bool head = i < count && k[j] != sentinel && (i == 0 || keys[i - 1] != k[j]);
            if (head) { out_k[u] = k[j]; out_v[u] = run; ++u; }
            run += w[j];
        }
        __syncthreads();
        // Pass 2: run ends turn the prefix into the run's sum.
        u = unique_carry + head_ex;
        run = w_carry + static_cast<W>(w_ex);
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            const i64 i = base + j;
            const bool head = i < count && k[j] != sentinel && (i == 0 || keys[i - 1] != k[j]);
            if (head) ++u;
            run += w[j];
            const bool end = i < count && k[j] != sentinel && (i + 1 == count || keys[i + 1] != k[j]);
            if (end) out_v[u - 1] = run - out_v[u - 1];
        }
        __syncthreads();
        unique_carry += heads_total;
        w_carry += static_cast<W>(wtotal);
    }
    return unique_carry;
}

// Rows with <= 32 entries: one warp per row, bitonic sort in registers.
template <typename W>
__global__ void __launch_bounds__(kThreads) segment_warp_kernel(i64 rows, const i32* __restrict__ list,
                                                                const i64* __restrict__ temp_off, u32 sentinel,
                                                                u32* tgt, W* wt, i64* row_len) {
    const int lane = threadIdx.x & 31;
    const i64 r = (static_cast<i64>(blockIdx.x) * kThreads + threadIdx.x) >> 5;
    if (r >= rows) return;
    const i32 c = list[r];
    const i64 s = temp_off[c];
    const int len = static_cast<int>(temp_off[c + 1] - s);
    u32 k = lane < len ? tgt[s + lane] : 0xffffffffu;
    W w = lane < len ? wt[s + lane] : W(0);
    warp_bitonic_sort(k, w);
    const u32 prev = __shfl_up_sync(0xffffffffu, k, 1);
    const bool valid = lane < len && k != sentinel;
    const bool head = valid && (lane == 0 || prev != k);
    // segmented inclusive sum over runs (runs are contiguous after sorting)
    W sum = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const W o = __shfl_up_sync(0xffffffffu, sum, d);
        const u32 ok = __shfl_up_sync(0xffffffffu, k, d);
        if (lane >= d && ok == k) sum += o;
    }
    const u32 next = __shfl_down_sync(0xffffffffu, k, 1);
    const bool end = valid && (lane == 31 || next != k);
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const int u = __popc(heads & lanemask_lt()) + (head ? 0 : -1);   // index of this lane's run
    __syncwarp();
    if (end) { tgt[s + u] = k; wt[s + u] = sum; }
    if (lane == 0) row_len[c] = __popc(heads);
}

// Rows with 33..kWarpSegCap entries: one warp per row, LSD radix sort with
// 8-bit digits in the warp's slice of shared memory (stable: equal digits
// keep their order through __match_any_sync ranks), then the runs of equal
// targets are summed 32 at a time with a carry between chunks.
template <typename W>
__global__ void __launch_bounds__(kThreads) segment_warp_radix_kernel(i64 rows, const i32* __restrict__ list,
                                                                      const i64* __restrict__ temp_off, u32 sentinel,
                                                                      int key_bits, u32* tgt, W* wt, i64* row_len) {
    extern __shared__ unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    W* vbase = reinterpret_cast<W*>(smem_raw) + warp * 2 * kWarpSegCap;
    u32* kbase = reinterpret_cast<u32*>(reinterpret_cast<W*>(smem_raw) + kWarps * 2 * kWarpSegCap) +
                 warp * (2 * kWarpSegCap + kRadix);
    W* v0 = vbase;
    W* v1 = vbase + kWarpSegCap;
    u32* k0 = kbase;
    u32* k1 = kbase + kWarpSegCap;
    u32* hist = kbase + 2 * kWarpSegCap;
    const i64 r = static_cast<i64>(blockIdx.x) * kWarps + warp;
    if (r >= rows) return;
    const i32 c = list[r];
    const i64 s = temp_off[c];
    const int len = static_cast<int>(temp_off[c + 1] - s);
    for (int i = lane; i < len; i += 32) { k0[i] = tgt[s + i]; v0[i] = wt[s + i]; }
    __syncwarp();
    for (int shift = 0; shift < key_bits; shift += 8) {
        for (int d = lane; d < kRadix; d += 32) hist[d] = 0;
        __syncwarp();
        for (int i = lane; i < len; i += 32) atomicAdd(&hist[(k0[i] >> shift) & (kRadix - 1)], 1u);
        __syncwarp();
        // exclusive scan of the 256 digit counts, 8 per lane
        u32 cnt[kRadix / 32];
        u32 tot = 0;
#pragma unroll
        for (int j = 0; j < kRadix / 32; ++j) { cnt[j] = hist[lane * (kRadix / 32) + j]; tot += cnt[j]; }
        u32 ex = warp_inclusive_sum(tot) - tot;
#pragma unroll
        for (int j = 0; j < kRadix / 32; ++j) { hist[lane * (kRadix / 32) + j] = ex; ex += cnt[j]; }
        __syncwarp();
        for (int base = 0; base < len; base += 32) {
            const int i = base + lane;
            const bool valid = i < len;
            const u32 key = valid ? k0[i] : 0u;
            const W val = valid ? v0[i] : W(0);
            const u32 dg = valid ? (key >> shift) & (kRadix - 1) : static_cast<u32>(kRadix);
            const unsigned peers = __match_any_sync(0xffffffffu, dg);
            const int leader = __ffs(peers) - 1;
            u32 b = (valid && lane == leader) ? hist[dg] : 0u;
            b = __shfl_sync(0xffffffffu, b, leader);
            if (valid) {
                const u32 pos = b + __popc(peers & lanemask_lt());
                k1[pos] = key;
                v1[pos] = val;
            }
            __syncwarp();
            if (valid && lane == leader) hist[dg] = b + __popc(peers);
            __syncwarp();
        }
        u32* tk = k0; k0 = k1; k1 = tk;
        W* tv = v0; v0 = v1; v1 = tv;
    }
    // runs of the sorted segment; the sentinel (internal edges) sorts last
    int u = 0;
    u32 carry_key = 0xffffffffu;
    W carry = 0;
    for (int base = 0; base < len; base += 32) {
        const int i = base + lane;
        const bool valid = i < len;
        const u32 key = valid ? k0[i] : sentinel;
        W sum = warp_run_sum(valid ? v0[i] : W(0), key);
        if (key == carry_key) sum += carry;
        const u32 prev = __shfl_up_sync(0xffffffffu, key, 1);
        u32 next = __shfl_down_sync(0xffffffffu, key, 1);
        if (lane == 31) next = i + 1 < len ? k0[i + 1] : sentinel;   // first key of the next chunk
        const bool real = valid && key != sentinel;
        const bool head = real && (lane == 0 ? key != carry_key : prev != key);
        const bool end = real && (i + 1 == len || next != key);
        const unsigned heads = __ballot_sync(0xffffffffu, head);
        if (end) {
            const int idx = u + __popc(heads & (lanemask_lt() | (1u << lane))) - 1;
            tgt[s + idx] = key;
            wt[s + idx] = sum;
        }
        u += __popc(heads);
        carry_key = __shfl_sync(0xffffffffu, key, 31);
        carry = __shfl_sync(0xffffffffu, sum, 31);
    }
    if (lane == 0) row_len[c] = u;
}

// Rows with kWarpSegCap+1..seg_smem_capacity entries: block per row, radix
// sort in a shared-memory buffer of `cap` entries (the class's bound).
template <typename W>
__global__ void __launch_bounds__(kThreads) segment_smem_kernel(i64 rows, const i32* __restrict__ list,
                                                                const i64* __restrict__ temp_off, u32 sentinel,
                                                                int key_bits, int cap, u32* tgt, W* wt, i64* row_len) {
    extern __shared__ unsigned char smem_raw[];
    W* w0 = reinterpret_cast<W*>(smem_raw);
    W* w1 = w0 + cap;
    u32* k0 = reinterpret_cast<u32*>(w1 + cap);
    u32* k1 = k0 + cap;
    __shared__ RankShared rank_sh;
    __shared__ RunShared<W> run_sh;
    const i64 r = blockIdx.x;
    if (r >= rows) return;
    const i32 c = list[r];
    const i64 s = temp_off[c];
    const i64 len = temp_off[c + 1] - s;
    // The row into shared memory with 128-bit loads: entries before the
    // first 16-byte boundary of the targets (tgt and wt are whole allocator
    // blocks, so tgt + s is 16-byte aligned when s is a multiple of 4, and wt
    // + s then too) and after the last whole group of four go by element.
    const u32* src_k = tgt + s;
    const W* src_w = wt + s;
    const i64 head = ((4 - (s & 3)) & 3) < len ? ((4 - (s & 3)) & 3) : len;
    const i64 groups = (len - head) / 4;
    for (i64 i = threadIdx.x; i < head; i += kThreads) { k0[i] = src_k[i]; w0[i] = src_w[i]; }
    for (i64 q = threadIdx.x; q < groups; q += kThreads) {
        const i64 i = head + 4 * q;
        const uint4 kk = *reinterpret_cast<const uint4*>(src_k + i);
        k0[i] = kk.x; k0[i + 1] = kk.y; k0[i + 2] = kk.z; k0[i + 3] = kk.w;
        if constexpr (sizeof(W) == 4) {
            const uint4 ww = *reinterpret_cast<const uint4*>(src_w + i);
            w0[i] = ww.x; w0[i + 1] = ww.y; w0[i + 2] = ww.z; w0[i + 3] = ww.w;
        } else {
            const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(src_w + i);
            const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(src_w + i + 2);
            w0[i] = a.x; w0[i + 1] = a.y; w0[i + 2] = b.x; w0[i + 3] = b.y;
        }
    }
    for (i64 i = head + 4 * groups + threadIdx.x; i < len; i += kThreads) { k0[i] = src_k[i]; w0[i] = src_w[i]; }
    __syncthreads();
    block_radix_sort_segment(k0, w0, k1, w1, len, 0, key_bits, rank_sh);
    const i64 u = block_reduce_runs(k0, w0, len, sentinel, tgt + s, wt + s, run_sh);
    if (threadIdx.x == 0) row_len[c] = u;
}

// Rows of the bitmap class on levels whose coarse id range spans more than
// kSortWindows bitmap windows: the bitmap kernel rescans the row once per
// window, so here one block sorts the row where it lies instead -- LSD radix
// passes ping-ponging between the row's segment and its alternate buffer
// (global memory, mostly L2-resident for rows of at most kGiantSeg entries),
// then its runs reduced into the alternate buffer.  Same output as
// segment_bitmap_kernel: rows sorted by target, duplicates summed, internal
// edges (the sentinel, which sorts last) dropped.
constexpr i64 kSortWindows = 4;

template <typename W>
__global__ void __launch_bounds__(kThreads) segment_sort_kernel(i64 rows, const i32* __restrict__ list,
                                                                const i64* __restrict__ temp_off,
                                                                const i64* __restrict__ alt_off, u32 sentinel,
                                                                int key_bits, u32* tgt, W* wt, u32* alt_k, W* alt_w,
                                                                i64* row_len) {
    __shared__ RankShared rank_sh;
    __shared__ RunShared<W> run_sh;
    const i64 r = blockIdx.x;
    if (r >= rows) return;
    const i32 c = list[r];
    const i64 s = temp_off[c];
    const i64 len = temp_off[c + 1] - s;
    u32* k_alt = alt_k + alt_off[r];
    W* w_alt = alt_w + alt_off[r];
    block_radix_sort_segment(tgt + s, wt + s, k_alt, w_alt, len, 0, key_bits, rank_sh);
    const i64 u = block_reduce_runs(tgt + s, wt + s, len, sentinel, k_alt, w_alt, run_sh);
    if (threadIdx.x == 0) row_len[c] = u;
}

// Rows above seg_smem_capacity entries: block per row, no sort.  The row's
// distinct targets are marked in a shared-memory bitmap over a window of the
// coarse id range; a target's output position is then the number of marked
// ids below it (a popcount prefix over 8-word groups), so the unique
// (target, weight) pairs land in ascending target order while the weights
// are summed by atomics.  Windows of kBitmapWindow ids are processed in
// ascending order, each with two passes over the row's entries.  Output goes
// to the row's alternate buffer (alt_off), which has room for all entries.
constexpr int kBitmapWindow = 1 << 19;                 // ids per window (64 KB of bits)
constexpr int kBitmapWords = kBitmapWindow / 32;
constexpr int kBitmapGroup = 8;                        // words per prefix entry
constexpr int kBitmapGroups = kBitmapWords / kBitmapGroup;

template <typename W>
__global__ void __launch_bounds__(kThreads) segment_bitmap_kernel(
    i64 rows, const i32* __restrict__ list, const i64* __restrict__ temp_off, const i64* __restrict__ alt_off,
    u32 sentinel, i64 id_count, const u32* __restrict__ tgt, const W* __restrict__ wt, u32* alt_k, W* alt_w,
    i64* row_len) {
    extern __shared__ unsigned char smem_raw[];
    u32* bits = reinterpret_cast<u32*>(smem_raw);
    u32* gpre = bits + kBitmapWords;
    __shared__ u32 scan_sh[kWarps + 1];
    const i64 r = blockIdx.x;
    if (r >= rows) return;
    const i32 c = list[r];
    const i64 s = temp_off[c];
    const i64 len = temp_off[c + 1] - s;
    u32* out_k = alt_k + alt_off[r];
    W* out_w = alt_w + alt_off[r];
    i64 unique = 0;
    for (i64 lo = 0; lo < id_count; lo += kBitmapWindow) {
        const i64 hi = lo + kBitmapWindow < id_count ? lo + kBitmapWindow : id_count;
        const int words = static_cast<int>((hi - lo + 31) >> 5);
        const int groups = (words + kBitmapGroup - 1) / kBitmapGroup;
        for (int i = threadIdx.x; i < groups * kBitmapGroup; i += kThreads) bits[i] = 0;
        __syncthreads();
        for (i64 i = threadIdx.x; i < len; i += kThreads) {
            const u32 t = tgt[s + i];
            if (t != sentinel && t >= lo && t < hi) {
                const u32 x = static_cast<u32>(t - lo);
                atomicOr(&bits[x >> 5], 1u << (x & 31));
            }
        }
        __syncthreads();
        // exclusive prefix of the groups' popcounts
        constexpr int kPer = kBitmapGroups / kThreads;   // groups per thread
        u32 cnt[kPer];
        u32 mine = 0;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int g = threadIdx.x * kPer + j;
            u32 pc = 0;
            if (g < groups) {
#pragma unroll
                for (int q = 0; q < kBitmapGroup; ++q) pc += __popc(bits[g * kBitmapGroup + q]);
            }
            cnt[j] = pc;
            mine += pc;
        }
        u32 total = 0;
        u32 run = block_exclusive_sum<u32>(mine, scan_sh, &total);
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int g = threadIdx.x * kPer + j;
            if (g < groups) gpre[g] = run;
            run += cnt[j];
        }
        for (i64 i = threadIdx.x; i < total; i += kThreads) out_w[unique + i] = W(0);
        __syncthreads();
        for (i64 i = threadIdx.x; i < len; i += kThreads) {
            const u32 t = tgt[s + i];
            if (t != sentinel && t >= lo && t < hi) {
                const u32 x = static_cast<u32>(t - lo);
                const int w = static_cast<int>(x >> 5);
                const int g = w / kBitmapGroup;
                u32 rank = gpre[g] + __popc(bits[w] & ((1u << (x & 31)) - 1u));
                for (int q = g * kBitmapGroup; q < w; ++q) rank += __popc(bits[q]);
                const i64 pos = unique + rank;
                out_k[pos] = t;
                if constexpr (sizeof(W) == 8)
                    atomicAdd(reinterpret_cast<unsigned long long*>(&out_w[pos]),
                              static_cast<unsigned long long>(wt[s + i]));
                else
                    atomicAdd(reinterpret_cast<unsigned*>(&out_w[pos]), static_cast<unsigned>(wt[s + i]));
            }
        }
        unique += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) row_len[c] = unique;
}

// Giant rows (more than kGiantSeg entries; the rows of hub clusters) would
// leave one block working long after the rest of the GPU is idle.  Their
// entries are cut into kGiantChunk-entry chunks spread over all SMs: one
// pass marks the targets in a global bitmap per row (coarse id range), a
// block per row scans the words' popcounts into per-8-word-group prefixes,
// and a second pass over the chunks writes each (target, weight) at its rank
// in the row's alternate buffer, summing weights with atomics.
constexpr i64 kGiantChunk = 8192;

struct SegChunk {
    i32 row;        // index among the giant rows
    i32 pad;
    i64 begin, end; // entry range in the scattered arrays
};

struct GiantChunkCount {
    const i32* list;
    const i64* temp_off;
    i64 count;
    __device__ i64 operator()(i64 i) const {
        if (i >= count) return 0;
        const i32 c = list[i];
        return (temp_off[c + 1] - temp_off[c] + kGiantChunk - 1) / kGiantChunk;
    }
};

__global__ void giant_chunks_kernel(i64 giants, const i32* __restrict__ list, const i64* __restrict__ temp_off,
                                    const i64* __restrict__ chunk_off, SegChunk* chunks) {
    const i64 g = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= giants) return;
    const i32 c = list[g];
    const i64 s = temp_off[c], e = temp_off[c + 1];
    for (i64 q = chunk_off[g]; q < chunk_off[g + 1]; ++q) {
        const i64 b = s + (q - chunk_off[g]) * kGiantChunk;
        chunks[q] = {static_cast<i32>(g), 0, b, b + kGiantChunk < e ? b + kGiantChunk : e};
    }
}

__global__ void __launch_bounds__(kThreads) giant_mark_kernel(const SegChunk* __restrict__ chunks,
                                                              const u32* __restrict__ tgt, u32 sentinel,
                                                              i64 words_per_row, u32* gbits) {
    const SegChunk ch = chunks[blockIdx.x];
    u32* bits = gbits + static_cast<i64>(ch.row) * words_per_row;
    for (i64 e = ch.begin + threadIdx.x; e < ch.end; e += kThreads) {
        const u32 t = tgt[e];
        if (t != sentinel) atomicOr(&bits[t >> 5], 1u << (t & 31));
    }
}

// Block per giant row: gpre[g] = marked ids in the row's words before group g
// (kBitmapGroup words per group); row_len = the row's marked ids.
__global__ void __launch_bounds__(kThreads) giant_scan_kernel(const i32* __restrict__ list, i64 words_per_row,
                                                              const u32* __restrict__ gbits, u32* gpre,
                                                              i64* row_len) {
    __shared__ u32 scan_sh[kWarps + 1];
    const i64 groups = (words_per_row + kBitmapGroup - 1) / kBitmapGroup;
    const u32* bits = gbits + static_cast<i64>(blockIdx.x) * words_per_row;
    u32* pre = gpre + static_cast<i64>(blockIdx.x) * groups;
    const i64 per = (groups + kThreads - 1) / kThreads;
    const i64 g0 = static_cast<i64>(threadIdx.x) * per;
    const i64 g1 = g0 + per < groups ? g0 + per : groups;
    auto group_count = [&](i64 g) {
        u32 pc = 0;
        for (i64 w = g * kBitmapGroup; w < (g + 1) * kBitmapGroup && w < words_per_row; ++w) pc += __popc(bits[w]);
        return pc;
    };
    u32 mine = 0;
    for (i64 g = g0; g < g1; ++g) mine += group_count(g);
    u32 total = 0;
    u32 run = block_exclusive_sum<u32>(mine, scan_sh, &total);
    for (i64 g = g0; g < g1; ++g) {
        pre[g] = run;
        run += group_count(g);
    }
    if (threadIdx.x == 0) row_len[list[blockIdx.x]] = total;
}

template <typename W>
__global__ void __launch_bounds__(kThreads) giant_place_kernel(const SegChunk* __restrict__ chunks,
                                                               const u32* __restrict__ tgt, const W* __restrict__ wt,
                                                               u32 sentinel, i64 words_per_row,
                                                               const u32* __restrict__ gbits,
                                                               const u32* __restrict__ gpre,
                                                               const i64* __restrict__ alt_off, u32* alt_k, W* alt_w) {
    const SegChunk ch = chunks[blockIdx.x];
    const i64 groups = (words_per_row + kBitmapGroup - 1) / kBitmapGroup;
    const u32* bits = gbits + static_cast<i64>(ch.row) * words_per_row;
    const u32* pre = gpre + static_cast<i64>(ch.row) * groups;
    u32* out_k = alt_k + alt_off[ch.row];
    W* out_w = alt_w + alt_off[ch.row];
    for (i64 e = ch.begin + threadIdx.x; e < ch.end; e += kThreads) {
        const u32 t = tgt[e];
        if (t == sentinel) continue;
        const i64 w = t >> 5;
        const i64 g = w / kBitmapGroup;
        u32 rank = pre[g] + __popc(bits[w] & ((1u << (t & 31)) - 1u));
        for (i64 q = g * kBitmapGroup; q < w; ++q) rank += __popc(bits[q]);
        out_k[rank] = t;
        if constexpr (sizeof(W) == 8)
            atomicAdd(reinterpret_cast<unsigned long long*>(&out_w[rank]), static_cast<unsigned long long>(wt[e]));
        else
            atomicAdd(reinterpret_cast<unsigned*>(&out_w[rank]), static_cast<unsigned>(wt[e]));
    }
}

// Classifies coarse rows by their number of scattered entries: counts[c]
// receives the rows of class c, counts[kRowClasses + c] their entries.
// `bitmap_from`: rows longer than this (up to kGiantSeg) take the bitmap
// ranking of class 5 whatever their class by length, since on levels with
// few coarse vertices a bitmap over the id range costs less than sorting.
__global__ void row_class_kernel(i64 rows, const i64* temp_off, i64 smem_cap, i64 bitmap_from, u64* keys, i32* vals,
                                 u64* counts) {
    __shared__ unsigned long long local[2 * kRowClasses];
    if (threadIdx.x < 2 * kRowClasses) local[threadIdx.x] = 0;
    __syncthreads();
    const i64 c = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c < rows) {
        const i64 l = temp_off[c + 1] - temp_off[c];
        const int k = l == 0 ? 0 : l <= 32 ? 1 : l <= kWarpSegCap ? 2 : (l > bitmap_from && l <= kGiantSeg) ? 5
                    : l <= kMidSegCap ? 3 : l <= smem_cap ? 4 : l <= kGiantSeg ? 5 : 6;
        keys[c] = static_cast<u64>(k);
        vals[c] = static_cast<i32>(c);
        atomicAdd(&local[k], 1ull);
        atomicAdd(&local[kRowClasses + k], static_cast<unsigned long long>(l));
    }
    __syncthreads();
    if (threadIdx.x < 2 * kRowClasses && local[threadIdx.x])
        atomicAdd(reinterpret_cast<unsigned long long*>(&counts[threadIdx.x]), local[threadIdx.x]);
}

template <typename O>
struct RowLenToO {
    const i64* len;
    __device__ O operator()(i64 i) const { return static_cast<O>(len[i]); }
};

struct BigRowLen {
    const i32* list;
    const i64* temp_off;
    i64 count;
    __device__ i64 operator()(i64 i) const {
        if (i >= count) return 0;
        const i32 c = list[i];
        return temp_off[c + 1] - temp_off[c];
    }
};

// Copy each row's unique entries from its segment to the final CSR; a warp
// per 32 rows in a virtual position space as in scatter_edges_kernel.  Rows
// whose segment exceeded the shared-memory capacity are copied from their
// alternate buffers by copy_big_rows_kernel.
template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) copy_rows_kernel(i64 rows, const i64* __restrict__ temp_off,
                                                             const O* __restrict__ coff, const u32* __restrict__ tgt,
                                                             const W* __restrict__ wt, i32* __restrict__ nbr,
                                                             W* __restrict__ ew) {
    const int lane = threadIdx.x & 31;
    const i64 r0 = ((static_cast<i64>(blockIdx.x) * kThreads + threadIdx.x) >> 5) * 32;
    if (r0 >= rows) return;
    const i64 r = r0 + lane;
    const bool has = r < rows;
    const i64 ds = has ? static_cast<i64>(coff[r]) : 0;
    i64 len = has ? static_cast<i64>(coff[r + 1]) - ds : 0;
    const i64 src = has ? temp_off[r] : 0;
    if (has && temp_off[r + 1] - src > seg_smem_capacity<W>()) len = 0;
    const i64 inc = warp_inclusive_sum(len);
    const i64 pre = inc - len;
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
        const i64 my_ds = __shfl_sync(0xffffffffu, ds, lo);
        const i64 my_src = __shfl_sync(0xffffffffu, src, lo);
        if (q < total) {
            nbr[my_ds + (q - my_pre)] = static_cast<i32>(tgt[my_src + (q - my_pre)]);
            ew[my_ds + (q - my_pre)] = wt[my_src + (q - my_pre)];
        }
    }
}

template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) copy_big_rows_kernel(const i32* __restrict__ list,
                                                                 const i64* __restrict__ alt_off,
                                                                 const O* __restrict__ coff,
                                                                 const u32* __restrict__ alt_k,
                                                                 const W* __restrict__ alt_w,
                                                                 i32* __restrict__ nbr, W* __restrict__ ew) {
    const i32 r = list[blockIdx.x];
    const i64 ds = coff[r], len = static_cast<i64>(coff[r + 1]) - ds, src = alt_off[blockIdx.x];
    for (i64 i = threadIdx.x; i < len; i += kThreads) {
        nbr[ds + i] = static_cast<i32>(alt_k[src + i]);
        ew[ds + i] = alt_w[src + i];
    }
}

}  // namespace gp
