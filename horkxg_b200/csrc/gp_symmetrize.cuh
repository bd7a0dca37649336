// Symmetrise and deduplicate a CSR on the GPU, with the semantics of the
// reference's external-memory tool (graph_untils/csr_symmetrize.cpp:277-538):
// every entry (v, u) with u != v stands for the undirected edge {u, v}; self
// loops are dropped and counted; the output holds both directions of every
// distinct edge, rows ascending by neighbour.
//
// The reference sorts (min, max) keys in disk runs, merges them, counts
// degrees and sorts again for the reverse direction.  Here the whole job is
// one device radix sort: each entry writes its two directed keys
// (v << b | u) and (u << b | v), b = bits of the vertex range, into slots 2e
// and 2e + 1 (a self loop writes two all-ones sentinels, which sort last);
// after the sort equal neighbours are adjacent, a flag-and-scan compaction
// keeps the first of each run, and the rows' lengths come from warp-
// aggregated counts of the sources.
#pragma once

#include "gp_prim.cuh"

namespace gp {

constexpr u64 kSymSentinel = ~0ULL;

// One warp per row: the two directed keys of every entry.
template <typename O>
__global__ void __launch_bounds__(kThreads) sym_keys_kernel(i64 n, const O* __restrict__ off,
                                                            const i32* __restrict__ nbr, int bits, u64* keys,
                                                            u64* self_loops) {
    const int lane = threadIdx.x & 31;
    const i64 warps_total = static_cast<i64>(gridDim.x) * kWarps;
    u64 loops = 0;
    for (i64 v = static_cast<i64>(blockIdx.x) * kWarps + (threadIdx.x >> 5); v < n; v += warps_total) {
        const i64 b = off[v], end = off[v + 1];
        for (i64 e = b + lane; e < end; e += 32) {
            const u64 u = static_cast<u64>(nbr[e]);
            if (u == static_cast<u64>(v)) {
                keys[2 * e] = kSymSentinel;
                keys[2 * e + 1] = kSymSentinel;
                ++loops;
            } else {
                keys[2 * e] = (static_cast<u64>(v) << bits) | u;
                keys[2 * e + 1] = (u << bits) | static_cast<u64>(v);
            }
        }
    }
    loops = warp_sum(loops);
    if (lane == 0 && loops) atomicAdd(reinterpret_cast<unsigned long long*>(self_loops), loops);
}

// R-MAT pairs generated on the device, drawn exactly as the host generator
// of this package draws them (horkxg_b200/csrc/gen.cpp, build_rmat): pair i,
// level l takes the uniform double of splitmix64(stream ^ splitmix64(64 i +
// l)) and descends into quadrant a | b | c | d; vertex ids then go through the
// seeded permutation `perm`.  Each pair writes its two directed keys (or two
// sentinels for a self loop), as sym_keys_kernel does for a CSR entry.
// splitmix64 is the published 64-bit mixer of Steele, Lea and Flood.
__host__ __device__ __forceinline__ u64 splitmix64(u64 x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

__global__ void rmat_keys_kernel(i64 pairs, int scale, double a, double ab, double abc, u64 stream,
                                 const u32* __restrict__ perm, int bits, u64* keys) {
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < pairs;
         i += static_cast<i64>(gridDim.x) * blockDim.x) {
        u32 s = 0, d = 0;
        for (int level = 0; level < scale; ++level) {
            const u64 x = splitmix64(stream ^ splitmix64(static_cast<u64>(i) * 64 + static_cast<u64>(level)));
            const double r = static_cast<double>(x >> 11) * (1.0 / 9007199254740992.0);
            s = (s << 1) | (r >= ab ? 1u : 0u);
            d = (d << 1) | (((r >= a && r < ab) || r >= abc) ? 1u : 0u);
        }
        const u64 ps = perm[s], pd = perm[d];
        keys[2 * i] = ps == pd ? kSymSentinel : (ps << bits) | pd;
        keys[2 * i + 1] = ps == pd ? kSymSentinel : (pd << bits) | ps;
    }
}

// Position of the first sentinel among sorted keys (= the count of keys
// that are not sentinels), into *first (preset to the key count).
__global__ void sym_first_sentinel_kernel(i64 count, const u64* __restrict__ keys, i64* first) {
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<i64>(gridDim.x) * blockDim.x)
        if (keys[i] == kSymSentinel && (i == 0 || keys[i - 1] != kSymSentinel)) *first = i;
}

// First key of each run among the `valid` sorted keys.
struct SymHead {
    const u64* keys;
    i64 valid;
    __device__ i64 operator()(i64 i) const { return i < valid && (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0; }
};

// Writes the neighbour of every run head at its rank and counts the row
// lengths (keys sorted by source, so a warp's heads mostly share a source:
// one atomic per source and warp).
template <typename N>
__global__ void sym_compact_kernel(i64 valid, const u64* __restrict__ keys, const i64* __restrict__ rank, int bits,
                                   N* out_nbr, i64* degree) {
    const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
    const i64 end = (valid + 31) / 32 * 32;   // whole warps, for the match below
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < end; i += stride) {
        const bool head = i < valid && (i == 0 || keys[i] != keys[i - 1]);
        const u64 key = i < valid ? keys[i] : 0;
        const i64 src = head ? static_cast<i64>(key >> bits) : -1;
        if (head) out_nbr[rank[i]] = static_cast<N>(key & ((1ULL << bits) - 1));
        const unsigned peers = __match_any_sync(0xffffffffu, src);
        if (head && (threadIdx.x & 31) == __ffs(peers) - 1)
            atomicAdd(reinterpret_cast<unsigned long long*>(&degree[src]), static_cast<unsigned long long>(__popc(peers)));
    }
}

}  // namespace gp
