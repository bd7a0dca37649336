// Incremental bucketed refinement (src/refine_incremental.cuh:7-361,
// src/refine.cu:52-142).  B200 layout:
//
// * the dense n x k affinity cache is u32 when the graph's total directed
//   edge weight fits 32 bits (halving the dominant HBM stream), else u64;
// * LP proposals append proposers to a list; the priority filter, the fused
//   cache+cut update and the commit then touch proposers/movers only;
// * list-driven kernels use a fixed grid with grid-stride loops so the host
//   never has to size a launch from a device count;
// * the rebalance ranks vertices inside a (source, gain bucket, section)
//   bucket either with atomics in arbitrary order (the reference's
//   behaviour) or, in deterministic mode, by (gain per weight descending,
//   vertex ascending) through a stable radix sort, which makes labels
//   bit-reproducible.
#pragma once

#include "gp_prim.cuh"
#include "gp_sclp.cuh"

namespace gp {

constexpr int kBalBuckets = 50, kBalSections = 16, kBalWidth = kBalBuckets * kBalSections;

struct RefineCounters {
    i64 proposers;
    i64 movers;
    long long delta;      // cut decrease of the last apply
    u64 directed_cut;
    i64 mover_degree;     // sum of the movers' degrees
    i64 big;              // movers of degree > kSplitDegree handed to apply_big_rows_kernel
    i64 big_degree;       // their degree sum
    i64 walked_degree;    // edges apply_cache_cut_kernel walked itself
    i64 hub_edges;        // edges of moving hubs walked by hub_apply_kernel
    i64 hub_chunks;       // their chunks
    i64 filter_degree;    // edges of the LP proposers below the hub degree (profiling only)
};

// Profiling only: the edges the priority filter walks (proposers' rows below
// the hub degree), into ctr->filter_degree.
template <typename O>
__global__ void filter_degree_kernel(const i32* __restrict__ list, const RefineCounters* ctr_in,
                                     const O* __restrict__ off, RefineCounters* ctr) {
    const i64 count = ctr_in->proposers;
    i64 sum = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i32 v = list[i];
        const i64 d = static_cast<i64>(off[v + 1]) - static_cast<i64>(off[v]);
        if (d <= kHubDegree) sum += d;
    }
    sum = warp_sum(sum);
    if ((threadIdx.x & 31) == 0 && sum)
        atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->filter_degree), static_cast<unsigned long long>(sum));
}

// Per-vertex proposal record written by the LP pass: the priority filter
// gathers one 16-byte record per neighbour instead of three arrays.
struct alignas(16) PropRec {
    i32 label;
    i32 target;   // -1: no proposal
    i64 gain;
};

__device__ __forceinline__ void cache_add(u32* p, u64 v) { atomicAdd(p, static_cast<u32>(v)); }
__device__ __forceinline__ void cache_add(u64* p, u64 v) { atomic_add_u64(p, v); }

// Exact directed cut, warp per vertex, one atomic per block
// (refine_cut_kernel, src/refine.cu:52-87).
template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) cut_kernel(i64 n, const O* __restrict__ off, const i32* __restrict__ nbr,
                                                       const W* __restrict__ ew, const i32* __restrict__ labels,
                                                       u64* out) {
    __shared__ u64 sh[kWarps + 1];
    const int lane = threadIdx.x & 31;
    u64 local = 0;
    const i64 warps_total = static_cast<i64>(gridDim.x) * kWarps;
    for (i64 v = static_cast<i64>(blockIdx.x) * kWarps + (threadIdx.x >> 5); v < n; v += warps_total) {
        const i64 b = off[v], end = off[v + 1];
        if (end - b > kHubDegree) continue;   // hub rows: chunked kernel
        const i32 s = labels[v];
        for (i64 e = b + lane; e < end; e += 32)
            if (labels[nbr[e]] != s) local += static_cast<u64>(weight_at(ew, e));
    }
    local = block_sum(local, sh);
    if (threadIdx.x == 0 && local) atomic_add_u64(out, local);
}

// Sum of `w` over the lanes that share this lane's `key` (the lanes of
// `peers`), the same value in every lane of the group.
template <typename C>
__device__ __forceinline__ u64 group_sum(unsigned peers, u64 w) {
    if constexpr (sizeof(C) == 4) {
        return __reduce_add_sync(peers, static_cast<u32>(w));
    } else {
        u64 sum = 0;
#pragma unroll
        for (int s = 0; s < 32; ++s) {
            const u64 x = __shfl_sync(0xffffffffu, w, s);
            if (peers & (1u << s)) sum += x;
        }
        return sum;
    }
}

// One vertex's k cache entries into registers, with 16-byte loads when the
// row is 16-byte aligned (k a multiple of 4 for 32-bit entries, of 2 for
// 64-bit entries); entries past k are left untouched.
template <typename C>
__device__ __forceinline__ void load_row(const C* row, int k, C (&vals)[32]) {
    if constexpr (sizeof(C) == 4) {
        if ((k & 3) == 0) {
            const uint4* r4 = reinterpret_cast<const uint4*>(row);
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (4 * q < k) {
                    const uint4 x = r4[q];
                    vals[4 * q] = x.x; vals[4 * q + 1] = x.y; vals[4 * q + 2] = x.z; vals[4 * q + 3] = x.w;
                }
            return;
        }
    } else {
        if ((k & 1) == 0) {
            const ulonglong2* r2 = reinterpret_cast<const ulonglong2*>(row);
#pragma unroll
            for (int q = 0; q < 16; ++q)
                if (2 * q < k) {
                    const ulonglong2 x = r2[q];
                    vals[2 * q] = x.x; vals[2 * q + 1] = x.y;
                }
            return;
        }
    }
#pragma unroll
    for (int p = 0; p < 32; ++p)
        if (p < k) vals[p] = row[p];
}

// incremental_build_affinity (src/refine_incremental.cuh:7-25).  A warp
// takes four consecutive vertices: rows of at most 32 entries are walked by
// 8 lanes each (up to four steps, all four rows at once), longer rows (up to
// the hub degree) by the whole warp one after the other.  Each row is summed
// in a private accumulator in shared memory: with a 32-bit cache (every sum
// fits 32 bits) every lane adds its edge with a 32-bit shared atomic; with a
// 64-bit cache lanes holding the same part are grouped with __match_any_sync
// and only the group leader adds their sum (measured at RMAT-24: the 32-bit
// atomics take 26% less time than the match, 64-bit shared atomics 45% more).
// The four cache rows, consecutive in memory, are then stored by the whole
// warp in one coalesced pass.  Hub rows are left to the chunked kernel
// (zero_hub_rows_kernel clears them after this one).
template <typename O, typename W, typename C>
__global__ void __launch_bounds__(kThreads) build_cache_kernel(i64 n, const O* __restrict__ off,
                                                               const i32* __restrict__ nbr, const W* __restrict__ ew,
                                                               const i32* __restrict__ labels, int k, C* cache) {
    __shared__ u64 rows[kWarps][4][32];
    u32 (*rows32)[4][32] = reinterpret_cast<u32 (*)[4][32]>(&rows[0][0][0]);   // C = u32: 32-bit accumulators
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane >> 3, gl = lane & 7;
    const i64 warps_total = static_cast<i64>(gridDim.x) * kWarps;
    for (i64 q = static_cast<i64>(blockIdx.x) * kWarps + warp; q * 4 < n; q += warps_total) {
        const i64 v = q * 4 + grp;
        i64 b = 0, deg = 0;
        if (v < n) {
            b = static_cast<i64>(off[v]);
            deg = static_cast<i64>(off[v + 1]) - b;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if constexpr (sizeof(C) == 4) rows32[warp][grp][gl + 8 * j] = 0;
            else rows[warp][grp][gl + 8 * j] = 0;
        }
        __syncwarp();
        const bool short_row = deg <= 32;
        const unsigned steps = __reduce_max_sync(0xffffffffu, short_row ? static_cast<unsigned>((deg + 7) >> 3) : 0u);
        for (unsigned r = 0; r < steps; ++r) {
            const i64 e = static_cast<i64>(r) * 8 + gl;
            int p = -1;
            u64 w = 0;
            if (short_row && e < deg) {
                const i32 u = nbr[b + e];
                if (u != v) { p = labels[u]; w = static_cast<u64>(weight_at(ew, b + e)); }
            }
            if constexpr (sizeof(C) == 4) {
                if (p >= 0) atomicAdd(&rows32[warp][grp][p], static_cast<u32>(w));
            } else {
                const unsigned peers = __match_any_sync(0xffffffffu, p < 0 ? -1 - grp : grp * 32 + p);
                const u64 sum = group_sum<C>(peers, w);
                if (p >= 0 && lane == __ffs(peers) - 1) rows[warp][grp][p] += sum;
            }
            __syncwarp();
        }
        // rows of 33..kHubDegree entries, one at a time by the whole warp
        unsigned longs = __ballot_sync(0xffffffffu, gl == 0 && !short_row && deg <= kHubDegree);
        while (longs) {
            const int src = __ffs(longs) - 1;
            longs &= longs - 1;
            const int g = src >> 3;
            const i64 lb = __shfl_sync(0xffffffffu, b, src), ld = __shfl_sync(0xffffffffu, deg, src);
            const i64 lv = q * 4 + g;
            for (i64 base = 0; base < ld; base += 32) {
                const i64 e = base + lane;
                int p = -1;
                u64 w = 0;
                if (e < ld) {
                    const i32 u = nbr[lb + e];
                    if (u != lv) { p = labels[u]; w = static_cast<u64>(weight_at(ew, lb + e)); }
                }
                if constexpr (sizeof(C) == 4) {
                    if (p >= 0) atomicAdd(&rows32[warp][g][p], static_cast<u32>(w));
                } else {
                    const unsigned peers = __match_any_sync(0xffffffffu, p);
                    const u64 sum = group_sum<C>(peers, w);
                    if (p >= 0 && lane == __ffs(peers) - 1) rows[warp][g][p] += sum;
                }
                __syncwarp();
            }
        }
        // the four rows are consecutive in the cache: entries [4qk, 4qk + 4k)
        const i64 first = q * 4;
        const int nrows = static_cast<int>(n - first < 4 ? n - first : 4);
        const unsigned hub_rows = __ballot_sync(0xffffffffu, gl == 0 && deg > kHubDegree);
        C* dst = cache + first * k;
        for (int i = lane; i < nrows * k; i += 32) {
            const int row = i / k;
            if (!(hub_rows & (1u << (row * 8)))) {
                if constexpr (sizeof(C) == 4) dst[i] = static_cast<C>(rows32[warp][row][i - row * k]);
                else dst[i] = static_cast<C>(rows[warp][row][i - row * k]);
            }
        }
        __syncwarp();
    }
}

// incremental_lp_proposals (src/refine_incremental.cuh:27-46); proposers
// are appended to `list`.
template <typename C>
__global__ void lp_proposals_kernel(i64 n, const C* __restrict__ cache, const i32* __restrict__ labels, int k,
                                    double filter, const u64* __restrict__ max_edge_weight, unsigned char* locks,
                                    i32* targets, i64* gains, PropRec* props, i32* list, RefineCounters* ctr) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    // the filter of refine_incremental.cuh:332-333, from the level's maximum
    // edge weight when it was computed on the device
    if (max_edge_weight) filter = *max_edge_weight <= 1 ? 0.25 : 0.75;
    bool propose = false;
    if (v < n) {
        i32 target = -1;
        i64 g = INT64_MIN;
        const i32 s = labels[v];
        if (locks[v]) {
            locks[v] = 0;
        } else {
            C vals[32];
            load_row(cache + v * k, k, vals);
            u64 best = 0, current = 0;
            int t = -1;
#pragma unroll
            for (int p = 0; p < 32; ++p) {
                if (p >= k) break;
                const u64 c = static_cast<u64>(vals[p]);
                if (p == s) current = c;
                else if (c > best) { best = c; t = p; }
            }
            if (t >= 0 &&
                (best >= current || current - best < static_cast<u64>(filter * static_cast<double>(current)))) {
                g = best >= current ? static_cast<i64>(best - current) : -static_cast<i64>(current - best);
                target = t;
                propose = true;
            }
        }
        targets[v] = target;
        gains[v] = g;
        props[v] = {s, target, g};
    }
    const u64 slot = warp_append(propose, reinterpret_cast<u64*>(&ctr->proposers));
    if (propose) list[slot] = static_cast<i32>(v);
}

// incremental_priority_filter (src/refine_incremental.cuh:48-67); movers are
// appended to `movers` and flagged.
template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) priority_filter_kernel(
    const i32* __restrict__ list, const RefineCounters* ctr_in, const O* __restrict__ off,
    const i32* __restrict__ nbr, const W* __restrict__ ew, const PropRec* __restrict__ props, unsigned char* flags,
    i32* movers, RefineCounters* ctr) {
    // A warp takes up to 32 proposers and walks their edges together; each
    // row's correction is summed in shared memory (hub rows: chunked kernel).
    __shared__ long long corr_sh[kWarps][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 count = ctr_in->proposers;
    const i64 warps = static_cast<i64>(gridDim.x) * kWarps;
    const int G = rows_per_warp(count, warps);
    for (i64 i0 = (static_cast<i64>(blockIdx.x) * kWarps + warp) * G; i0 < count; i0 += warps * G) {
        const i64 i = i0 + lane;
        const bool has = lane < G && i < count;
        const i32 v = has ? list[i] : 0;
        const i64 b = has ? static_cast<i64>(off[v]) : 0;
        const i64 deg = has ? static_cast<i64>(off[v + 1]) - b : 0;
        const bool hub = deg > kHubDegree;
        const PropRec me = has ? props[v] : PropRec{0, -1, 0};
        corr_sh[warp][lane] = 0;
        __syncwarp();
        warp_edge_walk(b, hub ? 0 : deg, [&](bool valid, int owner, i64 e) {
            const i32 ov = __shfl_sync(0xffffffffu, v, owner);
            const i32 s = __shfl_sync(0xffffffffu, me.label, owner);
            const i32 t = __shfl_sync(0xffffffffu, me.target, owner);
            const i64 g = __shfl_sync(0xffffffffu, me.gain, owner);
            long long c = 0;
            if (valid) {
                const i32 u = nbr[e];
                if (u != ov) {
                    const PropRec o = props[u];
                    if (o.target >= 0 && (o.gain > g || (o.gain == g && u < ov))) {
                        const auto w = static_cast<long long>(weight_at(ew, e));
                        c = w * ((o.target == t) - (o.target == s) - (o.label == t) + (o.label == s));
                    }
                }
            }
            const long long run = warp_run_sum(c, owner);
            const int next = __shfl_down_sync(0xffffffffu, owner, 1);
            if ((lane == 31 || next != owner) && run != 0) corr_sh[warp][owner] += run;
            __syncwarp();
        });
        const bool move = has && !hub && me.gain + corr_sh[warp][lane] >= 0;
        const u64 slot = warp_append(move, reinterpret_cast<u64*>(&ctr->movers));
        if (move) {
            flags[v] = 1;
            movers[slot] = v;
        }
        const i64 moved_degree = warp_sum(move ? deg : i64{0});
        if (lane == 0 && moved_degree)
            atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->mover_degree),
                      static_cast<unsigned long long>(moved_degree));
        __syncwarp();
    }
}

// incremental_update_cache_and_cut (src/refine_incremental.cuh:69-95) for
// one edge of mover v (label s, target t): the neighbour's cache row loses w
// at s and gains it at t; the cut change is counted once per undirected edge
// (the neighbour is not a mover, or has the larger id).
//
// Here over the edges [b, e1) of mover v, thread `tid` of `nthreads`
// taking every nthreads-th edge, kApplyBatch of them per step: the batch's
// neighbour ids are loaded first, then their flags and labels, then the cache
// updates issued, so a thread keeps kApplyBatch independent gather chains in
// flight instead of one.  Integer sums, so the result does not depend on the
// order.
constexpr int kApplyBatch = 4;

template <typename W, typename C>
__device__ __forceinline__ long long apply_edges_batched(i32 v, i32 s, i32 t, i64 b, i64 e1, int tid, int nthreads,
                                                         const i32* __restrict__ nbr, const W* __restrict__ ew,
                                                         const i32* __restrict__ labels,
                                                         const i32* __restrict__ targets,
                                                         const unsigned char* __restrict__ flags, int k, C* cache) {
    long long gain = 0;
    const i64 step = static_cast<i64>(nthreads);
    for (i64 e0 = b + tid; e0 < e1; e0 += kApplyBatch * step) {
        i32 u[kApplyBatch];
#pragma unroll
        for (int j = 0; j < kApplyBatch; ++j) {
            const i64 e = e0 + j * step;
            u[j] = e < e1 ? nbr[e] : v;   // past the row: treated as a self loop, skipped
        }
        bool fu[kApplyBatch];
        i32 lu[kApplyBatch];
#pragma unroll
        for (int j = 0; j < kApplyBatch; ++j) {
            fu[j] = false;
            lu[j] = 0;
            if (u[j] != v) {
                fu[j] = flags[u[j]] != 0;
                lu[j] = labels[u[j]];
            }
        }
#pragma unroll
        for (int j = 0; j < kApplyBatch; ++j) {
            if (u[j] == v) continue;
            const u64 w = static_cast<u64>(weight_at(ew, e0 + j * step));
            cache_add(&cache[static_cast<i64>(u[j]) * k + s], 0ULL - w);
            cache_add(&cache[static_cast<i64>(u[j]) * k + t], w);
            if (fu[j] && u[j] < v) continue;
            const i32 nn = fu[j] ? targets[u[j]] : lu[j];
            gain += static_cast<long long>(w) * ((s != lu[j]) - (t != nn));
        }
    }
    return gain;
}

// The same update over the edges of up to 32 movers, one per lane (v, s, t, first
// edge `begin`, `deg` edges; deg 0 for no mover), walked as warp_edge_walk
// walks them but kApplyBatch 32-edge steps at a time: each lane resolves its
// kApplyBatch positions (owning lane, edge) and loads their neighbour ids,
// then their flags and labels, before any cache update.
template <typename W, typename C>
__device__ __forceinline__ long long warp_apply_rows(i32 v, i32 s, i32 t, i64 begin, i64 deg,
                                                     const i32* __restrict__ nbr, const W* __restrict__ ew,
                                                     const i32* __restrict__ labels, const i32* __restrict__ targets,
                                                     const unsigned char* __restrict__ flags, int k, C* cache) {
    const int lane = threadIdx.x & 31;
    const i64 inc = warp_inclusive_sum(deg);
    const i64 pre = inc - deg;
    const i64 total = __shfl_sync(0xffffffffu, inc, 31);
    long long gain = 0;
    for (i64 base = 0; base < total; base += kApplyBatch * 32) {
        i32 ov[kApplyBatch], os[kApplyBatch], ot[kApplyBatch], u[kApplyBatch];
        i64 e[kApplyBatch];
#pragma unroll
        for (int j = 0; j < kApplyBatch; ++j) {
            const i64 q = base + j * 32 + lane;
            int lo = 0;
#pragma unroll
            for (int step = 16; step; step >>= 1) {
                const i64 probe = __shfl_sync(0xffffffffu, pre, lo + step);
                if (probe <= q) lo += step;
            }
            const i64 my_pre = __shfl_sync(0xffffffffu, pre, lo);
            const i64 my_begin = __shfl_sync(0xffffffffu, begin, lo);
            ov[j] = __shfl_sync(0xffffffffu, v, lo);
            os[j] = __shfl_sync(0xffffffffu, s, lo);
            ot[j] = __shfl_sync(0xffffffffu, t, lo);
            e[j] = my_begin + (q - my_pre);
            u[j] = q < total ? nbr[e[j]] : ov[j];   // past the last edge: treated as a self loop, skipped
        }
        bool fu[kApplyBatch];
        i32 lu[kApplyBatch];
#pragma unroll
        for (int j = 0; j < kApplyBatch; ++j) {
            fu[j] = false;
            lu[j] = 0;
            if (u[j] != ov[j]) {
                fu[j] = flags[u[j]] != 0;
                lu[j] = labels[u[j]];
            }
        }
#pragma unroll
        for (int j = 0; j < kApplyBatch; ++j) {
            if (u[j] == ov[j]) continue;
            const u64 w = static_cast<u64>(weight_at(ew, e[j]));
            cache_add(&cache[static_cast<i64>(u[j]) * k + os[j]], 0ULL - w);
            cache_add(&cache[static_cast<i64>(u[j]) * k + ot[j]], w);
            if (fu[j] && u[j] < ov[j]) continue;
            const i32 nn = fu[j] ? targets[u[j]] : lu[j];
            gain += static_cast<long long>(w) * ((os[j] != lu[j]) - (ot[j] != nn));
        }
    }
    return gain;
}

// Movers of degree above this are walked by a whole block
// (apply_big_rows_kernel): one warp would take deg/32 dependent steps, and the
// launch would wait for that one warp.
constexpr i64 kSplitDegree = 256;

template <typename O, typename W, typename C>
__global__ void __launch_bounds__(kThreads) apply_cache_cut_kernel(
    const i32* __restrict__ movers, const RefineCounters* ctr_in, const O* __restrict__ off,
    const i32* __restrict__ nbr, const W* __restrict__ ew, const i32* __restrict__ labels,
    const i32* __restrict__ targets, const unsigned char* __restrict__ flags, int k, C* cache, RefineCounters* ctr,
    i32* __restrict__ big) {
    // A warp takes up to 32 movers and walks their edges together (rows above
    // kSplitDegree: block kernel; hub rows: chunked kernel).  The cut delta is
    // summed per warp and added with one atomic per warp, so warps never wait
    // for each other.
    const int lane = threadIdx.x & 31;
    const i64 count = ctr_in->movers;
    const i64 warps = static_cast<i64>(gridDim.x) * kWarps;
    const int G = rows_per_warp(count, warps);
    long long gain = 0;
    for (i64 i0 = (static_cast<i64>(blockIdx.x) * kWarps + (threadIdx.x >> 5)) * G; i0 < count; i0 += warps * G) {
        const i64 i = i0 + lane;
        const bool has = lane < G && i < count;
        const i32 v = has ? movers[i] : 0;
        const i64 b = has ? static_cast<i64>(off[v]) : 0;
        i64 deg = has ? static_cast<i64>(off[v + 1]) - b : 0;
        const bool split = deg > kSplitDegree && deg <= kHubDegree;
        const u64 slot = warp_append(split, reinterpret_cast<u64*>(&ctr->big));
        if (split) big[slot] = v;
        const i64 big_degree = warp_sum(split ? deg : i64{0});
        if (lane == 0 && big_degree)
            atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->big_degree), static_cast<unsigned long long>(big_degree));
        if (deg > kSplitDegree) deg = 0;
        const i64 walked = warp_sum(deg);
        if (lane == 0 && walked)
            atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->walked_degree), static_cast<unsigned long long>(walked));
        const i32 s = has ? labels[v] : 0, t = has ? targets[v] : 0;
        gain += warp_apply_rows(v, s, t, b, deg, nbr, ew, labels, targets, flags, k, cache);
    }
    gain = warp_sum(gain);
    if (lane == 0 && gain) atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->delta), static_cast<unsigned long long>(gain));
}

// The movers set aside by apply_cache_cut_kernel (kSplitDegree < degree <=
// kHubDegree), one block per row over a grid-stride loop.
template <typename O, typename W, typename C>
__global__ void __launch_bounds__(kThreads) apply_big_rows_kernel(
    const i32* __restrict__ big, const RefineCounters* ctr_in, const O* __restrict__ off,
    const i32* __restrict__ nbr, const W* __restrict__ ew, const i32* __restrict__ labels,
    const i32* __restrict__ targets, const unsigned char* __restrict__ flags, int k, C* cache, RefineCounters* ctr) {
    __shared__ long long sh[kWarps + 1];
    const i64 count = ctr_in->big;
    long long gain = 0;
    for (i64 r = blockIdx.x; r < count; r += gridDim.x) {
        const i32 v = big[r];
        const i32 s = labels[v], t = targets[v];
        gain += apply_edges_batched(v, s, t, static_cast<i64>(off[v]), static_cast<i64>(off[v + 1]),
                                    static_cast<int>(threadIdx.x), kThreads, nbr, ew, labels, targets, flags, k,
                                    cache);
    }
    gain = block_sum(gain, sh);
    if (threadIdx.x == 0 && gain)
        atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->delta), static_cast<unsigned long long>(gain));
}

// incremental_commit (src/refine_incremental.cuh:97-109); also clears the
// mover flag so that `flags` is all-zero outside an apply.  Part-weight
// changes are summed per block in shared memory first: all movers hit the
// same k counters, so global atomics would serialise.
template <typename W>
__global__ void commit_kernel(const i32* __restrict__ movers, const RefineCounters* ctr_in,
                              i32* labels, const i32* __restrict__ targets, const W* __restrict__ vw, u64* pw,
                              unsigned char* locks, unsigned char* flags, int lp) {
    __shared__ unsigned long long delta[32];
    if (threadIdx.x < 32) delta[threadIdx.x] = 0;
    __syncthreads();
    const i64 count = ctr_in->movers;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i32 v = movers[i];
        const i32 s = labels[v], t = targets[v];
        const u64 w = static_cast<u64>(weight_at(vw, v));
        atomicAdd(&delta[s], 0ULL - w);
        atomicAdd(&delta[t], static_cast<unsigned long long>(w));
        labels[v] = t;
        if (lp) locks[v] = 1;
        flags[v] = 0;
    }
    __syncthreads();
    if (threadIdx.x < 32 && delta[threadIdx.x]) atomic_add_u64(&pw[threadIdx.x], delta[threadIdx.x]);
}

// Rebalance gain bucket (refine_incremental.cuh:167-171) restated with host
// thresholds 1.5^j: for g < 0, 25 + the smallest j with -g <= 1.5^j,
// clamped to [2, 49].
struct BucketThresholds { double t[48]; };   // j = -23 .. 24

__device__ __forceinline__ int gain_bucket(double g, const BucketThresholds& th) {
    if (g > 0) return 0;
    if (g == 0) return 1;
    const double a = -g;
    if (a <= th.t[0]) return 2;
    int lo = 1, hi = 47;   // smallest index in [1,47] with a <= t[idx], else 48
    if (a > th.t[47]) return 49;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a <= th.t[mid]) hi = mid; else lo = mid + 1;
    }
    return 25 + (lo - 23);
}

// Ranks of weighted items in per-key counters with one atomic per key and
// warp: the lanes that share a key take consecutive ranges in lane order, as
// if their atomicAdds had run back to back (the reference's ranks come from
// plain atomicAdds in scheduling order, so any such order is one it can
// produce).  All 32 lanes call it; key < 0 means no item.
__device__ __forceinline__ u64 warp_rank_add(int key, u64 w, bool unit, u64* counts) {
    const int lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const unsigned lower = peers & lanemask_lt();
    u64 before = 0, total = 0;
    if (unit) {
        before = static_cast<u64>(__popc(lower));
        total = static_cast<u64>(__popc(peers));
    } else {
#pragma unroll
        for (int s = 0; s < 32; ++s) {
            const u64 x = __shfl_sync(0xffffffffu, w, s);
            if ((peers >> s) & 1u) {
                total += x;
                if (s < lane) before += x;
            }
        }
    }
    const int leader = __ffs(peers) - 1;
    u64 base = 0;
    if (key >= 0 && lane == leader) base = atomic_add_u64(&counts[key], total);
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + before;
}

// incremental_rebalance_proposals + balance_source_histogram
// (src/refine_incremental.cuh:111-186).  Atomic mode ranks here; the
// deterministic mode appends candidates (ascending vertex order is restored by
// the scan-based compaction that follows).
// One rebalance candidate: the destination with slack that it is best
// connected to (ties: more slack), a zero-connection vertex spread over the
// parts with slack by a hashed ticket; returns the vertex's bucket
// (source part, gain-per-weight bucket, hashed section) or -1.
template <typename C, typename W>
__device__ __forceinline__ int rebalance_choice(i64 v, const C* __restrict__ cache, const i32* __restrict__ labels,
                                                const W* __restrict__ vw, int k, const u64* spw, u64 cap,
                                                const BucketThresholds& th, i32* targets, double* gpw, i32* bucket,
                                                u64& w) {
    targets[v] = -1;
    bucket[v] = -1;
    const i32 s = labels[v];
    if (spw[s] <= cap) return -1;
    w = static_cast<u64>(weight_at(vw, v));
    C vals[32];
    load_row(cache + v * k, k, vals);
    int best = -1;
    u64 best_conn = 0, best_slack = 0, current = 0;
#pragma unroll
    for (int p = 0; p < 32; ++p) {
        if (p >= k) break;
        const u64 value = static_cast<u64>(vals[p]);
        if (p == s) { current = value; continue; }
        const u64 pp = spw[p];
        if (pp >= cap || w > cap - pp) continue;
        const u64 slack = cap - pp;
        if (best < 0 || value > best_conn || (value == best_conn && slack > best_slack)) {
            best = p; best_conn = value; best_slack = slack;
        }
    }
    if (best >= 0 && best_conn == 0) {
        u64 total_slack = 0;
        for (int p = 0; p < k; ++p) {
            const u64 pp = spw[p];
            if (p != s && pp < cap && w <= cap - pp)
                total_slack = UINT64_MAX - total_slack < cap - pp ? UINT64_MAX : total_slack + cap - pp;
        }
        u64 ticket = static_cast<u64>(mix32(static_cast<u32>(v))) % total_slack;
        for (int p = 0; p < k; ++p) {
            const u64 pp = spw[p];
            if (p == s || pp >= cap || w > cap - pp) continue;
            const u64 slack = cap - pp;
            if (ticket < slack) { best = p; break; }
            ticket -= slack;
        }
    }
    if (best < 0) return -1;
    const double gain = best_conn >= current ? static_cast<double>(best_conn - current)
                                             : -static_cast<double>(current - best_conn);
    const double g = gain / static_cast<double>(w);
    targets[v] = best;
    gpw[v] = g;
    const int b = s * kBalWidth + gain_bucket(g, th) * kBalSections +
                  static_cast<int>(mix32(static_cast<u32>(v)) % kBalSections);
    bucket[v] = b;
    return b;
}

// The rebalance kernels run over list[0, n), or over list[0, *count) when
// `count` is given (the candidate count left on the device, no round trip);
// their grid-stride loops keep whole warps together for the warp ranks.
__device__ __forceinline__ i64 list_length(i64 n, const i64* count) { return count ? *count : n; }

// Over the candidate list (vertices of overloaded parts); part weights are
// staged in shared memory.
template <typename C, typename W>
__global__ void rebalance_proposals_kernel(i64 n, const i64* count, const i32* __restrict__ list,
                                           const C* __restrict__ cache, const i32* __restrict__ labels,
                                           const W* __restrict__ vw, int k, const u64* __restrict__ pw, u64 cap,
                                           BucketThresholds th, int deterministic, i32* targets, double* gpw,
                                           i32* bucket, u64* rank, u64* counts) {
    __shared__ u64 spw[32];
    if (threadIdx.x < 32) spw[threadIdx.x] = static_cast<int>(threadIdx.x) < k ? pw[threadIdx.x] : ~0ULL;
    __syncthreads();
    n = list_length(n, count);
    for (i64 base = static_cast<i64>(blockIdx.x) * blockDim.x; base < n; base += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 i = base + threadIdx.x;
        const i64 v = i < n ? (list ? list[i] : i) : 0;
        u64 w = 0;
        const int b = i < n ? rebalance_choice(v, cache, labels, vw, k, spw, cap, th, targets, gpw, bucket, w) : -1;
        if (!deterministic) {
            const u64 r = warp_rank_add(b, w, vw == nullptr, counts);
            if (b >= 0) rank[v] = r;
        }
    }
}

// balance_scan_buckets (src/refine_incremental.cuh:188-202): exclusive scan
// of the 800 buckets of each part, block per part.  The counts are left
// zero for the next ranking pass.
__global__ void __launch_bounds__(kThreads) bucket_scan_kernel(u64* counts, u64* offsets) {
    __shared__ u64 sh[kWarps + 1];
    constexpr int kPer = (kBalWidth + kThreads - 1) / kThreads;   // 4
    u64 vals[kPer];
    u64 local = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int b = threadIdx.x * kPer + i;
        vals[i] = b < kBalWidth ? counts[blockIdx.x * kBalWidth + b] : 0;
        if (b < kBalWidth) counts[blockIdx.x * kBalWidth + b] = 0;
        local += vals[i];
    }
    u64 run = block_exclusive_sum(local, sh, static_cast<u64*>(nullptr));
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int b = threadIdx.x * kPer + i;
        if (b < kBalWidth) offsets[blockIdx.x * kBalWidth + b] = run;
        run += vals[i];
    }
}

// balance_select_sources (src/refine_incremental.cuh:204-217)
template <typename W>
__global__ void select_sources_kernel(i64 n, const i64* count, const i32* __restrict__ list, i32* bucket, u64* rank,
                                      const u64* offsets, const u64* pw, u64 cap, const i32* targets, const W* vw,
                                      int deterministic, u64* counts) {
    n = list_length(n, count);
    for (i64 base = static_cast<i64>(blockIdx.x) * blockDim.x; base < n; base += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 i = base + threadIdx.x;
        const i64 v = i < n ? (list ? list[i] : i) : 0;
        int d = -1;
        if (i < n && bucket[v] >= 0) {
            const int b = bucket[v], s = b / kBalWidth;
            if (offsets[b] + rank[v] >= pw[s] - cap) {
                bucket[v] = -1;
            } else {
                d = targets[v] * kBalWidth + b % kBalWidth;
                bucket[v] = d;
            }
        }
        if (!deterministic) {
            const u64 r = warp_rank_add(d, i < n ? static_cast<u64>(weight_at(vw, v)) : 0, vw == nullptr, counts);
            if (d >= 0) rank[v] = r;
        }
    }
}

// balance_select_destinations (src/refine_incremental.cuh:219-232).
template <typename W>
__global__ void select_destinations_kernel(i64 n, const i64* count, const i32* __restrict__ list, const i32* bucket,
                                           const u64* rank, const u64* offsets, const u64* pw, u64 cap, const W* vw,
                                           unsigned char* flags, i32* movers, RefineCounters* ctr) {
    n = list_length(n, count);
    for (i64 base = static_cast<i64>(blockIdx.x) * blockDim.x; base < n; base += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 i = base + threadIdx.x;
        bool move = false;
        i64 v = 0;
        if (i < n) {
            v = list ? list[i] : i;
            const int b = bucket[v];
            if (b >= 0) {
                const u64 before = offsets[b] + rank[v];
                const u64 slack = cap - pw[b / kBalWidth];
                move = before <= slack && static_cast<u64>(weight_at(vw, v)) <= slack - before;
            }
        }
        const u64 slot = warp_append(move, reinterpret_cast<u64*>(&ctr->movers));
        if (move) {
            flags[v] = 1;
            movers[slot] = static_cast<i32>(v);
        }
    }
}

// Deterministic ranks: candidates (bucket >= 0) compacted in vertex order,
// sorted by (bucket asc, gain per weight desc); rank = weight prefix inside
// the bucket; counts = bucket totals.
struct HasBucket {
    const i32* bucket;
    const i32* list;   // candidate vertices (ascending), or null for all
    __device__ i64 operator()(i64 i) const { return bucket[list ? list[i] : i] >= 0 ? 1 : 0; }
};

__global__ void compact_bucket_kernel(i64 n, const i32* cand, const i32* bucket, const i64* pos, i32* list) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const i64 v = cand ? cand[i] : i;
    if (bucket[v] >= 0) list[pos[i]] = static_cast<i32>(v);
}

// Vertices of the parts above capacity: the only rebalance candidates, and a
// superset of them for the whole rebalance (destinations never exceed the
// capacity, so no part becomes overloaded and vertices only leave).
struct InOverloaded {
    const i32* labels;
    const u64* pw;
    u64 cap;
    __device__ i64 operator()(i64 v) const { return pw[labels[v]] > cap ? 1 : 0; }
};

__global__ void compact_overloaded_kernel(i64 n, const i32* labels, const u64* pw, u64 cap, const i64* pos,
                                          i32* list) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n && pw[labels[v]] > cap) list[pos[v]] = static_cast<i32>(v);
}

// mode 0: ~orderable(gpw) (desc); mode 1: bucket
__global__ void rank_keys_kernel(i64 count, const i32* list, const double* gpw, const i32* bucket, int mode, u64* keys) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const i32 v = list[i];
    if (mode == 0) {
        double g = gpw[v];
        if (g == 0.0) g = 0.0;
        const u64 b = static_cast<u64>(__double_as_longlong(g));
        const u64 ord = (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
        keys[i] = ~ord;
    } else {
        keys[i] = static_cast<u64>(bucket[v]);
    }
}

template <typename W>
struct ListWeight {
    const i32* list;
    const W* vw;
    __device__ u64 operator()(i64 i) const { return static_cast<u64>(weight_at(vw, list[i])); }
};

__global__ void bucket_heads_kernel(i64 count, const i32* list, const i32* bucket, const u64* excl, u64* bucket_base) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int b = bucket[list[i]];
    if (i == 0 || bucket[list[i - 1]] != b) bucket_base[b] = excl[i];
}

template <typename W>
__global__ void bucket_ranks_kernel(i64 count, const i32* list, const i32* bucket, const u64* excl,
                                    const u64* bucket_base, const W* vw, u64* rank, u64* counts) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const i32 v = list[i];
    const int b = bucket[v];
    rank[v] = excl[i] - bucket_base[b];
    if (i + 1 == count || bucket[list[i + 1]] != b)
        counts[b] = excl[i] + static_cast<u64>(weight_at(vw, v)) - bucket_base[b];
}

__global__ void project_kernel(i64 n, const i32* map, const i32* coarse, i32* fine) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n) fine[v] = coarse[map[v]];
}

template <typename W>
__global__ void max_weight_kernel(i64 m, const W* ew, u64* out) {
    u64 mx = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += static_cast<i64>(gridDim.x) * blockDim.x)
        mx = static_cast<u64>(ew[i]) > mx ? static_cast<u64>(ew[i]) : mx;
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0 && mx) atomic_max_u64(out, mx);
}

}  // namespace gp
