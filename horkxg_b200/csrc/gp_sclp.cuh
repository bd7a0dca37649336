// SCLP aggregation (size-constrained label propagation), the first stage of
// the partitioner.  Restates src/coarsen.cu:937-1659 with a B200 layout:
//
// * affinity + gain decode fused in one pass per degree class: 8-lane groups
//   (__match_any_sync) for deg <= 8, a warp for deg <= 32, a warp with a
//   512-slot shared hash for deg <= 256, a block with a 4096-slot shared hash
//   for deg <= 2048, and a block with an L2-resident global hash table for
//   hubs above that; the four u64 affinity arrays of the reference never hit
//   HBM;
// * admission without a global sort: every target's proposed weight
//   ("demand") is summed during the affinity pass; a proposal to a target
//   whose whole demand fits is accepted directly, and only proposals to
//   over-subscribed targets are ordered by (target, gain desc, tie desc,
//   vertex) with a stable LSD radix sort over the compacted list;
// * isolated packing, two-hop pairing and compaction as in the reference.
//
// The result (cluster map, coarse weights) is bit-identical to the
// reference's: every sum is exact integer arithmetic and every selection is a
// total order.
#pragma once

#include "gp_prim.cuh"

namespace gp {

constexpr i32 kInvalid = 0x7fffffff;     // SCLP_INVALID, src/coarsen.cu:201
constexpr int kMediumSlots = 512;        // warp hash, deg 33..256
constexpr int kLargeSlots = 4096;        // block hash, deg 257..2048
constexpr int kHubDegree = 2048;         // above: global hash

struct RoundParams {
    u32 role_salt;
    u32 tie_salt;
    u32 mover_threshold;
    int filter;      // role filtering (rounds 0-3); off for the two-hop pass
    int identity;    // clusters are the identity (round 0): skip the gather
    int two_hop;     // write favourites instead of LP proposals
    int sum32;       // every connection sum fits 32 bits (total edge weight < 2^32)
};

// Salts of src/coarsen.cu:1152-1157.
inline RoundParams make_round(u32 seed, int level, int round, bool filter, u32 mover_threshold) {
    RoundParams p;
    p.role_salt = seed ^ (static_cast<u32>(level) * 0x9e3779b9U) ^ (static_cast<u32>(round) * 0x85ebca6bU) ^ 0x27d4eb2dU;
    p.tie_salt = seed ^ (static_cast<u32>(level) * 0xc2b2ae35U) ^ (static_cast<u32>(round) * 0x165667b1U) ^ 0xd3a2646cU;
    p.mover_threshold = mover_threshold;
    p.filter = filter ? 1 : 0;
    p.identity = round == 0 ? 1 : 0;
    p.two_hop = 0;
    p.sum32 = 0;
    return p;
}

__device__ __forceinline__ bool is_mover(i32 c, const RoundParams& p) {
    return mix32(static_cast<u32>(c) ^ p.role_salt) < p.mover_threshold;
}

// With role filtering, a vertex whose own cluster is not a mover gets no
// proposal whatever its affinities (sclp_decode_gain_kernel,
// src/coarsen.cu:562-598), so its affinity pass is skipped altogether.
__device__ __forceinline__ bool role_blocked(i32 source, const RoundParams& p) {
    return p.filter && !is_mover(source, p);
}

// sclp_better_candidate, src/coarsen.cu:224-229
__device__ __forceinline__ bool better(u64 a, u64 ta, u64 b, u64 tb) {
    return a > b || (a == b && a != 0 && ta > tb);
}

__device__ __forceinline__ u64 tie_key(u32 v, i32 c, u32 tie_salt) {
    const u32 h = mix32(v ^ mix32(static_cast<u32>(c)) ^ tie_salt);
    return (static_cast<u64>(h) << 32) | (0xffffffffULL - static_cast<u32>(c));
}

struct SclpOut {
    i32* target;      // proposal / favourite, kInvalid if none
    u64* gain;
    u32* tie;
    u64* demand;      // per target cluster: proposed vertex weight
};

// sclp_decode_gain_kernel (src/coarsen.cu:562-598) + favourite selection
// (sclp_singleton_favorite_kernel, :682-692) + demand accumulation.
template <typename W>
__device__ __forceinline__ void decode_and_write(i32 v, i32 source, u64 current, u64 best, u64 best_tie,
                                                 const RoundParams& p, const W* vw, const u64* cw,
                                                 const SclpOut& out) {
    const bool can_move = !p.filter || is_mover(source, p);
    const u64 role_gain = can_move && best > current ? best - current : 0;
    i32 target = kInvalid;
    if (role_gain != 0) {
        const auto t = static_cast<i32>(0xffffffffULL - (best_tie & 0xffffffffULL));
        if (t >= 0 && t != source) target = t;
    }
    const u64 w = static_cast<u64>(weight_at(vw, v));
    if (p.two_hop && target != kInvalid && cw[source] != w) target = kInvalid;
    out.target[v] = target;
    if (target != kInvalid) {
        out.gain[v] = best - current;
        out.tie[v] = static_cast<u32>(best_tie >> 32);
        if (!p.two_hop) atomic_add_u64(&out.demand[target], w);
    }
}

// Reduce (current, best, tie) over `width` lanes (a power of two <= 32)
// using xor shuffles; all lanes end with the result.
__device__ __forceinline__ void group_reduce(u64& current, u64& best, u64& tie, int width, unsigned mask) {
    for (int o = width >> 1; o > 0; o >>= 1) {
        const u64 oc = __shfl_xor_sync(mask, current, o);
        const u64 ob = __shfl_xor_sync(mask, best, o);
        const u64 ot = __shfl_xor_sync(mask, tie, o);
        current = oc > current ? oc : current;
        if (better(ob, ot, best, tie)) { best = ob; tie = ot; }
    }
}

// deg <= G: one lane per edge, G lanes per vertex, equal clusters grouped by
// __match_any_sync (cf. sclp_affinity_low_match_kernel, :332-403).
template <int G, typename O, typename W>
__global__ void __launch_bounds__(kThreads) affinity_small_kernel(
    i64 count, const i32* __restrict__ list, const O* __restrict__ off, const i32* __restrict__ nbr,
    const W* __restrict__ ew, const W* __restrict__ vw, const i32* __restrict__ clusters,
    const u64* __restrict__ cw, RoundParams p, SclpOut out) {
    const int lane = threadIdx.x & 31;
    const int lig = lane & (G - 1);
    const unsigned mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
    const i64 gid = (static_cast<i64>(blockIdx.x) * kThreads + threadIdx.x) / G;
    const bool has_vertex = gid < count;
    const i32 v = has_vertex ? list[gid] : -1;
    const i32 source = has_vertex ? (p.identity ? v : clusters[v]) : -1;
    bool valid = false;
    i32 c = -1;
    u64 w = 0;
    if (has_vertex && !role_blocked(source, p)) {
        const i64 begin = off[v];
        const i64 deg = static_cast<i64>(off[v + 1]) - begin;
        if (lig < deg) {
            const i64 e = begin + lig;
            const i32 u = nbr[e];
            if (u != v) {
                valid = true;
                c = p.identity ? u : clusters[u];
                w = static_cast<u64>(weight_at(ew, e));
            }
        }
    }
    const unsigned peers = __match_any_sync(mask, valid ? c : -1);
    u64 conn = 0;
    if (p.sum32) {
        conn = __reduce_add_sync(peers, static_cast<u32>(w));
    } else {
        const int base = lane & ~(G - 1);
#pragma unroll
        for (int s = 0; s < G; ++s) {
            const u64 pw = __shfl_sync(mask, w, base + s);
            if (peers & (1u << (base + s))) conn += pw;
        }
    }
    const bool leader = valid && lane == __ffs(peers) - 1;
    u64 current = 0, best = 0, tie = 0;
    if (leader) {
        if (c == source) {
            current = conn;
        } else if (!p.filter || !is_mover(c, p)) {
            best = conn;
            tie = tie_key(static_cast<u32>(v), c, p.tie_salt);
        }
    }
    group_reduce(current, best, tie, G, mask);
    if (has_vertex && lig == 0) decode_and_write(v, source, current, best, tie, p, vw, cw, out);
}

// Shared/global open-addressing table insert (linear probing, key = cluster).
__device__ __forceinline__ void table_insert(i32* keys, u64* vals, u32 mask, i32 c, u64 w, u32* err) {
    u32 slot = mix32(static_cast<u32>(c)) & mask;
    for (u32 probe = 0; probe <= mask; ++probe) {
        const i32 found = atomicCAS(&keys[slot], -1, c);
        if (found == -1 || found == c) {
            atomic_add_u64(&vals[slot], w);
            return;
        }
        slot = (slot + 1) & mask;
    }
    set_error(err, kErrTableFull);
}

// Packed 8-byte slots for levels whose total edge weight fits 32 bits (every
// connection sum does): cluster + 1 in the low half (0 = empty), the sum in
// the high half.  A cluster not yet in the table is claimed together with its
// first weight by one 64-bit CAS; one already present takes one 32-bit add.
// Most neighbours of a vertex lie in distinct clusters, so most inserts cost
// one shared atomic instead of table_insert's two, and a slot takes 8 bytes
// instead of 12.
__device__ __forceinline__ void packed_insert(unsigned long long* slots, u32 mask, i32 c, u64 w, u32* err) {
    const u32 key = static_cast<u32>(c) + 1;
    const unsigned long long fresh = (static_cast<unsigned long long>(static_cast<u32>(w)) << 32) | key;
    u32 slot = mix32(static_cast<u32>(c)) & mask;
    for (u32 probe = 0; probe <= mask; ++probe) {
        const unsigned long long found = atomicCAS(&slots[slot], 0ULL, fresh);
        if (found == 0ULL) return;
        if (static_cast<u32>(found) == key) {
            atomicAdd(reinterpret_cast<u32*>(&slots[slot]) + 1, static_cast<u32>(w));
            return;
        }
        slot = (slot + 1) & mask;
    }
    set_error(err, kErrTableFull);
}

// Candidate of one table slot.
__device__ __forceinline__ void slot_candidate(i32 key, u64 conn, u32 v, i32 source, const RoundParams& p,
                                               u64& current, u64& best, u64& tie) {
    if (key < 0) return;
    if (key == source) { current = conn; return; }
    // a sum below the running best (or zero) never wins, whatever its tie
    // key: skip the mover test and the tie hash for it
    if (conn < best || conn == 0) return;
    if (p.filter && is_mover(key, p)) return;
    const u64 t = tie_key(v, key, p.tie_salt);
    if (better(conn, t, best, tie)) { best = conn; tie = t; }
}

// Warp per vertex, shared hash of kMediumSlots per warp (cf.
// sclp_affinity_medium_hash_kernel, :405-476).
// PACKED: 8-byte slots (packed_insert), for levels with p.sum32.
template <bool PACKED, typename O, typename W>
__global__ void __launch_bounds__(kThreads) affinity_warp_hash_kernel(
    i64 count, const i32* __restrict__ list, const O* __restrict__ off, const i32* __restrict__ nbr,
    const W* __restrict__ ew, const W* __restrict__ vw, const i32* __restrict__ clusters,
    const u64* __restrict__ cw, RoundParams p, SclpOut out, u32* err) {
    constexpr int kSlotBytes = PACKED ? 8 : 12;
    __shared__ __align__(16) unsigned char table_all[kWarps][kMediumSlots * kSlotBytes];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 gid = static_cast<i64>(blockIdx.x) * kWarps + warp;
    if (gid >= count) return;
    const i32 v = list[gid];
    const i32 source = p.identity ? v : clusters[v];
    if (role_blocked(source, p)) {
        if (lane == 0) out.target[v] = kInvalid;
        return;
    }
    auto* slots = reinterpret_cast<unsigned long long*>(table_all[warp]);   // PACKED
    u64* vals = reinterpret_cast<u64*>(table_all[warp]);                     // !PACKED
    i32* keys = reinterpret_cast<i32*>(vals + kMediumSlots);
    for (int s = lane; s < kMediumSlots; s += 32) {
        if constexpr (PACKED) { slots[s] = 0ULL; } else { keys[s] = -1; vals[s] = 0; }
    }
    __syncwarp();
    const i64 begin = off[v], end = off[v + 1];
    for (i64 e = begin + lane; e < end; e += 32) {
        const i32 u = nbr[e];
        if (u == v) continue;
        const i32 c = p.identity ? u : clusters[u];
        const u64 w = static_cast<u64>(weight_at(ew, e));
        if constexpr (PACKED) packed_insert(slots, kMediumSlots - 1, c, w, err);
        else table_insert(keys, vals, kMediumSlots - 1, c, w, err);
    }
    __syncwarp();
    u64 current = 0, best = 0, tie = 0;
    for (int s = lane; s < kMediumSlots; s += 32) {
        if constexpr (PACKED) {
            const unsigned long long x = slots[s];
            const u32 key = static_cast<u32>(x);
            if (key) slot_candidate(static_cast<i32>(key - 1), x >> 32, static_cast<u32>(v), source, p, current, best, tie);
        } else {
            slot_candidate(keys[s], vals[s], static_cast<u32>(v), source, p, current, best, tie);
        }
    }
    group_reduce(current, best, tie, 32, 0xffffffffu);
    if (lane == 0) decode_and_write(v, source, current, best, tie, p, vw, cw, out);
}

// Block-wide reduction of (current, best, tie); result valid in thread 0.
struct CandShared { u64 c[kWarps], b[kWarps], t[kWarps]; };
__device__ __forceinline__ void block_candidate_reduce(u64& current, u64& best, u64& tie, CandShared& sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    group_reduce(current, best, tie, 32, 0xffffffffu);
    if (lane == 0) { sh.c[warp] = current; sh.b[warp] = best; sh.t[warp] = tie; }
    __syncthreads();
    if (warp == 0) {
        current = lane < kWarps ? sh.c[lane] : 0;
        best = lane < kWarps ? sh.b[lane] : 0;
        tie = lane < kWarps ? sh.t[lane] : 0;
        group_reduce(current, best, tie, 32, 0xffffffffu);
    }
}

// Block per vertex with a kLargeSlots shared hash (PACKED: 8-byte slots,
// for levels with p.sum32; dynamic shared memory kLargeSlots * 8, else * 12).
template <bool PACKED, typename O, typename W>
__global__ void __launch_bounds__(kThreads) affinity_block_hash_kernel(
    i64 count, const i32* __restrict__ list, const O* __restrict__ off, const i32* __restrict__ nbr,
    const W* __restrict__ ew, const W* __restrict__ vw, const i32* __restrict__ clusters,
    const u64* __restrict__ cw, RoundParams p, SclpOut out, u32* err) {
    extern __shared__ unsigned char smem_raw[];
    auto* slots = reinterpret_cast<unsigned long long*>(smem_raw);   // PACKED
    u64* vals = reinterpret_cast<u64*>(smem_raw);                     // !PACKED
    i32* keys = reinterpret_cast<i32*>(vals + kLargeSlots);
    __shared__ CandShared red;
    const i64 gid = blockIdx.x;
    if (gid >= count) return;
    const i32 v = list[gid];
    const i32 source = p.identity ? v : clusters[v];
    if (role_blocked(source, p)) {
        if (threadIdx.x == 0) out.target[v] = kInvalid;
        return;
    }
    const i64 begin = off[v], end = off[v + 1];
    int nslots = 512;   // power of two >= 2 * degree (degree <= kHubDegree)
    while (nslots < 2 * (end - begin) && nslots < kLargeSlots) nslots <<= 1;
    for (int s = threadIdx.x; s < nslots; s += kThreads) {
        if constexpr (PACKED) { slots[s] = 0ULL; } else { keys[s] = -1; vals[s] = 0; }
    }
    __syncthreads();
    for (i64 e = begin + threadIdx.x; e < end; e += kThreads) {
        const i32 u = nbr[e];
        if (u == v) continue;
        const i32 c = p.identity ? u : clusters[u];
        const u64 w = static_cast<u64>(weight_at(ew, e));
        if constexpr (PACKED) packed_insert(slots, static_cast<u32>(nslots - 1), c, w, err);
        else table_insert(keys, vals, static_cast<u32>(nslots - 1), c, w, err);
    }
    __syncthreads();
    u64 current = 0, best = 0, tie = 0;
    for (int s = threadIdx.x; s < nslots; s += kThreads) {
        if constexpr (PACKED) {
            const unsigned long long x = slots[s];
            const u32 key = static_cast<u32>(x);
            if (key) slot_candidate(static_cast<i32>(key - 1), x >> 32, static_cast<u32>(v), source, p, current, best, tie);
        } else {
            slot_candidate(keys[s], vals[s], static_cast<u32>(v), source, p, current, best, tie);
        }
    }
    block_candidate_reduce(current, best, tie, red);
    if (threadIdx.x == 0) decode_and_write(v, source, current, best, tie, p, vw, cw, out);
}

// ---------------------------------------------------------------------------
// Per-level set-up: degree classes (lists in ascending vertex order).
// class 0: deg 0 (isolated); 1: 1..8; 2: 9..32; 3: 33..256; 4: 257..2048; 5: hubs
// ---------------------------------------------------------------------------
constexpr int kClasses = 6;

// counts[c] (u32) and edges[c] (u64, sum of degrees) per class.
template <typename O>
__global__ void degree_class_kernel(i64 n, const O* off, u64* keys, i32* vals, u32* counts, u64* edges) {
    __shared__ u32 local[kClasses];
    __shared__ unsigned long long local_edges[kClasses];
    if (threadIdx.x < kClasses) { local[threadIdx.x] = 0; local_edges[threadIdx.x] = 0; }
    __syncthreads();
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n) {
        const i64 d = static_cast<i64>(off[v + 1]) - off[v];
        const int c = d == 0 ? 0 : d <= 8 ? 1 : d <= 32 ? 2 : d <= 256 ? 3 : d <= kHubDegree ? 4 : 5;
        keys[v] = static_cast<u64>(c);
        vals[v] = static_cast<i32>(v);
        atomicAdd(&local[c], 1u);
        atomicAdd(&local_edges[c], static_cast<unsigned long long>(d));
    }
    __syncthreads();
    if (threadIdx.x < kClasses && local[threadIdx.x]) {
        atomicAdd(&counts[threadIdx.x], local[threadIdx.x]);
        atomic_add_u64(&edges[threadIdx.x], local_edges[threadIdx.x]);
    }
}



// Level statistics: total / maximum vertex weight and degree-class counts.
template <typename W>
__global__ void weight_stats_kernel(i64 n, const W* vw, u64* out /* [0]=sum [1]=max */) {
    __shared__ u64 sh[kWarps + 1];
    u64 s = 0, m = 0;
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x) {
        const u64 w = static_cast<u64>(weight_at(vw, v));
        s += w;
        m = w > m ? w : m;
    }
    s = block_sum(s, sh);
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0 && m) atomic_max_u64(&out[1], m);
    if (threadIdx.x == 0 && s) atomic_add_u64(&out[0], s);
}

// ---------------------------------------------------------------------------
// Admission (src/coarsen.cu:1086-1121,1334-1370,652-680)
// cls: 0 = no move, 1 = accept, 2 = contested (target over-subscribed)
// ---------------------------------------------------------------------------
__global__ void admission_classify_kernel(i64 n, const i32* target, const u64* demand, const u64* cw, u64 cap,
                                          const u64* gain, unsigned char* cls, u64* gmax) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const i32 t = target[v];
    unsigned char c = 0;
    if (t != kInvalid) {
        const u64 base = cw[t];
        if (base <= cap) {
            if (demand[t] <= cap - base) {
                c = 1;
            } else {
                c = 2;
                atomic_max_u64(gmax, gain[v]);
            }
        }
    }
    cls[v] = c;
}

// Two-hop candidates: every valid favourite is "contested" (needs order).
__global__ void favorite_classify_kernel(i64 n, const i32* target, const u64* gain, unsigned char* cls, u64* gmax) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const bool ok = target[v] != kInvalid;
    cls[v] = ok ? 2 : 0;
    if (ok) atomic_max_u64(gmax, gain[v]);
}

struct IsClass2 {
    const unsigned char* cls;
    __device__ i64 operator()(i64 i) const { return cls[i] == 2 ? 1 : 0; }
};

__global__ void compact_class2_kernel(i64 n, const unsigned char* cls, const i64* pos, i32* list) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n && cls[v] == 2) list[pos[v]] = static_cast<i32>(v);
}

// Sort keys for the order (target asc, gain desc, tie desc); vertex order is
// kept by stability (the list is in ascending vertex order).
// mode 0: full key  t << (gbits+32) | (gmax-gain) << 32 | ~tie
// mode 1: ~tie only;  mode 2: t << gbits | (gmax - gain);  mode 3: gmax-gain;  mode 4: t
__global__ void admission_keys_kernel(i64 count, const i32* list, const i32* target, const u64* gain, const u32* tie,
                                      u64 gmax, int gbits, int mode, u64* keys) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const i32 v = list[i];
    const u64 t = static_cast<u64>(static_cast<u32>(target[v]));
    const u64 rg = gmax - gain[v];
    const u64 rt = static_cast<u64>(~tie[v]);
    u64 k = 0;
    switch (mode) {
        case 0: k = (t << (gbits + 32)) | (rg << 32) | rt; break;
        case 1: k = rt; break;
        case 2: k = (t << gbits) | rg; break;
        case 3: k = rg; break;
        default: k = t; break;
    }
    keys[i] = k;
}

template <typename W>
struct SortedWeight {
    const i32* list;
    const W* vw;
    __device__ u64 operator()(i64 i) const { return static_cast<u64>(weight_at(vw, list[i])); }
};

// segment base of each target: the exclusive weight prefix at its first entry
__global__ void segment_heads_kernel(i64 count, const i32* list, const i32* target, const u64* excl, u64* segbase,
                                     int store_index) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const i32 t = target[list[i]];
    if (i == 0 || target[list[i - 1]] != t) segbase[t] = store_index ? static_cast<u64>(i) : excl[i];
}

template <typename W>
__global__ void contested_accept_kernel(i64 count, const i32* list, const i32* target, const u64* excl,
                                        const u64* segbase, const u64* cw, const W* vw, u64 cap, unsigned char* cls) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const i32 v = list[i];
    const i32 t = target[v];
    const u64 w = static_cast<u64>(weight_at(vw, v));
    const u64 prefix = excl[i] + w - segbase[t];
    const u64 base = cw[t];
    cls[v] = (base <= cap && prefix <= cap - base) ? 1 : 0;
}

template <typename W>
__global__ void sclp_commit_kernel(i64 n, const unsigned char* cls, const i32* target, const W* vw, i32* clusters,
                                   u64* cw) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n || cls[v] != 1) return;
    const i32 t = target[v];
    const i32 s = clusters[v];
    const u64 w = static_cast<u64>(weight_at(vw, v));
    atomic_add_u64(&cw[s], 0ULL - w);
    atomic_add_u64(&cw[t], w);
    clusters[v] = t;
}

__global__ void count_nonzero_kernel(i64 n, const u64* cw, u64* out) {
    __shared__ u64 sh[kWarps + 1];
    u64 c = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<i64>(gridDim.x) * blockDim.x)
        c += cw[i] != 0 ? 1 : 0;
    c = block_sum(c, sh);
    if (threadIdx.x == 0 && c) atomic_add_u64(out, c);
}

// ---------------------------------------------------------------------------
// Two-hop pairing (src/coarsen.cu:694-724,1461-1516)
// ---------------------------------------------------------------------------
template <typename W>
__global__ void pair_flags_kernel(i64 count, const i32* list, const i32* target, const u64* segstart, const W* vw,
                                  u64 cap, i64* flags) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const i32 v = list[i];
    const u64 rank = static_cast<u64>(i) - segstart[target[v]] + 1;
    const bool second = (rank & 1ULL) == 0ULL;
    i64 f = 0;
    if (second && i > 0) {
        const u64 prev = static_cast<u64>(weight_at(vw, list[i - 1]));
        f = prev <= cap - static_cast<u64>(weight_at(vw, v)) ? 1 : 0;
    }
    flags[i] = f;
}

template <typename W>
__global__ void pair_commit_kernel(i64 count, const i32* list, const i64* flags, const i64* positions, u64 budget,
                                   const W* vw, i32* clusters, u64* cw) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count || !flags[i] || static_cast<u64>(positions[i]) >= budget) return;
    const i32 v = list[i];
    const i32 s = clusters[v];
    const i32 t = clusters[list[i - 1]];
    if (s == t) return;
    const u64 w = static_cast<u64>(weight_at(vw, v));
    atomic_add_u64(&cw[s], 0ULL - w);
    atomic_add_u64(&cw[t], w);
    clusters[v] = t;
}

// ---------------------------------------------------------------------------
// Isolated packing (src/coarsen.cu:741-773,1410-1441)
// ---------------------------------------------------------------------------
__global__ void fill_i32_kernel(i64 n, i32* a, i32 value) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) a[i] = value;
}

template <typename W>
__global__ void isolated_rep_kernel(i64 count, const i32* iso, const u64* excl, const W* vw, u64 cap, i32* reps) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const i32 v = iso[i];
    const u64 incl = excl[i] + static_cast<u64>(weight_at(vw, v));
    const u64 first = (incl - static_cast<u64>(weight_at(vw, v))) / cap, last = (incl - 1) / cap;
    if (first == last) atomicMin(&reps[first], v);
}

template <typename W>
__global__ void isolated_commit_kernel(i64 count, const i32* iso, const u64* excl, const W* vw, u64 cap,
                                       const i32* reps, i32* clusters, u64* cw) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const i32 v = iso[i];
    const u64 w = static_cast<u64>(weight_at(vw, v));
    const u64 incl = excl[i] + w;
    const u64 first = (incl - w) / cap, last = (incl - 1) / cap;
    if (first != last) return;
    const i32 t = reps[first];
    if (t == v) return;
    clusters[v] = t;
    cw[v] = 0;
    atomic_add_u64(&cw[t], w);
}

// ---------------------------------------------------------------------------
// Compaction (src/coarsen.cu:726-731,775-780,151-158,1541-1577)
// ---------------------------------------------------------------------------
struct NonEmpty {
    const u64* cw;
    __device__ i32 operator()(i64 i) const { return cw[i] > 0 ? 1 : 0; }
};

template <typename W>
__global__ void compact_map_kernel(i64 n, const i32* clusters, const i32* compact, const W* vw, i32* map, W* cvw) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const i32 c = compact[clusters[v]];
    map[v] = c;
    atomic_add_w(&cvw[c], weight_at(vw, v));
}

template <typename W>
__global__ void coarse_weights_kernel(i64 n, const i32* map, const W* vw, W* cvw) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n) atomic_add_w(&cvw[map[v]], weight_at(vw, v));
}

template <typename W>
__global__ void cap_check_kernel(i64 n, const W* cvw, u64 cap, u32* err) {
    const i64 c = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c < n && static_cast<u64>(cvw[c]) > cap) set_error(err, kErrCapacity);
}

}  // namespace gp
