// Hub splitting.  Power-law graphs (RMAT) have vertices with 10^4-10^6
// neighbours; one warp or block per such vertex serialises a whole kernel
// behind the largest hub.  Every level therefore keeps a hub index: the
// vertices of degree > kHubThreshold, each cut into chunks of kChunkEdges
// edges.  Kernels that walk rows skip hubs in their per-vertex loops and
// handle hub chunks in a separate launch (one block per chunk), combining the
// per-hub partial results with atomics or a per-hub finalisation.
#pragma once

#include "gp_prim.cuh"
#include "gp_sclp.cuh"
#include "gp_refine.cuh"

namespace gp {

constexpr i64 kHubThreshold = 2048;   // the SCLP global-hash class boundary
constexpr i64 kChunkEdges = 2048;

struct Chunk {
    i32 v;       // vertex
    i32 hub;     // index in the hub list
    i64 begin;   // edge range
    i64 end;
};

template <typename O>
__device__ __forceinline__ bool is_hub(const O* off, i64 v) {
    return static_cast<i64>(off[v + 1]) - static_cast<i64>(off[v]) > kHubThreshold;
}

template <typename O>
struct HubFlag {
    const O* off;
    __device__ i64 operator()(i64 v) const { return is_hub(off, v) ? 1 : 0; }
};

template <typename O>
struct HubChunkCount {
    const O* off;
    __device__ i64 operator()(i64 v) const {
        const i64 d = static_cast<i64>(off[v + 1]) - static_cast<i64>(off[v]);
        return d > kHubThreshold ? (d + kChunkEdges - 1) / kChunkEdges : 0;
    }
};

template <typename O>
__global__ void hub_fill_kernel(i64 n, const O* off, const i64* hub_pos, const i64* chunk_pos, i32* hubs,
                                Chunk* chunks, i64* chunk_begin) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n || !is_hub(off, v)) return;
    const i64 h = hub_pos[v];
    hubs[h] = static_cast<i32>(v);
    chunk_begin[h] = chunk_pos[v];
    const i64 b = off[v], e = off[v + 1];
    i64 c = chunk_pos[v];
    for (i64 s = b; s < e; s += kChunkEdges, ++c)
        chunks[c] = {static_cast<i32>(v), static_cast<i32>(h), s, s + kChunkEdges < e ? s + kChunkEdges : e};
}

// ---------------------------------------------------------------------------
// SCLP affinity of hubs: chunked insertion into per-hub global tables with
// warp-level pre-aggregation (__match_any_sync on the cluster id), then a
// candidate pass over kSlotTile-slot tiles (table sizes are multiples of the
// tile, so tiles never straddle two tables), then a per-hub finalisation that
// merges the tiles and decodes the proposal.
// ---------------------------------------------------------------------------
// A slot holds key and value in one sector; key 0 is empty (cluster c is
// stored as c + 1), so a table is cleared by a memset.  Levels whose total
// edge weight fits in 32 bits use 8-byte slots (no per-cluster sum can
// overflow), others 16-byte slots; tables are about 1.3x the hub's degree,
// so the 8-byte form keeps the level-0 tables of large power-law graphs
// several times smaller and mostly resident in L2.
struct HubSlot {
    u32 key;
    u32 pad;
    u64 val;
    __device__ void add(u64 w) { atomic_add_u64(&val, w); }
    __device__ u64 value() const { return val; }
};

struct HubSlot32 {
    u32 key;
    u32 val;
    __device__ void add(u64 w) { atomicAdd(&val, static_cast<u32>(w)); }
    __device__ u64 value() const { return val; }
};

constexpr i64 kSlotTile = 1024;

// Table size of a hub: at least 1.3x its degree (load factor <= 0.77 even
// if every neighbour is in a different cluster), rounded up to whole tiles.
template <typename O>
struct HubTableSize {
    const i32* list;
    const O* off;
    i64 count;
    __device__ i64 operator()(i64 i) const {
        if (i >= count) return 0;
        const i32 v = list[i];
        const i64 d = static_cast<i64>(off[v + 1]) - off[v];
        const i64 want = d + (d * 3 + 9) / 10;
        return (want + kSlotTile - 1) / kSlotTile * kSlotTile;
    }
};

// Fixed-point range reduction of the hash onto [0, size) (size < 2^32).
__device__ __forceinline__ u32 slot_of(i32 c, u32 size) {
    return static_cast<u32>((static_cast<u64>(mix32(static_cast<u32>(c))) * size) >> 32);
}

template <typename S>
__device__ __forceinline__ void slot_insert(S* table, u32 size, i32 c, u64 w, u32* err) {
    const u32 key = static_cast<u32>(c) + 1;
    u32 slot = slot_of(c, size);
    for (u32 probe = 0; probe < size; ++probe) {
        const u32 found = atomicCAS(&table[slot].key, 0u, key);
        if (found == 0u || found == key) {
            table[slot].add(w);
            return;
        }
        if (++slot == size) slot = 0;
    }
    set_error(err, kErrTableFull);
}

// 8-byte slots: key and value are claimed together by one 64-bit CAS (an
// empty slot is the all-zero word), so a first insert is a single atomic; a
// slot that already holds the key takes a 32-bit add.
__device__ __forceinline__ void slot_insert(HubSlot32* table, u32 size, i32 c, u64 w, u32* err) {
    const u32 key = static_cast<u32>(c) + 1;
    const unsigned long long fresh = (static_cast<unsigned long long>(static_cast<u32>(w)) << 32) | key;
    u32 slot = slot_of(c, size);
    for (u32 probe = 0; probe < size; ++probe) {
        const unsigned long long found =
            atomicCAS(reinterpret_cast<unsigned long long*>(&table[slot]), 0ULL, fresh);
        if (found == 0ULL) return;
        if (static_cast<u32>(found) == key) {
            table[slot].add(w);
            return;
        }
        if (++slot == size) slot = 0;
    }
    set_error(err, kErrTableFull);
}

template <typename O, typename W, typename S>
__global__ void __launch_bounds__(kThreads) hub_insert_kernel(
    const Chunk* __restrict__ chunks, const i32* __restrict__ nbr, const W* __restrict__ ew,
    const i32* __restrict__ clusters, RoundParams p, const i64* __restrict__ table_off, S* table, u32* err) {
    const Chunk ch = chunks[blockIdx.x];
    if (role_blocked(p.identity ? ch.v : clusters[ch.v], p)) return;   // no proposal: nothing to count
    const int lane = threadIdx.x & 31;
    const i64 t0 = table_off[ch.hub];
    const u32 size = static_cast<u32>(table_off[ch.hub + 1] - t0);
    S* slots = table + t0;
    // The next edge's cluster is gathered before the current insert, so its
    // load latency overlaps the CAS round trip.
    auto gather = [&](i64 e, i32& c, u64& w) {
        c = -1;
        w = 0;
        if (e < ch.end) {
            const i32 u = nbr[e];
            if (u != ch.v) {
                c = p.identity ? u : clusters[u];
                w = static_cast<u64>(weight_at(ew, e));
            }
        }
    };
    i32 c_next;
    u64 w_next;
    gather(ch.begin + threadIdx.x, c_next, w_next);
    for (i64 base = ch.begin; base < ch.end; base += kThreads) {
        const i32 c = c_next;
        const u64 w = w_next;
        gather(base + kThreads + threadIdx.x, c_next, w_next);
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        u64 sum = 0;
        if (ew == nullptr) {
            sum = static_cast<u64>(__popc(peers));   // unit weights
        } else {
#pragma unroll
            for (int s = 0; s < 32; ++s) {
                const u64 pw = __shfl_sync(0xffffffffu, w, s);
                if (peers & (1u << s)) sum += pw;
            }
        }
        if (c >= 0 && lane == __ffs(peers) - 1) slot_insert(slots, size, c, sum, err);
    }
}

struct HubPartial { u64 current, best, tie; };

// ---------------------------------------------------------------------------
// SCLP affinity of hubs whose table fits in one CTA's shared memory (up to
// ~22K edges): one CTA per hub does the inserts, the candidate scan and the
// decode in one launch, so these tables never reach global memory and need
// neither a clearing memset nor a separate candidate pass.  8-byte slots
// (cluster + 1, 32-bit sum) claimed by one 64-bit CAS, as HubSlot32: used on
// levels whose total edge weight fits 32 bits.  Larger hubs keep the chunked
// global tables: one CTA walking 10^4-10^5 edges would be a long chain of
// dependent loads, where the chunks spread a hub over many CTAs.
// ---------------------------------------------------------------------------
// Three shapes: hubs whose table fits 42 KB (up to ~4.1K edges, most hubs of
// an RMAT level) run 512 threads with four CTAs per SM; up to 96 KB, 512
// threads with two CTAs per SM; up to the largest table one CTA can hold
// (~227 KB), 1024 threads with one CTA per SM.
constexpr int kHubSmallSlots = 5376;        // 42 KB
constexpr int kHubSmemSlots = 12288;        // 96 KB
constexpr int kHubSmemThreads = 512;
constexpr int kHubMidThreads = 1024;        // its table: what the device's per-CTA limit leaves (hub_mid_slots)

// Table slots for a hub of `degree` edges: at least 1.3x the degree (a hub
// has at most `degree` distinct neighbour clusters), whole 32-slot lines.
__host__ __device__ inline i64 hub_smem_slots(i64 degree) {
    const i64 want = degree + (degree * 3 + 9) / 10;
    return (want + 31) / 32 * 32;
}

template <int THREADS, typename O, typename W>
__global__ void __launch_bounds__(THREADS) hub_smem_kernel(
    const i32* __restrict__ hub_ids, const O* __restrict__ off, const i32* __restrict__ nbr,
    const W* __restrict__ ew, const W* __restrict__ vw, const i32* __restrict__ clusters,
    const u64* __restrict__ cw, RoundParams p, SclpOut out) {
    constexpr int kHubSmemWarps = THREADS / 32;
    constexpr int kHubSmemThreads = THREADS;
    extern __shared__ unsigned long long table[];   // hub_smem_slots(degree) entries
    __shared__ u64 red[3][kHubSmemWarps];
    const i32 v = hub_ids[blockIdx.x];
    const i32 source = clusters[v];
    if (role_blocked(source, p)) {
        if (threadIdx.x == 0) out.target[v] = kInvalid;
        return;
    }
    const i64 b = off[v], end = off[v + 1];
    const u32 size = static_cast<u32>(hub_smem_slots(end - b));
    for (u32 s = threadIdx.x; s < size; s += kHubSmemThreads) table[s] = 0ULL;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (i64 base = b; base < end; base += kHubSmemThreads) {
        const i64 e = base + threadIdx.x;
        i32 c = -1;
        u64 w = 0;
        if (e < end) {
            const i32 u = nbr[e];
            if (u != v) {
                c = clusters[u];
                w = static_cast<u64>(weight_at(ew, e));
            }
        }
        // Every lane inserts its own edge: the 32 neighbours of one step
        // rarely share a cluster, so a __match_any_sync pre-aggregation (and,
        // on weighted levels, its 32-shuffle group sum) cost more issue slots
        // than the shared-memory atomics it saved (measured: this kernel 20%
        // faster at RMAT-22 and RMAT-24 without it, identical hierarchies).
        if (c >= 0) {
            const u32 key = static_cast<u32>(c) + 1;
            const u64 sum = w;
            const unsigned long long fresh = (static_cast<unsigned long long>(static_cast<u32>(sum)) << 32) | key;
            u32 slot = slot_of(c, size);
            // at most size probes: the table has more slots than distinct keys
            for (u32 probe = 0; probe < size; ++probe) {
                const unsigned long long found = atomicCAS(&table[slot], 0ULL, fresh);
                if (found == 0ULL) break;
                if (static_cast<u32>(found) == key) {
                    atomicAdd(reinterpret_cast<u32*>(&table[slot]) + 1, static_cast<u32>(sum));
                    break;
                }
                if (++slot == size) slot = 0;
            }
        }
    }
    __syncthreads();
    u64 current = 0, best = 0, tie = 0;
    for (u32 s = threadIdx.x; s < size; s += kHubSmemThreads) {
        const unsigned long long x = table[s];
        const u32 key = static_cast<u32>(x);
        if (key) slot_candidate(static_cast<i32>(key - 1), x >> 32, static_cast<u32>(v), source, p, current, best, tie);
    }
    group_reduce(current, best, tie, 32, 0xffffffffu);
    const int warp = threadIdx.x >> 5;
    if (lane == 0) { red[0][warp] = current; red[1][warp] = best; red[2][warp] = tie; }
    __syncthreads();
    if (warp == 0) {
        current = lane < kHubSmemWarps ? red[0][lane] : 0;
        best = lane < kHubSmemWarps ? red[1][lane] : 0;
        tie = lane < kHubSmemWarps ? red[2][lane] : 0;
        group_reduce(current, best, tie, 32, 0xffffffffu);
        if (lane == 0) decode_and_write(v, source, current, best, tie, p, vw, cw, out);
    }
}

// Degree and first edge of every hub (for the host's split of the hubs into
// on-chip classes and global-table hubs, once per level).
template <typename O>
__global__ void hub_extent_kernel(i64 count, const i32* __restrict__ hubs, const O* __restrict__ off, i64* out) {
    const i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (h >= count) return;
    const i32 v = hubs[h];
    out[2 * h] = static_cast<i64>(off[v]);
    out[2 * h + 1] = static_cast<i64>(off[v + 1]) - static_cast<i64>(off[v]);
}

// Profiling only: the work an affinity pass over `list` really does, since
// vertices (and hubs) whose own cluster is not a mover are skipped.  out[0]
// counts the processed vertices, out[1] their edges, out[2] the slots of
// their hub tables (HubTableSize).
template <typename O>
__global__ void role_work_kernel(i64 count, const i32* __restrict__ list, const O* __restrict__ off,
                                 const i32* __restrict__ clusters, RoundParams p, u64* out) {
    u64 v_n = 0, e_n = 0, s_n = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i32 v = list[i];
        if (role_blocked(p.identity ? v : clusters[v], p)) continue;
        const i64 d = static_cast<i64>(off[v + 1]) - off[v];
        const i64 want = d + (d * 3 + 9) / 10;
        ++v_n;
        e_n += static_cast<u64>(d);
        s_n += static_cast<u64>((want + kSlotTile - 1) / kSlotTile * kSlotTile);
    }
    v_n = warp_sum(v_n); e_n = warp_sum(e_n); s_n = warp_sum(s_n);
    if ((threadIdx.x & 31) == 0 && v_n) {
        atomicAdd(reinterpret_cast<unsigned long long*>(out), static_cast<unsigned long long>(v_n));
        atomicAdd(reinterpret_cast<unsigned long long*>(out + 1), static_cast<unsigned long long>(e_n));
        atomicAdd(reinterpret_cast<unsigned long long*>(out + 2), static_cast<unsigned long long>(s_n));
    }
}

template <typename W, typename S>
__global__ void __launch_bounds__(kThreads) hub_candidates_kernel(
    i64 hubs, const i32* __restrict__ hub_list, const i64* __restrict__ table_off, S* table,
    const i32* __restrict__ clusters, RoundParams p, HubPartial* partials, i64 tile_base) {
    __shared__ CandShared red;
    __shared__ int hub_sh;
    const i64 tile = tile_base + blockIdx.x;  // tile_base offsets a launch over a sub-range of tables
    const i64 s0 = tile * kSlotTile;
    if (threadIdx.x == 0) {
        i64 lo = 0, hi = hubs - 1;   // last hub with table_off <= s0
        while (lo < hi) {
            const i64 mid = (lo + hi + 1) >> 1;
            if (table_off[mid] <= s0) lo = mid; else hi = mid - 1;
        }
        hub_sh = static_cast<int>(lo);
    }
    __syncthreads();
    const int h = hub_sh;
    const i32 v = hub_list[h];
    const i32 source = p.identity ? v : clusters[v];
    if (role_blocked(source, p)) return;   // empty table, no proposal
    u64 current = 0, best = 0, tie = 0;
    for (i64 s = s0 + threadIdx.x; s < s0 + kSlotTile; s += kThreads) {
        const S slot = table[s];
        if (slot.key) {
            slot_candidate(static_cast<i32>(slot.key - 1), slot.value(), static_cast<u32>(v), source, p, current, best,
                           tie);
            table[s] = S{};
        }
    }
    block_candidate_reduce(current, best, tie, red);
    if (threadIdx.x == 0) partials[tile] = {current, best, tie};
}

template <typename W>
__global__ void hub_finalize_kernel(i64 hubs, const i32* __restrict__ hub_list, const i64* __restrict__ table_off,
                                    const HubPartial* __restrict__ partials, const i32* __restrict__ clusters,
                                    const W* __restrict__ vw, const u64* __restrict__ cw, RoundParams p, SclpOut out) {
    const i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (h >= hubs) return;
    const i32 v = hub_list[h];
    const i32 source = p.identity ? v : clusters[v];
    u64 current = 0, best = 0, tie = 0;
    for (i64 t = table_off[h] / kSlotTile; t < table_off[h + 1] / kSlotTile; ++t) {
        const HubPartial q = partials[t];
        current = q.current > current ? q.current : current;
        if (better(q.best, q.tie, best, tie)) { best = q.best; tie = q.tie; }
    }
    decode_and_write(v, source, current, best, tie, p, vw, cw, out);
}

// ---------------------------------------------------------------------------
// Refinement and cut over hub chunks
// ---------------------------------------------------------------------------
template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) hub_cut_kernel(const Chunk* __restrict__ chunks,
                                                           const i32* __restrict__ nbr, const W* __restrict__ ew,
                                                           const i32* __restrict__ labels, u64* out) {
    __shared__ u64 sh[kWarps + 1];
    const Chunk ch = chunks[blockIdx.x];
    const i32 s = labels[ch.v];
    u64 local = 0;
    // four edges per thread and step: their neighbour ids, then their labels
    for (i64 e0 = ch.begin + threadIdx.x; e0 < ch.end; e0 += 4 * kThreads) {
        i32 u[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const i64 e = e0 + j * kThreads;
            u[j] = e < ch.end ? nbr[e] : -1;
        }
        i32 lu[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) lu[j] = u[j] >= 0 ? labels[u[j]] : s;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (lu[j] != s) local += static_cast<u64>(weight_at(ew, e0 + j * kThreads));
    }
    local = block_sum(local, sh);
    if (threadIdx.x == 0 && local) atomic_add_u64(out, local);
}

template <typename C>
__global__ void zero_hub_rows_kernel(i64 hubs, const i32* hub_list, int k, C* cache) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < hubs * k) cache[static_cast<i64>(hub_list[i / k]) * k + i % k] = 0;
}

template <typename W, typename C>
__global__ void __launch_bounds__(kThreads) hub_build_cache_kernel(const Chunk* __restrict__ chunks,
                                                                   const i32* __restrict__ nbr,
                                                                   const W* __restrict__ ew,
                                                                   const i32* __restrict__ labels, int k, C* cache) {
    __shared__ u64 rows[kWarps][32];
    u32 (*rows32)[32] = reinterpret_cast<u32 (*)[32]>(&rows[0][0]);   // C = u32: 32-bit accumulators
    const Chunk ch = chunks[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if constexpr (sizeof(C) == 4) rows32[warp][lane] = 0;
    else rows[warp][lane] = 0;
    __syncwarp();
    // each warp walks its own contiguous slice of the chunk
    const i64 len = ch.end - ch.begin;
    const i64 per = (len + kWarps - 1) / kWarps;
    const i64 lo = ch.begin + warp * per, hi = lo + per < ch.end ? lo + per : ch.end;
    // four 32-edge steps at a time: their neighbour ids, then their labels,
    // then the warp's match and row updates
    for (i64 base = lo; base < hi; base += 4 * 32) {
        i32 u[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const i64 e = base + j * 32 + lane;
            u[j] = e < hi ? nbr[e] : ch.v;
        }
        int p[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) p[j] = u[j] != ch.v ? labels[u[j]] : -1;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const u64 w = p[j] >= 0 ? static_cast<u64>(weight_at(ew, base + j * 32 + lane)) : 0;
            if constexpr (sizeof(C) == 4) {   // as build_cache_kernel: 32-bit shared atomics
                if (p[j] >= 0) atomicAdd(&rows32[warp][p[j]], static_cast<u32>(w));
            } else {
                const unsigned peers = __match_any_sync(0xffffffffu, p[j]);
                const u64 sum = group_sum<C>(peers, w);
                if (p[j] >= 0 && lane == __ffs(peers) - 1) rows[warp][p[j]] += sum;
            }
            __syncwarp();
        }
    }
    __syncthreads();
    if (threadIdx.x < k) {
        u64 t = 0;
        for (int w2 = 0; w2 < kWarps; ++w2) t += sizeof(C) == 4 ? rows32[w2][threadIdx.x] : rows[w2][threadIdx.x];
        if (t) cache_add(&cache[static_cast<i64>(ch.v) * k + threadIdx.x], t);
    }
}

// Partial priority corrections of hub proposers (incremental_priority_filter,
// src/refine_incremental.cuh:48-67), summed per hub.
template <typename W>
__global__ void __launch_bounds__(kThreads) hub_filter_kernel(const Chunk* __restrict__ chunks,
                                                              const i32* __restrict__ nbr, const W* __restrict__ ew,
                                                              const PropRec* __restrict__ props, long long* corr) {
    __shared__ long long sh[kWarps + 1];
    const Chunk ch = chunks[blockIdx.x];
    const i32 v = ch.v;
    const PropRec me = props[v];
    const i32 t = me.target;
    if (t < 0) return;
    const i32 s = me.label;
    const i64 g = me.gain;
    long long local = 0;
    for (i64 e = ch.begin + threadIdx.x; e < ch.end; e += kThreads) {
        const i32 u = nbr[e];
        if (u == v) continue;
        const PropRec o = props[u];
        if (o.target < 0) continue;
        if (!(o.gain > g || (o.gain == g && u < v))) continue;
        local += static_cast<long long>(weight_at(ew, e)) *
                 ((o.target == t) - (o.target == s) - (o.label == t) + (o.label == s));
    }
    local = block_sum(local, sh);
    if (threadIdx.x == 0 && local) atomicAdd(reinterpret_cast<unsigned long long*>(&corr[ch.hub]),
                                             static_cast<unsigned long long>(local));
}

template <typename O>
__global__ void hub_filter_finalize_kernel(i64 hubs, const i32* __restrict__ hub_list, const O* __restrict__ off,
                                           const i32* __restrict__ targets, const i64* __restrict__ gains,
                                           long long* corr, unsigned char* flags, i32* movers, RefineCounters* ctr) {
    const i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (h >= hubs) return;
    const i32 v = hub_list[h];
    const long long c = corr[h];
    corr[h] = 0;
    if (targets[v] < 0 || gains[v] + c < 0) return;
    flags[v] = 1;
    const unsigned long long slot = atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->movers), 1ULL);
    movers[slot] = v;
    atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->mover_degree),
              static_cast<unsigned long long>(static_cast<i64>(off[v + 1]) - static_cast<i64>(off[v])));
}

// Cache and cut update of the hub rows among the movers.  Most applies (the
// rebalance iterations) move no hub, so a launch of one block per chunk would
// mostly schedule blocks that exit at once.  Instead a grid of at most a few
// blocks per SM strides over the chunks: each block first tests the mover flag
// of up to 256 of its chunks in parallel, then walks the flagged chunks one
// after another with all its threads.
template <typename W, typename C>
__global__ void __launch_bounds__(kThreads) hub_apply_kernel(i64 nchunks, const Chunk* __restrict__ chunks,
                                                             const i32* __restrict__ nbr, const W* __restrict__ ew,
                                                             const i32* __restrict__ labels,
                                                             const i32* __restrict__ targets,
                                                             const unsigned char* __restrict__ flags, int k,
                                                             C* cache, RefineCounters* ctr) {
    __shared__ long long sh[kWarps + 1];
    __shared__ int todo[kThreads];
    __shared__ int ntodo;
    const i64 stride = gridDim.x;
    long long gain = 0;
    for (i64 base = blockIdx.x; base < nchunks; base += stride * kThreads) {
        if (threadIdx.x == 0) ntodo = 0;
        __syncthreads();
        const i64 mine = base + static_cast<i64>(threadIdx.x) * stride;
        if (mine < nchunks && flags[chunks[mine].v]) todo[atomicAdd(&ntodo, 1)] = static_cast<int>(threadIdx.x);
        __syncthreads();
        const int count = ntodo;
        if (threadIdx.x == 0 && count)
            atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->hub_chunks), static_cast<unsigned long long>(count));
        for (int j = 0; j < count; ++j) {
            const Chunk ch = chunks[base + static_cast<i64>(todo[j]) * stride];
            if (threadIdx.x == 0)
                atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->hub_edges),
                          static_cast<unsigned long long>(ch.end - ch.begin));
            const i32 v = ch.v;
            gain += apply_edges_batched(v, labels[v], targets[v], ch.begin, ch.end, static_cast<int>(threadIdx.x),
                                        kThreads, nbr, ew, labels, targets, flags, k, cache);
        }
        __syncthreads();
    }
    gain = block_sum(gain, sh);
    if (threadIdx.x == 0 && gain) atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->delta),
                                            static_cast<unsigned long long>(gain));
}

// ---------------------------------------------------------------------------
// Contraction scatter of hub rows: the row's segment base was reserved by the
// warp pass (hub_dst[hub]).
// ---------------------------------------------------------------------------
template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) hub_scatter_kernel(const Chunk* __restrict__ chunks,
                                                               const O* __restrict__ off,
                                                               const i32* __restrict__ nbr,
                                                               const W* __restrict__ ew, const i32* __restrict__ map,
                                                               const i64* __restrict__ hub_dst, u32 sentinel,
                                                               u32* __restrict__ tgt, W* __restrict__ wt) {
    const Chunk ch = chunks[blockIdx.x];
    const i32 c = map[ch.v];
    const i64 base = hub_dst[ch.hub] - static_cast<i64>(off[ch.v]);
    for (i64 e = ch.begin + threadIdx.x; e < ch.end; e += kThreads) {
        const i32 t = map[nbr[e]];
        tgt[base + e] = t == c ? sentinel : static_cast<u32>(t);
        wt[base + e] = weight_at(ew, e);
    }
}

}  // namespace gp

namespace gp {

// ---------------------------------------------------------------------------
// Identity rounds on duplicate-free rows: every neighbour is its own cluster,
// so a vertex's connection to cluster u is the weight of its single edge to u
// (the reference's singleton fast path, src/coarsen.cu:306-330,1158-1170).
// No table is needed; the best candidate is a max over edges.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void direct_candidate(i32 v, i32 u, u64 w, const RoundParams& p, u64& best, u64& tie) {
    if (u == v) return;
    if (p.filter && is_mover(u, p)) return;
    const u64 t = tie_key(static_cast<u32>(v), u, p.tie_salt);
    if (better(w, t, best, tie)) { best = w; tie = t; }
}

template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) affinity_direct_warp_kernel(
    i64 count, const i32* __restrict__ list, const O* __restrict__ off, const i32* __restrict__ nbr,
    const W* __restrict__ ew, const W* __restrict__ vw, const u64* __restrict__ cw, RoundParams p, SclpOut out) {
    const int lane = threadIdx.x & 31;
    const i64 gid = (static_cast<i64>(blockIdx.x) * kThreads + threadIdx.x) >> 5;
    if (gid >= count) return;
    const i32 v = list[gid];
    if (role_blocked(v, p)) {
        if (lane == 0) out.target[v] = kInvalid;
        return;
    }
    u64 current = 0, best = 0, tie = 0;
    for (i64 e = static_cast<i64>(off[v]) + lane; e < static_cast<i64>(off[v + 1]); e += 32)
        direct_candidate(v, nbr[e], static_cast<u64>(weight_at(ew, e)), p, best, tie);
    group_reduce(current, best, tie, 32, 0xffffffffu);
    if (lane == 0) decode_and_write(v, v, current, best, tie, p, vw, cw, out);
}

template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) affinity_direct_block_kernel(
    i64 count, const i32* __restrict__ list, const O* __restrict__ off, const i32* __restrict__ nbr,
    const W* __restrict__ ew, const W* __restrict__ vw, const u64* __restrict__ cw, RoundParams p, SclpOut out) {
    __shared__ CandShared red;
    const i32 v = list[blockIdx.x];
    if (role_blocked(v, p)) {
        if (threadIdx.x == 0) out.target[v] = kInvalid;
        return;
    }
    u64 current = 0, best = 0, tie = 0;
    for (i64 e = static_cast<i64>(off[v]) + threadIdx.x; e < static_cast<i64>(off[v + 1]); e += kThreads)
        direct_candidate(v, nbr[e], static_cast<u64>(weight_at(ew, e)), p, best, tie);
    block_candidate_reduce(current, best, tie, red);
    if (threadIdx.x == 0) decode_and_write(v, v, current, best, tie, p, vw, cw, out);
}

// Hubs: one partial per chunk, merged per hub by hub_chunk_finalize_kernel.
template <typename W>
__global__ void __launch_bounds__(kThreads) hub_direct_kernel(const Chunk* __restrict__ chunks,
                                                              const i32* __restrict__ nbr, const W* __restrict__ ew,
                                                              RoundParams p, HubPartial* partials) {
    __shared__ CandShared red;
    const Chunk ch = chunks[blockIdx.x];
    if (role_blocked(ch.v, p)) return;   // the hub's finalisation writes no proposal
    u64 current = 0, best = 0, tie = 0;
    for (i64 e = ch.begin + threadIdx.x; e < ch.end; e += kThreads)
        direct_candidate(ch.v, nbr[e], static_cast<u64>(weight_at(ew, e)), p, best, tie);
    block_candidate_reduce(current, best, tie, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = {current, best, tie};
}

template <typename W>
__global__ void hub_chunk_finalize_kernel(i64 hubs, const i32* __restrict__ hub_list,
                                          const i64* __restrict__ chunk_begin,
                                          const HubPartial* __restrict__ partials, const i32* __restrict__ clusters,
                                          const W* __restrict__ vw, const u64* __restrict__ cw, RoundParams p,
                                          SclpOut out) {
    const i64 h = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (h >= hubs) return;
    const i32 v = hub_list[h];
    const i32 source = p.identity ? v : clusters[v];
    u64 current = 0, best = 0, tie = 0;
    for (i64 c = chunk_begin[h]; c < chunk_begin[h + 1]; ++c) {
        const HubPartial q = partials[c];
        current = q.current > current ? q.current : current;
        if (better(q.best, q.tie, best, tie)) { best = q.best; tie = q.tie; }
    }
    decode_and_write(v, source, current, best, tie, p, vw, cw, out);
}

// Level-0 check of the reference's sorted-unique flag (src/coarsen.cu:44-70):
// rows strictly increasing.  Warp per non-hub row; hub rows by chunks.
template <typename O>
__global__ void __launch_bounds__(kThreads) unsorted_rows_kernel(i64 n, const O* __restrict__ off,
                                                                 const i32* __restrict__ nbr, u32* flag) {
    const int lane = threadIdx.x & 31;
    const i64 warps_total = static_cast<i64>(gridDim.x) * kWarps;
    bool bad = false;
    for (i64 v = static_cast<i64>(blockIdx.x) * kWarps + (threadIdx.x >> 5); v < n; v += warps_total) {
        const i64 b = off[v], e1 = off[v + 1];
        if (e1 - b > kHubDegree) continue;
        for (i64 e = b + 1 + lane; e < e1; e += 32) bad |= nbr[e] <= nbr[e - 1];
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flag, 1u);
}

template <typename O>
__global__ void __launch_bounds__(kThreads) hub_unsorted_kernel(const Chunk* __restrict__ chunks,
                                                                const O* __restrict__ off,
                                                                const i32* __restrict__ nbr, u32* flag) {
    const Chunk ch = chunks[blockIdx.x];
    const i64 row_begin = off[ch.v];
    bool bad = false;
    for (i64 e = ch.begin + threadIdx.x; e < ch.end; e += kThreads)
        if (e > row_begin) bad |= nbr[e] <= nbr[e - 1];
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1u);
}

}  // namespace gp
