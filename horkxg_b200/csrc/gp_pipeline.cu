// Host side of the B200 partitioner: input preparation, the coarsening level
// loop, the batched initial partition, the level-by-level projection and
// refinement, and the C ABI of include/gpart_b200.h.
//
// Pipeline semantics follow app/partition_main.cu:20-142,
// src/coarsen.cu:1906-2164, src/initial_partition_gpu.cu:170-276,
// src/refine.cu:423-646 and src/refine_incremental.cuh:235-361.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "gp_common.cuh"
#include "gp_prim.cuh"
#include "gp_sclp.cuh"
#include "gp_contract.cuh"
#include "gp_initial.cuh"
#include "gp_refine.cuh"
#include "gp_hub.cuh"
#include "gp_analyze.cuh"
#include "gp_symmetrize.cuh"

namespace gp {

void Device::check_errors() {
    u32 e = 0;
    fetch(*this, &e, err, 1);
    if (!e) return;
    GP_CUDA(cudaMemsetAsync(err, 0, sizeof(u32), stream));
    if (e & kErrTimeout) fail(GP_ETIMEOUT, "a bounded device wait timed out");
    if (e & kErrCapacity) fail(GP_ERUNTIME, "SCLP coarsening exceeded cluster capacity");
    if (e & kErrSplit) fail(GP_ERUNTIME, "GPU spectral split cannot satisfy capacity");
    if (e & kErrBalance) fail(GP_ERUNTIME, "GPU initializer infeasible balance");
    if (e & kErrCutUnderflow) fail(GP_ERUNTIME, "incremental cut underflow");
    if (e & kErrOddCut) fail(GP_ERUNTIME, "weighted CSR cut is not symmetric");
    if (e & kErrTableFull) fail(GP_ERUNTIME, "internal hash table overflow");
    fail(GP_EINVAL, "invalid graph input");
}

using Clock = std::chrono::steady_clock;
inline double seconds_since(Clock::time_point t) { return std::chrono::duration<double>(Clock::now() - t).count(); }

// include/partition_capacity.hpp:12-23
u64 partition_capacity(u64 total, int parts, double ratio) {
    if (parts < 2 || parts > 32 || !std::isfinite(ratio) || ratio < 1.0)
        fail(GP_EINVAL, "invalid partition capacity options");
    const long double raw = static_cast<long double>(total) * ratio / parts;
    if (!std::isfinite(raw) || raw >= static_cast<long double>(std::numeric_limits<u64>::max()))
        fail(GP_EOVERFLOW, "partition capacity exceeds uint64");
    const auto capacity = static_cast<u64>(std::floor(raw));
    if (capacity < total / static_cast<unsigned>(parts) + (total % parts != 0))
        fail(GP_EINVAL, "integer partition capacity cannot hold total weight");
    return capacity;
}

// ---------------------------------------------------------------------------
// Device graph (one hierarchy level)
// ---------------------------------------------------------------------------
template <typename T>
struct DGraph {
    using O = typename T::O;
    using W = typename T::W;
    i64 n = 0, m = 0;
    Buf<O> off;
    Buf<i32> nbr;
    Buf<W> ew, vw;
    bool unit_ew = true, unit_vw = true;
    const W* ewp() const { return unit_ew ? nullptr : ew.get(); }
    const W* vwp() const { return unit_vw ? nullptr : vw.get(); }
    // hub index (vertices of degree > kHubThreshold, chunked), built on demand
    struct Hubs {
        bool built = false;
        i64 count = 0, chunks = 0;
        Buf<i32> list;
        Buf<Chunk> chunk;
        Buf<i64> chunk_begin;   // per hub, count + 1 entries
        // SCLP affinity split (hub_split): the hubs whose table fits one
        // CTA's shared memory (chip_ids: small_count hubs of the 42 KB shape,
        // then chip_count of the 96 KB shape, then mid_count of the 227 KB
        // shape), and the hubs that keep global tables, with their own chunk
        // list (Chunk::hub indexes global_list)
        bool split_built = false;
        Buf<i32> chip_ids;
        i64 small_count = 0, chip_count = 0, mid_count = 0;
        i64 mid_slots = 0;   // table slots of the 1024-thread shape on this device
        i64 global_count = 0, global_chunks = 0;
        Buf<i32> global_list;
        Buf<Chunk> global_chunk;
    };
    mutable Hubs hubs;
    // rows free of duplicate neighbours: 1 yes, 0 no, -1 not yet checked
    mutable int unique_rows = -1;
    // vertices of degree in (256, 2048] (the refinement's block-walked
    // rows), from the degree classes of an aggregation; -1 unknown
    mutable i64 mid_rows = -1;
};
static_assert(kSplitDegree == 256, "mid_rows counts SCLP degree class 4, (256, kHubDegree]");

// known_count: the number of hub vertices when the caller already has it
// (the degree classes of an aggregation); 0 skips the scans.
template <typename T>
const typename DGraph<T>::Hubs& hub_index(Device& d, const DGraph<T>& g, i64 known_count = -1) {
    auto& h = g.hubs;
    if (h.built) return h;
    if (known_count == 0) {
        h.count = h.chunks = 0;
        h.built = true;
        return h;
    }
    using O = typename T::O;
    const i64 n = g.n;
    Buf<i64> hpos(d, static_cast<size_t>(n) + 1), cpos(d, static_cast<size_t>(n) + 1), tot(d, 2);
    exclusive_scan<i64>(d, HubFlag<O>{g.off.get()}, hpos.get(), n, tot.get());
    exclusive_scan<i64>(d, HubChunkCount<O>{g.off.get()}, cpos.get(), n, tot.get() + 1);
    i64 t[2];
    fetch(d, t, tot.get(), 2);
    h.count = t[0];
    h.chunks = t[1];
    if (h.count) {
        h.list = Buf<i32>(d, static_cast<size_t>(h.count));
        h.chunk = Buf<Chunk>(d, static_cast<size_t>(h.chunks));
        h.chunk_begin = Buf<i64>(d, static_cast<size_t>(h.count) + 1);
        launch(d, "hub_fill_kernel", hub_fill_kernel<O>, blocks_for(n, kThreads), kThreads, 0, n, g.off.get(),
               hpos.get(), cpos.get(), h.list.get(), h.chunk.get(), h.chunk_begin.get());
        GP_CUDA(cudaMemcpyAsync(h.chunk_begin.get() + h.count, tot.get() + 1, sizeof(i64), cudaMemcpyDeviceToDevice,
                                d.stream));
    }
    h.built = true;
    return h;
}

// Splits a level's hubs (once) into those of hub_smem_kernel and those that
// keep the global tables.
template <typename T>
const typename DGraph<T>::Hubs& hub_split(Device& d, const DGraph<T>& g) {
    using O = typename T::O;
    const auto& hubs = hub_index(d, g);
    auto& h = g.hubs;
    if (h.split_built) return h;
    std::vector<i64> ext(static_cast<size_t>(2 * hubs.count));
    std::vector<i32> ids(static_cast<size_t>(hubs.count));
    if (hubs.count) {
        Buf<i64> dev_ext(d, ext.size());
        launch(d, "hub_extent_kernel", hub_extent_kernel<O>, blocks_for(hubs.count, kThreads), kThreads, 0,
               hubs.count, hubs.list.get(), g.off.get(), dev_ext.get());
        GP_LAUNCH();
        to_host(d, ext.data(), dev_ext.get(), ext.size());
        to_host(d, ids.data(), hubs.list.get(), ids.size());
        d.sync();
    }
    // the largest table one CTA of the 1024-thread shape can hold: the
    // device's opt-in shared memory per block less the kernel's static part,
    // whole 32-slot lines
    int optin = 0;
    GP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d.device));
    cudaFuncAttributes fa{};
    GP_CUDA(cudaFuncGetAttributes(&fa, hub_smem_kernel<kHubMidThreads, O, typename T::W>));
    h.mid_slots = std::max<i64>(0, (static_cast<i64>(optin) - static_cast<i64>(fa.sharedSizeBytes)) / 8 / 32 * 32);
    std::vector<i32> small, chip, mid, glob;
    std::vector<Chunk> chunks;
    for (i64 i = 0; i < hubs.count; ++i) {
        const i64 begin = ext[2 * i], degree = ext[2 * i + 1];
        if (hub_smem_slots(degree) <= kHubSmallSlots) {
            small.push_back(ids[i]);
            continue;
        }
        if (hub_smem_slots(degree) <= kHubSmemSlots) {
            chip.push_back(ids[i]);
            continue;
        }
        if (hub_smem_slots(degree) <= h.mid_slots) {
            mid.push_back(ids[i]);
            continue;
        }
        const i32 gi = static_cast<i32>(glob.size());
        glob.push_back(ids[i]);
        for (i64 e = begin; e < begin + degree; e += kChunkEdges)
            chunks.push_back({ids[i], gi, e, std::min(e + kChunkEdges, begin + degree)});
    }
    h.small_count = static_cast<i64>(small.size());
    h.chip_count = static_cast<i64>(chip.size());
    h.mid_count = static_cast<i64>(mid.size());
    small.insert(small.end(), chip.begin(), chip.end());
    small.insert(small.end(), mid.begin(), mid.end());
    if (!small.empty()) {
        h.chip_ids = Buf<i32>(d, small.size());
        to_device(d, h.chip_ids.get(), small.data(), small.size());
    }
    h.global_count = static_cast<i64>(glob.size());
    h.global_chunks = static_cast<i64>(chunks.size());
    if (!glob.empty()) {
        h.global_list = Buf<i32>(d, glob.size());
        h.global_chunk = Buf<Chunk>(d, chunks.size());
        to_device(d, h.global_list.get(), glob.data(), glob.size());
        to_device(d, h.global_chunk.get(), chunks.data(), chunks.size());
    }
    d.sync();   // host vectors go out of scope
    h.split_built = true;
    return h;
}

// The reference's level-0 sortedness flag (src/coarsen.cu:44-70,1965): rows
// strictly increasing, hence duplicate-free.  Contracted levels are
// duplicate-free by construction.
template <typename T>
bool unique_rows(Device& d, const DGraph<T>& g) {
    if (g.unique_rows >= 0) return g.unique_rows == 1;
    using O = typename T::O;
    Buf<u32> flag(d, 1);
    flag.zero(d);
    launch(d, "unsorted_rows_kernel", unsorted_rows_kernel<O>, stride_grid(d, g.n * 32), kThreads, 0, g.n, g.off.get(),
           g.nbr.get(), flag.get());
    const auto& hubs = hub_index(d, g);
    if (hubs.count)
        launch(d, "hub_unsorted_kernel", hub_unsorted_kernel<O>, static_cast<int>(hubs.chunks), kThreads, 0,
               hubs.chunk.get(), g.off.get(), g.nbr.get(), flag.get());
    u32 f = 0;
    fetch(d, &f, flag.get(), 1);
    g.unique_rows = f ? 0 : 1;
    return g.unique_rows == 1;
}

struct Log {
    bool on = false;
    std::ostream& out = std::cout;
};

// Opt-in phase trace (environment variable GP_TRACE=1): synchronises the
// stream at each mark and prints the wall time since the previous mark to
// stderr.  For locating host stalls; off in normal runs.
struct Trace {
    bool on = std::getenv("GP_TRACE") != nullptr;
    std::chrono::steady_clock::time_point last = std::chrono::steady_clock::now();
    void mark(Device& d, const char* what, long long a = -1, long long b = -1) {
        if (!on) return;
        d.sync();
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "trace %-28s %8.3f ms", what, std::chrono::duration<double, std::milli>(now - last).count());
        if (a >= 0) std::fprintf(stderr, " (%lld)", a);
        if (b >= 0) std::fprintf(stderr, " (%lld)", b);
        std::fprintf(stderr, "\n");
        last = std::chrono::steady_clock::now();
    }
};
inline Trace& trace() { static Trace t; return t; }

__global__ void iota_kernel(i64 n, i32* a) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) a[i] = static_cast<i32>(i);
}

template <typename W>
__global__ void widen_weights_kernel(i64 n, const W* vw, u64* out) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<u64>(weight_at(vw, i));
}

template <typename W>
__global__ void sat_sum_kernel(i64 m, const W* w, u64* out) {
    __shared__ u64 sh[kWarps];
    u64 s = 0;
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const u64 x = static_cast<u64>(weight_at(w, i));
        s = ~0ULL - s < x ? ~0ULL : s + x;
    }
    for (int o = 16; o; o >>= 1) {
        const u64 x = __shfl_xor_sync(0xffffffffu, s, o);
        s = ~0ULL - s < x ? ~0ULL : s + x;
    }
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        s = 0;
        for (int i = 0; i < kWarps; ++i) s = ~0ULL - s < sh[i] ? ~0ULL : s + sh[i];
        if (s) {
            u64 prev = *reinterpret_cast<volatile u64*>(out);
            while (true) {
                const u64 next = ~0ULL - prev < s ? ~0ULL : prev + s;
                const u64 seen = atomic_cas_u64(out, prev, next);
                if (seen == prev) break;
                prev = seen;
            }
        }
    }
}

inline int stride_grid(Device& d, i64 items, int per_block = kThreads) {
    return static_cast<int>(std::min<i64>(blocks_for(items, per_block), d.grid_limit(8)));
}

// ---------------------------------------------------------------------------
// SCLP aggregation (src/coarsen.cu:937-1659)
// ---------------------------------------------------------------------------
template <typename T>
struct AggResult {
    Buf<i32> map;
    Buf<typename T::W> cvw;
    i64 coarse_n = 0;
    u64 cap = 0;
};

template <typename T>
struct SclpWork {
    Buf<i32> clusters, target, list, list_alt, clist, clist_alt;
    Buf<u64> cw, gain, demand, keys, keys_alt, excl, ckeys, ckeys_alt;
    Buf<u32> tie, ccount;
    Buf<unsigned char> cls;
    Buf<i64> pos, flags, positions, table_off;
    Buf<HubSlot> table;
    Buf<u64> scalars;
    u64 edge_total = 0;          // total directed edge weight of the first level (an upper bound below)
    bool edge_total_known = false;
    Buf<HubPartial> partials;
    void ensure(Device& d, i64 n) {
        const size_t s = static_cast<size_t>(n) + 1;
        clusters.ensure(d, s); target.ensure(d, s); list.ensure(d, s); list_alt.ensure(d, s);
        clist.ensure(d, s); clist_alt.ensure(d, s);
        cw.ensure(d, s); gain.ensure(d, s); demand.ensure(d, s); keys.ensure(d, s); keys_alt.ensure(d, s);
        excl.ensure(d, s); ckeys.ensure(d, s); ckeys_alt.ensure(d, s);
        tie.ensure(d, s); ccount.ensure(d, 8); cls.ensure(d, s);
        pos.ensure(d, s); flags.ensure(d, s); positions.ensure(d, s);
        scalars.ensure(d, 16);
    }
};

// Orders list[0, count) (ascending vertex ids) by (target asc, gain desc,
// tie desc); vertex order survives as the stable tie-break.
template <typename T>
void order_proposals(Device& d, SclpWork<T>& w, i64 n, i64 count, u64 gmax) {
    const int tbits = std::max(1, bit_width_u64(static_cast<u64>(std::max<i64>(1, n - 1))));
    const int gbits = std::max(1, bit_width_u64(gmax));
    auto keys = [&](int mode) {
        launch(d, "admission_keys_kernel", admission_keys_kernel, blocks_for(count, kThreads), kThreads, 0, 
            count, w.list.get(), w.target.get(), w.gain.get(), w.tie.get(), gmax, gbits, mode, w.keys.get());
        GP_LAUNCH();
    };
    auto sort = [&](int bits) {
        radix_sort<u64, i32>(d, w.keys.get(), w.list.get(), w.keys_alt.get(), w.list_alt.get(), count, 0, bits);
    };
    if (tbits + gbits + 32 <= 64) {
        keys(0); sort(tbits + gbits + 32);
    } else {
        keys(1); sort(32);
        if (tbits + gbits <= 64) { keys(2); sort(tbits + gbits); }
        else { keys(3); sort(gbits); keys(4); sort(tbits); }
    }
}

template <typename T>
void aggregate(Device& d, const DGraph<T>& g, SclpWork<T>& w, int parts, u32 seed, int level, int beta, bool pack,
               AggResult<T>& out, Log& log) {
    using O = typename T::O;
    using W = typename T::W;
    if (parts < 2 || parts > 32 || beta < 2) fail(GP_EINVAL, "invalid SCLP cluster capacity options");
    const i64 n = g.n;
    if (n <= 0 || n > std::numeric_limits<i32>::max())
        fail(GP_ERUNTIME, "SCLP coarsening received an unsupported graph size");
    w.ensure(d, n);
    const O* off = g.off.get();
    const i32* nbr = g.nbr.get();
    const W* ew = g.ewp();
    const W* vw = g.vwp();
    u64* sc = w.scalars.get();
    GP_CUDA(cudaMemsetAsync(sc, 0, 16 * sizeof(u64), d.stream));
    w.ccount.zero(d);
    launch(d, "weight_stats_kernel", weight_stats_kernel<W>, stride_grid(d, n), kThreads, 0, n, vw, sc);
    GP_LAUNCH();
    launch(d, "degree_class_kernel", degree_class_kernel<O>, blocks_for(n, kThreads), kThreads, 0, n, off, w.ckeys.get(),
           w.clist.get(), w.ccount.get(), sc + 8);
    GP_LAUNCH();
    radix_sort<u64, i32>(d, w.ckeys.get(), w.clist.get(), w.ckeys_alt.get(), w.clist_alt.get(), n, 0, 8);
    trace().mark(d, "agg.classes_launched", level);
    u64 stats[16];
    u32 cnt[kClasses];
    to_host(d, stats, sc, 16);
    fetch(d, cnt, w.ccount.get(), kClasses);
    const u64 total = stats[0], maxw = stats[1];
    const u64 denom = static_cast<u64>(beta) * static_cast<u64>(parts);
    const u64 cap = std::max(maxw, total / denom + (total % denom != 0 ? 1 : 0));
    i64 class_off[kClasses + 1] = {0};
    for (int c = 0; c < kClasses; ++c) class_off[c + 1] = class_off[c] + cnt[c];
    const i32* lists = w.clist.get();
    auto class_list = [&](int c) { return lists + class_off[c]; };

    trace().mark(d, "agg.classes_fetched", level);
    if (!w.edge_total_known) {
        if (ew) {
            Buf<u64> t(d, 1);
            t.zero(d);
            launch(d, "sat_sum_kernel", sat_sum_kernel<W>, stride_grid(d, g.m), kThreads, 0, g.m, ew, t.get());
            fetch(d, &w.edge_total, t.get(), 1);
        } else {
            w.edge_total = static_cast<u64>(g.m);
        }
        w.edge_total_known = true;
    }
    const int sum32 = w.edge_total <= 0xffffffffULL ? 1 : 0;
    g.mid_rows = static_cast<i64>(cnt[4]);
    const auto& hubs = hub_index(d, g, static_cast<i64>(cnt[5]));
    // hash-free affinity on identity rounds (rows without duplicates)
    const bool direct_ok = unique_rows(d, g);
    // global hash tables for hubs
    if (hubs.count != static_cast<i64>(cnt[5])) fail(GP_ERUNTIME, "hub index disagrees with degree classes");
    // Hubs whose table fits on chip (32-bit sums) run hub_smem_kernel; the
    // others keep per-hub tables in global memory.
    const bool chip = sum32 && hubs.count > 0 && d.hub_chip;
    if (chip) hub_split(d, g);
    const i64 gcount = chip ? hubs.global_count : hubs.count;
    const i64 gchunks = chip ? hubs.global_chunks : hubs.chunks;
    const i32* glist = chip ? hubs.global_list.get() : hubs.list.get();
    const Chunk* gchunk = chip ? hubs.global_chunk.get() : hubs.chunk.get();
    i64 table_total = 0;
    if (hubs.count > 0) {
        if (gcount > 0) {
            w.table_off.ensure(d, static_cast<size_t>(gcount) + 1);
            exclusive_scan<i64>(d, HubTableSize<O>{glist, off, gcount}, w.table_off.get(), gcount + 1,
                                reinterpret_cast<i64*>(sc + 4));
            fetch(d, &table_total, reinterpret_cast<i64*>(sc + 4), 1);
            w.table.ensure(d, static_cast<size_t>(table_total));
            GP_CUDA(cudaMemsetAsync(w.table.get(), 0, table_total * (sum32 ? sizeof(HubSlot32) : sizeof(HubSlot)),
                                    d.stream));
        }
        // the identity rounds' hub_direct_kernel writes one partial per chunk of every hub
        w.partials.ensure(d, static_cast<size_t>(std::max<i64>(table_total / kSlotTile, hubs.chunks)));
    }

    trace().mark(d, "agg.hub_tables", level);
    i32* clusters = w.clusters.get();
    u64* cw = w.cw.get();
    launch(d, "iota_kernel", iota_kernel, blocks_for(n, kThreads), kThreads, 0, n, clusters);
    launch(d, "widen_weights_kernel", widen_weights_kernel<W>, blocks_for(n, kThreads), kThreads, 0, n, vw, cw);
    launch(d, "fill_i32_kernel", fill_i32_kernel, blocks_for(n, kThreads), kThreads, 0, n, w.target.get(), kInvalid);
    GP_LAUNCH();
    SclpOut so{w.target.get(), w.gain.get(), w.tie.get(), w.demand.get()};

    // Algorithmic bytes of one affinity+decode pass over class c, counting
    // the work done (profiling only; measured by role_work_kernel): per
    // processed vertex offsets, list, cluster[v]/cluster weight reads and the
    // proposal writes; per edge of a processed vertex its neighbour, edge
    // weight and cluster gather (none at round 0); a skipped vertex reads its
    // cluster and writes an empty proposal.
    u64 work[kClasses][3] = {};
    u64 gwork[3] = {};   // the same for the hubs with global tables
    auto affinity_bytes = [&](int c, bool identity) {
        const double v = static_cast<double>(work[c][0]), e = static_cast<double>(work[c][1]);
        return v * (2 * sizeof(O) + 4 + 4 + 8 + 4 + 8 + 4 + 8) + (static_cast<double>(cnt[c]) - v) * 8 +
               e * (4 + (ew ? sizeof(W) : 0) + (identity ? 0 : 4));
    };
    auto affinity = [&](const RoundParams& p) {
        if (d.prof) {
            Buf<u64> cw_dev(d, 3 * kClasses);
            cw_dev.zero(d);
            for (int c = 1; c < kClasses; ++c)
                if (cnt[c])
                    launch(d, "role_work_kernel", role_work_kernel<O>, stride_grid(d, cnt[c]), kThreads, 0,
                           static_cast<i64>(cnt[c]), class_list(c), off, clusters, p, cw_dev.get() + 3 * c);
            fetch(d, &work[0][0], cw_dev.get(), 3 * kClasses);
            if (chip && gcount) {
                Buf<u64> gw(d, 3);
                gw.zero(d);
                launch(d, "role_work_kernel", role_work_kernel<O>, stride_grid(d, gcount), kThreads, 0, gcount, glist,
                       off, clusters, p, gw.get());
                fetch(d, gwork, gw.get(), 3);
            } else {
                for (int j = 0; j < 3; ++j) gwork[j] = work[5][j];
            }
            d.prof_bytes("affinity_small_kernel", affinity_bytes(1, p.identity) + affinity_bytes(2, p.identity));
            if (!(p.identity && direct_ok)) {   // the direct kernels of identity rounds carry no model
                d.prof_bytes("affinity_warp_hash_kernel", affinity_bytes(3, p.identity));
                d.prof_bytes("affinity_block_hash_kernel", affinity_bytes(4, p.identity));
            }
        }
        if (cnt[1])
            launch(d, "affinity_small_kernel", affinity_small_kernel<8, O, W>, blocks_for(static_cast<i64>(cnt[1]) * 8, kThreads), kThreads, 0, 
                cnt[1], class_list(1), off, nbr, ew, vw, clusters, cw, p, so);
        if (cnt[2])
            launch(d, "affinity_small_kernel", affinity_small_kernel<32, O, W>, blocks_for(static_cast<i64>(cnt[2]) * 32, kThreads), kThreads, 0, 
                cnt[2], class_list(2), off, nbr, ew, vw, clusters, cw, p, so);
        const bool direct = p.identity && direct_ok;
        if (cnt[3] && direct)
            launch(d, "affinity_direct_warp_kernel", affinity_direct_warp_kernel<O, W>,
                   blocks_for(static_cast<i64>(cnt[3]) * 32, kThreads), kThreads, 0, static_cast<i64>(cnt[3]),
                   class_list(3), off, nbr, ew, vw, cw, p, so);
        if (cnt[4] && direct)
            launch(d, "affinity_direct_block_kernel", affinity_direct_block_kernel<O, W>, static_cast<int>(cnt[4]),
                   kThreads, 0, static_cast<i64>(cnt[4]), class_list(4), off, nbr, ew, vw, cw, p, so);
        if (cnt[5] && direct) {
            launch(d, "hub_direct_kernel", hub_direct_kernel<W>, static_cast<int>(hubs.chunks), kThreads, 0,
                   hubs.chunk.get(), nbr, ew, p, w.partials.get());
            launch(d, "hub_chunk_finalize_kernel", hub_chunk_finalize_kernel<W>, blocks_for(hubs.count, kThreads),
                   kThreads, 0, hubs.count, hubs.list.get(), hubs.chunk_begin.get(), w.partials.get(), clusters, vw,
                   cw, p, so);
        }
        if (direct) return;
        // 8-byte table slots where every connection sum fits 32 bits
        if (cnt[3])
            launch(d, "affinity_warp_hash_kernel",
                   sum32 ? affinity_warp_hash_kernel<true, O, W> : affinity_warp_hash_kernel<false, O, W>,
                   blocks_for(cnt[3], kWarps), kThreads, 0, cnt[3], class_list(3), off, nbr, ew, vw, clusters, cw, p,
                   so, d.err);
        if (cnt[4]) {
            auto kernel = sum32 ? affinity_block_hash_kernel<true, O, W> : affinity_block_hash_kernel<false, O, W>;
            const int smem = kLargeSlots * (sum32 ? 8 : 12);
            GP_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            launch(d, "affinity_block_hash_kernel", kernel, static_cast<int>(cnt[4]), kThreads, smem, cnt[4],
                   class_list(4), off, nbr, ew, vw, clusters, cw, p, so, d.err);
        }
        if (cnt[5] && chip) {
            // per processed on-chip hub: its offsets, cluster and proposal
            // writes; per edge its neighbour, weight and cluster gather
            const double chip_edges = static_cast<double>(work[5][1] - gwork[1]);
            const double chip_hubs = static_cast<double>(work[5][0] - gwork[0]);
            d.prof_bytes("hub_smem_kernel", chip_hubs * (2 * sizeof(O) + 4 + 4 + 8 + 4 + 8) +
                                                chip_edges * (4 + 4 + (ew ? sizeof(W) : 0)));
            // the attribute is the largest size any launch of the kernel
            // uses (server slots share it across threads): never lowered
            const size_t smem512 = static_cast<size_t>(kHubSmemSlots) * sizeof(unsigned long long);
            auto k512 = hub_smem_kernel<kHubSmemThreads, O, W>;
            if (hubs.small_count || hubs.chip_count)
                GP_CUDA(cudaFuncSetAttribute(k512, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem512)));
            if (hubs.small_count)
                launch(d, "hub_smem_kernel", k512, static_cast<int>(hubs.small_count), kHubSmemThreads,
                       static_cast<size_t>(kHubSmallSlots) * sizeof(unsigned long long), hubs.chip_ids.get(), off,
                       nbr, ew, vw, clusters, cw, p, so);
            if (hubs.chip_count)
                launch(d, "hub_smem_kernel", k512, static_cast<int>(hubs.chip_count), kHubSmemThreads, smem512,
                       hubs.chip_ids.get() + hubs.small_count, off, nbr, ew, vw, clusters, cw, p, so);
            if (hubs.mid_count) {
                const size_t smem = static_cast<size_t>(hubs.mid_slots) * sizeof(unsigned long long);
                auto k = hub_smem_kernel<kHubMidThreads, O, W>;
                GP_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
                launch(d, "hub_smem_kernel", k, static_cast<int>(hubs.mid_count), kHubMidThreads, smem,
                       hubs.chip_ids.get() + hubs.small_count + hubs.chip_count, off, nbr, ew, vw, clusters, cw, p,
                       so);
            }
        }
        if (cnt[5] && gcount) {
            // chunk records of the global-table hubs; neighbour, weight and
            // cluster of each edge of the hubs that are not skipped; the
            // slots of their tables for the candidate pass
            d.prof_bytes("hub_insert_kernel", static_cast<double>(gwork[1]) * (4 + 4 + (ew ? sizeof(W) : 0)) +
                                                  static_cast<double>(gchunks) * sizeof(Chunk));
            auto hub_tables = [&](auto* table) {
                using S = std::remove_pointer_t<decltype(table)>;
                d.prof_bytes("hub_candidates_kernel", static_cast<double>(gwork[2]) * sizeof(S));
                launch(d, "hub_insert_kernel", hub_insert_kernel<O, W, S>, static_cast<int>(gchunks), kThreads, 0,
                       gchunk, nbr, ew, clusters, p, w.table_off.get(), table, d.err);
                launch(d, "hub_candidates_kernel", hub_candidates_kernel<W, S>,
                       static_cast<int>(table_total / kSlotTile), kThreads, 0, gcount, glist, w.table_off.get(), table,
                       clusters, p, w.partials.get(), i64{0});
            };
            if (sum32) hub_tables(reinterpret_cast<HubSlot32*>(w.table.get()));
            else hub_tables(w.table.get());
            launch(d, "hub_finalize_kernel", hub_finalize_kernel<W>, blocks_for(gcount, kThreads), kThreads, 0, gcount,
                   glist, w.table_off.get(), w.partials.get(), clusters, vw, cw, p, so);
        }
        GP_LAUNCH();
    };
    // compaction of cls == 2 into list (ascending) + count and gain maximum
    auto compact_contested = [&](i64& count, u64& gmax) {
        exclusive_scan<i64>(d, IsClass2{w.cls.get()}, w.pos.get(), n, reinterpret_cast<i64*>(sc + 2));
        launch(d, "compact_class2_kernel", compact_class2_kernel, blocks_for(n, kThreads), kThreads, 0, n, w.cls.get(), w.pos.get(),
                                                                                    w.list.get());
        GP_LAUNCH();
        u64 h[2];
        fetch(d, h, sc + 2, 2);
        count = static_cast<i64>(h[0]);
        gmax = h[1];
    };
    auto count_clusters = [&]() {
        GP_CUDA(cudaMemsetAsync(sc + 5, 0, sizeof(u64), d.stream));
        launch(d, "count_nonzero_kernel", count_nonzero_kernel, stride_grid(d, n), kThreads, 0, n, cw, sc + 5);
        GP_LAUNCH();
        u64 c;
        fetch(d, &c, sc + 5, 1);
        return static_cast<i64>(c);
    };
    auto sorted_weight_prefix = [&](i64 count) {
        exclusive_scan<u64>(d, SortedWeight<W>{w.list.get(), vw}, w.excl.get(), count);
    };

    i64 cluster_count = n;
    const i64 desired = (n + 1) / 2;
    int rounds = 0;
    for (int round = 0; round < 4; ++round) {
        if (static_cast<double>(cluster_count) <= 0.60 * n) break;
        const i64 removable = std::max<i64>(0, cluster_count - desired);
        const double fraction = std::min(0.50, static_cast<double>(removable) / static_cast<double>(cluster_count));
        const auto threshold = static_cast<u32>(fraction * 4294967296.0);
        RoundParams p = make_round(seed, level, round, true, threshold);
        p.sum32 = sum32;
        w.demand.zero(d);
        affinity(p);
        GP_CUDA(cudaMemsetAsync(sc + 3, 0, sizeof(u64), d.stream));
        launch(d, "admission_classify_kernel", admission_classify_kernel, blocks_for(n, kThreads), kThreads, 0, 
            n, w.target.get(), w.demand.get(), cw, cap, w.gain.get(), w.cls.get(), sc + 3);
        GP_LAUNCH();
        i64 contested = 0;
        u64 gmax = 0;
        compact_contested(contested, gmax);
        if (contested > 0) {
            order_proposals(d, w, n, contested, gmax);
            sorted_weight_prefix(contested);
            launch(d, "segment_heads_kernel", segment_heads_kernel, blocks_for(contested, kThreads), kThreads, 0, 
                contested, w.list.get(), w.target.get(), w.excl.get(), w.demand.get(), 0);
            launch(d, "contested_accept_kernel", contested_accept_kernel<W>, blocks_for(contested, kThreads), kThreads, 0, 
                contested, w.list.get(), w.target.get(), w.excl.get(), w.demand.get(), cw, vw, cap, w.cls.get());
            GP_LAUNCH();
        }
        launch(d, "sclp_commit_kernel", sclp_commit_kernel<W>, blocks_for(n, kThreads), kThreads, 0, n, w.cls.get(), w.target.get(), vw,
                                                                                 clusters, cw);
        GP_LAUNCH();
        cluster_count = count_clusters();
        trace().mark(d, "agg.round", round);
        ++rounds;
        if (log.on)
            log.out << "ml_gpu_sclp_round level=" << level << " round=" << round << " mover_fraction=" << fraction
                    << " clusters=" << cluster_count
                    << " contraction_ratio=" << static_cast<double>(cluster_count) / static_cast<double>(n) << '\n';
        if (static_cast<double>(cluster_count) <= 0.60 * n) break;
    }

    if (pack && cnt[0] > 1) {
        const i64 iso = cnt[0];
        exclusive_scan<u64>(d, SortedWeight<W>{class_list(0), vw}, w.excl.get(), iso);
        launch(d, "fill_i32_kernel", fill_i32_kernel, blocks_for(iso + 1, kThreads), kThreads, 0, iso + 1, w.list_alt.get(),
                                                                                   std::numeric_limits<i32>::max());
        launch(d, "isolated_rep_kernel", isolated_rep_kernel<W>, blocks_for(iso, kThreads), kThreads, 0, iso, class_list(0), w.excl.get(),
                                                                                    vw, cap, w.list_alt.get());
        launch(d, "isolated_commit_kernel", isolated_commit_kernel<W>, blocks_for(iso, kThreads), kThreads, 0, 
            iso, class_list(0), w.excl.get(), vw, cap, w.list_alt.get(), clusters, cw);
        GP_LAUNCH();
        cluster_count = count_clusters();
    }

    if (static_cast<double>(cluster_count) > 0.60 * n) {
        RoundParams p = make_round(seed, level, 4, false, 0);
        p.two_hop = 1;
        p.sum32 = sum32;
        affinity(p);
        GP_CUDA(cudaMemsetAsync(sc + 3, 0, sizeof(u64), d.stream));
        launch(d, "favorite_classify_kernel", favorite_classify_kernel, blocks_for(n, kThreads), kThreads, 0, n, w.target.get(), w.gain.get(),
                                                                                   w.cls.get(), sc + 3);
        GP_LAUNCH();
        i64 cand = 0;
        u64 gmax = 0;
        compact_contested(cand, gmax);
        if (cand > 0) {
            order_proposals(d, w, n, cand, gmax);
            launch(d, "segment_heads_kernel", segment_heads_kernel, blocks_for(cand, kThreads), kThreads, 0, 
                cand, w.list.get(), w.target.get(), w.excl.get(), w.demand.get(), 1);
            launch(d, "pair_flags_kernel", pair_flags_kernel<W>, blocks_for(cand, kThreads), kThreads, 0, 
                cand, w.list.get(), w.target.get(), w.demand.get(), vw, cap, w.flags.get());
            GP_LAUNCH();
            exclusive_scan_array<i64>(d, w.flags.get(), w.positions.get(), cand);
            const u64 budget = static_cast<u64>(std::max<i64>(0, cluster_count - desired));
            if (budget > 0) {
                launch(d, "pair_commit_kernel", pair_commit_kernel<W>, blocks_for(cand, kThreads), kThreads, 0, 
                    cand, w.list.get(), w.flags.get(), w.positions.get(), budget, vw, clusters, cw);
                GP_LAUNCH();
            }
        }
        cluster_count = count_clusters();
    }

    trace().mark(d, "agg.isolated_two_hop", level);
    // compaction
    Buf<i32> compact(d, static_cast<size_t>(n));
    exclusive_scan<i32>(d, NonEmpty{cw}, compact.get(), n, reinterpret_cast<i32*>(sc + 6));
    i32 coarse_n = 0;
    fetch(d, &coarse_n, reinterpret_cast<i32*>(sc + 6), 1);
    out.map = Buf<i32>(d, static_cast<size_t>(n));
    out.cvw = Buf<W>(d, static_cast<size_t>(std::max<i32>(coarse_n, 1)));
    out.cvw.zero(d);
    launch(d, "compact_map_kernel", compact_map_kernel<W>, blocks_for(n, kThreads), kThreads, 0, n, clusters, compact.get(), vw,
                                                                             out.map.get(), out.cvw.get());
    launch(d, "cap_check_kernel", cap_check_kernel<W>, blocks_for(coarse_n, kThreads), kThreads, 0, coarse_n, out.cvw.get(), cap, d.err);
    GP_LAUNCH();
    out.coarse_n = coarse_n;
    out.cap = cap;
    trace().mark(d, "agg.compaction", level);
    if (log.on)
        log.out << "ml_gpu_sclp level=" << level << " fine_vertices=" << n << " coarse_vertices=" << coarse_n
                << " contraction_ratio=" << static_cast<double>(coarse_n) / static_cast<double>(n) << " beta=" << beta
                << " cluster_cap=" << cap << " lp_rounds=" << rounds << " low_vertices=" << cnt[1]
                << " medium_vertices=" << cnt[2] + cnt[3] << " high_vertices=" << cnt[4] + cnt[5]
                << " isolated_vertices=" << cnt[0] << " seed=" << seed << '\n';
}

// ---------------------------------------------------------------------------
// Contraction (src/coarsen.cu:1674-1814)
// ---------------------------------------------------------------------------
template <typename T>
void contract(Device& d, const DGraph<T>& g, const i32* map, i64 coarse_n, Buf<typename T::W>&& cvw, DGraph<T>& out) {
    using O = typename T::O;
    using W = typename T::W;
    const i64 n = g.n, m = g.m;
    Buf<i64> fdeg(d, static_cast<size_t>(coarse_n) + 1);
    Buf<i64> temp_off(d, static_cast<size_t>(coarse_n) + 1);
    Buf<i64> cursor(d, static_cast<size_t>(coarse_n) + 1);
    Buf<i64> scal(d, 4);
    fdeg.zero(d);
    cursor.zero(d);
    launch(d, "row_fine_degree_kernel", row_fine_degree_kernel<O>, blocks_for(n, kThreads), kThreads, 0, n, g.off.get(), map, fdeg.get());
    GP_LAUNCH();
    exclusive_scan_array<i64>(d, fdeg.get(), temp_off.get(), coarse_n + 1);
    const u32 sentinel = static_cast<u32>(coarse_n);
    trace().mark(d, "contract.rows", coarse_n);
    Buf<u32> tgt(d, static_cast<size_t>(std::max<i64>(m, 1)));
    Buf<W> wt(d, static_cast<size_t>(std::max<i64>(m, 1)));
    const i64 warps = (n + 31) / 32;
    d.prof_bytes("scatter_edges_kernel", static_cast<double>(n + 1) * sizeof(O) + n * (4.0 + 8 + 8) +
                                             static_cast<double>(m) * (4 + 4 + 4 + (g.ewp() ? sizeof(W) : 0) + sizeof(W)));
    launch(d, "scatter_edges_kernel", scatter_edges_kernel<O, W>, blocks_for(warps * 32, kThreads), kThreads, 0, n,
           g.off.get(), g.nbr.get(), g.ewp(), map, temp_off.get(), cursor.get(), sentinel, tgt.get(), wt.get());
    const auto& hubs = hub_index(d, g);
    if (hubs.count) {
        Buf<i64> hub_dst(d, static_cast<size_t>(hubs.count));
        launch(d, "hub_reserve_kernel", hub_reserve_kernel<O>, blocks_for(hubs.count, kThreads), kThreads, 0,
               hubs.count, hubs.list.get(), g.off.get(), map, temp_off.get(), cursor.get(), hub_dst.get());
        launch(d, "hub_scatter_kernel", hub_scatter_kernel<O, W>, static_cast<int>(hubs.chunks), kThreads, 0,
               hubs.chunk.get(), g.off.get(), g.nbr.get(), g.ewp(), map, hub_dst.get(), sentinel, tgt.get(), wt.get());
    }
    GP_LAUNCH();
    trace().mark(d, "contract.scatter", m);
    // row classes
    Buf<u64> rk(d, static_cast<size_t>(coarse_n)), rk_alt(d, static_cast<size_t>(coarse_n));
    Buf<i32> rl(d, static_cast<size_t>(coarse_n)), rl_alt(d, static_cast<size_t>(coarse_n));
    Buf<u64> rc(d, 2 * kRowClasses);
    rc.zero(d);
    // A row is ranked by the bitmap of segment_bitmap_kernel instead of a
    // shared-memory sort once it is longer than coarse_n / 64: the bitmap
    // costs about coarse_n / 32 words per window plus two passes over the row,
    // the sort three passes with barriers; both give the same row.
    const i64 bitmap_from = std::max<i64>(kWarpSegCap, coarse_n / 64);
    launch(d, "row_class_kernel", row_class_kernel, blocks_for(coarse_n, kThreads), kThreads, 0, coarse_n,
           temp_off.get(), static_cast<i64>(seg_smem_capacity<W>()), bitmap_from, rk.get(), rl.get(), rc.get());
    GP_LAUNCH();
    radix_sort<u64, i32>(d, rk.get(), rl.get(), rk_alt.get(), rl_alt.get(), coarse_n, 0, 8);
    u64 rcnt[2 * kRowClasses];
    fetch(d, rcnt, rc.get(), 2 * kRowClasses);
    const u64* rent = rcnt + kRowClasses;   // entries per class
    i64 cstart[kRowClasses + 1] = {0};
    for (int k = 0; k < kRowClasses; ++k) cstart[k + 1] = cstart[k] + static_cast<i64>(rcnt[k]);
    // segment kernels read and write each scattered entry once (target + weight)
    auto seg_bytes = [&](int k) { return 2.0 * static_cast<double>(rent[k]) * (4 + sizeof(W)); };
    d.prof_bytes("segment_warp_kernel", seg_bytes(1));
    d.prof_bytes("segment_warp_radix_kernel", seg_bytes(2));
    d.prof_bytes("segment_smem_kernel", seg_bytes(3) + seg_bytes(4));
    const bool sort_big = (coarse_n + kBitmapWindow - 1) / kBitmapWindow > kSortWindows;
    d.prof_bytes(sort_big ? "segment_sort_kernel" : "segment_bitmap_kernel", seg_bytes(5));
    d.prof_bytes("giant_place_kernel", seg_bytes(6));
    Buf<i64> row_len(d, static_cast<size_t>(coarse_n) + 1);
    row_len.zero(d);
    const int key_bits = std::max(1, bit_width_u64(static_cast<u64>(coarse_n)));
    if (rcnt[1])
        launch(d, "segment_warp_kernel", segment_warp_kernel<W>, blocks_for(static_cast<i64>(rcnt[1]) * 32, kThreads),
               kThreads, 0, rcnt[1], rl.get() + cstart[1], temp_off.get(), sentinel, tgt.get(), wt.get(),
               row_len.get());
    if (rcnt[2]) {
        const size_t smem = static_cast<size_t>(kWarps) * (2 * kWarpSegCap * sizeof(W) +
                                                          (2 * kWarpSegCap + kRadix) * sizeof(u32));
        GP_CUDA(cudaFuncSetAttribute(segment_warp_radix_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
        launch(d, "segment_warp_radix_kernel", segment_warp_radix_kernel<W>,
               blocks_for(static_cast<i64>(rcnt[2]) * 32, kThreads), kThreads, smem, rcnt[2], rl.get() + cstart[2],
               temp_off.get(), sentinel, key_bits, tgt.get(), wt.get(), row_len.get());
    }
    for (int k = 3; k <= 4; ++k) {
        if (!rcnt[k]) continue;
        const int cap = k == 3 ? kMidSegCap : seg_smem_capacity<W>();
        const size_t smem = 2 * static_cast<size_t>(cap) * (sizeof(u32) + sizeof(W));
        GP_CUDA(cudaFuncSetAttribute(segment_smem_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(2 * static_cast<size_t>(seg_smem_capacity<W>()) *
                                                      (sizeof(u32) + sizeof(W)))));
        launch(d, "segment_smem_kernel", segment_smem_kernel<W>, static_cast<int>(rcnt[k]), kThreads, smem, rcnt[k],
               rl.get() + cstart[k], temp_off.get(), sentinel, key_bits, cap, tgt.get(), wt.get(), row_len.get());
    }
    GP_LAUNCH();
    // rows above seg_smem_capacity (classes 5 and 6, contiguous in the class
    // order) are written to alternate buffers
    const i64 c3 = cstart[5];
    const i64 big = static_cast<i64>(rcnt[5] + rcnt[6]);
    Buf<i64> alt_off;
    Buf<u32> ak;
    Buf<W> aw;
    if (big) {
        alt_off = Buf<i64>(d, static_cast<size_t>(big) + 1);
        exclusive_scan<i64>(d, BigRowLen{rl.get() + c3, temp_off.get(), big}, alt_off.get(), big + 1,
                            scal.get());
        i64 alt_total = 0;
        fetch(d, &alt_total, scal.get(), 1);
        ak = Buf<u32>(d, static_cast<size_t>(alt_total));
        aw = Buf<W>(d, static_cast<size_t>(alt_total));
    }
    if (rcnt[5] && sort_big) {
        launch(d, "segment_sort_kernel", segment_sort_kernel<W>, static_cast<int>(rcnt[5]), kThreads, 0,
               static_cast<i64>(rcnt[5]), rl.get() + c3, temp_off.get(), alt_off.get(), sentinel, key_bits, tgt.get(),
               wt.get(), ak.get(), aw.get(), row_len.get());
        GP_LAUNCH();
    } else if (rcnt[5]) {
        const size_t smem = (static_cast<size_t>(kBitmapWords) + kBitmapGroups) * sizeof(u32);
        GP_CUDA(cudaFuncSetAttribute(segment_bitmap_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
        launch(d, "segment_bitmap_kernel", segment_bitmap_kernel<W>, static_cast<int>(rcnt[5]), kThreads, smem,
               static_cast<i64>(rcnt[5]), rl.get() + c3, temp_off.get(), alt_off.get(), sentinel, coarse_n, tgt.get(),
               wt.get(), ak.get(), aw.get(), row_len.get());
        GP_LAUNCH();
    }
    if (rcnt[6]) {
        const i64 giants = static_cast<i64>(rcnt[6]);
        const i32* glist = rl.get() + cstart[6];
        const i64* galt = alt_off.get() + rcnt[5];
        Buf<i64> chunk_off(d, static_cast<size_t>(giants) + 1);
        exclusive_scan<i64>(d, GiantChunkCount{glist, temp_off.get(), giants}, chunk_off.get(), giants + 1,
                            scal.get());
        i64 gbase = 0, chunks_total = 0;
        fetch(d, &chunks_total, scal.get(), 1);
        fetch(d, &gbase, galt, 1);
        Buf<SegChunk> chunks(d, static_cast<size_t>(chunks_total));
        launch(d, "giant_chunks_kernel", giant_chunks_kernel, blocks_for(giants, kThreads), kThreads, 0, giants,
               glist, temp_off.get(), chunk_off.get(), chunks.get());
        const i64 wpr = (coarse_n + 31) / 32;
        const i64 groups = (wpr + kBitmapGroup - 1) / kBitmapGroup;
        Buf<u32> gbits(d, static_cast<size_t>(giants * wpr));
        Buf<u32> gpre(d, static_cast<size_t>(giants * groups));
        gbits.zero(d);
        GP_CUDA(cudaMemsetAsync(aw.get() + gbase, 0,
                                static_cast<size_t>(static_cast<i64>(ak.size()) - gbase) * sizeof(W), d.stream));
        launch(d, "giant_mark_kernel", giant_mark_kernel, static_cast<int>(chunks_total), kThreads, 0, chunks.get(),
               tgt.get(), sentinel, wpr, gbits.get());
        launch(d, "giant_scan_kernel", giant_scan_kernel, static_cast<int>(giants), kThreads, 0, glist, wpr,
               gbits.get(), gpre.get(), row_len.get());
        launch(d, "giant_place_kernel", giant_place_kernel<W>, static_cast<int>(chunks_total), kThreads, 0,
               chunks.get(), tgt.get(), wt.get(), sentinel, wpr, gbits.get(), gpre.get(), galt, ak.get(), aw.get());
        GP_LAUNCH();
    }
    trace().mark(d, "contract.segments", static_cast<long long>(rcnt[5]), static_cast<long long>(rcnt[6]));
    out.n = coarse_n;
    out.off = Buf<O>(d, static_cast<size_t>(coarse_n) + 1);
    exclusive_scan<O>(d, RowLenToO<O>{row_len.get()}, out.off.get(), coarse_n + 1, reinterpret_cast<O*>(scal.get() + 1));
    O cm = 0;
    fetch(d, &cm, reinterpret_cast<O*>(scal.get() + 1), 1);
    out.m = static_cast<i64>(cm);
    out.nbr = Buf<i32>(d, static_cast<size_t>(std::max<i64>(out.m, 1)));
    out.ew = Buf<W>(d, static_cast<size_t>(std::max<i64>(out.m, 1)));
    out.unit_ew = false;
    if (out.m > 0) {
        d.prof_bytes("copy_rows_kernel", static_cast<double>(coarse_n) * (sizeof(O) + 8) + 2.0 * out.m * (4 + sizeof(W)));
        launch(d, "copy_rows_kernel", copy_rows_kernel<O, W>, blocks_for(((coarse_n + 31) / 32) * 32, kThreads),
               kThreads, 0, coarse_n, temp_off.get(), out.off.get(), tgt.get(), wt.get(), out.nbr.get(), out.ew.get());
        if (big)
            launch(d, "copy_big_rows_kernel", copy_big_rows_kernel<O, W>, static_cast<int>(big), kThreads, 0,
                   rl.get() + c3, alt_off.get(), out.off.get(), ak.get(), aw.get(), out.nbr.get(), out.ew.get());
        GP_LAUNCH();
    }
    out.vw = std::move(cvw);
    out.unit_vw = false;
    out.unique_rows = 1;
    trace().mark(d, "contract.copy", out.m);
}

// ---------------------------------------------------------------------------
// Hierarchy
// ---------------------------------------------------------------------------
struct Opts {
    int parts = 4;
    double ratio = 1.03;
    u32 seed = 0;
    bool verify = false;
    bool deterministic = false;
    int beta = 0;
    bool pack = true;
    int max_levels = 24;
    int max_rounds = 32;
    double stop = 0.90;
    double growth = 2.0;
};

Opts to_opts(const gp_options* o) {
    Opts r;
    if (!o) return r;
    r.parts = o->parts;
    r.ratio = o->imbalance;
    r.seed = o->seed;
    r.verify = o->verify != 0;
    r.deterministic = o->deterministic != 0;
    r.beta = o->cluster_size_factor;
    r.pack = o->pack_isolated != 0;
    r.max_levels = o->max_levels;
    r.max_rounds = o->max_rounds;
    r.stop = o->stop_ratio;
    r.growth = o->growth_ratio;
    return r;
}

inline int production_beta(int parts) { return std::max(64, (512 + parts - 1) / parts); }

template <typename T>
struct Hierarchy {
    std::vector<DGraph<T>> levels;
    std::vector<Buf<i32>> maps;
    std::string stop_reason = "capacity_floor";
};

// ---------------------------------------------------------------------------
// --verify: checks of every coarsening step on the device, with the rules and
// messages of validate_coarsening_step (src/coarsen.cu:1835-1902).
// ---------------------------------------------------------------------------
template <typename O>
__global__ void check_offsets_kernel(i64 n, const O* off, i64 m, u32* err);
__global__ void check_neighbors_kernel(i64 m, const i32* nbr, i64 n, u32* err);
template <typename O, typename W>
__global__ void symmetry_kernel(i64 n, const O* off, const i32* nbr, const W* ew, u32* err);

enum VerifyFlag : u32 {
    kVerifyMapRange = 1u << 0,
    kVerifyCluster = 1u << 1,
    kVerifyCap = 1u << 2,
    kVerifySelfLoop = 1u << 3,
};

template <typename W>
__global__ void verify_map_kernel(i64 n, const i32* __restrict__ map, i64 coarse_n, const W* __restrict__ vw,
                                  u64* recomputed, u32* coverage, u32* flags) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const i32 c = map[v];
    if (c < 0 || c >= coarse_n) {
        atomicOr(flags, kVerifyMapRange);
        return;
    }
    atomic_add_u64(&recomputed[c], static_cast<u64>(weight_at(vw, v)));
    atomicAdd(&coverage[c], 1u);
}

template <typename W>
__global__ void verify_clusters_kernel(i64 coarse_n, const u64* __restrict__ recomputed,
                                       const u32* __restrict__ coverage, const W* __restrict__ cvw, u64 cap,
                                       u32* flags) {
    const i64 c = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= coarse_n) return;
    const u64 w = static_cast<u64>(weight_at(cvw, c));
    if (coverage[c] == 0 || recomputed[c] != w) atomicOr(flags, kVerifyCluster);
    if (w > cap) atomicOr(flags, kVerifyCap);
}

template <typename O>
__global__ void self_loop_kernel(i64 n, const O* __restrict__ off, const i32* __restrict__ nbr, u32* flags) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    for (i64 e = off[v]; e < static_cast<i64>(off[v + 1]); ++e)
        if (nbr[e] == v) {
            atomicOr(flags, kVerifySelfLoop);
            return;
        }
}

// Labels (c * 2654435761 + 17) mod 23 of coarse vertex c, through `map` for
// the fine level (map == nullptr: the coarse level itself).
__global__ void hashed_labels_kernel(i64 n, const i32* __restrict__ map, i32* labels) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const u64 c = map ? static_cast<u64>(map[v]) : static_cast<u64>(v);
    labels[v] = static_cast<i32>((c * 2654435761ULL + 17ULL) % 23ULL);
}

template <typename T>
u64 directed_cut(Device& d, const DGraph<T>& g, const i32* labels, u64* scratch);

template <typename T>
void verify_coarsening_step(Device& d, const DGraph<T>& fine, const DGraph<T>& coarse, const i32* map, u64 cap,
                            int level, Log& log) {
    using O = typename T::O;
    using W = typename T::W;
    if (coarse.n <= 0 || coarse.n > fine.n) fail(GP_ERUNTIME, "coarsening produced an invalid vertex count");
    Buf<u64> recomputed(d, static_cast<size_t>(coarse.n)), sums(d, 4);
    Buf<u32> coverage(d, static_cast<size_t>(coarse.n)), flags(d, 1);
    recomputed.zero(d);
    coverage.zero(d);
    sums.zero(d);
    flags.zero(d);
    launch(d, "verify_map_kernel", verify_map_kernel<W>, blocks_for(fine.n, kThreads), kThreads, 0, fine.n, map,
           coarse.n, fine.vwp(), recomputed.get(), coverage.get(), flags.get());
    launch(d, "weight_stats_kernel", weight_stats_kernel<W>, stride_grid(d, fine.n), kThreads, 0, fine.n, fine.vwp(),
           sums.get());
    launch(d, "weight_stats_kernel", weight_stats_kernel<W>, stride_grid(d, coarse.n), kThreads, 0, coarse.n,
           coarse.vwp(), sums.get() + 2);
    GP_LAUNCH();
    u32 f = 0;
    fetch(d, &f, flags.get(), 1);
    if (f & kVerifyMapRange) fail(GP_ERUNTIME, "coarsening map contains an out-of-range id");
    u64 st[4];
    fetch(d, st, sums.get(), 4);
    if (st[0] != st[2]) fail(GP_ERUNTIME, "coarsening did not conserve vertex weight");
    launch(d, "verify_clusters_kernel", verify_clusters_kernel<W>, blocks_for(coarse.n, kThreads), kThreads, 0,
           coarse.n, recomputed.get(), coverage.get(), coarse.vwp(), cap, flags.get());
    GP_LAUNCH();
    fetch(d, &f, flags.get(), 1);
    if (f & kVerifyCluster) fail(GP_ERUNTIME, "coarsening cluster weight mismatch");
    if (f & kVerifyCap) fail(GP_ERUNTIME, "coarse point exceeds configured weight cap");
    // strict CSR checks of the coarse level (validate_weighted_csr, src/graph.cpp:122-190)
    launch(d, "check_offsets_kernel", check_offsets_kernel<O>, blocks_for(coarse.n + 1, kThreads), kThreads, 0,
           coarse.n, coarse.off.get(), coarse.m, flags.get());
    if (coarse.m)
        launch(d, "check_neighbors_kernel", check_neighbors_kernel, stride_grid(d, coarse.m), kThreads, 0, coarse.m,
               coarse.nbr.get(), coarse.n, flags.get());
    GP_LAUNCH();
    fetch(d, &f, flags.get(), 1);
    if (f & kErrBadInput) fail(GP_ERUNTIME, "invalid weighted CSR shape");
    launch(d, "self_loop_kernel", self_loop_kernel<O>, blocks_for(coarse.n, kThreads), kThreads, 0, coarse.n,
           coarse.off.get(), coarse.nbr.get(), flags.get());
    launch(d, "symmetry_kernel", symmetry_kernel<O, W>, blocks_for(coarse.n, kThreads), kThreads, 0, coarse.n,
           coarse.off.get(), coarse.nbr.get(), coarse.ewp(), flags.get());
    GP_LAUNCH();
    fetch(d, &f, flags.get(), 1);
    if (f & kVerifySelfLoop) fail(GP_ERUNTIME, "contracted graph contains a self loop");
    if (f & kErrOddCut) fail(GP_ERUNTIME, "weighted CSR is not bidirectional");
    // the cut of hashed coarse labels equals the cut of their projection
    Buf<i32> fl(d, static_cast<size_t>(fine.n)), cl(d, static_cast<size_t>(coarse.n));
    launch(d, "hashed_labels_kernel", hashed_labels_kernel, blocks_for(fine.n, kThreads), kThreads, 0, fine.n, map,
           fl.get());
    launch(d, "hashed_labels_kernel", hashed_labels_kernel, blocks_for(coarse.n, kThreads), kThreads, 0, coarse.n,
           static_cast<const i32*>(nullptr), cl.get());
    GP_LAUNCH();
    const u64 fine_cut = directed_cut<T>(d, fine, fl.get(), sums.get());
    const u64 coarse_cut = directed_cut<T>(d, coarse, cl.get(), sums.get() + 2);
    if ((fine_cut & 1ULL) || (coarse_cut & 1ULL)) fail(GP_ERUNTIME, "weighted CSR cut is not symmetric");
    if (fine_cut != coarse_cut) fail(GP_ERUNTIME, "cut is not conserved by coarse projection");
    if (log.on)
        log.out << "ml_layer_verify level=" << level << " map=ok weights=ok csr=ok projection_cut=ok\n";
}

template <typename T>
void coarsen(Device& d, DGraph<T>&& input, const Opts& o, Hierarchy<T>& h, Log& log) {
    const int beta = o.beta > 0 ? o.beta : production_beta(o.parts);
    if (o.parts < 2 || o.parts > 32 || beta < 2 || o.max_levels < 0 || !std::isfinite(o.stop) || o.stop <= 0 || o.stop > 1)
        fail(GP_EINVAL, "invalid coarsening options");
    h.levels.clear();
    h.maps.clear();
    h.levels.reserve(static_cast<size_t>(o.max_levels) + 1);
    const i64 cutoff = std::max<i64>(32, static_cast<i64>(beta) * o.parts);
    DGraph<T> current = std::move(input);
    SclpWork<T> work;
    int level = 0;
    for (; level < o.max_levels && current.n > cutoff; ++level) {
        const u32 level_seed = o.seed + static_cast<u32>(level);
        if (log.on)
            log.out << "ml_coarsen_begin level=" << level << " vertices=" << current.n << " edges=" << current.m
                    << " method=sclp seed=" << level_seed << '\n';
        AggResult<T> agg;
        aggregate(d, current, work, o.parts, level_seed, level, beta, o.pack, agg, log);
        d.check_errors();
        const double ratio = static_cast<double>(agg.coarse_n) / static_cast<double>(current.n);
        if (agg.coarse_n >= current.n || ratio > o.stop) {
            if (log.on) log.out << "ml_coarsen_stop reason=insufficient_contraction\n";
            h.stop_reason = "insufficient_contraction";
            break;
        }
        DGraph<T> coarse;
        contract(d, current, agg.map.get(), agg.coarse_n, std::move(agg.cvw), coarse);
        if (log.on)
            log.out << "ml_gpu_contract_seconds level=" << level << " coarse_edges=" << coarse.m << '\n';
        if (o.verify) verify_coarsening_step(d, current, coarse, agg.map.get(), agg.cap, level, log);
        h.levels.push_back(std::move(current));
        h.maps.push_back(std::move(agg.map));
        current = std::move(coarse);
    }
    if (level == o.max_levels && current.n > cutoff) h.stop_reason = "max_levels";
    h.levels.push_back(std::move(current));
}

// ---------------------------------------------------------------------------
// Initial partition (src/initial_partition_gpu.cu:170-276)
// ---------------------------------------------------------------------------
struct DepthPlan {
    std::vector<InitTask> tasks;   // first_part, parts, children filled; data fields by the device
};

std::vector<DepthPlan> plan_tasks(int parts) {
    std::vector<DepthPlan> depths(1);
    depths[0].tasks.push_back({0, 0, 0, parts, 0, -1, -1});
    for (size_t dpt = 0; dpt < depths.size(); ++dpt) {
        DepthPlan next;
        for (auto& t : depths[dpt].tasks) {
            const int lp = t.parts / 2, rp = t.parts - lp;
            if (lp >= 2) { t.left_child = static_cast<i32>(next.tasks.size()); next.tasks.push_back({0, 0, t.first_part, lp, 0, -1, -1}); }
            if (rp >= 2) { t.right_child = static_cast<i32>(next.tasks.size()); next.tasks.push_back({0, 0, t.first_part + lp, rp, 0, -1, -1}); }
        }
        if (!next.tasks.empty()) depths.push_back(std::move(next));
    }
    return depths;
}

template <typename T>
void launch_diffusion(Device& d, const DGraph<T>& g, int ntasks, const InitTask* tasks, const i32* task_of_pos,
                      i32 positions, const i32* order, const i32* labels, u32 seed, int steps, float* deg, float* xa,
                      float* xb, Moments* contrib, float* x_out, u64* key, u32* bar, i64 max_degree = -1) {
    using O = typename T::O;
    using W = typename T::W;
    // Small graphs (max_degree known, every row within a warp's reach): one
    // thread-block cluster, same values, no grid barriers.
    if (d.small_diffusion && max_degree >= 0 && max_degree <= kHeavyRow && positions <= kSmallDiffN &&
        g.m <= kSmallDiffM && positions == g.n) {
        auto small = diffusion_small_kernel<O, W>;
        const size_t smem = small_diffusion_smem(positions);
        // the attribute is shared by every thread of the process (server
        // slots launch concurrently): always the largest size, never lowered
        GP_CUDA(cudaFuncSetAttribute(small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(small_diffusion_smem(kSmallDiffN))));
        // a power of two: one block per 1024 positions and per
        // kSmallDiffBlockEdges edges
        int cs = 1;
        while (cs < kSmallDiffCluster && (cs * kSmallDiffThreads < positions || cs * kSmallDiffBlockEdges < g.m)) cs *= 2;
        if (cs > 8) GP_CUDA(cudaFuncSetAttribute(small, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(kSmallDiffThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = d.stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cs;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        // a cluster that cannot be placed (too few free SMs in a GPC) leaves
        // the graph to the cooperative kernel, which computes the same values
        int placeable = 0;
        GP_CUDA(cudaOccupancyMaxActiveClusters(&placeable, small, &cfg));
        if (placeable > 0) {
            cudaEvent_t ev0 = nullptr;
            if (d.prof) { ev0 = d.event(); GP_CUDA(cudaEventRecord(ev0, d.stream)); }
            const O* off = g.off.get();
            GP_CUDA(cudaLaunchKernelEx(&cfg, small, ntasks, tasks, task_of_pos, positions, order, labels, off,
                                       g.nbr.get(), g.ewp(), seed, steps, x_out, key));
            ++d.launches;
            if (d.prof) {
                cudaEvent_t ev1 = d.event();
                GP_CUDA(cudaEventRecord(ev1, d.stream));
                auto& e = d.prof_table["diffusion_small_kernel"];
                e.pending.push_back({ev0, ev1});
                ++e.launches;
            }
            return;
        }
    }
    auto kernel = diffusion_kernel<O, W>;
    int per_sm = 0;
    GP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0));
    const int max_grid = std::max(1, per_sm) * d.sms;
    const int grid = std::max(1, std::min({max_grid, 2 * d.sms, blocks_for(positions, kWarps)}));
    GP_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(u32), d.stream));
    const O* off = g.off.get();
    const i32* nbr = g.nbr.get();
    const W* ew = g.ewp();
    u32* bar_counter = bar;
    u32* bar_gen = bar + 1;
    u32* err = d.err;
    void* args[] = {&ntasks, &tasks, &task_of_pos, &positions, &order, &labels, &off, &nbr, &ew, &seed, &steps,
                    &deg, &xa, &xb, &contrib, &x_out, &key, &bar_counter, &bar_gen, &err};
    cudaEvent_t ev0 = nullptr;
    if (d.prof) { ev0 = d.event(); GP_CUDA(cudaEventRecord(ev0, d.stream)); }
    GP_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kernel), grid, kThreads, args, 0, d.stream));
    ++d.launches;
    if (d.prof) {
        cudaEvent_t ev1 = d.event();
        GP_CUDA(cudaEventRecord(ev1, d.stream));
        auto& e = d.prof_table["diffusion_kernel"];
        e.pending.push_back({ev0, ev1});
        ++e.launches;
    }
}

// `trace` (optional, device, depths x n floats): for every recursion depth
// the normalised diffusion value of each vertex of an open task at that
// depth; the caller fills it with a marker beforehand.
template <typename T>
void initial_partition(Device& d, const DGraph<T>& g, int parts, double ratio, u32 seed, Buf<i32>& labels,
                       u64* initial_cut, Log& log, float* trace = nullptr) {
    using W = typename T::W;
    const i64 n64 = g.n;
    if (n64 <= 0 || n64 > std::numeric_limits<int>::max() - 255 || parts < 2 || parts > n64 || parts > 32 ||
        !std::isfinite(ratio) || ratio < 1.0)
        fail(GP_EINVAL, "invalid GPU initial partition input");
    const i32 n = static_cast<i32>(n64);
    Buf<u64> sc(d, 8);
    sc.zero(d);
    launch(d, "weight_stats_kernel", weight_stats_kernel<W>, stride_grid(d, n), kThreads, 0, n, g.vwp(), sc.get());
    launch(d, "sat_sum_kernel", sat_sum_kernel<W>, stride_grid(d, g.m), kThreads, 0, g.m, g.ewp(), sc.get() + 2);
    launch(d, "max_degree_kernel", max_degree_kernel<typename T::O>, stride_grid(d, n), kThreads, 0, n64, g.off.get(),
           sc.get() + 3);
    GP_LAUNCH();
    u64 st[4];
    fetch(d, st, sc.get(), 4);
    const u64 total = st[0], maxw = st[1], edge_total = st[2];
    const i64 max_degree = static_cast<i64>(st[3]);
    if (!total || total == ~0ULL || edge_total == ~0ULL)
        fail(GP_EOVERFLOW, "GPU initializer weight accumulation overflow");
    const u64 capacity = partition_capacity(total, parts, ratio);
    if (maxw > capacity) fail(GP_EINVAL, "a vertex exceeds partition capacity");

    labels = Buf<i32>(d, static_cast<size_t>(n));
    labels.zero(d);
    Buf<i32> order(d, static_cast<size_t>(n)), task_of_pos(d, static_cast<size_t>(n));
    launch(d, "iota_kernel", iota_kernel, blocks_for(n, kThreads), kThreads, 0, n, order.get());
    Buf<float> deg(d, static_cast<size_t>(n)), xa(d, static_cast<size_t>(n)), xb(d, static_cast<size_t>(n));
    Buf<Moments> contrib(d, static_cast<size_t>(n));
    Buf<u64> key(d, static_cast<size_t>(n)), key_alt(d, static_cast<size_t>(n)), prefix(d, static_cast<size_t>(n));
    Buf<u32> bar(d, 2);
    auto depths = plan_tasks(parts);
    depths[0].tasks[0].count = n;
    depths[0].tasks[0].weight = total;
    std::vector<Buf<InitTask>> dtasks;
    for (auto& dp : depths) {
        dtasks.emplace_back(d, dp.tasks.size());
        to_device(d, dtasks.back().get(), dp.tasks.data(), dp.tasks.size());
    }
    for (size_t dpt = 0; dpt < depths.size(); ++dpt) {
        const int nt = static_cast<int>(depths[dpt].tasks.size());
        GP_CUDA(cudaMemsetAsync(task_of_pos.get(), 0xff, n * sizeof(i32), d.stream));
        launch(d, "task_positions_kernel", task_positions_kernel, nt, kThreads, 0, nt, dtasks[dpt].get(), task_of_pos.get());
        GP_LAUNCH();
        float* x_out = trace ? trace + dpt * static_cast<size_t>(n) : nullptr;
        launch_diffusion(d, g, nt, dtasks[dpt].get(), task_of_pos.get(), n, order.get(), labels.get(), seed, 64,
                         deg.get(), xa.get(), xb.get(), contrib.get(), x_out, key.get(), bar.get(), max_degree);
        launch(d, "task_sort_kernel", task_sort_kernel, nt, kThreads, 0, nt, dtasks[dpt].get(), key.get(), key_alt.get(), order.get());
        InitTask* next = dpt + 1 < depths.size() ? dtasks[dpt + 1].get() : nullptr;
        launch(d, "task_split_kernel", task_split_kernel<W>, nt, kThreads, 0, nt, dtasks[dpt].get(), next, order.get(), g.vwp(), capacity,
                                                           prefix.get(), labels.get(), d.err);
        GP_LAUNCH();
    }
    d.check_errors();
    Buf<u64> loads(d, static_cast<size_t>(parts) + 1);
    loads.zero(d);
    launch(d, "part_weight_kernel", part_weight_kernel<W>, blocks_for(n, kThreads), kThreads, 0, n, labels.get(), g.vwp(), loads.get());
    launch(d, "cut_kernel", cut_kernel<typename T::O, W>, stride_grid(d, static_cast<i64>(n) * 32), kThreads, 0, n,
           g.off.get(), g.nbr.get(), g.ewp(), labels.get(), loads.get() + parts);
    {
        const auto& hubs = hub_index(d, g);
        if (hubs.count)
            launch(d, "hub_cut_kernel", hub_cut_kernel<typename T::O, W>, static_cast<int>(hubs.chunks), kThreads, 0,
                   hubs.chunk.get(), g.nbr.get(), g.ewp(), labels.get(), loads.get() + parts);
    }
    GP_LAUNCH();
    std::vector<u64> host(static_cast<size_t>(parts) + 1);
    fetch(d, host.data(), loads.get(), host.size());
    if (*std::max_element(host.begin(), host.begin() + parts) > capacity)
        fail(GP_ERUNTIME, "GPU initializer balance validation failed");
    if (initial_cut) *initial_cut = host[parts] / 2;
    if (log.on)
        log.out << "initial_partition_backend=gpu_spectral_batched_fp32\ncoarsest_vertices=" << n
                << "\ncoarsest_edge_entries=" << g.m << "\ninitial_partition_parts=" << parts
                << "\ninitial_partition_edgecut=" << host[parts] / 2 << '\n';
}

// ---------------------------------------------------------------------------
// Refinement (src/refine_incremental.cuh:235-361, src/refine.cu:423-646)
// ---------------------------------------------------------------------------
struct BucketThresholdsHost {
    BucketThresholds t;
    BucketThresholdsHost() { for (int j = -23; j <= 24; ++j) t.t[j + 23] = std::pow(1.5, j); }
};

template <typename T>
u64 directed_cut(Device& d, const DGraph<T>& g, const i32* labels, u64* scratch) {
    GP_CUDA(cudaMemsetAsync(scratch, 0, sizeof(u64), d.stream));
    d.prof_bytes("cut_kernel", static_cast<double>(g.n + 1) * sizeof(typename T::O) + g.n * 4.0 +
                                   static_cast<double>(g.m) * (4 + 4 + (g.ewp() ? sizeof(typename T::W) : 0)));
    launch(d, "cut_kernel", cut_kernel<typename T::O, typename T::W>, stride_grid(d, g.n * 32), kThreads, 0, g.n,
           g.off.get(), g.nbr.get(), g.ewp(), labels, scratch);
    const auto& hubs = hub_index(d, g);
    if (hubs.count)
        launch(d, "hub_cut_kernel", hub_cut_kernel<typename T::O, typename T::W>, static_cast<int>(hubs.chunks),
               kThreads, 0, hubs.chunk.get(), g.nbr.get(), g.ewp(), labels, scratch);
    GP_LAUNCH();
    u64 c = 0;
    fetch(d, &c, scratch, 1);
    return c;
}

template <typename T>
u64 undirected_cut(Device& d, const DGraph<T>& g, const i32* labels, u64* scratch) {
    const u64 c = directed_cut(d, g, labels, scratch);
    if (c & 1ULL) fail(GP_ERUNTIME, "refinement cut is not symmetric");
    return c / 2;
}

// The rebalance loop on the device (refine_incremental.cuh:303-330 runs it
// from the host, one round trip per iteration): a CUDA graph holds one
// conditional WHILE node whose body is the iteration's launches followed by
// rebalance_continue_kernel, which sums the iteration's counters here and
// sets the node's condition.
struct RebalanceLoop {
    long long delta;   // summed cut decrease of the iterations
    i64 accepted;      // summed movers
    int iterations;
    int stalled;       // the last iteration moved nothing
};

// One warp, after every iteration: continue while the iteration moved
// vertices, a part is above capacity and fewer than `limit` iterations ran
// (the host loop's conditions, so the loop ends after at most `limit`
// iterations whatever the data).
__global__ void rebalance_continue_kernel(cudaGraphConditionalHandle handle, const RefineCounters* ctr,
                                          const u64* pw, int k, u64 cap, int limit, RebalanceLoop* s) {
    const int lane = threadIdx.x & 31;
    u64 x = lane < k ? pw[lane] : 0;
    for (int o = 16; o; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (threadIdx.x != 0) return;
    const i64 moved = ctr->movers;
    const int it = ++s->iterations;
    s->delta += ctr->delta;
    s->accepted += moved;
    if (moved == 0) s->stalled = 1;
    cudaGraphSetConditional(handle, moved != 0 && x > cap && it < limit ? 1u : 0u);
}

// Rebalance iterations a level runs from the host before the adaptive mode
// captures its loop into a graph.
constexpr int kGraphLoopAfter = 8;

// The graph of one level's rebalance loop (its kernels' arguments are the
// level's buffers, so it is built once per level and launched after every
// LP round that leaves a part overloaded).
struct RebalanceGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t capturing = nullptr;   // set while the body is being captured
    u64 body_launches = 0;              // kernels per iteration
    RebalanceGraph() = default;
    RebalanceGraph(const RebalanceGraph&) = delete;
    RebalanceGraph& operator=(const RebalanceGraph&) = delete;
    ~RebalanceGraph() {
        if (capturing) {   // an exception left the capture open: close it, keep nothing
            cudaGraph_t body = nullptr;
            cudaStreamEndCapture(capturing, &body);
            cudaGetLastError();
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

struct RefineWork {
    Buf<unsigned char> cache_raw;
    Buf<i32> targets, list, movers, saved_labels, clist, clist_alt, cand;
    Buf<i64> gains, pos;
    Buf<PropRec> props;
    Buf<unsigned char> locks, flags;
    Buf<double> gpw;
    Buf<i32> bucket;
    Buf<u64> rank, counts, offsets, saved_pw, excl, keys, keys_alt, bucket_base, scratch;
    Buf<RefineCounters> ctr;
    void ensure(Device& d, i64 n, int k, size_t cache_bytes) {
        const size_t s = static_cast<size_t>(n) + 1;
        cache_raw.ensure(d, cache_bytes);
        targets.ensure(d, s); list.ensure(d, s); movers.ensure(d, s); saved_labels.ensure(d, s);
        clist.ensure(d, s); clist_alt.ensure(d, s); cand.ensure(d, s);
        gains.ensure(d, s); pos.ensure(d, s); props.ensure(d, s);
        locks.ensure(d, s); flags.ensure(d, s);
        gpw.ensure(d, s); bucket.ensure(d, s);
        rank.ensure(d, s); excl.ensure(d, s); keys.ensure(d, s); keys_alt.ensure(d, s);
        counts.ensure(d, static_cast<size_t>(k) * kBalWidth);
        offsets.ensure(d, static_cast<size_t>(k) * kBalWidth);
        bucket_base.ensure(d, static_cast<size_t>(k) * kBalWidth);
        saved_pw.ensure(d, 32);
        scratch.ensure(d, 8);
        ctr.ensure(d, 1);
    }
};

// known_cut: the cut of `labels` when the caller has it (a projection keeps
// the cut of the coarser level's result), else kUnknownCut.
constexpr u64 kUnknownCut = ~0ULL;

template <typename T, typename C>
gp_refine_stats refine_level(Device& d, const DGraph<T>& g, RefineWork& w, i32* labels, u64* pw,
                             std::vector<u64>& host_pw, int k, u64 cap, int rounds, bool deterministic, bool verify,
                             u64 known_cut) {
    using O = typename T::O;
    using W = typename T::W;
    const i64 n = g.n;
    w.ensure(d, n, k, static_cast<size_t>(n) * k * sizeof(C));
    C* cache = reinterpret_cast<C*>(w.cache_raw.get());
    const O* off = g.off.get();
    const i32* nbr = g.nbr.get();
    const W* ew = g.ewp();
    const W* vw = g.vwp();
    RefineCounters* ctr = w.ctr.get();
    static const BucketThresholdsHost thresholds;
    gp_refine_stats st{};
    w.locks.zero(d);
    w.flags.zero(d);
    const auto& hubs = hub_index(d, g);
    double build_bytes = 0;
    if (d.prof) {
        // offsets; neighbour, weight and label of every edge of a row below
        // the hub degree (hub rows are built by the chunked kernel); the
        // cache rows written
        i64 hub_edges = 0;
        if (hubs.count) {
            std::vector<i64> ext(static_cast<size_t>(2 * hubs.count));
            Buf<i64> dev_ext(d, ext.size());
            launch(d, "hub_extent_kernel", hub_extent_kernel<O>, blocks_for(hubs.count, kThreads), kThreads, 0,
                   hubs.count, hubs.list.get(), off, dev_ext.get());
            to_host(d, ext.data(), dev_ext.get(), ext.size());
            d.sync();
            for (i64 i = 0; i < hubs.count; ++i) hub_edges += ext[2 * i + 1];
        }
        build_bytes = static_cast<double>(n + 1) * sizeof(O) +
                      static_cast<double>(g.m - hub_edges) * (4 + 4 + (ew ? sizeof(W) : 0)) +
                      static_cast<double>(n - hubs.count) * k * sizeof(C);
        d.prof_bytes("build_cache_kernel", build_bytes);
    }
    launch(d, "build_cache_kernel", build_cache_kernel<O, W, C>, stride_grid(d, n * 8), kThreads, 0, n, off, nbr, ew,
           labels, k, cache);
    Buf<long long> hub_corr;
    if (hubs.count) {
        launch(d, "zero_hub_rows_kernel", zero_hub_rows_kernel<C>, blocks_for(hubs.count * k, kThreads), kThreads, 0,
               hubs.count, hubs.list.get(), k, cache);
        launch(d, "hub_build_cache_kernel", hub_build_cache_kernel<W, C>, static_cast<int>(hubs.chunks), kThreads, 0,
               hubs.chunk.get(), nbr, ew, labels, k, cache);
        hub_corr = Buf<long long>(d, static_cast<size_t>(hubs.count));
        hub_corr.zero(d);
    }
    GP_LAUNCH();
    u64 current_cut = known_cut != kUnknownCut ? known_cut : undirected_cut(d, g, labels, w.scratch.get());
    st.initial_cut = current_cut;
    u64 best_cut = current_cut;
    auto checkpoint = [&]() {
        GP_CUDA(cudaMemcpyAsync(w.saved_labels.get(), labels, n * sizeof(i32), cudaMemcpyDeviceToDevice, d.stream));
        GP_CUDA(cudaMemcpyAsync(w.saved_pw.get(), pw, k * sizeof(u64), cudaMemcpyDeviceToDevice, d.stream));
    };
    checkpoint();
    auto maximum = [&]() { return *std::max_element(host_pw.begin(), host_pw.end()); };
    // maximum edge weight decides the LP filter (refine_incremental.cuh:332-333);
    // for weighted levels it stays on the device (w.scratch[7]) and the LP
    // kernel derives the filter from it
    const double filter = 0.25;
    const u64* max_edge_weight = nullptr;
    if (ew) {
        GP_CUDA(cudaMemsetAsync(w.scratch.get() + 7, 0, sizeof(u64), d.stream));
        launch(d, "max_weight_kernel", max_weight_kernel<W>, stride_grid(d, g.m), kThreads, 0, g.m, ew,
               w.scratch.get() + 7);
        GP_LAUNCH();
        max_edge_weight = w.scratch.get() + 7;
    }
    struct Stats { RefineCounters c; u64 pw[32]; };
    static_assert(sizeof(Stats) <= Device::kPinnedBytes, "stats fit the pinned staging buffer");
    auto build_cache = [&]() {
        d.prof_bytes("build_cache_kernel", build_bytes);
        launch(d, "build_cache_kernel", build_cache_kernel<O, W, C>, stride_grid(d, n * 8), kThreads, 0, n, off, nbr,
               ew, labels, k, cache);
        if (hubs.count) {
            launch(d, "zero_hub_rows_kernel", zero_hub_rows_kernel<C>, blocks_for(hubs.count * k, kThreads), kThreads,
                   0, hubs.count, hubs.list.get(), k, cache);
            launch(d, "hub_build_cache_kernel", hub_build_cache_kernel<W, C>, static_cast<int>(hubs.chunks), kThreads,
                   0, hubs.chunk.get(), nbr, ew, labels, k, cache);
        }
    };
    // Applies the listed movers.  When the LP movers' edges outnumber m/8,
    // updating the affinity cache edge by edge (two random atomics per edge)
    // costs more than rebuilding it with one streaming pass, and the cut is
    // then recounted exactly instead of being updated by the per-edge deltas;
    // both routes give the same cache and the same cut.  (Rebalance moves
    // stay edge by edge: measured, the rebuild plus recount does not pay
    // there.)  The kernels read the mover count from the device, so a
    // rebalance apply needs no round trip before its launch: its grids are
    // sized for an upper bound of its movers.
    i64 ncand = 0;   // rebalance candidates in w.cand (vertices of overloaded parts, ascending)
    // the apply and commit launches for at most `bound` movers (the kernels
    // read the count from ctr)
    auto apply_launches = [&](bool lp, i64 bound, bool rebuild) {
        if (!rebuild) {
            // w.list (the LP proposers) is free once the movers are selected:
            // it takes the movers of degree above kSplitDegree
            launch(d, "apply_cache_cut_kernel", apply_cache_cut_kernel<O, W, C>, stride_grid(d, bound * 32),
                   kThreads, 0, w.movers.get(), ctr, off, nbr, ew, labels, w.targets.get(), w.flags.get(), k, cache,
                   ctr, w.list.get());
            if (g.mid_rows != 0)   // no row between kSplitDegree and the hub degree: nothing set aside
                launch(d, "apply_big_rows_kernel", apply_big_rows_kernel<O, W, C>,
                   static_cast<int>(std::min<i64>(std::max<i64>(bound, 1), d.grid_limit(4))), kThreads, 0,
                   w.list.get(), ctr, off, nbr, ew, labels, w.targets.get(), w.flags.get(), k, cache, ctr);
            if (hubs.count)
                launch(d, "hub_apply_kernel", hub_apply_kernel<W, C>,
                       static_cast<int>(std::min<i64>(hubs.chunks, d.grid_limit(8))), kThreads, 0,
                       hubs.chunks, hubs.chunk.get(), nbr, ew, labels, w.targets.get(), w.flags.get(), k, cache, ctr);
        }
        launch(d, "commit_kernel", commit_kernel<W>, stride_grid(d, bound), kThreads, 0, w.movers.get(), ctr, labels,
               w.targets.get(), vw, pw, w.locks.get(), w.flags.get(), lp ? 1 : 0);
        if (rebuild) build_cache();
    };
    // the cut after a decrease of `delta` (a negative delta raises it)
    auto apply_delta = [&](long long delta) {
        if (delta >= 0) {
            if (static_cast<u64>(delta) > current_cut) fail(GP_ERUNTIME, "incremental cut underflow");
            current_cut -= static_cast<u64>(delta);
        } else {
            current_cut += static_cast<u64>(-delta);
        }
    };
    auto finish_apply = [&](bool lp) -> i64 {
        RefineCounters c0{};
        const bool read_first = lp || d.prof || trace().on;
        if (read_first) {
            fetch(d, &c0, ctr, 1);
            if (c0.movers == 0) return 0;
        }
        const i64 bound = read_first ? c0.movers : ncand;
        const bool rebuild = lp && c0.mover_degree > g.m / 8;
        trace().mark(d, lp ? "refine.select_lp" : "refine.select_balance", n);
        apply_launches(lp, bound, rebuild);
        trace().mark(d, rebuild ? "refine.rebuild" : "refine.apply", c0.movers, c0.mover_degree);
        // counters and part weights straight into the pinned staging buffer,
        // one wait for both
        Stats h;
        {
            auto* staged = reinterpret_cast<Stats*>(d.pinned);
            GP_CUDA(cudaMemcpyAsync(&staged->c, ctr, sizeof(RefineCounters), cudaMemcpyDeviceToHost, d.stream));
            GP_CUDA(cudaMemcpyAsync(staged->pw, pw, k * sizeof(u64), cudaMemcpyDeviceToHost, d.stream));
            d.sync();
            std::memcpy(&h, staged, sizeof(Stats));
        }
        if (d.prof && !rebuild) {
            // per mover: offsets, label and target; per mover edge: neighbour,
            // weight, the neighbour's label and two read-modify-writes of the cache
            const double per_mover = 2 * sizeof(O) + 4 + 4 + 4;
            const double per_edge = 4 + 4 + (ew ? sizeof(W) : 0) + 4 * sizeof(C);
            d.prof_bytes("apply_cache_cut_kernel", static_cast<double>(h.c.movers - h.c.big) * per_mover +
                                                       static_cast<double>(h.c.walked_degree) * per_edge);
            d.prof_bytes("apply_big_rows_kernel",
                         static_cast<double>(h.c.big) * per_mover + static_cast<double>(h.c.big_degree) * per_edge);
            // every chunk record and the mover flag of its hub; the edges of
            // the moving hubs' chunks
            if (hubs.count)
                d.prof_bytes("hub_apply_kernel", static_cast<double>(hubs.chunks) * (sizeof(Chunk) + 1) +
                                                     static_cast<double>(h.c.hub_chunks) * 8 +
                                                     static_cast<double>(h.c.hub_edges) * per_edge);
        }
        if (rebuild) current_cut = undirected_cut(d, g, labels, w.scratch.get());
        else apply_delta(h.c.delta);
        std::copy(h.pw, h.pw + k, host_pw.begin());
        st.accepted += static_cast<u64>(h.c.movers);
        if (verify) {
            const u64 recount = undirected_cut(d, g, labels, w.scratch.get());
            if (recount != current_cut) fail(GP_ERUNTIME, "incremental cut differs from CSR scan");
        }
        return h.c.movers;
    };
    auto deterministic_ranks = [&]() {
        // candidates in ascending vertex order, sorted by (bucket, gpw desc)
        exclusive_scan<i64>(d, HasBucket{w.bucket.get(), w.cand.get()}, w.pos.get(), ncand,
                            reinterpret_cast<i64*>(w.scratch.get() + 1));
        launch(d, "compact_bucket_kernel", compact_bucket_kernel, blocks_for(ncand, kThreads), kThreads, 0, ncand,
               w.cand.get(), w.bucket.get(), w.pos.get(), w.clist.get());
        GP_LAUNCH();
        i64 count = 0;
        fetch(d, &count, reinterpret_cast<i64*>(w.scratch.get() + 1), 1);
        w.counts.zero(d);
        if (count == 0) return;
        launch(d, "rank_keys_kernel", rank_keys_kernel, blocks_for(count, kThreads), kThreads, 0, count, w.clist.get(), w.gpw.get(),
                                                                                w.bucket.get(), 0, w.keys.get());
        GP_LAUNCH();
        radix_sort<u64, i32>(d, w.keys.get(), w.clist.get(), w.keys_alt.get(), w.clist_alt.get(), count, 0, 64);
        launch(d, "rank_keys_kernel", rank_keys_kernel, blocks_for(count, kThreads), kThreads, 0, count, w.clist.get(), w.gpw.get(),
                                                                                w.bucket.get(), 1, w.keys.get());
        GP_LAUNCH();
        radix_sort<u64, i32>(d, w.keys.get(), w.clist.get(), w.keys_alt.get(), w.clist_alt.get(), count, 0,
                             std::max(1, bit_width_u64(static_cast<u64>(k) * kBalWidth)));
        exclusive_scan<u64>(d, ListWeight<W>{w.clist.get(), vw}, w.excl.get(), count);
        launch(d, "bucket_heads_kernel", bucket_heads_kernel, blocks_for(count, kThreads), kThreads, 0, count, w.clist.get(), w.bucket.get(),
                                                                                   w.excl.get(), w.bucket_base.get());
        launch(d, "bucket_ranks_kernel", bucket_ranks_kernel<W>, blocks_for(count, kThreads), kThreads, 0, 
            count, w.clist.get(), w.bucket.get(), w.excl.get(), w.bucket_base.get(), vw, w.rank.get(), w.counts.get());
        GP_LAUNCH();
    };
    // The rebalance loop as one graph launch: the iterations' launches are
    // captured once per level into the body of a WHILE node, and
    // rebalance_continue_kernel decides on the device whether another
    // iteration runs.  One round trip at the end reads the summed counters
    // and the part weights.
    RebalanceGraph rgraph;
    Buf<RebalanceLoop> loop_state;
    int host_iterations = 0;   // rebalance iterations of this level run by the host loop
    auto rebalance_on_device = [&](const auto& select, int limit) -> bool {
        if (!rgraph.exec) {
            loop_state = Buf<RebalanceLoop>(d, 1);
            GP_CUDA(cudaGraphCreate(&rgraph.graph, 0));
            cudaGraphConditionalHandle handle = 0;
            GP_CUDA(cudaGraphConditionalHandleCreate(&handle, rgraph.graph, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams p{};
            p.type = cudaGraphNodeTypeConditional;
            p.conditional.handle = handle;
            p.conditional.type = cudaGraphCondTypeWhile;
            p.conditional.size = 1;
            cudaGraphNode_t node = nullptr;
            GP_CUDA(cudaGraphAddNode(&node, rgraph.graph, nullptr, 0, &p));
            // thread-local capture: other threads (a server's slots) keep
            // allocating while this one captures
            GP_CUDA(cudaStreamBeginCaptureToGraph(d.stream, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
            rgraph.capturing = d.stream;
            const u64 before = d.launches;
            select();
            apply_launches(false, ncand, false);
            launch(d, "rebalance_continue_kernel", rebalance_continue_kernel, 1, 32, 0, handle, ctr, pw, k, cap, limit,
                   loop_state.get());
            rgraph.body_launches = d.launches - before;
            d.launches = before;
            cudaGraph_t body = nullptr;
            rgraph.capturing = nullptr;
            GP_CUDA(cudaStreamEndCapture(d.stream, &body));
            GP_CUDA(cudaGraphInstantiate(&rgraph.exec, rgraph.graph, 0));
        }
        GP_CUDA(cudaMemsetAsync(loop_state.get(), 0, sizeof(RebalanceLoop), d.stream));
        GP_CUDA(cudaGraphLaunch(rgraph.exec, d.stream));
        struct LoopStats { RebalanceLoop s; u64 pw[32]; };
        static_assert(sizeof(LoopStats) <= Device::kPinnedBytes, "loop stats fit the pinned staging buffer");
        LoopStats h;
        {
            auto* staged = reinterpret_cast<LoopStats*>(d.pinned);
            GP_CUDA(cudaMemcpyAsync(&staged->s, loop_state.get(), sizeof(RebalanceLoop), cudaMemcpyDeviceToHost,
                                    d.stream));
            GP_CUDA(cudaMemcpyAsync(staged->pw, pw, k * sizeof(u64), cudaMemcpyDeviceToHost, d.stream));
            d.sync();
            std::memcpy(&h, staged, sizeof(LoopStats));
        }
        if (h.s.iterations < 1 || h.s.iterations > limit) fail(GP_ERUNTIME, "rebalance graph iteration count");
        d.launches += static_cast<u64>(h.s.iterations) * rgraph.body_launches;
        st.admission_iterations += h.s.iterations;
        st.accepted += static_cast<u64>(h.s.accepted);
        apply_delta(h.s.delta);
        std::copy(h.pw, h.pw + k, host_pw.begin());
        if (verify) {
            const u64 recount = undirected_cut(d, g, labels, w.scratch.get());
            if (recount != current_cut) fail(GP_ERUNTIME, "incremental cut differs from CSR scan");
        }
        if (h.s.stalled) return false;
        return maximum() <= cap;
    };
    auto rebalance = [&]() -> bool {
        if (maximum() <= cap) return true;
        i64* cand_count = reinterpret_cast<i64*>(w.scratch.get() + 6);
        exclusive_scan<i64>(d, InOverloaded{labels, pw, cap}, w.pos.get(), n, cand_count);
        launch(d, "compact_overloaded_kernel", compact_overloaded_kernel, blocks_for(n, kThreads), kThreads, 0, n,
               labels, pw, cap, w.pos.get(), w.cand.get());
        // The candidate count stays on the device unless the host needs it
        // (the deterministic ranks size their sorts by it): the kernels read
        // it, and the grids are sized for the level's n.
        const bool host_count = deterministic || d.prof || trace().on;
        if (host_count) fetch(d, &ncand, cand_count, 1);
        else ncand = n;
        const i64* dev_count = host_count ? nullptr : cand_count;
        const int cgrid = host_count ? blocks_for(std::max<i64>(ncand, 1), kThreads) : stride_grid(d, n);
        w.counts.zero(d);   // bucket_scan_kernel leaves the counts zero for the next pass
        // one iteration's launches up to the movers (refine_incremental.cuh:303-326)
        auto select = [&]() {
            GP_CUDA(cudaMemsetAsync(ctr, 0, sizeof(RefineCounters), d.stream));
            launch(d, "rebalance_proposals_kernel", rebalance_proposals_kernel<C, W>, cgrid, kThreads, 0, ncand,
                   dev_count, w.cand.get(), cache, labels, vw, k, pw, cap, thresholds.t, deterministic ? 1 : 0, w.targets.get(),
                   w.gpw.get(), w.bucket.get(), w.rank.get(), w.counts.get());
            GP_LAUNCH();
            if (deterministic) deterministic_ranks();
            launch(d, "bucket_scan_kernel", bucket_scan_kernel, k, kThreads, 0, w.counts.get(), w.offsets.get());
            launch(d, "select_sources_kernel", select_sources_kernel<W>, cgrid, kThreads, 0, ncand, dev_count,
                   w.cand.get(),
                   w.bucket.get(), w.rank.get(), w.offsets.get(), pw, cap, w.targets.get(), vw, deterministic ? 1 : 0,
                   w.counts.get());
            GP_LAUNCH();
            if (deterministic) deterministic_ranks();
            launch(d, "bucket_scan_kernel", bucket_scan_kernel, k, kThreads, 0, w.counts.get(), w.offsets.get());
            launch(d, "select_destinations_kernel", select_destinations_kernel<W>, cgrid, kThreads, 0, ncand,
                   dev_count, w.cand.get(), w.bucket.get(), w.rank.get(), w.offsets.get(), pw, cap, vw, w.flags.get(),
                   w.movers.get(), ctr);
            GP_LAUNCH();
        };
        const int limit = 2 * k + 4;
        // Building the graph costs a few hundred microseconds per level, about
        // the host round trips of ten iterations: mode 1 captures once this
        // level's host loop has run kGraphLoopAfter iterations, mode 2 at once.
        if (!host_count && (d.graph_loops == 2 || (d.graph_loops == 1 && (rgraph.exec ||
                                                                           host_iterations >= kGraphLoopAfter))))
            return rebalance_on_device(select, limit);
        for (int it = 0; it < limit && maximum() > cap; ++it) {
            ++st.admission_iterations;
            ++host_iterations;
            select();
            const i64 moved = finish_apply(false);
            if (!moved) return false;
        }
        return maximum() <= cap;
    };
    int stale = 0, empty = 0;
    for (int phase = 0; phase < rounds && stale < 3; ++phase) {
        st.rounds = phase + 1;
        GP_CUDA(cudaMemsetAsync(ctr, 0, sizeof(RefineCounters), d.stream));
        d.prof_bytes("lp_proposals_kernel", static_cast<double>(n) * (k * sizeof(C) + 4 + 1 + 4 + 8));
        launch(d, "lp_proposals_kernel", lp_proposals_kernel<C>, blocks_for(n, kThreads), kThreads, 0, n, cache, labels, k,
               filter, max_edge_weight, w.locks.get(), w.targets.get(), w.gains.get(), w.props.get(), w.list.get(), ctr);
        if (d.prof) {
            // per proposer its list entry, offsets, record and flag; per edge
            // of a proposer below the hub degree its neighbour, weight and
            // the neighbour's 16-byte proposal record (filter_degree)
            RefineCounters pc{};
            launch(d, "filter_degree_kernel", filter_degree_kernel<O>, stride_grid(d, n), kThreads, 0, w.list.get(),
                   ctr, off, ctr);
            fetch(d, &pc, ctr, 1);
            d.prof_bytes("priority_filter_kernel",
                         static_cast<double>(pc.proposers) * (4 + 2 * sizeof(O) + sizeof(PropRec) + 1) +
                             static_cast<double>(pc.filter_degree) * (4 + (ew ? sizeof(W) : 0) + sizeof(PropRec)));
        }
        launch(d, "priority_filter_kernel", priority_filter_kernel<O, W>, stride_grid(d, n * 32), kThreads, 0,
               w.list.get(), ctr, off, nbr, ew, w.props.get(), w.flags.get(), w.movers.get(), ctr);
        if (hubs.count) {
            launch(d, "hub_filter_kernel", hub_filter_kernel<W>, static_cast<int>(hubs.chunks), kThreads, 0,
                   hubs.chunk.get(), nbr, ew, w.props.get(), hub_corr.get());
            launch(d, "hub_filter_finalize_kernel", hub_filter_finalize_kernel<O>, blocks_for(hubs.count, kThreads),
                   kThreads, 0, hubs.count, hubs.list.get(), off, w.targets.get(), w.gains.get(), hub_corr.get(),
                   w.flags.get(), w.movers.get(), ctr);
        }
        GP_LAUNCH();
        const i64 count = finish_apply(true);
        st.proposals += static_cast<u64>(count);
        if (!count) {
            if (++empty >= 2) break;
            ++stale;
            continue;
        }
        empty = 0;
        if (!rebalance()) { ++st.admission_fallbacks; break; }
        ++stale;
        if (current_cut < best_cut) {
            if (static_cast<long double>(current_cut) < 0.999L * best_cut) stale = 0;
            best_cut = current_cut;
            checkpoint();
        }
    }
    GP_CUDA(cudaMemcpyAsync(labels, w.saved_labels.get(), n * sizeof(i32), cudaMemcpyDeviceToDevice, d.stream));
    GP_CUDA(cudaMemcpyAsync(pw, w.saved_pw.get(), k * sizeof(u64), cudaMemcpyDeviceToDevice, d.stream));
    fetch(d, host_pw.data(), pw, static_cast<size_t>(k));
    st.final_cut = undirected_cut(d, g, labels, w.scratch.get());
    st.final_max_part_weight = maximum();
    if (st.final_cut != best_cut || st.final_cut > st.initial_cut || maximum() > cap)
        fail(GP_ERUNTIME, "incremental refinement postcondition failed");
    return st;
}

// Total directed edge weight of a level, saturated at 2^64 - 1 (m for unit
// weights, without a pass over the edges).
template <typename T>
u64 directed_total(Device& d, const DGraph<T>& g) {
    if (!g.ewp()) return static_cast<u64>(g.m);
    Buf<u64> s(d, 1);
    s.zero(d);
    launch(d, "sat_sum_kernel", sat_sum_kernel<typename T::W>, stride_grid(d, g.m), kThreads, 0, g.m, g.ewp(), s.get());
    GP_LAUNCH();
    u64 total = 0;
    fetch(d, &total, s.get(), 1);
    return total;
}

// The affinity cache can hold 32-bit sums when the level's total directed
// edge weight fits in 32 bits (whatever the graph width): no row sum can
// exceed it.
template <typename T>
bool narrow_cache(const DGraph<T>& g, Device& d) { return directed_total(d, g) <= 0xffffffffULL; }

// validate_refinement_gain_range (src/refine.cu:346-383): only the big width
// can exceed INT64_MAX/2 in total directed weight.
template <typename T>
void check_gain_range(u64 directed_total) {
    if (sizeof(typename T::W) == 8 && directed_total > static_cast<u64>(INT64_MAX) / 2)
        fail(GP_EOVERFLOW, "refinement signed gain range exceeded");
}

// range_checked: the caller ran check_gain_range on a level at least as heavy
// (a contraction only drops internal edges, so coarser levels weigh less).
template <typename T>
gp_refine_stats refine_dispatch(Device& d, const DGraph<T>& g, RefineWork& w, i32* labels, u64* pw,
                                std::vector<u64>& host_pw, int k, u64 cap, int rounds, bool det, bool verify, bool narrow,
                                bool range_checked = false, u64 known_cut = kUnknownCut) {
    if (!range_checked && sizeof(typename T::W) == 8) check_gain_range<T>(directed_total(d, g));
    if (narrow) return refine_level<T, u32>(d, g, w, labels, pw, host_pw, k, cap, rounds, det, verify, known_cut);
    return refine_level<T, u64>(d, g, w, labels, pw, host_pw, k, cap, rounds, det, verify, known_cut);
}

template <typename T>
void part_weights(Device& d, const DGraph<T>& g, const i32* labels, int k, u64* pw, std::vector<u64>& host) {
    GP_CUDA(cudaMemsetAsync(pw, 0, k * sizeof(u64), d.stream));
    launch(d, "part_weight_kernel", part_weight_kernel<typename T::W>, blocks_for(g.n, kThreads), kThreads, 0, g.n, labels, g.vwp(), pw);
    GP_LAUNCH();
    host.assign(static_cast<size_t>(k), 0);
    fetch(d, host.data(), pw, static_cast<size_t>(k));
}

struct UncoarsenResult {
    u64 cut = 0;
    u64 total_edge_weight = 0;
    std::vector<u64> pw;
};

// refine_hierarchy_impl (src/refine.cu:423-646) + uncoarsen_impl's report
// (src/uncoarsen.cu:39-97).  Consumes the hierarchy's levels.
template <typename T>
void uncoarsen(Device& d, Hierarchy<T>& h, Buf<i32>& labels, const Opts& o, u64 cap, UncoarsenResult& r, Log& log) {
    const int k = o.parts;
    RefineWork work;
    Buf<u64> pw(d, 32);
    std::vector<u64> host_pw;
    auto& coarsest = h.levels.back();
    // The finest level is the heaviest (a contraction only drops internal
    // edges), so its total decides the cache width and the gain range of
    // every level, and it is the reported total edge weight.
    const u64 directed = directed_total(d, h.levels.front());
    const bool narrow = directed <= 0xffffffffULL;
    part_weights(d, coarsest, labels.get(), k, pw.get(), host_pw);
    if (*std::max_element(host_pw.begin(), host_pw.end()) > cap)
        fail(GP_EINVAL, "initial refinement partition is imbalanced");
    check_gain_range<T>(directed);
    auto st = refine_dispatch(d, coarsest, work, labels.get(), pw.get(), host_pw, k, cap, o.max_rounds,
                              o.deterministic, o.verify, narrow, true);
    u64 last_cut = st.final_cut;
    i64 last_refined = coarsest.n;
    if (log.on)
        log.out << "refine_coarsest vertices=" << coarsest.n << " initial_cut=" << st.initial_cut
                << " final_cut=" << st.final_cut << " rounds=" << st.rounds << '\n';
    for (size_t lv = h.levels.size() - 1; lv > 0; --lv) {
        const size_t fine_level = lv - 1;
        auto& fine = h.levels[fine_level];
        Buf<i32> fine_labels(d, static_cast<size_t>(fine.n));
        launch(d, "project_kernel", project_kernel, blocks_for(fine.n, kThreads), kThreads, 0, fine.n, h.maps[fine_level].get(),
                                                                                labels.get(), fine_labels.get());
        GP_LAUNCH();
        labels = std::move(fine_labels);
        h.levels.pop_back();
        h.maps.pop_back();
        if (o.verify) {
            std::vector<u64> check;
            Buf<u64> pw2(d, 32);
            part_weights(d, fine, labels.get(), k, pw2.get(), check);
            const u64 c = undirected_cut(d, fine, labels.get(), work.scratch.get());
            if (c != last_cut || check != host_pw)
                fail(GP_ERUNTIME, "GPU projection failed cut or part-weight preservation");
        }
        const bool refine_this = fine_level == 0 || static_cast<double>(fine.n) >= o.growth * static_cast<double>(last_refined);
        gp_refine_stats ls{};
        if (refine_this) {
            ls = refine_dispatch(d, fine, work, labels.get(), pw.get(), host_pw, k, cap, o.max_rounds,
                                 o.deterministic, o.verify, narrow, true, last_cut);
            last_refined = fine.n;
        } else {
            ls.initial_cut = ls.final_cut = last_cut;
            ls.final_max_part_weight = *std::max_element(host_pw.begin(), host_pw.end());
        }
        last_cut = ls.final_cut;
        if (log.on)
            log.out << "uncoarsen_level=" << fine_level << " vertices=" << fine.n << " edge_entries=" << fine.m
                    << " projection_cut=" << ls.initial_cut << " refine_rounds=" << ls.rounds
                    << " refine_proposals=" << ls.proposals << " refine_accepted=" << ls.accepted
                    << " admission_iterations=" << ls.admission_iterations
                    << " admission_fallbacks=" << ls.admission_fallbacks << " refined_cut=" << ls.final_cut
                    << " refined_max_part_weight=" << ls.final_max_part_weight << '\n';
    }
    if (directed & 1ULL) fail(GP_ERUNTIME, "symmetric graph has odd directed edge weight");
    r.cut = last_cut;
    r.total_edge_weight = directed / 2;
    r.pw = host_pw;
}

// ---------------------------------------------------------------------------
// Input preparation: upload, narrowing and validation on the GPU with the
// rules and messages of src/graph.cpp:47-190.
// ---------------------------------------------------------------------------
// Offsets narrowed to the width's type and shifted down by `base` (the first
// edge of an instance inside a packed multi-graph CSR; 0 otherwise).
template <typename I, typename O>
__global__ void narrow_offsets_kernel(i64 n, const I* in, i64 base, O* out, i64 m, u32* err) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i > n) return;
    const i64 x = static_cast<i64>(in[i]) - base;
    if (x < 0 || x > m || (i > 0 && x < static_cast<i64>(in[i - 1]) - base)) set_error(err, kErrBadInput);
    out[i] = static_cast<O>(x);
}

__global__ void narrow_neighbors_kernel(i64 m, const i64* in, i32* out, i64 n, u32* err) {
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += static_cast<i64>(gridDim.x) * blockDim.x) {
        const i64 x = in[i];
        if (x < 0 || x >= n) set_error(err, kErrBadInput);
        out[i] = static_cast<i32>(x);
    }
}

template <typename O>
__global__ void check_offsets_kernel(i64 n, const O* off, i64 m, u32* err) {
    const i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i > n) return;
    const i64 x = static_cast<i64>(off[i]);
    if (x < 0 || x > m || (i > 0 && x < static_cast<i64>(off[i - 1])) || (i == 0 && x != 0) || (i == n && x != m))
        set_error(err, kErrBadInput);
}

__global__ void check_neighbors_kernel(i64 m, const i32* nbr, i64 n, u32* err) {
    for (i64 i = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += static_cast<i64>(gridDim.x) * blockDim.x)
        if (nbr[i] < 0 || nbr[i] >= n) set_error(err, kErrBadInput);
}

// --verify: every entry (v,u,w) has a reverse entry (u,v,w) found by binary
// search in u's row (validate_weighted_csr, src/graph.cpp:164-190).
template <typename O, typename W>
__global__ void symmetry_kernel(i64 n, const O* off, const i32* nbr, const W* ew, u32* err) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    for (i64 e = off[v]; e < static_cast<i64>(off[v + 1]); ++e) {
        const i32 u = nbr[e];
        i64 lo = off[u], hi = off[u + 1];
        while (lo < hi) {
            const i64 mid = lo + (hi - lo) / 2;
            if (nbr[mid] < v) lo = mid + 1; else hi = mid;
        }
        if (lo == static_cast<i64>(off[u + 1]) || nbr[lo] != v || weight_at(ew, e) != weight_at(ew, lo)) {
            set_error(err, kErrOddCut);
            return;
        }
    }
}

// `gi` describes the graph to partition; for one instance of a packed CSR its
// pointers are already advanced to the instance and `base` is the value of
// its first offset, which is subtracted from every offset.
template <typename T>
void prepare_graph(Device& d, const gp_graph* gi, DGraph<T>& g, bool verify, i64 base = 0) {
    using O = typename T::O;
    using W = typename T::W;
    if (!gi) fail(GP_EINVAL, "null graph");
    const i64 n = gi->n, m = gi->m;
    if (n < 0 || m < 0) fail(GP_EINVAL, "invalid graph size");
    if constexpr (std::is_same_v<T, Std>) {
        if (n > std::numeric_limits<i32>::max() || m > std::numeric_limits<i32>::max())
            fail(GP_ERUNTIME, "graph exceeds standard CSR limits; use gpart_coarsen_big");
    } else if (n > std::numeric_limits<i32>::max()) {
        fail(GP_ERUNTIME, "graph vertex ids exceed configured graph type");
    }
    const bool on_dev = gi->memory == GP_MEMORY_DEVICE;
    const cudaMemcpyKind kind = on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    g.n = n;
    g.m = m;
    // Device input in the width's own types is used in place (borrowed):
    // a resident graph is partitioned without a copy.
    // index64: 0 = arrays in the width's types, 1 = int64 offsets and
    // neighbours (the reference's file arrays), 2 = int64 offsets with int32
    // neighbours (a packed multi-graph CSR).  Device arrays in the width's
    // own types are used in place (borrowed): a resident graph is partitioned
    // without a copy.
    if (gi->index64 < 0 || gi->index64 > 2) fail(GP_EINVAL, "invalid index width");
    const bool nbr64 = gi->index64 == 1;
    const bool borrow_off = on_dev && gi->index64 == 0 && base == 0;
    const bool borrow_nbr = on_dev && !nbr64;
    if (borrow_off) g.off.borrow(static_cast<O*>(const_cast<void*>(gi->offsets)), static_cast<size_t>(n) + 1);
    else g.off = Buf<O>(d, static_cast<size_t>(n) + 1);
    if (borrow_nbr) g.nbr.borrow(static_cast<i32*>(const_cast<void*>(gi->neighbors)), static_cast<size_t>(m));
    else g.nbr = Buf<i32>(d, static_cast<size_t>(std::max<i64>(m, 1)));
    // device input is narrowed in place; host input goes through one staging buffer
    Buf<i64> stage;
    if (!on_dev && (gi->index64 != 0 || base != 0))
        stage = Buf<i64>(d, static_cast<size_t>(std::max<i64>(n + 1, nbr64 ? m : 0)));
    if (!borrow_off) {
        if (gi->index64 != 0) {
            const i64* src = static_cast<const i64*>(gi->offsets);
            if (!on_dev) {
                GP_CUDA(cudaMemcpyAsync(stage.get(), gi->offsets, (n + 1) * sizeof(i64), kind, d.stream));
                src = stage.get();
            }
            launch(d, "narrow_offsets_kernel", narrow_offsets_kernel<i64, O>, blocks_for(n + 1, kThreads), kThreads,
                   0, n, src, base, g.off.get(), m, d.err);
        } else if (base != 0) {
            const O* src = static_cast<const O*>(gi->offsets);
            if (!on_dev) {
                GP_CUDA(cudaMemcpyAsync(stage.get(), gi->offsets, (n + 1) * sizeof(O), kind, d.stream));
                src = reinterpret_cast<const O*>(stage.get());
            }
            launch(d, "narrow_offsets_kernel", narrow_offsets_kernel<O, O>, blocks_for(n + 1, kThreads), kThreads, 0,
                   n, src, base, g.off.get(), m, d.err);
        } else {
            GP_CUDA(cudaMemcpyAsync(g.off.get(), gi->offsets, (n + 1) * sizeof(O), kind, d.stream));
        }
        GP_LAUNCH();
    }
    if (!borrow_nbr && m) {
        if (nbr64) {
            const i64* src = static_cast<const i64*>(gi->neighbors);
            if (!on_dev) {
                GP_CUDA(cudaMemcpyAsync(stage.get(), gi->neighbors, m * sizeof(i64), kind, d.stream));
                src = stage.get();
            }
            launch(d, "narrow_neighbors_kernel", narrow_neighbors_kernel, stride_grid(d, m), kThreads, 0, m, src,
                   g.nbr.get(), n, d.err);
            GP_LAUNCH();
        } else {
            GP_CUDA(cudaMemcpyAsync(g.nbr.get(), gi->neighbors, m * sizeof(i32), kind, d.stream));
        }
    }
    launch(d, "check_offsets_kernel", check_offsets_kernel<O>, blocks_for(n + 1, kThreads), kThreads, 0, n, g.off.get(), m, d.err);
    if (!nbr64 && m) launch(d, "check_neighbors_kernel", check_neighbors_kernel, stride_grid(d, m), kThreads, 0, m, g.nbr.get(), n, d.err);
    GP_LAUNCH();
    g.unit_ew = gi->edge_weights == nullptr;
    g.unit_vw = gi->vertex_weights == nullptr;
    if (!g.unit_ew) {
        if (on_dev) {
            g.ew.borrow(static_cast<W*>(const_cast<void*>(gi->edge_weights)), static_cast<size_t>(m));
        } else {
            g.ew = Buf<W>(d, static_cast<size_t>(std::max<i64>(m, 1)));
            if (m) GP_CUDA(cudaMemcpyAsync(g.ew.get(), gi->edge_weights, m * sizeof(W), kind, d.stream));
        }
    }
    if (!g.unit_vw) {
        if (on_dev) {
            g.vw.borrow(static_cast<W*>(const_cast<void*>(gi->vertex_weights)), static_cast<size_t>(n));
        } else {
            g.vw = Buf<W>(d, static_cast<size_t>(std::max<i64>(n, 1)));
            if (n) GP_CUDA(cudaMemcpyAsync(g.vw.get(), gi->vertex_weights, n * sizeof(W), kind, d.stream));
        }
    }
    if (verify && n)
        launch(d, "symmetry_kernel", symmetry_kernel<O, W>, blocks_for(n, kThreads), kThreads, 0, n, g.off.get(), g.nbr.get(), g.ewp(), d.err);
    GP_LAUNCH();
    u32 e = 0;
    fetch(d, &e, d.err, 1);
    if (e) {
        GP_CUDA(cudaMemsetAsync(d.err, 0, sizeof(u32), d.stream));
        if (e & kErrOddCut) fail(GP_ERUNTIME, "weighted CSR is not bidirectional");
        fail(GP_ERUNTIME, "weighted CSR shape is invalid (offsets not monotone or neighbor out of range)");
    }
}

// Per-part counts of the reference's analyzer (graph_untils/
// analyze_partition.cpp:425-499) into `out` (kAnalyzeFields x parts, the
// layout of gp_analyze.cuh).  `labels` is a device array of n entries.
template <typename T>
void analyze_parts(Device& d, const DGraph<T>& g, const i32* labels, int parts, std::vector<u64>& out) {
    using O = typename T::O;
    using W = typename T::W;
    if (parts < 1 || parts > kAnalyzeMaxParts) fail(GP_EINVAL, "parts must be between 1 and 1024");
    const size_t cells = static_cast<size_t>(kAnalyzeFields) * static_cast<size_t>(parts);
    Buf<u64> acc(d, cells);
    acc.zero(d);
    const size_t smem = cells * sizeof(u64);
    auto rows = analyze_rows_kernel<O, W>;
    auto hubs_k = analyze_hub_kernel<W>;
    GP_CUDA(cudaFuncSetAttribute(rows, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    GP_CUDA(cudaFuncSetAttribute(hubs_k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    if (g.n) {
        // offsets, neighbour ids, their labels, weights, and each vertex's label
        d.prof_bytes("analyze_rows_kernel", static_cast<double>(g.n + 1) * sizeof(O) +
                                                static_cast<double>(g.m) * (8.0 + (g.ewp() ? sizeof(W) : 0)) +
                                                static_cast<double>(g.n) * 4.0);
        launch(d, "analyze_rows_kernel", rows, stride_grid(d, g.n * 32), kThreads, smem, g.n, g.off.get(), g.nbr.get(),
               g.ewp(), labels, parts, acc.get(), d.err);
        const auto& hubs = hub_index(d, g);
        if (hubs.count)
            launch(d, "analyze_hub_kernel", hubs_k, static_cast<int>(hubs.chunks), kThreads, smem, hubs.chunk.get(),
                   g.nbr.get(), g.ewp(), labels, parts, acc.get(), d.err);
        GP_LAUNCH();
    }
    d.check_errors();
    out.resize(cells);
    fetch(d, out.data(), acc.get(), cells);
}

// Sorts the directed keys (sentinels last), keeps the first of each run and
// writes the symmetric CSR: offsets (n + 1, device) and neighbours (device,
// `capacity` entries).  Returns the number of output entries; when it exceeds
// `capacity` nothing is written.
template <typename N>
i64 symmetrize_keys(Device& d, Buf<u64>& keys, Buf<u64>& alt, i64 total_keys, i64 valid, i64 n, int bits,
                    i64* out_off, N* out_nbr, i64 capacity, bool sorted) {
    if (!sorted) radix_sort<u64, i32>(d, keys.get(), nullptr, alt.get(), nullptr, total_keys, 0, 2 * bits);
    Buf<i64> rank(d, static_cast<size_t>(std::max<i64>(valid, 1))), tot(d, 1);
    exclusive_scan<i64>(d, SymHead{keys.get(), valid}, rank.get(), valid, tot.get());
    i64 out_m = 0;
    fetch(d, &out_m, tot.get(), 1);
    if (out_m > capacity) return out_m;
    Buf<i64> degree(d, static_cast<size_t>(std::max<i64>(n, 1)));
    degree.zero(d);
    if (valid)
        launch(d, "sym_compact_kernel", sym_compact_kernel<N>, stride_grid(d, valid), kThreads, 0, valid, keys.get(),
               rank.get(), bits, out_nbr, degree.get());
    exclusive_scan<i64>(d, ArrayInput<i64>{degree.get()}, out_off, n, out_off + n);
    GP_LAUNCH();
    return out_m;
}

// The symmetric CSR from 2m directed keys of which `valid` are not
// sentinels, into the caller's arrays (host or device), with the sizes in
// `info`; GP_EINVAL when `capacity` is too small.  `sorted`: the keys are
// sorted already.
void emit_symmetric(Device& d, Buf<u64>& keys, Buf<u64>& alt, i64 total_keys, i64 valid, i64 n, int bits, u64 self,
                    bool on_dev, i64* offsets_out, void* neighbors_out, int neighbor_bytes, i64 capacity,
                    gp_symmetrize_info* info, bool sorted = false);

inline int symmetrize_bits(i64 n) { return std::max(1, bit_width_u64(static_cast<u64>(std::max<i64>(n, 1) - 1))); }

void emit_symmetric(Device& d, Buf<u64>& keys, Buf<u64>& alt, i64 total_keys, i64 valid, i64 n, int bits, u64 self,
                    bool on_dev, i64* offsets_out, void* neighbors_out, int neighbor_bytes, i64 capacity,
                    gp_symmetrize_info* info, bool sorted) {
    Buf<i64> off_tmp;
    Buf<unsigned char> nbr_tmp;
    i64* off_dev = offsets_out;
    void* nbr_dev = neighbors_out;
    const i64 cap_dev = on_dev ? capacity : std::min<i64>(capacity, valid);
    if (!on_dev) {
        off_tmp = Buf<i64>(d, static_cast<size_t>(n) + 1);
        nbr_tmp = Buf<unsigned char>(d, static_cast<size_t>(std::max<i64>(cap_dev, 1)) * neighbor_bytes);
        off_dev = off_tmp.get();
        nbr_dev = nbr_tmp.get();
    }
    const i64 out_m = neighbor_bytes == 8
                          ? symmetrize_keys<i64>(d, keys, alt, total_keys, valid, n, bits, off_dev,
                                                 static_cast<i64*>(nbr_dev), cap_dev, sorted)
                          : symmetrize_keys<i32>(d, keys, alt, total_keys, valid, n, bits, off_dev,
                                                 static_cast<i32*>(nbr_dev), cap_dev, sorted);
    if (info) *info = gp_symmetrize_info{static_cast<int64_t>(self), out_m / 2, out_m};
    if (out_m > capacity)
        fail(GP_EINVAL, "neighbor capacity " + std::to_string(capacity) + " is below the " + std::to_string(out_m) +
                            " entries of the symmetric CSR");
    if (!on_dev) {
        to_host(d, offsets_out, off_dev, static_cast<size_t>(n) + 1);
        GP_CUDA(cudaMemcpyAsync(neighbors_out, nbr_dev, static_cast<size_t>(out_m) * neighbor_bytes,
                                cudaMemcpyDeviceToHost, d.stream));
    }
    d.sync();
}

template <typename T>
void host_level_copy(Device& d, const DGraph<T>& g, const i32* map, i64 map_n, std::vector<i64>& off,
                     std::vector<i32>& nbr, std::vector<u64>& ew, std::vector<u64>& vw, std::vector<i32>& mp) {
    using O = typename T::O;
    using W = typename T::W;
    std::vector<O> o(static_cast<size_t>(g.n) + 1);
    to_host(d, o.data(), g.off.get(), o.size());
    nbr.resize(static_cast<size_t>(g.m));
    to_host(d, nbr.data(), g.nbr.get(), nbr.size());
    std::vector<W> e, v;
    if (g.ewp()) { e.resize(static_cast<size_t>(g.m)); to_host(d, e.data(), g.ewp(), e.size()); }
    if (g.vwp()) { v.resize(static_cast<size_t>(g.n)); to_host(d, v.data(), g.vwp(), v.size()); }
    mp.resize(static_cast<size_t>(map ? map_n : 0));
    if (map) to_host(d, mp.data(), map, mp.size());
    d.sync();
    off.assign(o.begin(), o.end());
    ew.resize(static_cast<size_t>(g.m));
    vw.resize(static_cast<size_t>(g.n));
    for (i64 i = 0; i < g.m; ++i) ew[i] = g.ewp() ? static_cast<u64>(e[i]) : 1;
    for (i64 i = 0; i < g.n; ++i) vw[i] = g.vwp() ? static_cast<u64>(v[i]) : 1;
}

// ---------------------------------------------------------------------------
// Allocation-free spectral initial partition.
//
// Some callers cannot allocate device memory: a process whose device memory
// is owned by another allocator (a framework's pool that accounts for every
// byte, where a raw cudaMalloc bypasses its budget and can fail or fragment
// it), and latency-bound callers for which cudaMalloc's implicit
// synchronisation and unpredictable cost are not acceptable.  For small
// graphs -- the coarsest level of a hierarchy, at most kStaticMaxVertices
// vertices -- the recursive bisection runs entirely in a fixed scratch array
// that every GPU loading this library holds until exit.  The kernels are the
// ones of initial_partition(); only the memory comes from the array.
// ---------------------------------------------------------------------------
constexpr i64 kStaticMaxVertices = 65536;
constexpr size_t kStaticScratchBytes = size_t{4} << 20;   // 4 MiB
constexpr int kStaticMaxDepths = 6;
constexpr int kStaticMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct StaticScratch {
    u32* err;
    u32* bar;
    u64* stats;
    u64* loads;
    InitTask* tasks;   // kStaticMaxDepths x kMaxInitTasks
    i32* order;
    i32* task_of_pos;
    float* deg;
    float* xa;
    float* xb;
    Moments* contrib;
    u64* key;
    u64* key_alt;
    u64* prefix;
};

inline StaticScratch carve_static(unsigned char* base) {
    size_t at = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + at;
        at += (bytes + 255) & ~size_t{255};
        return p;
    };
    const size_t n = static_cast<size_t>(kStaticMaxVertices);
    StaticScratch s;
    s.err = reinterpret_cast<u32*>(take(sizeof(u32)));
    s.bar = reinterpret_cast<u32*>(take(2 * sizeof(u32)));
    s.stats = reinterpret_cast<u64*>(take(8 * sizeof(u64)));
    s.loads = reinterpret_cast<u64*>(take(33 * sizeof(u64)));
    s.tasks = reinterpret_cast<InitTask*>(take(kStaticMaxDepths * kMaxInitTasks * sizeof(InitTask)));
    s.order = reinterpret_cast<i32*>(take(n * sizeof(i32)));
    s.task_of_pos = reinterpret_cast<i32*>(take(n * sizeof(i32)));
    s.deg = reinterpret_cast<float*>(take(n * sizeof(float)));
    s.xa = reinterpret_cast<float*>(take(n * sizeof(float)));
    s.xb = reinterpret_cast<float*>(take(n * sizeof(float)));
    s.contrib = reinterpret_cast<Moments*>(take(n * sizeof(Moments)));
    s.key = reinterpret_cast<u64*>(take(n * sizeof(u64)));
    s.key_alt = reinterpret_cast<u64*>(take(n * sizeof(u64)));
    s.prefix = reinterpret_cast<u64*>(take(n * sizeof(u64)));
    if (at > kStaticScratchBytes) fail(GP_ERUNTIME, "static scratch layout exceeds its array");
    return s;
}

// Device address of the scratch array on the current device, looked up once
// per device with cudaGetSymbolAddress (a host-side reference to the array
// is not a device address).
inline unsigned char* static_scratch_address() {
    static std::mutex mutex;
    static unsigned char* address[kStaticMaxDevices] = {};
    int dev = 0;
    GP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kStaticMaxDevices) fail(GP_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(mutex);
    if (!address[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) fail(GP_ECUDA, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        address[dev] = static_cast<unsigned char*>(p);
    }
    return address[dev];
}

template <typename T>
void initial_partition_static(const gp_graph* gi, int parts, double ratio, u32 seed, i32* labels,
                              cudaStream_t stream) {
    using O = typename T::O;
    using W = typename T::W;
    if (!gi || gi->memory != GP_MEMORY_DEVICE || gi->index64)
        fail(GP_EINVAL, "the graph must be in device memory in the width's own types");
    if (!labels) fail(GP_EINVAL, "labels must be a device array of n entries");
    const i64 n64 = gi->n;
    if (n64 > kStaticMaxVertices)
        fail(GP_EINVAL, "graph has " + std::to_string(n64) + " vertices; the allocation-free initial partition "
                        "supports at most " + std::to_string(kStaticMaxVertices));
    if (n64 <= 0 || gi->m < 0 || parts < 2 || parts > n64 || parts > 32 || !std::isfinite(ratio) || ratio < 1.0)
        fail(GP_EINVAL, "invalid GPU initial partition input");
    if constexpr (std::is_same_v<T, Std>) {
        if (gi->m > std::numeric_limits<i32>::max()) fail(GP_EINVAL, "graph exceeds standard CSR limits");
    }
    const i32 n = static_cast<i32>(n64);
    const StaticScratch sc = carve_static(static_scratch_address());

    // A Device without an allocator: launches, stream and error word only.
    Device d;
    GP_CUDA(cudaGetDevice(&d.device));
    GP_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, d.device));
    d.stream = stream;
    d.err = sc.err;
    auto read = [&](void* host, const void* dev, size_t bytes) {
        GP_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, stream));
        GP_CUDA(cudaStreamSynchronize(stream));
    };
    // The array keeps the previous call's contents: clear what starts at zero.
    GP_CUDA(cudaMemsetAsync(sc.err, 0, sizeof(u32), stream));
    GP_CUDA(cudaMemsetAsync(sc.stats, 0, 8 * sizeof(u64), stream));
    GP_CUDA(cudaMemsetAsync(sc.loads, 0, 33 * sizeof(u64), stream));
    GP_CUDA(cudaMemsetAsync(labels, 0, static_cast<size_t>(n) * sizeof(i32), stream));

    DGraph<T> g;   // borrowed views of the caller's arrays
    g.n = n64;
    g.m = gi->m;
    g.off.borrow(static_cast<O*>(const_cast<void*>(gi->offsets)), static_cast<size_t>(n) + 1);
    g.nbr.borrow(static_cast<i32*>(const_cast<void*>(gi->neighbors)), static_cast<size_t>(gi->m));
    g.unit_ew = gi->edge_weights == nullptr;
    g.unit_vw = gi->vertex_weights == nullptr;
    if (!g.unit_ew) g.ew.borrow(static_cast<W*>(const_cast<void*>(gi->edge_weights)), static_cast<size_t>(gi->m));
    if (!g.unit_vw) g.vw.borrow(static_cast<W*>(const_cast<void*>(gi->vertex_weights)), static_cast<size_t>(n));

    // The caller's CSR is read in place, so check its shape before any kernel
    // follows an offset or a neighbour id: offsets monotone from 0 to m, ids
    // in [0, n).  The checks record a flag and never read out of bounds.
    launch(d, "check_offsets_kernel", check_offsets_kernel<O>, blocks_for(n64 + 1, kThreads), kThreads, 0, n64,
           g.off.get(), g.m, sc.err);
    if (g.m)
        launch(d, "check_neighbors_kernel", check_neighbors_kernel, stride_grid(d, g.m), kThreads, 0, g.m, g.nbr.get(),
               n64, sc.err);
    u32 shape_err = 0;
    read(&shape_err, sc.err, sizeof(shape_err));
    if (shape_err)
        fail(GP_EINVAL, "weighted CSR shape is invalid (offsets not monotone from 0 to m or neighbor out of range)");

    launch(d, "weight_stats_kernel", weight_stats_kernel<W>, stride_grid(d, n), kThreads, 0, n, g.vwp(), sc.stats);
    launch(d, "sat_sum_kernel", sat_sum_kernel<W>, stride_grid(d, g.m), kThreads, 0, g.m, g.ewp(), sc.stats + 2);
    u64 st[3];
    read(st, sc.stats, sizeof(st));
    const u64 total = st[0], maxw = st[1], edge_total = st[2];
    if (!total || total == ~0ULL || edge_total == ~0ULL)
        fail(GP_EOVERFLOW, "GPU initializer weight accumulation overflow");
    const u64 capacity = partition_capacity(total, parts, ratio);
    if (maxw > capacity) fail(GP_EINVAL, "a vertex exceeds partition capacity");

    auto depths = plan_tasks(parts);
    if (static_cast<int>(depths.size()) > kStaticMaxDepths) fail(GP_ERUNTIME, "task tree deeper than expected");
    depths[0].tasks[0].count = n;
    depths[0].tasks[0].weight = total;
    for (size_t dpt = 0; dpt < depths.size(); ++dpt)
        GP_CUDA(cudaMemcpyAsync(sc.tasks + dpt * kMaxInitTasks, depths[dpt].tasks.data(),
                                depths[dpt].tasks.size() * sizeof(InitTask), cudaMemcpyHostToDevice, stream));
    launch(d, "iota_kernel", iota_kernel, blocks_for(n, kThreads), kThreads, 0, n, sc.order);
    for (size_t dpt = 0; dpt < depths.size(); ++dpt) {
        const int nt = static_cast<int>(depths[dpt].tasks.size());
        InitTask* tasks = sc.tasks + dpt * kMaxInitTasks;
        GP_CUDA(cudaMemsetAsync(sc.task_of_pos, 0xff, static_cast<size_t>(n) * sizeof(i32), stream));
        launch(d, "task_positions_kernel", task_positions_kernel, nt, kThreads, 0, nt, tasks, sc.task_of_pos);
        launch_diffusion(d, g, nt, tasks, sc.task_of_pos, n, sc.order, labels, seed, 64, sc.deg, sc.xa, sc.xb,
                         sc.contrib, nullptr, sc.key, sc.bar);
        launch(d, "task_sort_kernel", task_sort_kernel, nt, kThreads, 0, nt, tasks, sc.key, sc.key_alt, sc.order);
        InitTask* next = dpt + 1 < depths.size() ? sc.tasks + (dpt + 1) * kMaxInitTasks : nullptr;
        launch(d, "task_split_kernel", task_split_kernel<W>, nt, kThreads, 0, nt, tasks, next, sc.order, g.vwp(),
               capacity, sc.prefix, labels, sc.err);
    }
    launch(d, "part_weight_kernel", part_weight_kernel<W>, blocks_for(n, kThreads), kThreads, 0, n, labels, g.vwp(),
           sc.loads);
    u32 e = 0;
    read(&e, sc.err, sizeof(e));
    if (e & kErrTimeout) fail(GP_ETIMEOUT, "a bounded device wait timed out");
    if (e & kErrSplit) fail(GP_ERUNTIME, "GPU spectral split cannot satisfy capacity");
    if (e & kErrBalance) fail(GP_ERUNTIME, "GPU initializer infeasible balance");
    if (e) fail(GP_ERUNTIME, "device error during the initial partition");
    u64 loads[32];
    read(loads, sc.loads, static_cast<size_t>(parts) * sizeof(u64));
    if (*std::max_element(loads, loads + parts) > capacity) fail(GP_ERUNTIME, "GPU initializer balance validation failed");
}

}  // namespace gp

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct gp_ctx {
    gp::Device dev;
    std::string error;
};

struct gp_hierarchy {
    struct Level {
        std::vector<int64_t> off;
        std::vector<int32_t> nbr;
        std::vector<uint64_t> ew, vw;
        std::vector<int32_t> map;   // to the next level
    };
    std::vector<Level> levels;
    std::string stop_reason;
};

namespace {

template <typename F>
gp_status guarded(gp_ctx* ctx, F&& f) {
    try {
        f();
        if (ctx) ctx->error.clear();
        return GP_OK;
    } catch (const gp::Error& e) {
        if (ctx) ctx->error = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->error = "host allocation failed";
        return GP_ENOMEM;
    } catch (const std::exception& e) {
        if (ctx) ctx->error = e.what();
        return GP_ERUNTIME;
    }
}

template <typename F>
void with_width(const gp_graph* g, F&& f) {
    if (!g) gp::fail(GP_EINVAL, "null graph");
    if (g->width == GP_WIDTH_BIG) f(gp::Big{});
    else if (g->width == GP_WIDTH_STANDARD) f(gp::Std{});
    else gp::fail(GP_EINVAL, "invalid graph width");
}

}  // namespace

extern "C" {

void gp_options_default(gp_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->parts = 4;
    o->cluster_size_factor = 0;
    o->imbalance = 1.03;
    o->seed = 0;
    o->pack_isolated = 1;
    o->max_levels = 24;
    o->max_rounds = 32;
    o->stop_ratio = 0.90;
    o->growth_ratio = 2.0;
}

gp_status gp_ctx_create(int device, gp_ctx** out) {
    if (!out) return GP_EINVAL;
    auto ctx = std::make_unique<gp_ctx>();
    const gp_status s = guarded(ctx.get(), [&] {
        auto& d = ctx->dev;
        d.device = device;
        GP_CUDA(cudaSetDevice(device));
        GP_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device));
        size_t free_bytes = 0;
        GP_CUDA(cudaMemGetInfo(&free_bytes, &d.total_bytes));   // once: the query costs milliseconds
        GP_CUDA(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
        GP_CUDA(cudaMalloc(&d.err, 64));
        GP_CUDA(cudaMemset(d.err, 0, 64));
        GP_CUDA(cudaMallocHost(&d.pinned, gp::Device::kPinnedBytes));
    });
    if (s != GP_OK) {
        *out = nullptr;
        return s;
    }
    *out = ctx.release();
    return GP_OK;
}

void gp_ctx_destroy(gp_ctx* ctx) {
    if (!ctx) return;
    auto& d = ctx->dev;
    cudaSetDevice(d.device);
    if (d.stream) cudaStreamSynchronize(d.stream);
    d.release_cached();
    for (auto& kv : d.live) d.driver_free(kv.first);
    d.live.clear();
    for (auto e : d.event_pool) cudaEventDestroy(e);
    if (d.sync_event) cudaEventDestroy(d.sync_event);
    if (d.err) cudaFree(d.err);
    if (d.pinned) cudaFreeHost(d.pinned);
    if (d.stream) cudaStreamDestroy(d.stream);
    delete ctx;
}

const char* gp_ctx_error(const gp_ctx* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

gp_status gp_ctx_set_device_share(gp_ctx* ctx, int share) {
    if (!ctx || share < 1) return GP_EINVAL;
    ctx->dev.share = share;
    return GP_OK;
}

gp_status gp_ctx_set_small_diffusion(gp_ctx* ctx, int enable) {
    if (!ctx) return GP_EINVAL;
    ctx->dev.small_diffusion = enable != 0;
    return GP_OK;
}

gp_status gp_ctx_set_hub_tables(gp_ctx* ctx, int on_chip) {
    if (!ctx) return GP_EINVAL;
    ctx->dev.hub_chip = on_chip != 0;
    return GP_OK;
}

gp_status gp_ctx_set_graph_loops(gp_ctx* ctx, int mode) {
    if (!ctx || mode < 0 || mode > 2) return GP_EINVAL;
    ctx->dev.graph_loops = mode;
    return GP_OK;
}

gp_status gp_ctx_set_sync_mode(gp_ctx* ctx, int blocking) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        auto& d = ctx->dev;
        GP_CUDA(cudaSetDevice(d.device));
        if (blocking && !d.sync_event)
            GP_CUDA(cudaEventCreateWithFlags(&d.sync_event, cudaEventBlockingSync | cudaEventDisableTiming));
        d.blocking_sync = blocking != 0;
    });
}

gp_status gp_partition_capacity(uint64_t total, int parts, double ratio, uint64_t* out) {
    return guarded(nullptr, [&] { *out = gp::partition_capacity(total, parts, ratio); });
}

}  // extern "C"

namespace {

// The whole pipeline on one graph; `graph` may be a view of one instance of a
// packed CSR, whose offsets start at `base` instead of 0.
gp_status partition_impl(gp_ctx* ctx, const gp_graph* graph, gp::i64 base, const gp_options* options,
                         int32_t* labels, gp_report* report) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        const gp::Opts o = gp::to_opts(options);
        gp::Log log;
        log.on = options && options->log;
        gp_report rep{};
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            rep.n = graph->n;
            rep.m = graph->m;
            gp::partition_capacity(static_cast<gp::u64>(graph->n), o.parts, o.ratio);
            if (!d.pressure) {
                // a graph projected to take more than half the device reuses
                // cached blocks by exact size class only (Device::cached_for)
                const gp::u64 fp = gp_footprint_bytes(graph->n, graph->m, o.parts, graph->width,
                                                      graph->index64 && graph->memory == GP_MEMORY_HOST);
                if (fp > d.total_bytes / 2) d.pressure = true;
            }
            const auto prep_start = gp::Clock::now();
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, o.verify, base);
            d.sync();
            rep.prepare_seconds = gp::seconds_since(prep_start);
            // algorithm_total_seconds scope (app/partition_main.cu:67-93)
            const auto t0 = gp::Clock::now();
            gp::u64 total = 0;
            {
                gp::Buf<gp::u64> s(d, 2);
                s.zero(d);
                launch(d, "weight_stats_kernel", gp::weight_stats_kernel<typename T::W>, gp::stride_grid(d, g.n), gp::kThreads, 0, 
                    g.n, g.vwp(), s.get());
                GP_LAUNCH();
                gp::fetch(d, &total, s.get(), 1);
            }
            const gp::u64 cap = gp::partition_capacity(total, o.parts, o.ratio);
            gp::Hierarchy<T> h;
            gp::coarsen<T>(d, std::move(g), o, h, log);
            d.sync();
            const auto t1 = gp::Clock::now();
            rep.levels = static_cast<int32_t>(h.levels.size());
            rep.coarsest_n = h.levels.back().n;
            gp::Buf<gp::i32> lab;
            gp::initial_partition<T>(d, h.levels.back(), o.parts, o.ratio, o.seed, lab, &rep.initial_cut, log);
            d.sync();
            const auto t2 = gp::Clock::now();
            gp::UncoarsenResult ur;
            gp::uncoarsen<T>(d, h, lab, o, cap, ur, log);
            d.sync();
            const auto t3 = gp::Clock::now();
            h.levels.clear();
            h.maps.clear();
            d.sync();
            const auto t4 = gp::Clock::now();
            if (gp::trace().on)
                std::fprintf(stderr, "trace allocations %llu calls (%llu from the driver), %.3f ms in the allocator\n",
                             static_cast<unsigned long long>(d.alloc_calls),
                             static_cast<unsigned long long>(d.driver_allocs), d.alloc_ms);
            rep.coarsen_seconds = std::chrono::duration<double>(t1 - t0).count();
            rep.initial_seconds = std::chrono::duration<double>(t2 - t1).count();
            rep.uncoarsen_seconds = std::chrono::duration<double>(t3 - t2).count();
            rep.free_seconds = std::chrono::duration<double>(t4 - t3).count();
            rep.algorithm_seconds = std::chrono::duration<double>(t4 - t0).count();
            rep.cut = ur.cut;
            rep.capacity = cap;
            rep.total_edge_weight = ur.total_edge_weight;
            for (size_t i = 0; i < ur.pw.size() && i < 32; ++i) rep.part_weights[i] = ur.pw[i];
            if (labels) {
                const bool dev_out = graph->memory == GP_MEMORY_DEVICE;
                GP_CUDA(cudaMemcpyAsync(labels, lab.get(), graph->n * sizeof(int32_t),
                                        dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, d.stream));
            }
            lab.reset();
            d.sync();
            if (log.on) {
                const gp::u64 mx = ur.pw.empty() ? 0 : *std::max_element(ur.pw.begin(), ur.pw.end());
                std::cout << std::setprecision(10) << "final_edge_cut=" << ur.cut << '\n'
                          << "final_cut_ratio="
                          << (ur.total_edge_weight == 0 ? 0.0 : static_cast<double>(ur.cut) / ur.total_edge_weight)
                          << '\n'
                          << "final_max_part_weight=" << mx << '\n'
                          << "final_imbalance="
                          << (total == 0 ? 0.0 : static_cast<double>(mx) * o.parts / static_cast<double>(total)) << '\n';
            }
        });
        if (report) *report = rep;
    });
}

}  // namespace

extern "C" {

gp_status gp_partition(gp_ctx* ctx, const gp_graph* graph, const gp_options* options, int32_t* labels,
                       gp_report* report) {
    return partition_impl(ctx, graph, 0, options, labels, report);
}

gp_status gp_partition_range(gp_ctx* ctx, const gp_graph* packed, int64_t vertex_begin, int64_t vertex_end,
                             const gp_options* options, int32_t* labels, gp_report* report) {
    if (!ctx) return GP_EINVAL;
    gp_graph view{};
    gp::i64 base = 0;
    const gp_status s = guarded(ctx, [&] {
        if (!packed) gp::fail(GP_EINVAL, "null graph");
        if (vertex_begin < 0 || vertex_end < vertex_begin || vertex_end > packed->n)
            gp::fail(GP_EINVAL, "instance range outside the packed graph");
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        const bool wide = packed->index64 || packed->width == GP_WIDTH_BIG;
        const size_t osize = wide ? 8 : 4;
        const size_t isize = packed->index64 == 1 ? 8 : 4;
        const size_t wsize = packed->width == GP_WIDTH_BIG ? 8 : 4;
        const auto* off = static_cast<const unsigned char*>(packed->offsets);
        auto read_offset = [&](gp::i64 v) -> gp::i64 {
            unsigned char raw[8] = {};
            if (packed->memory == GP_MEMORY_DEVICE)
                GP_CUDA(cudaMemcpy(raw, off + v * osize, osize, cudaMemcpyDeviceToHost));
            else
                std::memcpy(raw, off + v * osize, osize);
            if (wide) { int64_t x; std::memcpy(&x, raw, 8); return x; }
            int32_t x;
            std::memcpy(&x, raw, 4);
            return x;
        };
        const gp::i64 first = read_offset(vertex_begin), last = read_offset(vertex_end);
        if (first < 0 || last < first || last > packed->m)
            gp::fail(GP_ERUNTIME, "weighted CSR shape is invalid (offsets not monotone or neighbor out of range)");
        base = first;
        view = *packed;
        view.n = vertex_end - vertex_begin;
        view.m = last - first;
        view.offsets = off + vertex_begin * osize;
        view.neighbors = static_cast<const unsigned char*>(packed->neighbors) + base * isize;
        if (packed->edge_weights)
            view.edge_weights = static_cast<const unsigned char*>(packed->edge_weights) + base * wsize;
        if (packed->vertex_weights)
            view.vertex_weights = static_cast<const unsigned char*>(packed->vertex_weights) + vertex_begin * wsize;
    });
    if (s != GP_OK) return s;
    return partition_impl(ctx, &view, base, options, labels, report);
}

gp_status gp_ctx_memory(gp_ctx* ctx, uint64_t* live, uint64_t* cached, uint64_t* peak, int reset_peak) {
    if (!ctx) return GP_EINVAL;
    auto& d = ctx->dev;
    if (live) *live = d.live_bytes;
    if (cached) *cached = d.cached_bytes;
    if (peak) *peak = d.peak_bytes;
    if (reset_peak) d.peak_bytes = d.live_bytes;
    return GP_OK;
}

gp_status gp_ctx_allocator_stats(gp_ctx* ctx, uint64_t* requests, uint64_t* driver_allocs, uint64_t* cache_frees,
                                 double* host_ms) {
    if (!ctx) return GP_EINVAL;
    if (requests) *requests = ctx->dev.alloc_calls;
    if (driver_allocs) *driver_allocs = ctx->dev.driver_allocs;
    if (cache_frees) *cache_frees = ctx->dev.cache_frees;
    if (host_ms) *host_ms = ctx->dev.alloc_ms;
    return GP_OK;
}

gp_status gp_ctx_trim(gp_ctx* ctx) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        ctx->dev.release_cached();
    });
}

gp_status gp_aggregate(gp_ctx* ctx, const gp_graph* graph, int parts, uint32_t seed, int level,
                       int cluster_size_factor, int pack_isolated, int32_t* map, int64_t* coarse_n,
                       uint64_t* cluster_cap) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, false);
            gp::SclpWork<T> w;
            gp::AggResult<T> r;
            gp::Log log;
            gp::aggregate<T>(d, g, w, parts, seed, level, cluster_size_factor, pack_isolated != 0, r, log);
            d.check_errors();
            if (map) gp::to_host(d, map, r.map.get(), static_cast<size_t>(g.n));
            d.sync();
            if (coarse_n) *coarse_n = r.coarse_n;
            if (cluster_cap) *cluster_cap = r.cap;
        });
    });
}

gp_status gp_contract(gp_ctx* ctx, const gp_graph* graph, const int32_t* map, int64_t coarse_n, int64_t* offsets,
                      int32_t* neighbors, uint64_t* edge_weights, uint64_t* vertex_weights, int64_t* coarse_m) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            using W = typename T::W;
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, false);
            if (coarse_n <= 0 || coarse_n > g.n) gp::fail(GP_EINVAL, "invalid coarse vertex count");
            gp::Buf<gp::i32> dmap(d, static_cast<size_t>(g.n));
            gp::to_device(d, dmap.get(), map, static_cast<size_t>(g.n));
            gp::Buf<W> cvw(d, static_cast<size_t>(coarse_n));
            cvw.zero(d);
            launch(d, "coarse_weights_kernel", gp::coarse_weights_kernel<W>, gp::blocks_for(g.n, gp::kThreads), gp::kThreads, 0, 
                g.n, dmap.get(), g.vwp(), cvw.get());
            GP_LAUNCH();
            gp::DGraph<T> c;
            gp::contract<T>(d, g, dmap.get(), coarse_n, std::move(cvw), c);
            std::vector<int64_t> off;
            std::vector<int32_t> nbr, mp;
            std::vector<uint64_t> ew, vw;
            gp::host_level_copy<T>(d, c, nullptr, 0, off, nbr, ew, vw, mp);
            std::copy(off.begin(), off.end(), offsets);
            std::copy(nbr.begin(), nbr.end(), neighbors);
            std::copy(ew.begin(), ew.end(), edge_weights);
            std::copy(vw.begin(), vw.end(), vertex_weights);
            *coarse_m = c.m;
        });
    });
}

gp_status gp_coarsen(gp_ctx* ctx, const gp_graph* graph, const gp_options* options, gp_hierarchy** out) {
    if (!ctx || !out) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        const gp::Opts o = gp::to_opts(options);
        gp::Log log;
        log.on = options && options->log;
        auto res = std::make_unique<gp_hierarchy>();
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, o.verify);
            gp::Hierarchy<T> h;
            gp::coarsen<T>(d, std::move(g), o, h, log);
            res->stop_reason = h.stop_reason;
            for (size_t i = 0; i < h.levels.size(); ++i) {
                gp_hierarchy::Level L;
                const gp::i32* mp = i < h.maps.size() ? h.maps[i].get() : nullptr;
                gp::host_level_copy<T>(d, h.levels[i], mp, h.levels[i].n, L.off, L.nbr, L.ew, L.vw, L.map);
                res->levels.push_back(std::move(L));
            }
        });
        *out = res.release();
    });
}

int32_t gp_hierarchy_levels(const gp_hierarchy* h) { return h ? static_cast<int32_t>(h->levels.size()) : 0; }

gp_status gp_hierarchy_level(const gp_hierarchy* h, int level, int64_t* n, int64_t* m, int64_t* offsets,
                             int32_t* neighbors, uint64_t* edge_weights, uint64_t* vertex_weights,
                             int32_t* map_to_next) {
    if (!h || level < 0 || level >= static_cast<int>(h->levels.size())) return GP_EINVAL;
    const auto& L = h->levels[level];
    if (n) *n = static_cast<int64_t>(L.vw.size());
    if (m) *m = static_cast<int64_t>(L.nbr.size());
    if (offsets) std::copy(L.off.begin(), L.off.end(), offsets);
    if (neighbors) std::copy(L.nbr.begin(), L.nbr.end(), neighbors);
    if (edge_weights) std::copy(L.ew.begin(), L.ew.end(), edge_weights);
    if (vertex_weights) std::copy(L.vw.begin(), L.vw.end(), vertex_weights);
    if (map_to_next) std::copy(L.map.begin(), L.map.end(), map_to_next);
    return GP_OK;
}

gp_status gp_hierarchy_write(const gp_hierarchy* h, const char* path) {
    if (!h || !path) return GP_EINVAL;
    return guarded(nullptr, [&] {
        const std::string tmp = std::string(path) + ".tmp";
        {
            std::ofstream o(tmp, std::ios::binary | std::ios::trunc);
            if (!o) gp::fail(GP_ERUNTIME, "cannot open hierarchy temporary file");
            auto put = [&](int32_t v) { o.write(reinterpret_cast<const char*>(&v), 4); };
            put(static_cast<int32_t>(h->levels.size()));
            for (size_t i = 0; i < h->levels.size(); ++i) {
                const auto& L = h->levels[i];
                if (L.vw.size() > static_cast<size_t>(INT32_MAX) || L.nbr.size() > static_cast<size_t>(INT32_MAX))
                    gp::fail(GP_ERUNTIME, "hierarchy export requires 32-bit dimensions");
                put(static_cast<int32_t>(L.vw.size()));
                put(static_cast<int32_t>(L.nbr.size()));
                for (auto x : L.off) put(static_cast<int32_t>(x));
                for (auto x : L.nbr) put(x);
                for (auto x : L.ew) {
                    if (x > static_cast<uint64_t>(INT32_MAX)) gp::fail(GP_ERUNTIME, "hierarchy edge weight exceeds int32");
                    put(static_cast<int32_t>(x));
                }
                for (auto x : L.vw) {
                    if (x > static_cast<uint64_t>(INT32_MAX)) gp::fail(GP_ERUNTIME, "hierarchy vertex weight exceeds int32");
                    put(static_cast<int32_t>(x));
                }
                if (i > 0) for (auto x : h->levels[i - 1].map) put(x);
            }
            o.flush();
            if (!o) gp::fail(GP_ERUNTIME, "failed while writing hierarchy");
        }
        if (std::rename(tmp.c_str(), path) != 0) gp::fail(GP_ERUNTIME, "cannot commit hierarchy output");
    });
}

void gp_hierarchy_free(gp_hierarchy* h) { delete h; }

gp_status gp_initial_partition(gp_ctx* ctx, const gp_graph* graph, int parts, double ratio, uint32_t seed,
                               int32_t* labels) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, false);
            gp::Buf<gp::i32> lab;
            gp::Log log;
            gp::initial_partition<T>(d, g, parts, ratio, seed, lab, nullptr, log);
            gp::to_host(d, labels, lab.get(), static_cast<size_t>(g.n));
            d.sync();
        });
    });
}

gp_status gp_initial_partition_trace(gp_ctx* ctx, const gp_graph* graph, int parts, double ratio, uint32_t seed,
                                     int32_t* labels, float* trace, int32_t trace_depths, int32_t* depths) {
    if (!ctx || !depths) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        const int needed = static_cast<int>(gp::plan_tasks(std::max(2, std::min(parts, 32))).size());
        *depths = needed;
        if (trace && trace_depths < needed) gp::fail(GP_EINVAL, "trace holds fewer depths than the task tree");
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, false);
            const size_t cells = static_cast<size_t>(needed) * static_cast<size_t>(std::max<gp::i64>(g.n, 1));
            gp::Buf<float> dev_trace;
            if (trace) {
                dev_trace = gp::Buf<float>(d, cells);
                GP_CUDA(cudaMemsetAsync(dev_trace.get(), 0xff, cells * sizeof(float), d.stream));   // NaN marker
            }
            gp::Buf<gp::i32> lab;
            gp::Log log;
            gp::initial_partition<T>(d, g, parts, ratio, seed, lab, nullptr, log, trace ? dev_trace.get() : nullptr);
            gp::to_host(d, labels, lab.get(), static_cast<size_t>(g.n));
            if (trace) gp::to_host(d, trace, dev_trace.get(), static_cast<size_t>(needed) * static_cast<size_t>(g.n));
            d.sync();
        });
    });
}

gp_status gp_diffusion(gp_ctx* ctx, const gp_graph* graph, const int32_t* labels, int group, uint32_t seed, int steps,
                       float* x) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, false);
            const gp::i32 n = static_cast<gp::i32>(g.n);
            std::vector<gp::i32> members;
            for (gp::i32 v = 0; v < n; ++v) if (labels[v] == group) members.push_back(v);
            if (members.empty()) gp::fail(GP_EINVAL, "empty diffusion group");
            gp::Buf<gp::i32> dl(d, static_cast<size_t>(n)), order(d, static_cast<size_t>(n)), top(d, static_cast<size_t>(n));
            gp::to_device(d, dl.get(), labels, static_cast<size_t>(n));
            std::vector<gp::i32> ord(members);
            std::vector<gp::i32> tp(static_cast<size_t>(n), -1);
            for (size_t i = 0; i < members.size(); ++i) tp[i] = 0;
            ord.resize(static_cast<size_t>(n), 0);
            gp::to_device(d, order.get(), ord.data(), ord.size());
            gp::to_device(d, top.get(), tp.data(), tp.size());
            gp::InitTask task{0, static_cast<gp::i32>(members.size()), group, 2, 0, -1, -1};
            gp::Buf<gp::InitTask> dt(d, 1);
            gp::to_device(d, dt.get(), &task, 1);
            gp::Buf<float> deg(d, n), xa(d, n), xb(d, n), xo(d, n);
            gp::Buf<gp::Moments> contrib(d, n);
            gp::Buf<gp::u64> key(d, n);
            gp::Buf<gp::u32> bar(d, 2);
            xo.zero(d);
            gp::Buf<gp::u64> md(d, 1);
            md.zero(d);
            gp::launch(d, "max_degree_kernel", gp::max_degree_kernel<typename T::O>, gp::stride_grid(d, g.n), gp::kThreads,
                       0, g.n, g.off.get(), md.get());
            gp::u64 max_degree = 0;
            gp::fetch(d, &max_degree, md.get(), 1);
            gp::launch_diffusion<T>(d, g, 1, dt.get(), top.get(), n, order.get(), dl.get(), seed, steps, deg.get(),
                                    xa.get(), xb.get(), contrib.get(), xo.get(), key.get(), bar.get(),
                                    static_cast<gp::i64>(max_degree));
            d.check_errors();
            gp::to_host(d, x, xo.get(), static_cast<size_t>(n));
            d.sync();
        });
    });
}

gp_status gp_refine(gp_ctx* ctx, const gp_graph* graph, int32_t* labels, int parts, double ratio, int max_rounds,
                    int deterministic, gp_refine_stats* stats) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        if (parts < 2 || parts > 32 || max_rounds < 0 || max_rounds > 64 || !std::isfinite(ratio) || ratio < 1.0 ||
            !graph || graph->n <= 0)
            gp::fail(GP_EINVAL, "invalid refinement options");
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, false);
            for (gp::i64 v = 0; v < g.n; ++v)
                if (labels[v] < 0 || labels[v] >= parts) gp::fail(GP_EINVAL, "refinement partition has an invalid part id");
            gp::Buf<gp::i32> lab(d, static_cast<size_t>(g.n));
            gp::to_device(d, lab.get(), labels, static_cast<size_t>(g.n));
            gp::Buf<gp::u64> pw(d, 32);
            std::vector<gp::u64> host_pw;
            gp::part_weights<T>(d, g, lab.get(), parts, pw.get(), host_pw);
            gp::u64 total = 0;
            for (auto x : host_pw) total += x;
            const gp::u64 cap = gp::partition_capacity(total, parts, ratio);
            if (*std::max_element(host_pw.begin(), host_pw.end()) > cap)
                gp::fail(GP_EINVAL, "initial refinement partition is imbalanced");
            gp::RefineWork w;
            const bool narrow = gp::narrow_cache(g, d);
            auto st = gp::refine_dispatch<T>(d, g, w, lab.get(), pw.get(), host_pw, parts, cap, max_rounds,
                                             deterministic != 0, false, narrow);
            gp::to_host(d, labels, lab.get(), static_cast<size_t>(g.n));
            d.sync();
            if (stats) *stats = st;
        });
    });
}

uint64_t gp_launch_count(const gp_ctx* ctx) { return ctx ? ctx->dev.launches : 0; }
uint64_t gp_sync_count(const gp_ctx* ctx) { return ctx ? ctx->dev.syncs : 0; }

gp_status gp_initial_partition_static(const gp_graph* graph, int parts, double ratio, uint32_t seed, int32_t* labels,
                                      void* stream, char* message, uint64_t message_capacity) {
    std::string what;
    gp_status status = GP_OK;
    try {
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            gp::initial_partition_static<T>(graph, parts, ratio, seed, labels, static_cast<cudaStream_t>(stream));
        });
    } catch (const gp::Error& e) {
        status = e.status;
        what = e.what();
    } catch (const std::exception& e) {
        status = GP_ERUNTIME;
        what = e.what();
    }
    if (message && message_capacity) {
        const size_t k = std::min<size_t>(what.size(), static_cast<size_t>(message_capacity) - 1);
        std::memcpy(message, what.data(), k);
        message[k] = 0;
    }
    return status;
}

void* gp_ctx_stream(const gp_ctx* ctx) { return ctx ? static_cast<void*>(ctx->dev.stream) : nullptr; }

gp_status gp_profile_enable(gp_ctx* ctx, int on) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        auto& d = ctx->dev;
        d.prof_resolve();
        d.prof_table.clear();
        d.prof = on != 0;
    });
}

gp_status gp_profile_dump(gp_ctx* ctx, char* buffer, uint64_t capacity) {
    if (!ctx || !buffer || capacity == 0) return GP_EINVAL;
    return guarded(ctx, [&] {
        auto& d = ctx->dev;
        d.prof_resolve();
        std::ostringstream os;
        os << std::setprecision(12);
        for (const auto& kv : d.prof_table)
            os << kv.first << ' ' << kv.second.launches << ' ' << kv.second.ms << ' ' << kv.second.bytes << '\n';
        const std::string s = os.str();
        const size_t n = std::min<size_t>(s.size(), static_cast<size_t>(capacity) - 1);
        std::memcpy(buffer, s.data(), n);
        buffer[n] = 0;
    });
}

gp_status gp_analyze(gp_ctx* ctx, const gp_graph* graph, const int32_t* labels, int parts, gp_part_stats* per_part,
                     gp_analysis* summary) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        if (!labels) gp::fail(GP_EINVAL, "null labels");
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, false);
            const gp::i32* dev_labels = labels;
            gp::Buf<gp::i32> lab;
            if (graph->memory != GP_MEMORY_DEVICE) {
                lab = gp::Buf<gp::i32>(d, static_cast<size_t>(std::max<gp::i64>(g.n, 1)));
                gp::to_device(d, lab.get(), labels, static_cast<size_t>(g.n));
                dev_labels = lab.get();
            }
            std::vector<gp::u64> c;
            try {
                gp::analyze_parts<T>(d, g, dev_labels, parts, c);
            } catch (const gp::Error& e) {
                if (e.status == GP_EINVAL && std::string(e.what()) == "invalid graph input")
                    gp::fail(GP_EINVAL, "partition id outside [0, parts)");
                throw;
            }
            // analyze_partition.cpp:466-499
            gp_analysis a{};
            a.parts = parts;
            const double np = static_cast<double>(parts);
            a.min_vertices = a.min_edge_set = ~0ULL;
            for (int q = 0; q < parts; ++q) {
                gp_part_stats st{c[q], c[parts + q], c[2 * parts + q], c[3 * parts + q], c[4 * parts + q],
                                 c[5 * parts + q], c[6 * parts + q]};
                if (per_part) per_part[q] = st;
                a.directed_edge_cut += st.outgoing_cut_edges;
                a.weighted_directed_edge_cut += st.weighted_outgoing;
                const gp::u64 edge_set = st.internal_edges + st.outgoing_cut_edges + st.incoming_cut_edges;
                const gp::u64 local = st.outgoing_cut_edges + st.incoming_cut_edges;
                const gp::u64 wlocal = st.weighted_outgoing + st.weighted_incoming;
                a.avg_local_cut += static_cast<double>(local);
                a.weighted_avg_local_cut += static_cast<double>(wlocal);
                a.max_local_cut = std::max(a.max_local_cut, local);
                a.weighted_max_local_cut = std::max(a.weighted_max_local_cut, wlocal);
                a.min_vertices = std::min(a.min_vertices, st.vertices);
                a.max_vertices = std::max(a.max_vertices, st.vertices);
                a.min_edge_set = std::min(a.min_edge_set, edge_set);
                a.max_edge_set = std::max(a.max_edge_set, edge_set);
            }
            a.avg_local_cut /= np;
            a.weighted_avg_local_cut /= np;
            auto deviation = [](double value, double average) {
                if (average <= 0.0) return value == 0.0 ? 0.0 : std::numeric_limits<double>::infinity();
                return std::abs(value - average) / average;
            };
            auto imbalance = [](double max_value, double average) { return average > 0.0 ? max_value / average : 0.0; };
            a.vertex_avg = static_cast<double>(g.n) / np;
            a.edge_set_avg = static_cast<double>(static_cast<gp::u64>(g.m) + a.directed_edge_cut) / np;
            a.vertex_imbalance = imbalance(static_cast<double>(a.max_vertices), a.vertex_avg);
            a.vertex_max_deviation = std::max(deviation(static_cast<double>(a.max_vertices), a.vertex_avg),
                                              deviation(static_cast<double>(a.min_vertices), a.vertex_avg));
            a.edge_set_imbalance = imbalance(static_cast<double>(a.max_edge_set), a.edge_set_avg);
            a.edge_set_max_deviation = std::max(deviation(static_cast<double>(a.max_edge_set), a.edge_set_avg),
                                                deviation(static_cast<double>(a.min_edge_set), a.edge_set_avg));
            if (summary) *summary = a;
        });
    });
}

gp_status gp_symmetrize(gp_ctx* ctx, const gp_graph* graph, int64_t* offsets_out, void* neighbors_out,
                        int32_t neighbor_bytes, int64_t capacity, gp_symmetrize_info* info) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        if (neighbor_bytes != 4 && neighbor_bytes != 8) gp::fail(GP_EINVAL, "neighbor_bytes must be 4 or 8");
        if (!offsets_out || !neighbors_out || capacity < 0) gp::fail(GP_EINVAL, "null output or negative capacity");
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, false);
            const gp::i64 n = g.n, m = g.m;
            const int bits = gp::symmetrize_bits(n);
            gp::Buf<gp::u64> keys(d, static_cast<size_t>(std::max<gp::i64>(2 * m, 1)));
            gp::Buf<gp::u64> alt(d, static_cast<size_t>(std::max<gp::i64>(2 * m, 1)));
            gp::Buf<gp::u64> loops(d, 1);
            loops.zero(d);
            if (m)
                gp::launch(d, "sym_keys_kernel", gp::sym_keys_kernel<typename T::O>, gp::stride_grid(d, n * 32),
                           gp::kThreads, 0, n, g.off.get(), g.nbr.get(), bits, keys.get(), loops.get());
            GP_LAUNCH();
            gp::u64 self = 0;
            gp::fetch(d, &self, loops.get(), 1);
            gp::emit_symmetric(d, keys, alt, 2 * m, 2 * (m - static_cast<gp::i64>(self)), n, bits, self,
                               graph->memory == GP_MEMORY_DEVICE, offsets_out, neighbors_out, neighbor_bytes, capacity,
                               info);
        });
    });
}

gp_status gp_generate_rmat(gp_ctx* ctx, int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                           int32_t memory, int64_t* offsets_out, void* neighbors_out, int32_t neighbor_bytes,
                           int64_t capacity, gp_symmetrize_info* info) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        if (scale < 1 || scale > 30 || edge_factor < 1 || !(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
            gp::fail(GP_EINVAL, "invalid rmat parameters");
        if (neighbor_bytes != 4 && neighbor_bytes != 8) gp::fail(GP_EINVAL, "neighbor_bytes must be 4 or 8");
        if (!offsets_out || !neighbors_out || capacity < 0) gp::fail(GP_EINVAL, "null output or negative capacity");
        auto& d = ctx->dev;
        const gp::i64 n = gp::i64{1} << scale;
        const gp::i64 pairs = n * edge_factor;
        // the streams and the seeded Fisher-Yates relabelling of the host
        // generator (horkxg_b200/csrc/gen.cpp, build_rmat)
        const gp::u64 stream = gp::splitmix64(seed * 0x100000001b3ULL + 0x5851f42d4c957f2dULL);
        std::vector<gp::u32> perm(static_cast<size_t>(n));
        for (gp::i64 v = 0; v < n; ++v) perm[v] = static_cast<gp::u32>(v);
        const gp::u64 pstream = gp::splitmix64(stream ^ 0xa0761d6478bd642fULL);
        for (gp::i64 v = n - 1; v > 0; --v) {
            const gp::u64 j = gp::splitmix64(pstream ^ static_cast<gp::u64>(v)) % static_cast<gp::u64>(v + 1);
            std::swap(perm[v], perm[j]);
        }
        gp::Buf<gp::u32> dperm(d, static_cast<size_t>(n));
        gp::to_device(d, dperm.get(), perm.data(), perm.size());
        const int bits = gp::symmetrize_bits(n);
        gp::Buf<gp::u64> keys(d, static_cast<size_t>(2 * pairs)), alt(d, static_cast<size_t>(2 * pairs));
        gp::launch(d, "rmat_keys_kernel", gp::rmat_keys_kernel, gp::stride_grid(d, pairs), gp::kThreads, 0, pairs,
                   scale, a, a + b, a + b + c, stream, dperm.get(), bits, keys.get());
        GP_LAUNCH();
        d.sync();   // the host permutation goes out of scope
        // self loops are the pairs whose keys are sentinels: counted from the
        // sorted keys (they sort last)
        gp::radix_sort<gp::u64, gp::i32>(d, keys.get(), nullptr, alt.get(), nullptr, 2 * pairs, 0, 2 * bits);
        gp::Buf<gp::i64> first(d, 1);
        const gp::i64 all_keys = 2 * pairs;
        gp::to_device(d, first.get(), &all_keys, 1);
        gp::launch(d, "sym_first_sentinel_kernel", gp::sym_first_sentinel_kernel, gp::stride_grid(d, 2 * pairs),
                   gp::kThreads, 0, 2 * pairs, keys.get(), first.get());
        GP_LAUNCH();
        gp::i64 valid = 0;
        gp::fetch(d, &valid, first.get(), 1);
        gp::emit_symmetric(d, keys, alt, 2 * pairs, valid, n, bits, static_cast<gp::u64>((2 * pairs - valid) / 2),
                           memory == GP_MEMORY_DEVICE, offsets_out, neighbors_out, neighbor_bytes, capacity, info,
                           true);
    });
}

gp_status gp_cut(gp_ctx* ctx, const gp_graph* graph, const int32_t* labels, int parts, uint64_t* directed_cut,
                 uint64_t* loads) {
    if (!ctx) return GP_EINVAL;
    return guarded(ctx, [&] {
        GP_CUDA(cudaSetDevice(ctx->dev.device));
        if (parts < 1 || parts > 32) gp::fail(GP_EINVAL, "invalid parts");
        with_width(graph, [&](auto tag) {
            using T = decltype(tag);
            auto& d = ctx->dev;
            gp::DGraph<T> g;
            gp::prepare_graph<T>(d, graph, g, false);
            for (gp::i64 v = 0; v < g.n; ++v)
                if (labels[v] < 0 || labels[v] >= parts) gp::fail(GP_EINVAL, "invalid label");
            gp::Buf<gp::i32> lab(d, static_cast<size_t>(std::max<gp::i64>(g.n, 1)));
            gp::to_device(d, lab.get(), labels, static_cast<size_t>(g.n));
            gp::Buf<gp::u64> s(d, 2);
            const gp::u64 c = gp::directed_cut<T>(d, g, lab.get(), s.get());
            if (directed_cut) *directed_cut = c;
            if (loads) {
                gp::Buf<gp::u64> pw(d, 32);
                std::vector<gp::u64> host;
                gp::part_weights<T>(d, g, lab.get(), parts, pw.get(), host);
                std::copy(host.begin(), host.end(), loads);
            }
        });
    });
}

}  // extern "C"
