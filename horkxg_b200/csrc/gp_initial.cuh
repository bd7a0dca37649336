// Recursive weighted spectral bisection on the coarsest graph
// (src/initial_partition_gpu.cu:170-276), batched by recursion depth:
//
// * every open task of one depth runs its 64 lazy-diffusion steps in ONE
//   cooperative kernel; vertices are spread over all SMs (warp per vertex),
//   one bounded grid barrier per step; the per-task weighted moments are
//   reduced redundantly by every block in a fixed order (deterministic), and
//   the normalisation is folded into the next step's reads;
// * the split sort by (x, vertex id) is one launch: a block per task sorts its
//   slice with an LSD radix sort on (orderable x << 32 | id);
// * the weight-prefix split, its capacity checks and the child task
//   descriptors are computed on the device (block per task): the host never
//   waits inside the recursion.
//
// The diffusion is FP32 (the reference uses FP64); each diffusion vector is
// checked against the FP64 oracle within 1e-5 relative L2.
#pragma once

#include <cooperative_groups.h>

#include "gp_prim.cuh"

namespace gp {

struct InitTask {
    i32 begin;
    i32 count;
    i32 first_part;
    i32 parts;
    u64 weight;
    i32 left_child;    // index in the next depth's task array, -1 = leaf
    i32 right_child;
};

struct Moments { float mass, sum, squares; };
struct alignas(16) Moments4 { float mass, sum, squares, pad; };   // one 16-byte store

// Bounded grid barrier for cooperative launches: gives up after ~2^24 polls
// and records kErrTimeout (the kernel then finishes with garbage values that
// the host discards).
__device__ __forceinline__ void grid_barrier(u32* counter, volatile u32* generation, u32* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const u32 gen = *generation;
        __threadfence();
        const u32 arrived = atomicAdd(counter, 1u);
        if (arrived == gridDim.x - 1) {
            *counter = 0;
            __threadfence();
            atomicAdd(const_cast<u32*>(generation), 1u);
        } else {
            u32 polls = 0;
            while (*generation == gen) {
                if (++polls > (1u << 24)) { set_error(err, kErrTimeout); break; }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

constexpr int kMaxInitTasks = 16;   // tasks per depth for k <= 32

struct NormShared {
    float mean[kMaxInitTasks];
    float scale[kMaxInitTasks];
    float red[3][kWarps];
};

// Every block computes every task's (mean, scale) from the per-position
// contributions in the same order: deterministic and identical everywhere.
// Only the first kWarps warps take part, so blocks larger than kThreads get
// the same result.
// The tasks are reduced side by side: `wpt` warps per task, each warp over a
// lane-strided slice with an xor-shuffle tree, then one thread per task adds
// its warps' partials in warp order.
template <typename Rec>
__device__ void compute_norms(int tasks, const InitTask* task, const Rec* contrib, NormShared& sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int wpt = kWarps;
    while (wpt > 1 && tasks * wpt > kWarps) wpt >>= 1;
    const int per_round = kWarps / wpt;
    for (int t0 = 0; t0 < tasks; t0 += per_round) {
        const int t = t0 + warp / wpt;
        const int part = warp % wpt;
        float m = 0.f, s = 0.f, q = 0.f;
        if (warp < kWarps && t < tasks) {
            const i32 b = task[t].begin, c = task[t].count;
            for (i32 i = part * 32 + lane; i < c; i += wpt * 32) {
                const Rec x = contrib[b + i];
                m += x.mass; s += x.sum; q += x.squares;
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                m += __shfl_xor_sync(0xffffffffu, m, o);
                s += __shfl_xor_sync(0xffffffffu, s, o);
                q += __shfl_xor_sync(0xffffffffu, q, o);
            }
        }
        if (lane == 0 && warp < kWarps) { sh.red[0][warp] = m; sh.red[1][warp] = s; sh.red[2][warp] = q; }
        __syncthreads();
        if (threadIdx.x < per_round && t0 + static_cast<int>(threadIdx.x) < tasks) {
            float M = 0.f, S = 0.f, Q = 0.f;
            for (int w = threadIdx.x * wpt; w < (static_cast<int>(threadIdx.x) + 1) * wpt; ++w) {
                M += sh.red[0][w]; S += sh.red[1][w]; Q += sh.red[2][w];
            }
            const float mean = S / M;
            const float var = fmaxf(0.f, Q / M - mean * mean);
            sh.mean[t0 + threadIdx.x] = mean;
            sh.scale[t0 + threadIdx.x] = var > 1e-30f ? 1.0f / sqrtf(var) : 1.0f;
        }
        __syncthreads();
    }
}

// Rows longer than this are reduced by a whole block (fixed tree), shorter
// ones by one warp, so the step time is not set by the densest row.  Coarsest
// levels of power-law graphs are nearly complete (degrees in the thousands),
// and a block reduction per row costs more than a warp walking the row.
constexpr i64 kHeavyRow = 4096;

// Sum over a row range of f(e) restricted to the group, with four
// independent loads in flight per lane.  `stride` is the number of lanes
// cooperating on the row (32 or kThreads).
template <typename O, typename W, typename F>
__device__ __forceinline__ float row_sum(i64 begin, i64 end, int lane, int stride, const i32* __restrict__ nbr,
                                         const i32* __restrict__ labels, i32 group, const W* __restrict__ ew, F f) {
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    i64 e = begin + lane;
    for (; e + 3 * stride < end; e += 4 * stride) {
        const i32 u0 = nbr[e], u1 = nbr[e + stride], u2 = nbr[e + 2 * stride], u3 = nbr[e + 3 * stride];
        const bool g0 = labels[u0] == group, g1 = labels[u1] == group, g2 = labels[u2] == group,
                   g3 = labels[u3] == group;
        if (g0) a0 += static_cast<float>(weight_at(ew, e)) * f(u0);
        if (g1) a1 += static_cast<float>(weight_at(ew, e + stride)) * f(u1);
        if (g2) a2 += static_cast<float>(weight_at(ew, e + 2 * stride)) * f(u2);
        if (g3) a3 += static_cast<float>(weight_at(ew, e + 3 * stride)) * f(u3);
    }
    for (; e < end; e += stride) {
        const i32 u = nbr[e];
        if (labels[u] == group) a0 += static_cast<float>(weight_at(ew, e)) * f(u);
    }
    return (a0 + a1) + (a2 + a3);
}

struct One { __device__ float operator()(i32) const { return 1.f; } };
struct Normalised {
    const float* x;
    float mean, scale;
    __device__ float operator()(i32 u) const { return (x[u] - mean) * scale; }
};

// spectral_start + 64 x (normalize, spectral_step) + normalize
// (src/initial_partition_gpu.cu:81-142,206-229) for all tasks of one depth.
// x_out[v] receives the final normalised value; key[p] the sort key of
// position p.
template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) diffusion_kernel(
    int tasks, const InitTask* __restrict__ task, const i32* __restrict__ task_of_pos, i32 positions,
    const i32* __restrict__ order, const i32* __restrict__ labels, const O* __restrict__ off,
    const i32* __restrict__ nbr, const W* __restrict__ ew, u32 seed, int steps, float* deg, float* xa, float* xb,
    Moments* contrib, float* x_out, u64* key, u32* bar_counter, u32* bar_gen, u32* err) {
    __shared__ NormShared sh;
    __shared__ float red[kWarps + 1];
    const int lane = threadIdx.x & 31;
    const i32 warps_total = static_cast<i32>(gridDim.x) * kWarps;
    const i32 warp_id = static_cast<i32>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
    // start: degree restricted to the group, x0 = hash, moment contributions
    auto start_row = [&](i32 p, float d) {
        const i32 v = order[p];
        const i32 group = task[task_of_pos[p]].first_part;
        const u32 h = mix32(static_cast<u32>(v) ^ (seed ^ static_cast<u32>(group)));
        const float a = static_cast<float>(static_cast<double>(h) / 4294967296.0 - 0.5);
        deg[v] = d;
        xa[v] = a;
        const float mass = d > 0.f ? d : 1.f;
        contrib[p] = {mass, mass * a, mass * a * a};
    };
    for (i32 p = blockIdx.x; p < positions; p += gridDim.x) {   // heavy rows: block per row
        const i32 t = task_of_pos[p];
        if (t < 0) continue;
        const i32 v = order[p];
        const i64 b = off[v], e = off[v + 1];
        if (e - b <= kHeavyRow) continue;
        const float d = block_sum(row_sum<O, W>(b, e, threadIdx.x, kThreads, nbr, labels, task[t].first_part, ew, One{}), red);
        if (threadIdx.x == 0) start_row(p, d);
    }
    for (i32 p = warp_id; p < positions; p += warps_total) {      // light rows: warp per row
        const i32 t = task_of_pos[p];
        if (t < 0) continue;
        const i32 v = order[p];
        const i64 b = off[v], e = off[v + 1];
        if (e - b > kHeavyRow) continue;
        const float d = warp_sum(row_sum<O, W>(b, e, lane, 32, nbr, labels, task[t].first_part, ew, One{}));
        if (lane == 0) start_row(p, d);
    }
    float* x = xa;
    float* y = xb;
    for (int it = 0; it <= steps; ++it) {
        grid_barrier(bar_counter, bar_gen, err);
        compute_norms(tasks, task, contrib, sh);
        if (it == steps) break;
        auto step_row = [&](i32 p, i32 t, float s) {
            const i32 v = order[p];
            const float d = deg[v];
            const float xv = (x[v] - sh.mean[t]) * sh.scale[t];
            const float a = d > 0.f ? 0.5f * (xv + s / d) : xv;
            y[v] = a;
            const float mass = d > 0.f ? d : 1.f;
            contrib[p] = {mass, mass * a, mass * a * a};
        };
        for (i32 p = blockIdx.x; p < positions; p += gridDim.x) {
            const i32 t = task_of_pos[p];
            if (t < 0) continue;
            const i32 v = order[p];
            const i64 b = off[v], e = off[v + 1];
            if (e - b <= kHeavyRow) continue;
            const float s = block_sum(row_sum<O, W>(b, e, threadIdx.x, kThreads, nbr, labels, task[t].first_part, ew,
                                                    Normalised{x, sh.mean[t], sh.scale[t]}), red);
            if (threadIdx.x == 0) step_row(p, t, s);
        }
        for (i32 p = warp_id; p < positions; p += warps_total) {
            const i32 t = task_of_pos[p];
            if (t < 0) continue;
            const i32 v = order[p];
            const i64 b = off[v], e = off[v + 1];
            if (e - b > kHeavyRow) continue;
            const float s = warp_sum(row_sum<O, W>(b, e, lane, 32, nbr, labels, task[t].first_part, ew,
                                                   Normalised{x, sh.mean[t], sh.scale[t]}));
            if (lane == 0) step_row(p, t, s);
        }
        float* tmp = x; x = y; y = tmp;
    }
    // final normalisation + sort keys
    for (i32 p = static_cast<i32>(blockIdx.x) * kThreads + threadIdx.x; p < positions; p += static_cast<i32>(gridDim.x) * kThreads) {
        const i32 t = task_of_pos[p];
        if (t < 0) continue;
        const i32 v = order[p];
        float a = (x[v] - sh.mean[t]) * sh.scale[t];
        if (a == 0.f) a = 0.f;   // canonical +0 so that -0 and +0 tie (then id decides)
        if (x_out) x_out[v] = a;
        const u32 b = __float_as_uint(a);
        const u32 ord = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
        key[p] = (static_cast<u64>(ord) << 32) | static_cast<u32>(v);
    }
}

// ---------------------------------------------------------------------------
// Small coarsest graphs: the same diffusion in ONE thread-block cluster of up
// to kSmallDiffCluster blocks (1024 threads each; at least one block per 1024
// positions, so each thread owns at most one row, and one per
// kSmallDiffBlockEdges edges, for dense graphs whose rows go to warps), every
// per-vertex and
// per-position array in shared memory and the hardware cluster barrier in
// place of the grid barrier (no cooperative launch, no polling).  Each block
// owns the positions p with p % cluster size == its rank.  The new values of
// its rows are written into every block's shared memory (distributed shared
// memory), their moment contributions into block 0's only; block 0 runs
// compute_norms and sends the per-task mean and scale to the others.  It
// computes exactly the values of diffusion_kernel, operation for operation:
// * rows of more than 32 edges are summed by a warp with the same row_sum and
//   warp_sum;
// * rows of at most 32 edges are summed by one thread: in row_sum (stride 32)
//   each lane then holds at most one edge, so the thread forms the 32 lane
//   values and adds them in the butterfly order of warp_sum;
// * the moments use compute_norms on the first kWarps warps.
// Rows of more than kHeavyRow edges (block sums) are not taken: the host
// sends such graphs to diffusion_kernel.
// ---------------------------------------------------------------------------
constexpr int kSmallDiffThreads = 1024;
constexpr int kSmallDiffWarps = kSmallDiffThreads / 32;
constexpr int kSmallDiffCluster = 16;      // largest cluster (a non-portable size above 8)
constexpr i32 kSmallDiffN = 4096;          // positions (= vertices of the coarsest graph)
constexpr i64 kSmallDiffBlockEdges = 131072;                         // edges per block and step
constexpr i64 kSmallDiffM = kSmallDiffCluster * kSmallDiffBlockEdges;   // edges
constexpr i32 kThreadRowMax = 32;          // rows summed by a single thread

// Lane 0's result of warp_sum over the 32 lane values lane(l), l = 0..31.
template <typename L>
__device__ __forceinline__ float butterfly_sum(L lane) {
    float r[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) r[l] = lane(l);
#pragma unroll
    for (int o = 16; o; o >>= 1) {
#pragma unroll
        for (int l = 0; l < o; ++l) r[l] = r[l] + r[l + o];
    }
    return r[0];
}

inline size_t small_diffusion_smem(i32 n) {
    // moment records (per position; used in block 0), x, y, degree
    // (vertex-indexed floats), labels, position records {vertex,
    // degree << 8 | task} and the list of rows summed by warps
    return static_cast<size_t>(n) * (sizeof(Moments4) + 3 * sizeof(float) + 4 * sizeof(i32));
}

template <typename O, typename W>
__global__ void __launch_bounds__(kSmallDiffThreads) diffusion_small_kernel(
    int tasks, const InitTask* __restrict__ task, const i32* __restrict__ task_of_pos, i32 positions,
    const i32* __restrict__ order, const i32* __restrict__ labels_g, const O* __restrict__ off,
    const i32* __restrict__ nbr, const W* __restrict__ ew, u32 seed, int steps, float* x_out, u64* key) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = static_cast<int>(cluster.block_rank());
    const int cs = static_cast<int>(cluster.num_blocks());
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const i32 n = positions;
    Moments4* contrib = reinterpret_cast<Moments4*>(smem_raw);
    float* xa = reinterpret_cast<float*>(contrib + n);
    float* xb = xa + n;
    float* deg = xb + n;
    i32* labels = reinterpret_cast<i32*>(deg + n);
    i32* pv = labels + n;
    i32* pdt = pv + n;
    i32* heavy = pdt + n;
    __shared__ NormShared sh;
    __shared__ float norm_mean[kMaxInitTasks], norm_scale[kMaxInitTasks];
    __shared__ int nheavy;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) nheavy = 0;
    for (i32 v = threadIdx.x; v < n; v += kSmallDiffThreads) labels[v] = labels_g[v];
    __syncthreads();
    const i32 first = rank + cs * static_cast<i32>(threadIdx.x);
    const i32 stride = cs * kSmallDiffThreads;
    for (i32 p = first; p < n; p += stride) {
        const i32 t = task_of_pos[p];
        const i32 v = order[p];
        const i32 dg = static_cast<i32>(off[v + 1] - off[v]);
        pv[p] = v;
        pdt[p] = t < 0 ? -1 : (dg << 8) | t;
        if (t >= 0 && dg > kThreadRowMax) heavy[atomicAdd(&nheavy, 1)] = p;
    }
    cluster.sync();   // every block has started: its shared memory may be written
    const int nh = nheavy;
    Moments4* contrib0 = cluster.map_shared_rank(contrib, 0);
    // a row's new value goes to every block, its moment record to block 0
    auto put = [&](float* xlocal, i32 p, i32 v, float mass, float a) {
        for (int r = 0; r < cs; ++r) cluster.map_shared_rank(xlocal, r)[v] = a;
        contrib0[p] = Moments4{mass, mass * a, mass * a * a, 0.f};
    };
    auto start_row = [&](i32 p, float d) {
        const i32 v = pv[p];
        const i32 group = task[pdt[p] & 0xff].first_part;
        const u32 h = mix32(static_cast<u32>(v) ^ (seed ^ static_cast<u32>(group)));
        const float a = static_cast<float>(static_cast<double>(h) / 4294967296.0 - 0.5);
        deg[v] = d;
        put(xa, p, v, d > 0.f ? d : 1.f, a);
    };
    // row sum of f over the group, as diffusion_kernel forms it: lane l of
    // row_sum holds edge l alone, a0 = 0 + w * f(u) if u is in the group,
    // and returns (a0 + a1) + (a2 + a3) with a1 = a2 = a3 = 0
    auto sum_thread = [&](i32 p, auto f) {
        const i32 v = pv[p];
        const i64 b = static_cast<i64>(off[v]);
        const int dg = pdt[p] >> 8;
        const i32 group = task[pdt[p] & 0xff].first_part;
        return butterfly_sum([&](int l) {
            float a0 = 0.f;
            if (l < dg) {
                const i32 u = nbr[b + l];
                if (labels[u] == group) a0 += static_cast<float>(weight_at(ew, b + l)) * f(u);
            }
            const float a1 = 0.f, a2 = 0.f, a3 = 0.f;
            return (a0 + a1) + (a2 + a3);
        });
    };
    auto sum_warp = [&](i32 p, auto f) {
        const i32 v = pv[p];
        const i64 b = static_cast<i64>(off[v]);
        const i64 e = b + (pdt[p] >> 8);
        const i32 group = task[pdt[p] & 0xff].first_part;
        return warp_sum(row_sum<O, W>(b, e, lane, 32, nbr, labels, group, ew, f));
    };
    for (i32 p = first; p < n; p += stride)
        if (pdt[p] >= 0 && (pdt[p] >> 8) <= kThreadRowMax) start_row(p, sum_thread(p, One{}));
    for (int h = warp; h < nh; h += kSmallDiffWarps) {
        const float d = sum_warp(heavy[h], One{});
        if (lane == 0) start_row(heavy[h], d);
    }
    float* x = xa;
    float* y = xb;
    for (int it = 0; it <= steps; ++it) {
        cluster.sync();                       // all records of the step are in block 0
        if (rank == 0) {
            compute_norms(tasks, task, contrib, sh);
            if (threadIdx.x < static_cast<unsigned>(tasks))
                for (int r = 0; r < cs; ++r) {
                    cluster.map_shared_rank(norm_mean, r)[threadIdx.x] = sh.mean[threadIdx.x];
                    cluster.map_shared_rank(norm_scale, r)[threadIdx.x] = sh.scale[threadIdx.x];
                }
        }
        cluster.sync();                       // mean and scale are everywhere
        if (it == steps) break;
        auto step_row = [&](i32 p, float s) {
            const i32 v = pv[p];
            const int t = pdt[p] & 0xff;
            const float d = deg[v];
            const float xv = (x[v] - norm_mean[t]) * norm_scale[t];
            const float a = d > 0.f ? 0.5f * (xv + s / d) : xv;
            put(y, p, v, d > 0.f ? d : 1.f, a);
        };
        for (i32 p = first; p < n; p += stride) {
            if (pdt[p] < 0 || (pdt[p] >> 8) > kThreadRowMax) continue;
            const int t = pdt[p] & 0xff;
            step_row(p, sum_thread(p, Normalised{x, norm_mean[t], norm_scale[t]}));
        }
        for (int h = warp; h < nh; h += kSmallDiffWarps) {
            const i32 p = heavy[h];
            const int t = pdt[p] & 0xff;
            const float s = sum_warp(p, Normalised{x, norm_mean[t], norm_scale[t]});
            if (lane == 0) step_row(p, s);
        }
        float* tmp = x; x = y; y = tmp;
    }
    // no shared memory of another block is touched after the last cluster.sync
    for (i32 p = first; p < n; p += stride) {
        if (pdt[p] < 0) continue;
        const int t = pdt[p] & 0xff;
        const i32 v = pv[p];
        float a = (x[v] - norm_mean[t]) * norm_scale[t];
        if (a == 0.f) a = 0.f;
        if (x_out) x_out[v] = a;
        const u32 bits = __float_as_uint(a);
        const u32 ord = (bits & 0x80000000u) ? ~bits : (bits | 0x80000000u);
        key[p] = (static_cast<u64>(ord) << 32) | static_cast<u32>(v);
    }
}

template <typename O>
__global__ void max_degree_kernel(i64 n, const O* off, u64* out) {
    u64 m = 0;
    for (i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<i64>(gridDim.x) * blockDim.x) {
        const u64 dg = static_cast<u64>(off[v + 1] - off[v]);
        m = dg > m ? dg : m;
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0 && m) atomic_max_u64(out, m);
}

__global__ void task_positions_kernel(int tasks, const InitTask* task, i32* task_of_pos) {
    const int t = blockIdx.x;
    if (t >= tasks) return;
    for (i32 i = threadIdx.x; i < task[t].count; i += kThreads) task_of_pos[task[t].begin + i] = t;
}

// Block per task: sort its slice by (x, id) and rewrite `order`.
__global__ void __launch_bounds__(kThreads) task_sort_kernel(int tasks, const InitTask* task, u64* key, u64* key_alt,
                                                             i32* order) {
    __shared__ RankShared sh;
    const int t = blockIdx.x;
    if (t >= tasks) return;
    const i32 b = task[t].begin, c = task[t].count;
    block_radix_sort_segment<u64, u32>(key + b, nullptr, key_alt + b, nullptr, c, 0, 64, sh);
    for (i32 i = threadIdx.x; i < c; i += kThreads) order[b + i] = static_cast<i32>(key[b + i] & 0xffffffffu);
}

// floor(w * num / den) exactly (w * num fits in 128 bits).
__device__ __forceinline__ u64 mul_div_floor(u64 w, u64 num, u64 den) {
    const unsigned __int128 p = static_cast<unsigned __int128>(w) * num;
    return static_cast<u64>(p / den);
}

// Weight-prefix split, src/initial_partition_gpu.cu:231-254, block per task.
template <typename W>
__global__ void __launch_bounds__(kThreads) task_split_kernel(int tasks, const InitTask* task, InitTask* next,
                                                              const i32* order, const W* vw, u64 capacity,
                                                              u64* prefix, i32* labels, u32* err) {
    __shared__ i64 scan_sh[kWarps + 1];
    __shared__ int boundary_sh;
    __shared__ u64 left_weight_sh;
    const int t = blockIdx.x;
    if (t >= tasks) return;
    const InitTask tk = task[t];
    const i32 b = tk.begin, c = tk.count;
    u64 carry = 0;
    for (i32 base = 0; base < c; base += kThreads) {
        const i32 i = base + threadIdx.x;
        const u64 w = i < c ? static_cast<u64>(weight_at(vw, order[b + i])) : 0;
        i64 total;
        const i64 ex = block_exclusive_sum<i64>(static_cast<i64>(w), scan_sh, &total);
        if (i < c) prefix[b + i] = carry + static_cast<u64>(ex) + w;
        carry += static_cast<u64>(total);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int left_parts = tk.parts / 2, right_parts = tk.parts - left_parts;
        const u64 W_ = tk.weight;
        const u64 target = mul_div_floor(W_, static_cast<u64>(left_parts), static_cast<u64>(tk.parts));
        const u64 left_limit = capacity > W_ / left_parts ? W_ : capacity * left_parts;
        const u64 right_limit = capacity > W_ / right_parts ? W_ : capacity * right_parts;
        const u64 min_left = W_ > right_limit ? W_ - right_limit : 0;
        // lower_bound over the inclusive prefix
        i32 lo = 0, hi = c;
        while (lo < hi) {
            const i32 mid = lo + (hi - lo) / 2;
            if (prefix[b + mid] < target) lo = mid + 1; else hi = mid;
        }
        int boundary = lo + 1;
        boundary = max(left_parts, min(c - right_parts, boundary));
        u64 lw = prefix[b + boundary - 1];
        if (lw > left_limit && boundary > left_parts) { --boundary; lw = prefix[b + boundary - 1]; }
        if (lw < min_left && boundary < c - right_parts) { ++boundary; lw = prefix[b + boundary - 1]; }
        if (lw > left_limit || lw < min_left) set_error(err, kErrSplit);
        boundary_sh = boundary;
        left_weight_sh = lw;
        const u64 rw = W_ - lw;
        if (tk.left_child >= 0) {
            InitTask& L = next[tk.left_child];
            L.begin = b; L.count = boundary; L.weight = lw;
        } else if (lw > capacity) {
            set_error(err, kErrBalance);
        }
        if (tk.right_child >= 0) {
            InitTask& R = next[tk.right_child];
            R.begin = b + boundary; R.count = c - boundary; R.weight = rw;
        } else if (rw > capacity) {
            set_error(err, kErrBalance);
        }
    }
    __syncthreads();
    const int boundary = boundary_sh;
    const int left_parts = tk.parts / 2;
    for (i32 i = threadIdx.x; i < c; i += kThreads)
        labels[order[b + i]] = i < boundary ? tk.first_part : tk.first_part + left_parts;
}

// Part weights + cut terms of the initial partition (part_weights,
// cut_terms, src/initial_partition_gpu.cu:154-167).
template <typename W>
__global__ void part_weight_kernel(i64 n, const i32* labels, const W* vw, u64* loads) {
    const i64 v = static_cast<i64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v < n) atomic_add_u64(&loads[labels[v]], static_cast<u64>(weight_at(vw, v)));
}

}  // namespace gp
