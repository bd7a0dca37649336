// Partition analysis on the GPU: the per-part figures of the reference's CPU
// analyzer (graph_untils/analyze_partition.cpp:425-499) from the original CSR
// and a label array -- vertex counts, internal directed entries, outgoing and
// incoming cut entries, each also summed by edge weight.  The summary figures
// (imbalances, deviations, local cuts) follow on the host from these.
//
// Layout of the 7 x parts counters: vertices, internal, outgoing, incoming,
// weighted internal, weighted outgoing, weighted incoming.  Each block
// accumulates them in shared memory and adds them to the global counters
// once, so a launch makes 7 x parts global atomics per block.
#pragma once

#include "gp_prim.cuh"
#include "gp_hub.cuh"

namespace gp {

constexpr int kAnalyzeMaxParts = 1024;
constexpr int kAnalyzeFields = 7;

__device__ __forceinline__ u64 lane_group_sum(unsigned peers, u64 w) {
    u64 sum = 0;
#pragma unroll
    for (int s = 0; s < 32; ++s) {
        const u64 x = __shfl_sync(0xffffffffu, w, s);
        if (peers & (1u << s)) sum += x;
    }
    return sum;
}

// Adds one 32-edge slice of a row whose source part is `sp`: internal and
// outgoing entries go to the caller's running sums, incoming entries to the
// destination parts' counters (one shared atomic per distinct part in the
// warp).  Every lane of the warp calls it.
template <typename W>
__device__ __forceinline__ void analyze_slice(i64 e, i64 end, int sp, const i32* __restrict__ nbr,
                                              const W* __restrict__ ew, const i32* __restrict__ labels, int parts,
                                              u64* s_in, u64* s_win, u64& ni, u64& no, u64& wi, u64& wo,
                                              bool& bad) {
    int dp = -1;
    u64 w = 0;
    if (e < end) {
        const i32 u = nbr[e];
        const int q = labels[u];
        w = static_cast<u64>(weight_at(ew, e));
        if (q < 0 || q >= parts) {
            bad = true;
        } else if (q == sp) {
            ++ni;
            wi += w;
        } else {
            ++no;
            wo += w;
            dp = q;
        }
    }
    const unsigned peers = __match_any_sync(0xffffffffu, dp);
    const u64 wsum = ew ? lane_group_sum(peers, dp >= 0 ? w : 0) : static_cast<u64>(__popc(peers));
    if (dp >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&s_in[dp]), static_cast<unsigned long long>(__popc(peers)));
        atomicAdd(reinterpret_cast<unsigned long long*>(&s_win[dp]), static_cast<unsigned long long>(wsum));
    }
}

__device__ __forceinline__ void analyze_flush(u64* sh, int parts, u64* out) {
    __syncthreads();
    for (int i = threadIdx.x; i < kAnalyzeFields * parts; i += kThreads)
        if (sh[i]) atomicAdd(reinterpret_cast<unsigned long long*>(&out[i]), static_cast<unsigned long long>(sh[i]));
}

// One warp per vertex over the rows of at most kHubDegree entries (hub rows
// are walked by analyze_hub_kernel); every vertex is counted here.
template <typename O, typename W>
__global__ void __launch_bounds__(kThreads) analyze_rows_kernel(i64 n, const O* __restrict__ off,
                                                                const i32* __restrict__ nbr, const W* __restrict__ ew,
                                                                const i32* __restrict__ labels, int parts, u64* out,
                                                                u32* err) {
    extern __shared__ u64 sh[];
    for (int i = threadIdx.x; i < kAnalyzeFields * parts; i += kThreads) sh[i] = 0;
    __syncthreads();
    u64* s_vert = sh;
    u64* s_int = sh + parts;
    u64* s_out = sh + 2 * parts;
    u64* s_in = sh + 3 * parts;
    u64* s_wint = sh + 4 * parts;
    u64* s_wout = sh + 5 * parts;
    u64* s_win = sh + 6 * parts;
    const int lane = threadIdx.x & 31;
    bool bad = false;
    const i64 warps_total = static_cast<i64>(gridDim.x) * kWarps;
    for (i64 v = static_cast<i64>(blockIdx.x) * kWarps + (threadIdx.x >> 5); v < n; v += warps_total) {
        const int sp = labels[v];
        if (sp < 0 || sp >= parts) {
            bad = true;
            continue;
        }
        if (lane == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&s_vert[sp]), 1ULL);
        const i64 b = off[v], end = off[v + 1];
        if (end - b > kHubDegree) continue;
        u64 ni = 0, no = 0, wi = 0, wo = 0;
        for (i64 base = b; base < end; base += 32)
            analyze_slice(base + lane, end, sp, nbr, ew, labels, parts, s_in, s_win, ni, no, wi,
                          wo, bad);
        ni = warp_sum(ni);
        no = warp_sum(no);
        if (ew) {
            wi = warp_sum(wi);
            wo = warp_sum(wo);
        } else {
            wi = ni;
            wo = no;
        }
        if (lane == 0) {
            if (ni) {
                atomicAdd(reinterpret_cast<unsigned long long*>(&s_int[sp]), static_cast<unsigned long long>(ni));
                atomicAdd(reinterpret_cast<unsigned long long*>(&s_wint[sp]), static_cast<unsigned long long>(wi));
            }
            if (no) {
                atomicAdd(reinterpret_cast<unsigned long long*>(&s_out[sp]), static_cast<unsigned long long>(no));
                atomicAdd(reinterpret_cast<unsigned long long*>(&s_wout[sp]), static_cast<unsigned long long>(wo));
            }
        }
    }
    if (bad) set_error(err, kErrBadInput);
    analyze_flush(sh, parts, out);
}

// Hub rows, one block per 2048-entry chunk.  Vertex counts are not touched
// (analyze_rows_kernel counted every vertex).
template <typename W>
__global__ void __launch_bounds__(kThreads) analyze_hub_kernel(const Chunk* __restrict__ chunks,
                                                               const i32* __restrict__ nbr, const W* __restrict__ ew,
                                                               const i32* __restrict__ labels, int parts, u64* out,
                                                               u32* err) {
    extern __shared__ u64 sh[];
    __shared__ u64 red[kWarps + 1];
    for (int i = threadIdx.x; i < kAnalyzeFields * parts; i += kThreads) sh[i] = 0;
    __syncthreads();
    const Chunk ch = chunks[blockIdx.x];
    const int sp = labels[ch.v];
    if (sp < 0 || sp >= parts) {
        if (threadIdx.x == 0) set_error(err, kErrBadInput);
        return;
    }
    bool bad = false;
    u64 ni = 0, no = 0, wi = 0, wo = 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // each warp walks its own contiguous slice of the chunk
    const i64 len = ch.end - ch.begin;
    const i64 per = (len + kWarps - 1) / kWarps;
    const i64 lo = ch.begin + warp * per, hi = lo + per < ch.end ? lo + per : ch.end;
    for (i64 base = lo; base < hi; base += 32)
        analyze_slice(base + lane, hi, sp, nbr, ew, labels, parts, sh + 3 * parts, sh + 6 * parts, ni, no, wi,
                      wo, bad);
    if (bad) set_error(err, kErrBadInput);
    ni = block_sum(ni, red);
    no = block_sum(no, red);
    wi = block_sum(wi, red);
    wo = block_sum(wo, red);
    if (threadIdx.x == 0) {
        sh[parts + sp] += ni;
        sh[2 * parts + sp] += no;
        sh[4 * parts + sp] += ew ? wi : ni;
        sh[5 * parts + sp] += ew ? wo : no;
    }
    analyze_flush(sh, parts, out);
}

}  // namespace gp
