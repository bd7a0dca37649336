// Test infrastructure: CPU restatement of horkxg's multilevel partitioner.
//
// This file is the oracle for the B200 build.  It is loaded only by tests/,
// by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, always as
// the checker; the product never links or calls it.  Every function cites the
// reference file:line it restates (paths relative to the reference project).
// Integer arithmetic follows the reference exactly; the spectral diffusion is
// FP64 (the reference's own precision), against which the build's FP32
// diffusion is compared.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

thread_local std::string g_error;

struct InvalidArg : std::runtime_error { using std::runtime_error::runtime_error; };
struct Overflow : std::runtime_error { using std::runtime_error::runtime_error; };

using u64 = std::uint64_t;
using u32 = std::uint32_t;
using i64 = std::int64_t;
using i32 = std::int32_t;

// src/coarsen.cu:112-118 (identical mixer in refine.cu:38-44 and
// initial_partition_gpu.cu:36-39).
inline u32 mix32(u32 x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    return x ^ (x >> 16);
}

struct Graph {
    i64 n = 0;
    std::vector<i64> off;
    std::vector<i32> nbr;
    std::vector<u64> ew;
    std::vector<u64> vw;
    i64 m() const { return static_cast<i64>(nbr.size()); }
};

Graph make_graph(i64 n, const i64* offsets, const i32* neighbors, const u64* ew, const u64* vw) {
    if (n < 0 || !offsets) throw InvalidArg("invalid graph");
    Graph g;
    g.n = n;
    g.off.assign(offsets, offsets + n + 1);
    const i64 m = g.off[n];
    if (g.off[0] != 0 || m < 0) throw InvalidArg("invalid CSR endpoints");
    for (i64 v = 0; v < n; ++v)
        if (g.off[v] > g.off[v + 1]) throw InvalidArg("nonmonotone CSR offsets");
    g.nbr.assign(neighbors, neighbors + m);
    for (i32 u : g.nbr)
        if (u < 0 || u >= n) throw InvalidArg("invalid neighbor id");
    if (ew) g.ew.assign(ew, ew + m); else g.ew.assign(static_cast<size_t>(m), 1);
    if (vw) g.vw.assign(vw, vw + n); else g.vw.assign(static_cast<size_t>(n), 1);
    return g;
}

// include/partition_capacity.hpp:12-23
u64 partition_capacity(u64 total, int parts, double ratio) {
    if (parts < 2 || parts > 32 || !std::isfinite(ratio) || ratio < 1.0)
        throw InvalidArg("invalid partition capacity options");
    const long double raw = static_cast<long double>(total) * ratio / parts;
    if (!std::isfinite(raw) || raw >= static_cast<long double>(std::numeric_limits<u64>::max()))
        throw Overflow("partition capacity exceeds uint64");
    const auto capacity = static_cast<u64>(std::floor(raw));
    if (capacity < total / static_cast<unsigned>(parts) + (total % parts != 0))
        throw InvalidArg("integer partition capacity cannot hold total weight");
    return capacity;
}

// ---------------------------------------------------------------------------
// SCLP aggregation: src/coarsen.cu:937-1659
// ---------------------------------------------------------------------------
constexpr i32 kInvalid = 0x7fffffff;  // SCLP_INVALID, coarsen.cu:201

struct Proposals {
    std::vector<i32> target;
    std::vector<u64> gain;
    std::vector<u32> tie;
};

// sclp_better_candidate, coarsen.cu:224-229
inline bool better(u64 a, u64 ta, u64 b, u64 tb) {
    return a > b || (a == b && a != 0 && ta > tb);
}

// Affinity + gain decode for every vertex: the semantics shared by the
// singleton, low, medium and high kernels (coarsen.cu:306-560) and
// sclp_decode_gain_kernel (coarsen.cu:562-598).  Connections are exact u64
// sums per neighbouring cluster (self loops skipped); the best non-mover
// cluster is the maximum of (connection, tie) with tie =
// mix32(v ^ mix32(c) ^ tie_salt) << 32 | (0xffffffff - c).
Proposals form_proposals(const Graph& g, const std::vector<i32>& clusters, u32 seed,
                         int level, int round, bool filter, u32 mover_threshold) {
    const u32 role_salt = seed ^ (static_cast<u32>(level) * 0x9e3779b9U) ^
                          (static_cast<u32>(round) * 0x85ebca6bU) ^ 0x27d4eb2dU;
    const u32 tie_salt = seed ^ (static_cast<u32>(level) * 0xc2b2ae35U) ^
                         (static_cast<u32>(round) * 0x165667b1U) ^ 0xd3a2646cU;
    auto is_mover = [&](i32 c) { return mix32(static_cast<u32>(c) ^ role_salt) < mover_threshold; };
    Proposals p;
    p.target.assign(static_cast<size_t>(g.n), kInvalid);
    p.gain.assign(static_cast<size_t>(g.n), 0);
    p.tie.assign(static_cast<size_t>(g.n), 0);
    std::unordered_map<i32, u64> conn;
    for (i64 v = 0; v < g.n; ++v) {
        conn.clear();
        for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
            const i32 u = g.nbr[e];
            if (u == v) continue;
            conn[clusters[u]] += g.ew[e];
        }
        const i32 source = clusters[v];
        u64 current = 0, best = 0, best_tie = 0;
        for (const auto& [c, w] : conn) {
            if (c == source) { current = w; continue; }
            if (filter && is_mover(c)) continue;
            const u32 h = mix32(static_cast<u32>(v) ^ mix32(static_cast<u32>(c)) ^ tie_salt);
            const u64 tie = (static_cast<u64>(h) << 32) | (0xffffffffULL - static_cast<u32>(c));
            if (better(w, tie, best, best_tie)) { best = w; best_tie = tie; }
        }
        const bool can_move = !filter || is_mover(source);
        const u64 role_gain = can_move && best > current ? best - current : 0;
        if (role_gain == 0) continue;
        const auto target = static_cast<i32>(0xffffffffULL - (best_tie & 0xffffffffULL));
        if (target < 0 || target == source) continue;
        p.target[v] = target;
        p.gain[v] = best - current;
        p.tie[v] = static_cast<u32>(best_tie >> 32);
    }
    return p;
}

// build_admission_order, coarsen.cu:1086-1121: valid proposals sorted by
// (target asc, gain desc, tie desc, vertex asc).
std::vector<i32> admission_order(const std::vector<i32>& targets, const std::vector<u64>& gains,
                                 const std::vector<u32>& ties) {
    std::vector<i32> order;
    for (i64 v = 0; v < static_cast<i64>(targets.size()); ++v)
        if (targets[v] != kInvalid) order.push_back(static_cast<i32>(v));
    std::sort(order.begin(), order.end(), [&](i32 a, i32 b) {
        if (targets[a] != targets[b])
            return static_cast<u32>(targets[a]) < static_cast<u32>(targets[b]);
        if (gains[a] != gains[b]) return gains[a] > gains[b];
        if (ties[a] != ties[b]) return ties[a] > ties[b];
        return a < b;
    });
    return order;
}

i64 count_nonzero(const std::vector<u64>& w) {
    return static_cast<i64>(std::count_if(w.begin(), w.end(), [](u64 x) { return x != 0; }));
}

struct AggregateResult {
    std::vector<i32> map;
    std::vector<u64> coarse_vw;
    i64 coarse_n = 0;
    u64 cap = 0;
};

AggregateResult aggregate(const Graph& g, int parts, u32 seed, int level, int beta, bool pack) {
    if (parts < 2 || parts > 32 || beta < 2) throw InvalidArg("invalid SCLP cluster capacity options");
    const i64 n = g.n;
    if (n <= 0 || n > std::numeric_limits<i32>::max())
        throw std::runtime_error("SCLP coarsening received an unsupported graph size");
    // coarsen.cu:953-963
    u64 total = 0, maxw = 0;
    for (u64 w : g.vw) { total += w; maxw = std::max(maxw, w); }
    const u64 denom = static_cast<u64>(beta) * static_cast<u64>(parts);
    const u64 avg_cap = total / denom + (total % denom != 0 ? 1 : 0);
    const u64 cap = std::max(maxw, avg_cap);

    std::vector<i32> clusters(static_cast<size_t>(n));
    std::iota(clusters.begin(), clusters.end(), 0);
    std::vector<u64> cw(g.vw.begin(), g.vw.end());

    i64 cluster_count = n;
    const i64 desired = (n + 1) / 2;
    // Round loop, coarsen.cu:1305-1408
    for (int round = 0; round < 4; ++round) {
        if (static_cast<double>(cluster_count) <= 0.60 * n) break;
        const i64 removable = std::max<i64>(0, cluster_count - desired);
        const double fraction = std::min(0.50, static_cast<double>(removable) /
                                                   static_cast<double>(cluster_count));
        const auto threshold = static_cast<u32>(fraction * 4294967296.0);
        const auto p = form_proposals(g, clusters, seed, level, round, true, threshold);
        const auto order = admission_order(p.target, p.gain, p.tie);
        if (!order.empty()) {
            // inclusive_scan_by_key + sclp_commit_kernel, coarsen.cu:1336-1360,652-680
            const std::vector<u64> base(cw);
            std::vector<std::pair<i32, i32>> moves;
            u64 prefix = 0;
            for (size_t i = 0; i < order.size(); ++i) {
                const i32 v = order[i];
                const i32 t = p.target[v];
                if (i == 0 || p.target[order[i - 1]] != t) prefix = 0;
                prefix += g.vw[v];
                if (base[t] <= cap && prefix <= cap - base[t]) moves.push_back({v, t});
            }
            for (auto [v, t] : moves) {
                cw[clusters[v]] -= g.vw[v];
                cw[t] += g.vw[v];
                clusters[v] = t;
            }
        }
        cluster_count = count_nonzero(cw);
        if (static_cast<double>(cluster_count) <= 0.60 * n) break;
    }

    // Isolated packing, coarsen.cu:1410-1441,741-773
    if (pack) {
        std::vector<i32> isolated;
        for (i64 v = 0; v < n; ++v)
            if (g.off[v] == g.off[v + 1]) isolated.push_back(static_cast<i32>(v));
        const auto count = static_cast<i64>(isolated.size());
        if (count > 1) {
            std::vector<u64> prefix(static_cast<size_t>(count));
            u64 run = 0;
            for (i64 i = 0; i < count; ++i) { run += g.vw[isolated[i]]; prefix[i] = run; }
            const u64 total_iso = prefix[count - 1];
            std::vector<i32> reps(static_cast<size_t>(total_iso / cap + (total_iso % cap != 0)),
                                  std::numeric_limits<i32>::max());
            for (i64 i = 0; i < count; ++i) {
                const i32 v = isolated[i];
                const u64 first = (prefix[i] - g.vw[v]) / cap, last = (prefix[i] - 1) / cap;
                if (first == last) reps[first] = std::min(reps[first], v);
            }
            for (i64 i = 0; i < count; ++i) {
                const i32 v = isolated[i];
                const u64 first = (prefix[i] - g.vw[v]) / cap, last = (prefix[i] - 1) / cap;
                if (first != last) continue;
                const i32 t = reps[first];
                if (t == v) continue;
                clusters[v] = t;
                cw[v] = 0;
                cw[t] += g.vw[v];
            }
            cluster_count = count_nonzero(cw);
        }
    }

    // Two-hop pairing, coarsen.cu:1443-1539,682-724
    if (static_cast<double>(cluster_count) > 0.60 * n) {
        const auto p = form_proposals(g, clusters, seed, level, 4, false, 0);
        std::vector<i32> favorites(static_cast<size_t>(n), kInvalid);
        for (i64 v = 0; v < n; ++v)
            favorites[v] = cw[clusters[v]] == g.vw[v] ? p.target[v] : kInvalid;
        const auto order = admission_order(favorites, p.gain, p.tie);
        const i64 cand = static_cast<i64>(order.size());
        if (cand > 0) {
            std::vector<u64> rank(static_cast<size_t>(cand));
            for (i64 i = 0; i < cand; ++i)
                rank[i] = (i > 0 && favorites[order[i]] == favorites[order[i - 1]]) ? rank[i - 1] + 1 : 1;
            std::vector<int> flag(static_cast<size_t>(cand));
            for (i64 i = 0; i < cand; ++i) {
                const bool second = (rank[i] & 1ULL) == 0ULL;
                flag[i] = second && i > 0 && g.vw[order[i - 1]] <= cap - g.vw[order[i]] ? 1 : 0;
            }
            u64 pair_count = 0;
            for (int f : flag) pair_count += static_cast<u64>(f);
            const u64 budget = static_cast<u64>(std::max<i64>(0, cluster_count - desired));
            if (std::min(pair_count, budget) > 0) {
                u64 position = 0;
                std::vector<std::pair<i32, i32>> moves;
                for (i64 i = 0; i < cand; ++i) {
                    if (!flag[i]) continue;
                    const u64 pos = position++;
                    if (pos >= budget) continue;
                    const i32 v = order[i];
                    const i32 s = clusters[v];
                    const i32 t = clusters[order[i - 1]];
                    if (s == t) continue;
                    moves.push_back({v, t});
                }
                for (auto [v, t] : moves) {
                    cw[clusters[v]] -= g.vw[v];
                    cw[t] += g.vw[v];
                    clusters[v] = t;
                }
            }
        }
        cluster_count = count_nonzero(cw);
    }

    // Compaction, coarsen.cu:1541-1577
    AggregateResult out;
    out.cap = cap;
    out.coarse_n = cluster_count;
    std::vector<i32> compact(static_cast<size_t>(n));
    i32 run = 0;
    for (i64 c = 0; c < n; ++c) { compact[c] = run; run += cw[c] > 0 ? 1 : 0; }
    out.map.resize(static_cast<size_t>(n));
    out.coarse_vw.assign(static_cast<size_t>(cluster_count), 0);
    for (i64 v = 0; v < n; ++v) {
        out.map[v] = compact[clusters[v]];
        out.coarse_vw[out.map[v]] += g.vw[v];
    }
    u64 maxc = 0;
    for (u64 w : out.coarse_vw) maxc = std::max(maxc, w);
    if (maxc > cap) throw std::runtime_error("SCLP coarsening exceeded cluster capacity");
    return out;
}

// contract_typed, coarsen.cu:1674-1814
Graph contract(const Graph& fine, const std::vector<i32>& map, i64 coarse_n,
               const std::vector<u64>& coarse_vw) {
    std::vector<std::vector<std::pair<i32, u64>>> rows(static_cast<size_t>(coarse_n));
    for (i64 v = 0; v < fine.n; ++v) {
        const i32 s = map[v];
        for (i64 e = fine.off[v]; e < fine.off[v + 1]; ++e) {
            const i32 t = map[fine.nbr[e]];
            if (s != t) rows[s].push_back({t, fine.ew[e]});
        }
    }
    Graph g;
    g.n = coarse_n;
    g.off.assign(static_cast<size_t>(coarse_n) + 1, 0);
    for (i64 c = 0; c < coarse_n; ++c) {
        auto& r = rows[c];
        std::sort(r.begin(), r.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (size_t i = 0; i < r.size(); ++i) {
            if (i > 0 && r[i].first == r[i - 1].first) { g.ew.back() += r[i].second; continue; }
            g.nbr.push_back(r[i].first);
            g.ew.push_back(r[i].second);
        }
        g.off[c + 1] = static_cast<i64>(g.nbr.size());
        std::vector<std::pair<i32, u64>>().swap(r);
    }
    g.vw = coarse_vw;
    return g;
}

struct Hierarchy {
    std::vector<Graph> levels;
    std::vector<std::vector<i32>> maps;
};

// coarsen_impl, coarsen.cu:1906-2164
Hierarchy coarsen(Graph input, int parts, u32 seed, int beta, bool pack, int max_levels, double stop) {
    if (parts < 2 || parts > 32 || beta < 2 || max_levels < 0 || !std::isfinite(stop) || stop <= 0 || stop > 1)
        throw InvalidArg("invalid coarsening options");
    Hierarchy h;
    const i64 cutoff = std::max<i64>(32, static_cast<i64>(beta) * parts);
    Graph current = std::move(input);
    for (int level = 0; level < max_levels && current.n > cutoff; ++level) {
        const u32 level_seed = seed + static_cast<u32>(level);
        auto agg = aggregate(current, parts, level_seed, level, beta, pack);
        const double ratio = static_cast<double>(agg.coarse_n) / static_cast<double>(current.n);
        if (agg.coarse_n >= current.n || ratio > stop) break;
        Graph coarse = contract(current, agg.map, agg.coarse_n, agg.coarse_vw);
        h.levels.push_back(std::move(current));
        h.maps.push_back(std::move(agg.map));
        current = std::move(coarse);
    }
    h.levels.push_back(std::move(current));
    return h;
}

// ---------------------------------------------------------------------------
// Spectral initial partition, src/initial_partition_gpu.cu:36-276 (FP64)
// ---------------------------------------------------------------------------
struct Norm { double mean, scale; };

Norm moments(const std::vector<i32>& ids, const std::vector<double>& deg, const std::vector<double>& x) {
    double mass = 0, sum = 0, sq = 0;
    for (i32 v : ids) {
        const double d = deg[v] > 0 ? deg[v] : 1.0;
        mass += d; sum += d * x[v]; sq += d * x[v] * x[v];
    }
    const double mean = sum / mass;
    const double variance = std::fmax(0.0, sq / mass - mean * mean);
    return {mean, variance > 1e-30 ? 1.0 / std::sqrt(variance) : 1.0};
}

// spectral_start + 64 x {normalize, spectral_step} + final normalize
// (initial_partition_gpu.cu:81-142,210-229)
void diffuse(const Graph& g, const std::vector<i32>& labels, const std::vector<i32>& ids,
             int group, u32 seed, int steps, std::vector<double>& x) {
    std::vector<double> deg(static_cast<size_t>(g.n), 0.0), y(static_cast<size_t>(g.n), 0.0);
    for (i32 v : ids) {
        double d = 0;
        for (i64 e = g.off[v]; e < g.off[v + 1]; ++e)
            if (labels[g.nbr[e]] == group) d += static_cast<double>(g.ew[e]);
        deg[v] = d;
        x[v] = static_cast<double>(mix32(static_cast<u32>(v) ^ seed)) / 4294967296.0 - 0.5;
    }
    Norm nm = moments(ids, deg, x);
    for (int it = 0; it <= steps; ++it) {
        for (i32 v : ids) x[v] = (x[v] - nm.mean) * nm.scale;
        if (it == steps) break;
        for (i32 v : ids) {
            double s = 0;
            for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
                const i32 u = g.nbr[e];
                if (labels[u] == group) s += static_cast<double>(g.ew[e]) * x[u];
            }
            const double d = deg[v];
            y[v] = d > 0 ? 0.5 * (x[v] + s / d) : x[v];
        }
        for (i32 v : ids) x[v] = y[v];
        nm = moments(ids, deg, x);
    }
}

// With `trace` (depths x n FP32 values, as gp_initial_partition_trace
// returns them) each task is ordered by the traced value of its depth instead
// of the FP64 diffusion, so that the split rules are checked on exactly the
// vector the device sorted; the FP64 diffusion is still computed for every
// task and the largest relative L2 distance between the two is reported in
// *max_rel_l2.
std::vector<i32> initial_partition(const Graph& g, int parts, double ratio, u32 seed,
                                   const float* trace = nullptr, int trace_depths = 0,
                                   double* max_rel_l2 = nullptr) {
    const i64 n = g.n;
    if (n <= 0 || n > std::numeric_limits<int>::max() - 255 || parts < 2 || parts > n || parts > 32 ||
        !std::isfinite(ratio) || ratio < 1.0)
        throw InvalidArg("invalid GPU initial partition input");
    auto checked = [](u64 a, u64 b) { return ~u64{0} - a < b ? ~u64{0} : a + b; };
    u64 total = 0, edge_total = 0, maxw = 0;
    for (u64 w : g.vw) { total = checked(total, w); maxw = std::max(maxw, w); }
    for (u64 w : g.ew) edge_total = checked(edge_total, w);
    if (!total || total == ~u64{0} || edge_total == ~u64{0})
        throw Overflow("GPU initializer weight accumulation overflow");
    const u64 capacity = partition_capacity(total, parts, ratio);
    if (maxw > capacity) throw InvalidArg("a vertex exceeds partition capacity");
    std::vector<i32> labels(static_cast<size_t>(n), 0), order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), 0);
    std::vector<double> x(static_cast<size_t>(n), 0.0);
    struct Task { int begin, count, first_part, parts; u64 weight; int depth; };
    std::vector<Task> tasks{{0, static_cast<int>(n), 0, parts, total, 0}};
    if (max_rel_l2) *max_rel_l2 = 0.0;
    while (!tasks.empty()) {
        const Task t = tasks.back();
        tasks.pop_back();
        if (t.parts == 1) {
            if (t.weight > capacity) throw std::runtime_error("GPU initializer infeasible balance");
            continue;
        }
        std::vector<i32> ids(order.begin() + t.begin, order.begin() + t.begin + t.count);
        diffuse(g, labels, ids, t.first_part, seed ^ static_cast<u32>(t.first_part), 64, x);
        if (trace) {
            if (t.depth >= trace_depths) throw std::runtime_error("trace has fewer depths than the task tree");
            const float* row = trace + static_cast<size_t>(t.depth) * static_cast<size_t>(n);
            double diff = 0, norm = 0;
            for (i32 v : ids) {
                const float f = row[v];
                if (f != f) throw std::runtime_error("trace has no value for a vertex of an open task");
                diff += (static_cast<double>(f) - x[v]) * (static_cast<double>(f) - x[v]);
                norm += x[v] * x[v];
                x[v] = static_cast<double>(f);
            }
            if (max_rel_l2 && norm > 1e-24) *max_rel_l2 = std::max(*max_rel_l2, std::sqrt(diff / norm));
        }
        std::sort(ids.begin(), ids.end(), [&](i32 a, i32 b) { return x[a] < x[b] || (x[a] == x[b] && a < b); });
        std::copy(ids.begin(), ids.end(), order.begin() + t.begin);
        std::vector<u64> prefix(static_cast<size_t>(t.count));
        u64 run = 0;
        for (int i = 0; i < t.count; ++i) { run += g.vw[ids[i]]; prefix[i] = run; }
        // initial_partition_gpu.cu:233-248
        const int left_parts = t.parts / 2, right_parts = t.parts - left_parts;
        const u64 target = static_cast<u64>(static_cast<long double>(t.weight) * left_parts / t.parts);
        const u64 left_limit = capacity > t.weight / left_parts ? t.weight : capacity * left_parts;
        const u64 right_limit = capacity > t.weight / right_parts ? t.weight : capacity * right_parts;
        const u64 min_left = t.weight > right_limit ? t.weight - right_limit : 0;
        int boundary = static_cast<int>(std::lower_bound(prefix.begin(), prefix.end(), target) - prefix.begin()) + 1;
        boundary = std::max(left_parts, std::min(t.count - right_parts, boundary));
        u64 left_weight = prefix[boundary - 1];
        if (left_weight > left_limit && boundary > left_parts) { --boundary; left_weight = prefix[boundary - 1]; }
        if (left_weight < min_left && boundary < t.count - right_parts) { ++boundary; left_weight = prefix[boundary - 1]; }
        if (left_weight > left_limit || left_weight < min_left)
            throw std::runtime_error("GPU spectral split cannot satisfy capacity");
        for (int i = 0; i < t.count; ++i)
            labels[ids[i]] = i < boundary ? t.first_part : t.first_part + left_parts;
        tasks.push_back({t.begin + boundary, t.count - boundary, t.first_part + left_parts, right_parts,
                         t.weight - left_weight, t.depth + 1});
        tasks.push_back({t.begin, boundary, t.first_part, left_parts, left_weight, t.depth + 1});
    }
    std::vector<u64> loads(static_cast<size_t>(parts), 0);
    for (i64 v = 0; v < n; ++v) loads[labels[v]] += g.vw[v];
    if (*std::max_element(loads.begin(), loads.end()) > capacity)
        throw std::runtime_error("GPU initializer balance validation failed");
    return labels;
}

// ---------------------------------------------------------------------------
// Refinement, src/refine_incremental.cuh:7-361 and src/refine.cu:52-142
// ---------------------------------------------------------------------------
u64 directed_cut(const Graph& g, const std::vector<i32>& labels) {
    u64 d = 0;
    for (i64 v = 0; v < g.n; ++v)
        for (i64 e = g.off[v]; e < g.off[v + 1]; ++e)
            if (labels[v] != labels[g.nbr[e]]) d += g.ew[e];
    return d;
}

u64 undirected_cut(const Graph& g, const std::vector<i32>& labels) {
    const u64 d = directed_cut(g, labels);
    if (d & 1ULL) throw std::runtime_error("refinement cut is not symmetric");
    return d / 2;
}

// Rebalance gain bucket (refine_incremental.cuh:167-171) restated with
// thresholds 1.5^j computed once on the host: for g < 0 the bucket is
// 25 + the smallest j with -g <= 1.5^j, clamped to [2, 49].
struct BucketThresholds {
    double t[48];  // j = -23 .. 24
    BucketThresholds() { for (int j = -23; j <= 24; ++j) t[j + 23] = std::pow(1.5, j); }
    int bucket(double g) const {
        if (g > 0) return 0;
        if (g == 0) return 1;
        const double a = -g;
        if (a <= t[0]) return 2;
        for (int j = -22; j <= 24; ++j) if (a <= t[j + 23]) return 25 + j;
        return 49;
    }
};

constexpr int kBuckets = 50, kSections = 16, kWidth = kBuckets * kSections;

struct RefineState {
    const Graph& g;
    int k;
    u64 cap;
    std::vector<i32>& labels;
    std::vector<u64> cache;
    std::vector<u64> pw;
    std::vector<i32> targets, flags, locks;
    std::vector<i64> gains;
    u64 current_cut = 0;
    or_refine_stats stats{};
    BucketThresholds thresholds;

    RefineState(const Graph& graph, std::vector<i32>& l, int parts, u64 capacity)
        : g(graph), k(parts), cap(capacity), labels(l) {
        const i64 n = g.n;
        cache.assign(static_cast<size_t>(n) * k, 0);
        pw.assign(static_cast<size_t>(k), 0);
        for (i64 v = 0; v < n; ++v) pw[labels[v]] += g.vw[v];
        targets.assign(static_cast<size_t>(n), -1);
        flags.assign(static_cast<size_t>(n), 0);
        locks.assign(static_cast<size_t>(n), 0);
        gains.assign(static_cast<size_t>(n), 0);
        // incremental_build_affinity, refine_incremental.cuh:7-25
        for (i64 v = 0; v < n; ++v)
            for (i64 e = g.off[v]; e < g.off[v + 1]; ++e)
                if (g.nbr[e] != v) cache[v * k + labels[g.nbr[e]]] += g.ew[e];
    }
    u64 maximum() const { return *std::max_element(pw.begin(), pw.end()); }

    // incremental_update_cache_and_cut + incremental_commit (:69-109)
    void apply(const std::vector<i32>& movers, bool lp) {
        i64 delta = 0;
        for (i32 v : movers) {
            const i32 s = labels[v], t = targets[v];
            for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
                const i32 u = g.nbr[e];
                if (u == v) continue;
                const u64 w = g.ew[e];
                cache[static_cast<i64>(u) * k + s] -= w;
                cache[static_cast<i64>(u) * k + t] += w;
                if (!flags[u] || u > v) {
                    const i32 nn = flags[u] ? targets[u] : labels[u];
                    delta += static_cast<i64>(w) * ((s != labels[u]) - (t != nn));
                }
            }
        }
        for (i32 v : movers) {
            pw[labels[v]] -= g.vw[v];
            pw[targets[v]] += g.vw[v];
            labels[v] = targets[v];
            if (lp) locks[v] = 1;
        }
        if (delta >= 0) {
            if (static_cast<u64>(delta) > current_cut) throw std::runtime_error("incremental cut underflow");
            current_cut -= static_cast<u64>(delta);
        } else {
            current_cut += static_cast<u64>(-delta);
        }
        stats.accepted += movers.size();
    }

    // Rebalance loop (:111-232, :303-330) with deterministic ranks.
    bool rebalance() {
        const i64 n = g.n;
        for (int it = 0; it < 2 * k + 4 && maximum() > cap; ++it) {
            ++stats.admission_iterations;
            std::vector<double> gpw(static_cast<size_t>(n), 0.0);
            std::vector<int> bucket(static_cast<size_t>(n), -1);
            for (i64 v = 0; v < n; ++v) {
                targets[v] = -1;
                const i32 s = labels[v];
                const u64 w = g.vw[v];
                if (pw[s] <= cap) continue;
                int best = -1;
                u64 best_conn = 0, best_slack = 0;
                for (int p = 0; p < k; ++p) {
                    if (p == s || pw[p] >= cap || w > cap - pw[p]) continue;
                    const u64 value = cache[v * k + p];
                    const u64 slack = cap - pw[p];
                    if (best < 0 || value > best_conn || (value == best_conn && slack > best_slack)) {
                        best = p; best_conn = value; best_slack = slack;
                    }
                }
                if (best >= 0 && best_conn == 0) {
                    u64 total_slack = 0;
                    for (int p = 0; p < k; ++p)
                        if (p != s && pw[p] < cap && w <= cap - pw[p])
                            total_slack = UINT64_MAX - total_slack < cap - pw[p] ? UINT64_MAX : total_slack + cap - pw[p];
                    u64 ticket = static_cast<u64>(mix32(static_cast<u32>(v))) % total_slack;
                    for (int p = 0; p < k; ++p) {
                        if (p == s || pw[p] >= cap || w > cap - pw[p]) continue;
                        const u64 slack = cap - pw[p];
                        if (ticket < slack) { best = p; break; }
                        ticket -= slack;
                    }
                }
                if (best >= 0) {
                    const u64 current = cache[v * k + s];
                    const double gain = best_conn >= current ? static_cast<double>(best_conn - current)
                                                             : -static_cast<double>(current - best_conn);
                    gpw[v] = gain / static_cast<double>(w);
                    targets[v] = best;
                    bucket[v] = s * kWidth + thresholds.bucket(gpw[v]) * kSections +
                                static_cast<int>(mix32(static_cast<u32>(v)) % kSections);
                }
            }
            auto ranked = [&](const std::vector<int>& b, std::vector<u64>& rank, std::vector<u64>& offsets) {
                std::vector<i32> order;
                for (i64 v = 0; v < n; ++v) if (b[v] >= 0) order.push_back(static_cast<i32>(v));
                std::sort(order.begin(), order.end(), [&](i32 a, i32 c) {
                    if (b[a] != b[c]) return b[a] < b[c];
                    if (gpw[a] != gpw[c]) return gpw[a] > gpw[c];
                    return a < c;
                });
                std::vector<u64> counts(static_cast<size_t>(k) * kWidth, 0);
                for (size_t i = 0; i < order.size(); ++i) {
                    const i32 v = order[i];
                    rank[v] = counts[b[v]];
                    counts[b[v]] += g.vw[v];
                }
                offsets.assign(counts.size(), 0);
                for (int p = 0; p < k; ++p) {
                    u64 run = 0;
                    for (int j = 0; j < kWidth; ++j) { offsets[p * kWidth + j] = run; run += counts[p * kWidth + j]; }
                }
            };
            std::vector<u64> rank(static_cast<size_t>(n), 0), offsets;
            ranked(bucket, rank, offsets);
            for (i64 v = 0; v < n; ++v) {
                if (bucket[v] < 0) continue;
                const int b = bucket[v], s = b / kWidth;
                if (offsets[b] + rank[v] >= pw[s] - cap) { bucket[v] = -1; continue; }
                bucket[v] = targets[v] * kWidth + b % kWidth;
            }
            ranked(bucket, rank, offsets);
            std::vector<i32> movers;
            for (i64 v = 0; v < n; ++v) {
                flags[v] = 0;
                const int b = bucket[v];
                if (b < 0) continue;
                const u64 before = offsets[b] + rank[v];
                const u64 slack = cap - pw[b / kWidth];
                flags[v] = before <= slack && g.vw[v] <= slack - before;
                if (flags[v]) movers.push_back(static_cast<i32>(v));
            }
            if (movers.empty()) return false;
            apply(movers, false);
        }
        return maximum() <= cap;
    }

    void run(int rounds) {
        const i64 n = g.n;
        current_cut = undirected_cut(g, labels);
        stats.initial_cut = current_cut;
        u64 best_cut = current_cut;
        std::vector<i32> saved_labels(labels);
        std::vector<u64> saved_pw(pw);
        u64 maxe = 0;
        for (u64 w : g.ew) maxe = std::max(maxe, w);
        const double filter = maxe <= 1 ? 0.25 : 0.75;
        int stale = 0, empty = 0;
        for (int phase = 0; phase < rounds && stale < 3; ++phase) {
            stats.rounds = phase + 1;
            // incremental_lp_proposals (:27-46)
            for (i64 v = 0; v < n; ++v) {
                targets[v] = -1;
                gains[v] = INT64_MIN;
                if (locks[v]) { locks[v] = 0; continue; }
                const i32 s = labels[v];
                u64 best = 0;
                int target = -1;
                for (int p = 0; p < k; ++p)
                    if (p != s && cache[v * k + p] > best) { best = cache[v * k + p]; target = p; }
                const u64 current = cache[v * k + s];
                if (target >= 0 && (best >= current || current - best < static_cast<u64>(filter * current))) {
                    targets[v] = target;
                    gains[v] = best >= current ? static_cast<i64>(best - current) : -static_cast<i64>(current - best);
                }
            }
            // incremental_priority_filter (:48-67)
            std::vector<i32> movers;
            for (i64 v = 0; v < n; ++v) {
                flags[v] = 0;
                if (targets[v] < 0) continue;
                const i32 s = labels[v], t = targets[v];
                const i64 gain = gains[v];
                long long corr = 0;
                for (i64 e = g.off[v]; e < g.off[v + 1]; ++e) {
                    const i32 u = g.nbr[e];
                    if (u == v || targets[u] < 0 || !(gains[u] > gain || (gains[u] == gain && u < v))) continue;
                    const auto w = static_cast<long long>(g.ew[e]);
                    corr += w * ((targets[u] == t) - (targets[u] == s) - (labels[u] == t) + (labels[u] == s));
                }
                flags[v] = gain + corr >= 0;
                if (flags[v]) movers.push_back(static_cast<i32>(v));
            }
            stats.proposals += movers.size();
            if (movers.empty()) { if (++empty >= 2) break; ++stale; continue; }
            empty = 0;
            apply(movers, true);
            if (!rebalance()) { ++stats.admission_fallbacks; break; }
            ++stale;
            if (current_cut < best_cut) {
                if (static_cast<long double>(current_cut) < 0.999L * best_cut) stale = 0;
                best_cut = current_cut;
                saved_labels = labels;
                saved_pw = pw;
            }
        }
        labels = saved_labels;
        pw = saved_pw;
        stats.final_cut = undirected_cut(g, labels);
        stats.final_max_part_weight = maximum();
        if (stats.final_cut != best_cut || stats.final_cut > stats.initial_cut || maximum() > cap)
            throw std::runtime_error("incremental refinement postcondition failed");
    }
};

or_refine_stats refine(const Graph& g, std::vector<i32>& labels, int parts, double ratio, int rounds) {
    if (parts < 2 || parts > 32 || rounds < 0 || rounds > 64 || !std::isfinite(ratio) || ratio < 1.0 || g.n <= 0)
        throw InvalidArg("invalid refinement options");
    u64 total = 0;
    std::vector<u64> loads(static_cast<size_t>(parts), 0);
    for (i64 v = 0; v < g.n; ++v) {
        if (labels[v] < 0 || labels[v] >= parts) throw InvalidArg("refinement partition has an invalid part id");
        loads[labels[v]] += g.vw[v];
        total += g.vw[v];
    }
    const u64 cap = partition_capacity(total, parts, ratio);
    if (*std::max_element(loads.begin(), loads.end()) > cap)
        throw InvalidArg("initial refinement partition is imbalanced");
    RefineState st(g, labels, parts, cap);
    st.run(rounds);
    return st.stats;
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const InvalidArg& e) {
        g_error = e.what(); return 1;
    } catch (const Overflow& e) {
        g_error = e.what(); return 3;
    } catch (const std::exception& e) {
        g_error = e.what(); return 2;
    }
}

}  // namespace

struct or_hier { Hierarchy h; };

extern "C" {

const char* or_last_error(void) { return g_error.c_str(); }

int or_partition_capacity(uint64_t total, int parts, double ratio, uint64_t* out) {
    return guarded([&] { *out = partition_capacity(total, parts, ratio); });
}

int or_recount(int64_t n, const int64_t* offsets, const int32_t* neighbors,
               const uint64_t* edge_weights, const uint64_t* vertex_weights,
               const int32_t* labels, int parts, int threads,
               uint64_t* directed_cut_out, uint64_t* loads) {
    return guarded([&] {
        if (parts < 1 || parts > 32) throw InvalidArg("invalid parts");
        if (n < 0 || offsets[0] != 0) throw InvalidArg("invalid CSR endpoints");
        for (int64_t v = 0; v < n; ++v) {
            if (offsets[v] > offsets[v + 1]) throw InvalidArg("nonmonotone CSR offsets");
            if (labels[v] < 0 || labels[v] >= parts) throw InvalidArg("invalid label");
        }
        std::fill(loads, loads + parts, 0);
        for (int64_t v = 0; v < n; ++v) loads[labels[v]] += vertex_weights ? vertex_weights[v] : 1;
        const int t = std::max(1, std::min(threads, 64));
        std::vector<u64> part(static_cast<size_t>(t), 0);
        std::vector<int> bad(static_cast<size_t>(t), 0);
        std::vector<std::thread> pool;
        for (int i = 0; i < t; ++i) {
            pool.emplace_back([&, i] {
                const int64_t lo = n * i / t, hi = n * (i + 1) / t;
                u64 local = 0;
                for (int64_t v = lo; v < hi; ++v)
                    for (int64_t e = offsets[v]; e < offsets[v + 1]; ++e) {
                        const int32_t u = neighbors[e];
                        if (u < 0 || u >= n) { bad[i] = 1; continue; }
                        if (labels[v] != labels[u]) local += edge_weights ? edge_weights[e] : 1;
                    }
                part[i] = local;
            });
        }
        for (auto& th : pool) th.join();
        for (int b : bad) if (b) throw InvalidArg("invalid neighbor id");
        u64 d = 0;
        for (u64 x : part) d += x;
        *directed_cut_out = d;
    });
}

int or_aggregate(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                 const uint64_t* edge_weights, const uint64_t* vertex_weights,
                 int parts, uint32_t seed, int level, int beta, int pack_isolated,
                 int32_t* map, int64_t* coarse_n, uint64_t* cap) {
    return guarded([&] {
        const Graph g = make_graph(n, offsets, neighbors, edge_weights, vertex_weights);
        auto r = aggregate(g, parts, seed, level, beta, pack_isolated != 0);
        std::copy(r.map.begin(), r.map.end(), map);
        *coarse_n = r.coarse_n;
        *cap = r.cap;
    });
}

int or_contract(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                const uint64_t* edge_weights, const uint64_t* vertex_weights,
                const int32_t* map, int64_t coarse_n,
                int64_t* coarse_offsets, int32_t* coarse_neighbors,
                uint64_t* coarse_edge_weights, uint64_t* coarse_vertex_weights,
                int64_t* coarse_m) {
    return guarded([&] {
        const Graph g = make_graph(n, offsets, neighbors, edge_weights, vertex_weights);
        std::vector<i32> mp(map, map + n);
        std::vector<u64> cvw(static_cast<size_t>(coarse_n), 0);
        for (i64 v = 0; v < n; ++v) {
            if (mp[v] < 0 || mp[v] >= coarse_n) throw InvalidArg("map id out of range");
            cvw[mp[v]] += g.vw[v];
        }
        const Graph c = contract(g, mp, coarse_n, cvw);
        std::copy(c.off.begin(), c.off.end(), coarse_offsets);
        std::copy(c.nbr.begin(), c.nbr.end(), coarse_neighbors);
        std::copy(c.ew.begin(), c.ew.end(), coarse_edge_weights);
        std::copy(c.vw.begin(), c.vw.end(), coarse_vertex_weights);
        *coarse_m = c.m();
    });
}

int or_coarsen(int64_t n, const int64_t* offsets, const int32_t* neighbors,
               const uint64_t* edge_weights, const uint64_t* vertex_weights,
               int parts, uint32_t seed, int beta, int pack_isolated,
               int max_levels, double stop_ratio, or_hier** out) {
    return guarded([&] {
        if (beta < 0) beta = std::max(64, (512 + parts - 1) / parts);
        auto g = make_graph(n, offsets, neighbors, edge_weights, vertex_weights);
        auto* h = new or_hier;
        try {
            h->h = coarsen(std::move(g), parts, seed, beta, pack_isolated != 0, max_levels, stop_ratio);
        } catch (...) { delete h; throw; }
        *out = h;
    });
}

int or_hier_levels(const or_hier* h) { return static_cast<int>(h->h.levels.size()); }

void or_hier_level_size(const or_hier* h, int level, int64_t* n, int64_t* m) {
    *n = h->h.levels[level].n;
    *m = h->h.levels[level].m();
}

void or_hier_level_copy(const or_hier* h, int level, int64_t* offsets, int32_t* neighbors,
                        uint64_t* edge_weights, uint64_t* vertex_weights, int32_t* map_to_next) {
    const Graph& g = h->h.levels[level];
    std::copy(g.off.begin(), g.off.end(), offsets);
    std::copy(g.nbr.begin(), g.nbr.end(), neighbors);
    std::copy(g.ew.begin(), g.ew.end(), edge_weights);
    std::copy(g.vw.begin(), g.vw.end(), vertex_weights);
    if (map_to_next && level + 1 < static_cast<int>(h->h.levels.size()))
        std::copy(h->h.maps[level].begin(), h->h.maps[level].end(), map_to_next);
}

// Same byte layout as the reference's write_hierarchy (include/hierarchy.hpp:42-126).
int or_hier_write(const or_hier* h, const char* path) {
    return guarded([&] {
        std::ofstream o(path, std::ios::binary | std::ios::trunc);
        if (!o) throw std::runtime_error("cannot open hierarchy output");
        auto put = [&](int32_t v) { o.write(reinterpret_cast<const char*>(&v), 4); };
        put(static_cast<int32_t>(h->h.levels.size()));
        for (size_t i = 0; i < h->h.levels.size(); ++i) {
            const Graph& g = h->h.levels[i];
            put(static_cast<int32_t>(g.n));
            put(static_cast<int32_t>(g.m()));
            for (i64 x : g.off) put(static_cast<int32_t>(x));
            for (i32 x : g.nbr) put(x);
            for (u64 x : g.ew) put(static_cast<int32_t>(x));
            for (u64 x : g.vw) put(static_cast<int32_t>(x));
            if (i > 0) for (i32 x : h->h.maps[i - 1]) put(x);
        }
        if (!o) throw std::runtime_error("failed while writing hierarchy");
    });
}

void or_hier_free(or_hier* h) { delete h; }

int or_diffusion(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                 const uint64_t* edge_weights, const int32_t* labels, int group,
                 uint32_t seed, int steps, double* x_out) {
    return guarded([&] {
        const Graph g = make_graph(n, offsets, neighbors, edge_weights, nullptr);
        std::vector<i32> lab(labels, labels + n), ids;
        for (i64 v = 0; v < n; ++v) if (lab[v] == group) ids.push_back(static_cast<i32>(v));
        std::vector<double> x(static_cast<size_t>(n), 0.0);
        diffuse(g, lab, ids, group, seed ^ static_cast<u32>(group), steps, x);
        std::copy(x.begin(), x.end(), x_out);
    });
}

int or_initial_partition(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                         const uint64_t* edge_weights, const uint64_t* vertex_weights,
                         int parts, double ratio, uint32_t seed, int32_t* labels) {
    return guarded([&] {
        const Graph g = make_graph(n, offsets, neighbors, edge_weights, vertex_weights);
        const auto l = initial_partition(g, parts, ratio, seed);
        std::copy(l.begin(), l.end(), labels);
    });
}

int or_initial_partition_replay(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                                const uint64_t* edge_weights, const uint64_t* vertex_weights,
                                int parts, double ratio, uint32_t seed, const float* trace,
                                int trace_depths, int32_t* labels, double* max_rel_l2) {
    return guarded([&] {
        const Graph g = make_graph(n, offsets, neighbors, edge_weights, vertex_weights);
        const auto l = initial_partition(g, parts, ratio, seed, trace, trace_depths, max_rel_l2);
        std::copy(l.begin(), l.end(), labels);
    });
}

int or_refine(int64_t n, const int64_t* offsets, const int32_t* neighbors,
              const uint64_t* edge_weights, const uint64_t* vertex_weights,
              int32_t* labels, int parts, double ratio, int max_rounds,
              or_refine_stats* stats) {
    return guarded([&] {
        const Graph g = make_graph(n, offsets, neighbors, edge_weights, vertex_weights);
        std::vector<i32> l(labels, labels + n);
        const auto s = refine(g, l, parts, ratio, max_rounds);
        std::copy(l.begin(), l.end(), labels);
        if (stats) *stats = s;
    });
}

int or_partition_from(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                      const uint64_t* edge_weights, const uint64_t* vertex_weights,
                      int parts, double ratio, uint32_t seed, const int32_t* coarsest_labels,
                      int64_t coarsest_n, int32_t* labels, uint64_t* cut) {
    return guarded([&] {
        auto g = make_graph(n, offsets, neighbors, edge_weights, vertex_weights);
        u64 total = 0;
        for (u64 w : g.vw) total += w;
        partition_capacity(total, parts, ratio);
        const int beta = std::max(64, (512 + parts - 1) / parts);
        Hierarchy h = coarsen(std::move(g), parts, seed, beta, true, 24, 0.90);
        std::vector<i32> cur;
        if (coarsest_labels) {
            if (coarsest_n != h.levels.back().n) throw InvalidArg("coarsest labels do not match the coarsest level");
            cur.assign(coarsest_labels, coarsest_labels + coarsest_n);
        } else {
            cur = initial_partition(h.levels.back(), parts, ratio, seed);
        }
        refine(h.levels.back(), cur, parts, ratio, 32);
        i64 last_refined = h.levels.back().n;
        for (size_t lv = h.levels.size() - 1; lv > 0; --lv) {
            const size_t fine_level = lv - 1;
            const Graph& fine = h.levels[fine_level];
            std::vector<i32> proj(static_cast<size_t>(fine.n));
            for (i64 v = 0; v < fine.n; ++v) proj[v] = cur[h.maps[fine_level][v]];
            cur = std::move(proj);
            if (fine_level == 0 || static_cast<double>(fine.n) >= 2.0 * static_cast<double>(last_refined)) {
                refine(fine, cur, parts, ratio, 32);
                last_refined = fine.n;
            }
        }
        std::copy(cur.begin(), cur.end(), labels);
        *cut = undirected_cut(h.levels.front(), cur);
    });
}

int or_partition(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                 const uint64_t* edge_weights, const uint64_t* vertex_weights,
                 int parts, double ratio, uint32_t seed, int32_t* labels, uint64_t* cut) {
    return or_partition_from(n, offsets, neighbors, edge_weights, vertex_weights, parts, ratio, seed, nullptr, 0,
                             labels, cut);
}

}  // extern "C"
