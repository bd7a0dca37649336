// Synthetic graph generators for the partitioner's workloads.
//
// Every generator writes the partitioner's input format: native-endian int64
// CSR offsets (n+1) and int64 neighbour ids (m), symmetric, rows sorted and
// free of self loops and duplicate entries (the semantics of the reference's
// graph_untils/csr_symmetrize.cpp:277-538).  All generators are deterministic
// functions of their parameters and seed; they use a counter-based splitmix64
// stream so the multithreaded output does not depend on the thread count.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

using u64 = std::uint64_t;
using i64 = std::int64_t;
using u32 = std::uint32_t;

thread_local std::string g_error;

inline u64 splitmix64(u64 x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// Uniform double in [0,1) from stream `s`, draw `i`.
inline double uniform(u64 s, u64 i) {
    return static_cast<double>(splitmix64(s ^ splitmix64(i)) >> 11) * (1.0 / 9007199254740992.0);
}

int thread_count() {
    const unsigned hw = std::thread::hardware_concurrency();
    return static_cast<int>(std::max(1u, std::min(hw, 64u)));
}

template <typename F>
void parallel_for(i64 count, F&& f) {
    const int t = thread_count();
    std::vector<std::thread> pool;
    for (int i = 0; i < t; ++i) {
        pool.emplace_back([&, i] {
            const i64 lo = count * i / t, hi = count * (i + 1) / t;
            f(lo, hi);
        });
    }
    for (auto& th : pool) th.join();
}

void write_file(const std::string& path, const void* data, size_t bytes) {
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + tmp);
    const char* p = static_cast<const char*>(data);
    size_t done = 0;
    while (done < bytes) {
        const size_t chunk = std::min<size_t>(bytes - done, size_t{1} << 28);
        if (std::fwrite(p + done, 1, chunk, f) != chunk) { std::fclose(f); throw std::runtime_error("short write " + tmp); }
        done += chunk;
    }
    if (std::fclose(f) != 0) throw std::runtime_error("cannot close " + tmp);
    if (std::rename(tmp.c_str(), path.c_str()) != 0) throw std::runtime_error("cannot rename " + tmp);
}

// Build a symmetric, sorted, duplicate-free CSR from undirected pairs.
void pairs_to_csr(i64 n, const std::vector<u32>& src, const std::vector<u32>& dst,
                  std::vector<i64>& offsets, std::vector<i64>& indices) {
    const i64 pairs = static_cast<i64>(src.size());
    std::vector<std::atomic<u32>> degree(static_cast<size_t>(n));
    parallel_for(n, [&](i64 lo, i64 hi) { for (i64 v = lo; v < hi; ++v) degree[v].store(0, std::memory_order_relaxed); });
    parallel_for(pairs, [&](i64 lo, i64 hi) {
        for (i64 i = lo; i < hi; ++i) {
            if (src[i] == dst[i]) continue;
            degree[src[i]].fetch_add(1, std::memory_order_relaxed);
            degree[dst[i]].fetch_add(1, std::memory_order_relaxed);
        }
    });
    std::vector<i64> raw_off(static_cast<size_t>(n) + 1, 0);
    for (i64 v = 0; v < n; ++v) raw_off[v + 1] = raw_off[v] + degree[v].load(std::memory_order_relaxed);
    std::vector<u32> raw(static_cast<size_t>(raw_off[n]));
    std::vector<std::atomic<i64>> cursor(static_cast<size_t>(n));
    parallel_for(n, [&](i64 lo, i64 hi) { for (i64 v = lo; v < hi; ++v) cursor[v].store(raw_off[v], std::memory_order_relaxed); });
    parallel_for(pairs, [&](i64 lo, i64 hi) {
        for (i64 i = lo; i < hi; ++i) {
            const u32 a = src[i], b = dst[i];
            if (a == b) continue;
            raw[cursor[a].fetch_add(1, std::memory_order_relaxed)] = b;
            raw[cursor[b].fetch_add(1, std::memory_order_relaxed)] = a;
        }
    });
    std::vector<i64> unique_deg(static_cast<size_t>(n), 0);
    parallel_for(n, [&](i64 lo, i64 hi) {
        for (i64 v = lo; v < hi; ++v) {
            auto b = raw.begin() + raw_off[v], e = raw.begin() + raw_off[v + 1];
            std::sort(b, e);
            unique_deg[v] = std::unique(b, e) - b;
        }
    });
    offsets.assign(static_cast<size_t>(n) + 1, 0);
    for (i64 v = 0; v < n; ++v) offsets[v + 1] = offsets[v] + unique_deg[v];
    indices.resize(static_cast<size_t>(offsets[n]));
    parallel_for(n, [&](i64 lo, i64 hi) {
        for (i64 v = lo; v < hi; ++v)
            for (i64 j = 0; j < unique_deg[v]; ++j) indices[offsets[v] + j] = raw[raw_off[v] + j];
    });
}

struct Csr {
    std::vector<i64> off, idx;
};

void emit(const Csr& g, const char* indptr_path, const char* indices_path, i64* n_out, i64* m_out) {
    write_file(indptr_path, g.off.data(), g.off.size() * sizeof(i64));
    write_file(indices_path, g.idx.data(), g.idx.size() * sizeof(i64));
    *n_out = static_cast<i64>(g.off.size()) - 1;
    *m_out = static_cast<i64>(g.idx.size());
}

template <typename F>
int guarded(F&& f) {
    try { f(); return 0; } catch (const std::exception& e) { g_error = e.what(); return 1; }
}

template <typename F>
void* hold(F&& build, i64* n, i64* m) {
    try {
        auto* g = new Csr(build());
        *n = static_cast<i64>(g->off.size()) - 1;
        *m = static_cast<i64>(g->idx.size());
        return g;
    } catch (const std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}


// 2D 5-point grid, vertex id = row * nx + column.
Csr build_grid2d(i64 nx, i64 ny) {
    {
        if (nx < 1 || ny < 1) throw std::runtime_error("invalid grid");
        const i64 nv = nx * ny;
        std::vector<i64> off(static_cast<size_t>(nv) + 1, 0), idx;
        for (i64 v = 0; v < nv; ++v) {
            const i64 x = v % nx, y = v / nx;
            off[v + 1] = off[v] + (x > 0) + (x + 1 < nx) + (y > 0) + (y + 1 < ny);
        }
        idx.resize(static_cast<size_t>(off[nv]));
        parallel_for(nv, [&](i64 lo, i64 hi) {
            for (i64 v = lo; v < hi; ++v) {
                const i64 x = v % nx, y = v / nx;
                i64 p = off[v];
                if (y > 0) idx[p++] = v - nx;
                if (x > 0) idx[p++] = v - 1;
                if (x + 1 < nx) idx[p++] = v + 1;
                if (y + 1 < ny) idx[p++] = v + nx;
            }
        });
        return Csr{std::move(off), std::move(idx)};
    }
}

// 3D 7-point grid, vertex id = (z * ny + y) * nx + x.
Csr build_grid3d(i64 nx, i64 ny, i64 nz) {
    {
        if (nx < 1 || ny < 1 || nz < 1) throw std::runtime_error("invalid grid");
        const i64 plane = nx * ny, nv = plane * nz;
        std::vector<i64> off(static_cast<size_t>(nv) + 1, 0), idx;
        for (i64 v = 0; v < nv; ++v) {
            const i64 x = v % nx, y = (v / nx) % ny, z = v / plane;
            off[v + 1] = off[v] + (x > 0) + (x + 1 < nx) + (y > 0) + (y + 1 < ny) + (z > 0) + (z + 1 < nz);
        }
        idx.resize(static_cast<size_t>(off[nv]));
        parallel_for(nv, [&](i64 lo, i64 hi) {
            for (i64 v = lo; v < hi; ++v) {
                const i64 x = v % nx, y = (v / nx) % ny, z = v / plane;
                i64 p = off[v];
                if (z > 0) idx[p++] = v - plane;
                if (y > 0) idx[p++] = v - nx;
                if (x > 0) idx[p++] = v - 1;
                if (x + 1 < nx) idx[p++] = v + 1;
                if (y + 1 < ny) idx[p++] = v + nx;
                if (z + 1 < nz) idx[p++] = v + plane;
            }
        });
        return Csr{std::move(off), std::move(idx)};
    }
}

// R-MAT with 2^scale vertices and edge_factor * 2^scale generated pairs,
// quadrant probabilities (a, b, c, 1-a-b-c); vertex ids are relabelled by a
// seeded random permutation; pairs are symmetrised with self loops and
// duplicates removed.
Csr build_rmat(int scale, int edge_factor, double a, double b, double c, u64 seed) {
    {
        if (scale < 1 || scale > 30 || edge_factor < 1) throw std::runtime_error("invalid rmat");
        const i64 nv = i64{1} << scale;
        const i64 pairs = nv * edge_factor;
        const u64 stream = splitmix64(seed * 0x100000001b3ULL + 0x5851f42d4c957f2dULL);
        std::vector<u32> src(static_cast<size_t>(pairs)), dst(static_cast<size_t>(pairs));
        const double ab = a + b, abc = a + b + c;
        parallel_for(pairs, [&](i64 lo, i64 hi) {
            for (i64 i = lo; i < hi; ++i) {
                u32 s = 0, d = 0;
                for (int level = 0; level < scale; ++level) {
                    const double r = uniform(stream, static_cast<u64>(i) * 64 + static_cast<u64>(level));
                    const u32 bs = r >= ab ? 1u : 0u;
                    const u32 bd = (r >= a && r < ab) || r >= abc ? 1u : 0u;
                    s = (s << 1) | bs;
                    d = (d << 1) | bd;
                }
                src[i] = s;
                dst[i] = d;
            }
        });
        // Seeded Fisher-Yates relabelling.
        std::vector<u32> perm(static_cast<size_t>(nv));
        for (i64 v = 0; v < nv; ++v) perm[v] = static_cast<u32>(v);
        const u64 pstream = splitmix64(stream ^ 0xa0761d6478bd642fULL);
        for (i64 v = nv - 1; v > 0; --v) {
            const u64 j = splitmix64(pstream ^ static_cast<u64>(v)) % static_cast<u64>(v + 1);
            std::swap(perm[v], perm[j]);
        }
        parallel_for(pairs, [&](i64 lo, i64 hi) {
            for (i64 i = lo; i < hi; ++i) { src[i] = perm[src[i]]; dst[i] = perm[dst[i]]; }
        });
        std::vector<i64> off, idx;
        pairs_to_csr(nv, src, dst, off, idx);
        return Csr{std::move(off), std::move(idx)};
    }
}

// Random geometric graph: nv points uniform in the unit square, an edge for
// every pair at Euclidean distance < radius.  Vertices are numbered in
// row-major cell order (cells of side >= radius), which keeps neighbours
// close in id space as spatial generators usually do.
Csr build_rgg(i64 nv, double radius, u64 seed) {
    {
        if (nv < 1 || !(radius > 0)) throw std::runtime_error("invalid rgg");
        const u64 stream = splitmix64(seed * 0x9e3779b97f4a7c15ULL + 0x2545f4914f6cdd1dULL);
        std::vector<double> px(static_cast<size_t>(nv)), py(static_cast<size_t>(nv));
        parallel_for(nv, [&](i64 lo, i64 hi) {
            for (i64 i = lo; i < hi; ++i) {
                px[i] = uniform(stream, static_cast<u64>(i) * 2);
                py[i] = uniform(stream, static_cast<u64>(i) * 2 + 1);
            }
        });
        const i64 cells = std::max<i64>(1, std::min<i64>(static_cast<i64>(1.0 / radius), 1 << 15));
        auto cell_of = [&](double x) { return std::min<i64>(cells - 1, static_cast<i64>(x * cells)); };
        std::vector<i64> count(static_cast<size_t>(cells * cells) + 1, 0);
        std::vector<i64> cell(static_cast<size_t>(nv));
        for (i64 i = 0; i < nv; ++i) { cell[i] = cell_of(py[i]) * cells + cell_of(px[i]); ++count[cell[i] + 1]; }
        for (i64 c = 0; c < cells * cells; ++c) count[c + 1] += count[c];
        std::vector<i64> order(static_cast<size_t>(nv));
        {
            std::vector<i64> cur(count.begin(), count.end() - 1);
            for (i64 i = 0; i < nv; ++i) order[cur[cell[i]]++] = i;
        }
        // New id = position in cell order.
        std::vector<double> qx(static_cast<size_t>(nv)), qy(static_cast<size_t>(nv));
        for (i64 j = 0; j < nv; ++j) { qx[j] = px[order[j]]; qy[j] = py[order[j]]; }
        const double r2 = radius * radius;
        std::vector<std::vector<i64>> rows(static_cast<size_t>(nv));
        parallel_for(nv, [&](i64 lo, i64 hi) {
            for (i64 v = lo; v < hi; ++v) {
                const i64 cx = cell_of(qx[v]), cy = cell_of(qy[v]);
                auto& row = rows[v];
                for (i64 dy = -1; dy <= 1; ++dy) {
                    const i64 y = cy + dy;
                    if (y < 0 || y >= cells) continue;
                    for (i64 dx = -1; dx <= 1; ++dx) {
                        const i64 x = cx + dx;
                        if (x < 0 || x >= cells) continue;
                        const i64 c = y * cells + x;
                        for (i64 u = count[c]; u < count[c + 1]; ++u) {
                            if (u == v) continue;
                            const double ddx = qx[u] - qx[v], ddy = qy[u] - qy[v];
                            if (ddx * ddx + ddy * ddy < r2) row.push_back(u);
                        }
                    }
                }
                std::sort(row.begin(), row.end());
            }
        });
        std::vector<i64> off(static_cast<size_t>(nv) + 1, 0), idx;
        for (i64 v = 0; v < nv; ++v) off[v + 1] = off[v] + static_cast<i64>(rows[v].size());
        idx.resize(static_cast<size_t>(off[nv]));
        parallel_for(nv, [&](i64 lo, i64 hi) {
            for (i64 v = lo; v < hi; ++v) std::copy(rows[v].begin(), rows[v].end(), idx.begin() + off[v]);
        });
        return Csr{std::move(off), std::move(idx)};
    }
}


}  // namespace

extern "C" {

const char* gp_gen_last_error(void) { return g_error.c_str(); }

int gp_gen_grid2d(i64 nx, i64 ny, const char* indptr_path, const char* indices_path, i64* n, i64* m) {
    return guarded([&] { emit(build_grid2d(nx, ny), indptr_path, indices_path, n, m); });
}

int gp_gen_grid3d(i64 nx, i64 ny, i64 nz, const char* indptr_path, const char* indices_path, i64* n, i64* m) {
    return guarded([&] { emit(build_grid3d(nx, ny, nz), indptr_path, indices_path, n, m); });
}

int gp_gen_rmat(int scale, int edge_factor, double a, double b, double c, u64 seed,
                const char* indptr_path, const char* indices_path, i64* n, i64* m) {
    return guarded([&] { emit(build_rmat(scale, edge_factor, a, b, c, seed), indptr_path, indices_path, n, m); });
}

int gp_gen_rgg(i64 nv, double radius, u64 seed, const char* indptr_path, const char* indices_path,
               i64* n, i64* m) {
    return guarded([&] { emit(build_rgg(nv, radius, seed), indptr_path, indices_path, n, m); });
}

// In-memory variants: the graph is kept in a handle; gp_gen_copy writes its
// offsets (int64) and neighbours (int32 or int64) into caller arrays.
void* gp_gen_grid2d_new(i64 nx, i64 ny, i64* n, i64* m) {
    return hold([&] { return build_grid2d(nx, ny); }, n, m);
}

void* gp_gen_rmat_new(int scale, int edge_factor, double a, double b, double c, u64 seed, i64* n, i64* m) {
    return hold([&] { return build_rmat(scale, edge_factor, a, b, c, seed); }, n, m);
}

void* gp_gen_rgg_new(i64 nv, double radius, u64 seed, i64* n, i64* m) {
    return hold([&] { return build_rgg(nv, radius, seed); }, n, m);
}

int gp_gen_copy(const void* handle, i64* offsets, void* neighbors, int neighbor_bytes) {
    return guarded([&] {
        const auto* g = static_cast<const Csr*>(handle);
        if (!g || (neighbor_bytes != 4 && neighbor_bytes != 8)) throw std::runtime_error("invalid copy");
        if (offsets) std::copy(g->off.begin(), g->off.end(), offsets);
        if (!neighbors) return;
        if (neighbor_bytes == 8) {
            std::copy(g->idx.begin(), g->idx.end(), static_cast<i64*>(neighbors));
        } else {
            auto* out = static_cast<std::int32_t*>(neighbors);
            parallel_for(static_cast<i64>(g->idx.size()), [&](i64 lo, i64 hi) {
                for (i64 i = lo; i < hi; ++i) out[i] = static_cast<std::int32_t>(g->idx[i]);
            });
        }
    });
}

void gp_gen_free(void* handle) { delete static_cast<Csr*>(handle); }

}  // extern "C"
