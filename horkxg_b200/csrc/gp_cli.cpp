// Drop-in drivers for the reference's command lines.
//
//   gpart_partition_{standard,big} <indptr.bin> <indices.bin> <parts>
//       <partition.out> [imbalance_ratio=1.03] [seed=0] [--verify]
//     (app/partition_main.cu:20-142: same grammar, files, stdout keys,
//      timer scopes and exit codes: usage -> 2, any failure -> 1 with a
//      "gpart_partition: " message on stderr)
//
//   gpart_coarsen_{standard,big} <indptr.bin> <indices.bin> <parts>
//       <hierarchy.out> [seed=0] [stop_contraction_ratio=0.90]
//       [max_levels=24] [--verify]
//     (app/coarsen_main.cu:13-79: library defaults beta=256, no isolated
//      packing; the reference's write_hierarchy file layout)
//
// Compiled twice, with GP_DRIVER_WIDTH = GP_WIDTH_STANDARD or GP_WIDTH_BIG.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>
#include <algorithm>

#include "../../include/gpart_b200.h"

#ifndef GP_DRIVER_WIDTH
#define GP_DRIVER_WIDTH GP_WIDTH_STANDARD
#endif

namespace {

// Page-locked staging for the input arrays (fast H2D); plain host memory
// when page-locking is unavailable.
struct Pinned {
    void* p = nullptr;
    bool pinned = false;
    explicit Pinned(size_t bytes) {
        if (!bytes) return;
        if (cudaMallocHost(&p, bytes) == cudaSuccess) {
            pinned = true;
        } else {
            cudaGetLastError();
            p = std::malloc(bytes);
            if (!p) throw std::runtime_error("cannot allocate host memory");
        }
    }
    ~Pinned() {
        if (!p) return;
        if (pinned) cudaFreeHost(p); else std::free(p);
    }
    int64_t* i64() const { return static_cast<int64_t*>(p); }
};

int64_t element_count(const std::string& path) {
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) throw std::runtime_error("cannot open " + path);
    const auto bytes = in.tellg();
    if (bytes < 0 || bytes % 8 != 0) throw std::runtime_error("invalid binary size " + path);
    return static_cast<int64_t>(bytes / 8);
}

void read_all(const std::string& path, int64_t* dst, int64_t count) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    int64_t done = 0;
    while (done < count) {
        const size_t chunk = static_cast<size_t>(std::min<int64_t>(count - done, int64_t{1} << 24));
        const size_t got = std::fread(dst + done, sizeof(int64_t), chunk, f);
        if (got != chunk) { std::fclose(f); throw std::runtime_error("cannot read " + path); }
        done += static_cast<int64_t>(got);
    }
    std::fclose(f);
}

struct Input {
    int64_t n = 0, m = 0;
    Pinned* off = nullptr;
    Pinned* idx = nullptr;
    ~Input() { delete off; delete idx; }
};

// src/graph.cpp:47-122 (host part: sizes, endpoints, limits).  Narrowing,
// monotonicity and neighbour ranges are checked on the GPU.
void load(const std::string& indptr, const std::string& indices, Input& in) {
    const int64_t offsets = element_count(indptr);
    const int64_t edges = element_count(indices);
    if (offsets < 1) throw std::runtime_error("empty CSR indptr");
    const int64_t n = offsets - 1;
    if (GP_DRIVER_WIDTH == GP_WIDTH_STANDARD) {
        if (n > std::numeric_limits<int32_t>::max() || edges > std::numeric_limits<int32_t>::max())
            throw std::runtime_error("graph exceeds standard CSR limits; use gpart_coarsen_big");
    } else if (n > std::numeric_limits<int32_t>::max()) {
        throw std::runtime_error("graph vertex ids exceed configured graph type");
    }
    in.off = new Pinned(static_cast<size_t>(offsets) * 8);
    in.idx = new Pinned(static_cast<size_t>(std::max<int64_t>(edges, 1)) * 8);
    read_all(indptr, in.off->i64(), offsets);
    if (in.off->i64()[0] != 0 || in.off->i64()[n] != edges) throw std::runtime_error("CSR offsets do not match indices");
    read_all(indices, in.idx->i64(), edges);
    in.n = n;
    in.m = edges;
    std::cout << "vertices=" << n << " edge_entries=" << edges << " device_count=1\n";
}

void check(gp_status s, gp_ctx* ctx) {
    if (s != GP_OK) throw std::runtime_error(ctx ? gp_ctx_error(ctx) : "operation failed");
}

int partition_main(int argc, char** argv) {
    const auto wall_start = std::chrono::steady_clock::now();
    bool verify = false;
    int pos = argc;
    while (pos > 1) {
        if (std::string(argv[pos - 1]) == "--verify") verify = true;
        else break;
        --pos;
    }
    if (pos < 5 || pos > 7) {
        std::cerr << "Usage: " << argv[0] << " <indptr.bin> <indices.bin> <parts> <partition.out>"
                  << " [imbalance_ratio=1.03] [seed] [--verify]\n";
        return 2;
    }
    gp_ctx* ctx = nullptr;
    try {
        const int parts = std::stoi(argv[3]);
        const double imbalance = pos >= 6 ? std::stod(argv[5]) : 1.03;
        const auto seed = pos >= 7 ? static_cast<uint32_t>(std::stoul(argv[6])) : 0U;
        const auto load_start = std::chrono::steady_clock::now();
        Input in;
        load(argv[1], argv[2], in);
        uint64_t cap = 0;
        if (gp_partition_capacity(static_cast<uint64_t>(in.n), parts, imbalance, &cap) != GP_OK) {
            // reproduce the reference's messages through a throwaway context-free call
            throw std::runtime_error(parts < 2 || parts > 32 || !(imbalance >= 1.0)
                                         ? "invalid partition capacity options"
                                         : "integer partition capacity cannot hold total weight");
        }
        const auto load_end = std::chrono::steady_clock::now();
        std::cout << "verify=" << (verify ? 1 : 0) << '\n';
        gp_options o;
        gp_options_default(&o);
        o.parts = parts;
        o.imbalance = imbalance;
        o.seed = seed;
        o.verify = verify ? 1 : 0;
        o.log = 1;
        if (const char* det = std::getenv("GP_DETERMINISTIC")) o.deterministic = std::atoi(det) != 0;
        std::cout << "pipeline_mode=incremental_bucket cluster_size_factor=" << std::max(64, (512 + parts - 1) / parts)
                  << " pack_isolated=1\n";
        check(gp_ctx_create(0, &ctx), ctx);
        gp_graph g{};
        g.n = in.n;
        g.m = in.m;
        g.width = GP_DRIVER_WIDTH;
        g.memory = GP_MEMORY_HOST;
        g.index64 = 1;
        g.offsets = in.off->p;
        g.neighbors = in.idx->p;
        std::vector<int32_t> labels(static_cast<size_t>(in.n));
        gp_report rep{};
        const auto call_start = std::chrono::steady_clock::now();
        check(gp_partition(ctx, &g, &o, labels.data(), &rep), ctx);
        const double call_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - call_start).count();
        const auto output_start = std::chrono::steady_clock::now();
        std::ofstream out(argv[4], std::ios::binary | std::ios::trunc);
        if (!out) throw std::runtime_error("cannot open partition output");
        out.write(reinterpret_cast<const char*>(labels.data()), static_cast<std::streamsize>(labels.size() * 4));
        out.close();
        if (!out) throw std::runtime_error("cannot write partition output");
        const auto output_end = std::chrono::steady_clock::now();
        const double input_seconds = std::chrono::duration<double>(load_end - load_start).count();
        const double output_seconds = std::chrono::duration<double>(output_end - output_start).count();
        const double d2h = std::max(0.0, call_seconds - rep.prepare_seconds - rep.algorithm_seconds);
        std::cout << std::setprecision(10) << "partition_timing input_load_seconds=" << input_seconds
                  << " coarsen_seconds=" << rep.coarsen_seconds
                  << " initial_partition_seconds=" << rep.initial_seconds
                  << " uncoarsen_seconds=" << rep.uncoarsen_seconds
                  << " input_prepare_seconds=" << rep.prepare_seconds
                  << " hierarchy_free_seconds=" << rep.free_seconds
                  << " final_partition_d2h_seconds=" << d2h
                  << " timing_scope=jet_device_input_to_device_partition"
                  << " partition_output_seconds=" << output_seconds
                  << " partition_total_seconds=" << rep.algorithm_seconds
                  << " algorithm_total_seconds=" << rep.algorithm_seconds
                  << " wall_total_seconds="
                  << std::chrono::duration<double>(output_end - wall_start).count() << '\n';
        gp_ctx_destroy(ctx);
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "gpart_partition: " << e.what() << '\n';
        gp_ctx_destroy(ctx);
        return 1;
    }
}

int coarsen_main(int argc, char** argv) {
    int pos = argc;
    const bool verify = argc > 1 && std::string(argv[argc - 1]) == "--verify";
    if (verify) --pos;
    if (pos < 5 || pos > 8) {
        std::cerr << "Usage: " << argv[0] << " <indptr.bin> <indices.bin> <parts> <hierarchy.out>"
                  << " [seed=0] [stop_contraction_ratio=0.90] [max_levels=24] [--verify]\n";
        return 2;
    }
    gp_ctx* ctx = nullptr;
    gp_hierarchy* h = nullptr;
    try {
        const int parts = std::stoi(argv[3]);
        const uint32_t seed = pos >= 6 ? static_cast<uint32_t>(std::stoul(argv[5])) : 0U;
        const double stop = pos >= 7 ? std::stod(argv[6]) : 0.90;
        const int max_levels = pos >= 8 ? std::stoi(argv[7]) : 24;
        if (parts < 2 || parts > 32) throw std::runtime_error("parts must be between 2 and 32");
        if (stop <= 0.0 || stop > 1.0) throw std::runtime_error("invalid coarsening stop ratio");
        if (max_levels <= 0 || max_levels > 200) throw std::runtime_error("invalid coarsening max levels");
        Input in;
        load(argv[1], argv[2], in);
        gp_options o;
        gp_options_default(&o);
        o.parts = parts;
        o.seed = seed;
        o.stop_ratio = stop;
        o.max_levels = max_levels;
        o.verify = verify ? 1 : 0;
        o.cluster_size_factor = 256;   // kBeta, include/coarsen.hpp:15
        o.pack_isolated = 0;
        o.log = 1;
        check(gp_ctx_create(0, &ctx), ctx);
        gp_graph g{};
        g.n = in.n;
        g.m = in.m;
        g.width = GP_DRIVER_WIDTH;
        g.memory = GP_MEMORY_HOST;
        g.index64 = 1;
        g.offsets = in.off->p;
        g.neighbors = in.idx->p;
        const auto t0 = std::chrono::steady_clock::now();
        check(gp_coarsen(ctx, &g, &o, &h), ctx);
        const bool skip = std::getenv("ML_SKIP_HIERARCHY_EXPORT") != nullptr;
        if (!skip && gp_hierarchy_write(h, argv[4]) != GP_OK) throw std::runtime_error("cannot write hierarchy");
        int64_t cn = 0;
        gp_hierarchy_level(h, gp_hierarchy_levels(h) - 1, &cn, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
        std::cout << "ml_hierarchy_levels=" << gp_hierarchy_levels(h) << " coarsest_vertices=" << cn
                  << " stop_contraction_ratio=" << stop << " method=sclp\n";
        std::cout << "ml_total_seconds=" << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
                  << " hierarchy=" << (skip ? "skipped" : argv[4]) << " coarsen_only=1 method=sclp graph_type="
                  << (GP_DRIVER_WIDTH == GP_WIDTH_BIG ? "big" : "standard") << '\n';
        gp_hierarchy_free(h);
        gp_ctx_destroy(ctx);
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "gpart_coarsen: " << e.what() << '\n';
        gp_hierarchy_free(h);
        gp_ctx_destroy(ctx);
        return 1;
    }
}

}  // namespace

int main(int argc, char** argv) {
    const std::string self = argv[0];
    if (self.find("coarsen") != std::string::npos) return coarsen_main(argc, argv);
    return partition_main(argc, argv);
}
