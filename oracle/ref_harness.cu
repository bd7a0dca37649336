// Test-infrastructure harness linked against the reference's own compiled
// objects (built by oracle/Makefile into oracle/_ref/).  It is a checker, never
// part of the product: it dumps the reference's SCLP hierarchy for the
// production coarsening options so that the hierarchy produced by the
// B200 build can be compared with it bit for bit.
//
// Usage:
//   ref_hierarchy_<variant> <indptr.bin> <indices.bin> <parts> <seed>
//                           <cluster_size_factor> <pack_isolated 0|1>
//                           <hierarchy.out> [max_levels=24] [stop_ratio=0.90]
//
// cluster_size_factor < 0 selects the production value
// max(64, ceil(512/parts)) used by app/partition_main.cu:53-55.
// The file format is the reference's write_hierarchy (include/hierarchy.hpp:42-126).
#include "coarsen.hpp"
#include "graph.hpp"
#include "graph_types.hpp"
#include "hierarchy.hpp"

#include <algorithm>
#include <cstdint>
#include <iostream>
#include <stdexcept>
#include <string>

int main(int argc, char** argv) {
    try {
        if (argc < 8 || argc > 10) {
            std::cerr << "usage: " << argv[0]
                      << " indptr indices parts seed beta pack_isolated out"
                         " [max_levels] [stop_ratio]\n";
            return 2;
        }
        using Types = gpart::ActiveTypes;
        const int parts = std::stoi(argv[3]);
        const auto seed = static_cast<std::uint32_t>(std::stoul(argv[4]));
        int beta = std::stoi(argv[5]);
        if (beta < 0) beta = std::max(64, (512 + parts - 1) / parts);
        const bool pack = std::stoi(argv[6]) != 0;
        auto graph = gpart::load_weighted_graph<Types>(argv[1], argv[2]);
        gpart::CoarsenOptions options;
        options.parts = parts;
        options.seed = seed;
        options.cluster_size_factor = beta;
        options.pack_isolated = pack;
        if (argc >= 9) options.max_levels = std::stoi(argv[8]);
        if (argc >= 10) options.stop_contraction_ratio = std::stod(argv[9]);
        auto hierarchy = gpart::coarsen<Types>(graph, options);
        gpart::write_hierarchy(hierarchy, argv[7]);
        std::cout << "ref_hierarchy levels=" << hierarchy.levels.size()
                  << " stop_reason=" << hierarchy.stop_reason << '\n';
        return 0;
    } catch (const std::exception& error) {
        std::cerr << "ref_harness: " << error.what() << '\n';
        return 1;
    }
}
