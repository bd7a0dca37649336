/* Test infrastructure: CPU restatement of horkxg's partition pipeline.
 *
 * This library is the checker for the B200 build.  Only tests/, the smoke()
 * check and bench.py's CPU-baseline leg load it; the product never does.
 * Each function names the reference file:line it restates.
 *
 * Graph arguments: n vertices, CSR offsets (int64, n+1), neighbours (int32, m),
 * edge weights (uint64, m; NULL = unit) and vertex weights (uint64, n;
 * NULL = unit).  Status codes: 0 ok, 1 invalid argument, 2 runtime
 * (infeasible / postcondition), 3 overflow.
 */
#ifndef GP_ORACLE_H
#define GP_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

const char* or_last_error(void);

/* include/partition_capacity.hpp:12-23 */
int or_partition_capacity(uint64_t total, int parts, double ratio, uint64_t* out);

/* tools/verify_partition.py:22-65 and src/graph.cpp:192-212: exact directed
 * cut (all directed entries whose endpoints differ, weighted) and per-part
 * vertex-weight loads.  Multithreaded. */
int or_recount(int64_t n, const int64_t* offsets, const int32_t* neighbors,
               const uint64_t* edge_weights, const uint64_t* vertex_weights,
               const int32_t* labels, int parts, int threads,
               uint64_t* directed_cut, uint64_t* loads);

/* One SCLP aggregation (src/coarsen.cu:937-1659).  Writes map[n]; returns the
 * coarse vertex count and the cluster cap. */
int or_aggregate(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                 const uint64_t* edge_weights, const uint64_t* vertex_weights,
                 int parts, uint32_t seed, int level, int beta, int pack_isolated,
                 int32_t* map, int64_t* coarse_n, uint64_t* cap);

/* Contraction (src/coarsen.cu:1674-1814): coarse CSR with rows sorted by
 * target, internal edges dropped, parallel edges summed.  The caller sizes
 * coarse arrays with m (an upper bound); *coarse_m receives the edge count. */
int or_contract(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                const uint64_t* edge_weights, const uint64_t* vertex_weights,
                const int32_t* map, int64_t coarse_n,
                int64_t* coarse_offsets, int32_t* coarse_neighbors,
                uint64_t* coarse_edge_weights, uint64_t* coarse_vertex_weights,
                int64_t* coarse_m);

/* Full coarsening (src/coarsen.cu:1906-2164).  beta < 0 selects the
 * production factor max(64, ceil(512/parts)) (app/partition_main.cu:53-55). */
typedef struct or_hier or_hier;
int or_coarsen(int64_t n, const int64_t* offsets, const int32_t* neighbors,
               const uint64_t* edge_weights, const uint64_t* vertex_weights,
               int parts, uint32_t seed, int beta, int pack_isolated,
               int max_levels, double stop_ratio, or_hier** out);
int or_hier_levels(const or_hier* h);
void or_hier_level_size(const or_hier* h, int level, int64_t* n, int64_t* m);
void or_hier_level_copy(const or_hier* h, int level, int64_t* offsets,
                        int32_t* neighbors, uint64_t* edge_weights,
                        uint64_t* vertex_weights, int32_t* map_to_next);
int or_hier_write(const or_hier* h, const char* path);
void or_hier_free(or_hier* h);

/* FP64 lazy diffusion of one bisection task
 * (src/initial_partition_gpu.cu:81-142,206-229): vertices with
 * labels[v]==group take part; x0 = hash(v ^ (seed ^ group))/2^32 - 1/2;
 * `steps` steps of y = d>0 ? (x + D^-1 A x)/2 : x, each preceded by the
 * weighted mean/variance normalisation; x_out[v] is the final normalised value
 * (0 outside the group). */
int or_diffusion(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                 const uint64_t* edge_weights, const int32_t* labels, int group,
                 uint32_t seed, int steps, double* x_out);

/* Recursive spectral bisection (src/initial_partition_gpu.cu:170-276), FP64. */
int or_initial_partition(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                         const uint64_t* edge_weights, const uint64_t* vertex_weights,
                         int parts, double ratio, uint32_t seed, int32_t* labels);

/* The same recursion, each task ordered by a traced FP32 vector (depths x n,
 * NaN outside open tasks) instead of the FP64 diffusion; *max_rel_l2 gets the
 * largest relative L2 distance between a task's traced and FP64 vectors. */
int or_initial_partition_replay(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                                const uint64_t* edge_weights, const uint64_t* vertex_weights,
                                int parts, double ratio, uint32_t seed, const float* trace,
                                int trace_depths, int32_t* labels, double* max_rel_l2);

typedef struct {
    int rounds;
    uint64_t proposals, accepted, initial_cut, final_cut, final_max_part_weight;
    int admission_iterations, admission_fallbacks;
} or_refine_stats;

/* Incremental bucketed refinement (src/refine_incremental.cuh:235-361) with
 * the deterministic in-bucket ranking: inside each rebalance bucket vertices
 * are ranked by (gain per weight descending, vertex id ascending). */
int or_refine(int64_t n, const int64_t* offsets, const int32_t* neighbors,
              const uint64_t* edge_weights, const uint64_t* vertex_weights,
              int32_t* labels, int parts, double ratio, int max_rounds,
              or_refine_stats* stats);

/* Whole pipeline: coarsen (production options) -> FP64 initial partition ->
 * level-by-level projection and refinement (src/refine.cu:423-646).
 * Returns the final undirected cut. */
int or_partition(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                 const uint64_t* edge_weights, const uint64_t* vertex_weights,
                 int parts, double ratio, uint32_t seed, int32_t* labels,
                 uint64_t* cut);

/* or_partition starting from given labels of the coarsest level (coarsest_n
 * entries) instead of the FP64 initial partition (NULL = compute it). */
int or_partition_from(int64_t n, const int64_t* offsets, const int32_t* neighbors,
                      const uint64_t* edge_weights, const uint64_t* vertex_weights,
                      int parts, double ratio, uint32_t seed, const int32_t* coarsest_labels,
                      int64_t coarsest_n, int32_t* labels, uint64_t* cut);

#ifdef __cplusplus
}
#endif
#endif
