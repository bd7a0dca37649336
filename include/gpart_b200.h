/*
 * gpart_b200.h - C ABI of the B200-native multilevel k-way graph partitioner.
 *
 * The library replaces the partition path behind the reference's
 * gpart_partition_standard / gpart_partition_big drivers
 * (app/partition_main.cu:20-142): SCLP coarsening, recursive spectral
 * bisection and incremental bucketed refinement, from CSR to int32 labels.
 * Every entry point is plain C: pointers, sizes and status codes, no C++ or
 * torch types.  A context owns one CUDA stream and a memory pool on one GPU;
 * it is not thread-safe (one context per host thread, as the reference's
 * scratch pool is thread_local, include/detail/scratch_pool.hpp:35).
 *
 * Status codes follow the reference's exception classes:
 *   GP_EINVAL    <- std::invalid_argument (bad input, infeasible capacity)
 *   GP_ERUNTIME  <- std::runtime_error   (spectral split infeasible, SCLP cap
 *                                         exceeded, postconditions)
 *   GP_EOVERFLOW <- std::overflow_error  (weight ranges)
 * plus GP_ECUDA / GP_ENOMEM / GP_ETIMEOUT for device failures.
 */
#ifndef GPART_B200_H
#define GPART_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gp_status {
    GP_OK = 0,
    GP_EINVAL = 1,
    GP_ERUNTIME = 2,
    GP_EOVERFLOW = 3,
    GP_ECUDA = 4,
    GP_ETIMEOUT = 5,
    GP_ENOMEM = 6
} gp_status;

/* Graph widths: the reference's StandardTypes / BigTypes
 * (include/graph_types.hpp:7-17). */
enum { GP_WIDTH_STANDARD = 0, GP_WIDTH_BIG = 1 };
/* Where the arrays of a gp_graph live. */
enum { GP_MEMORY_HOST = 0, GP_MEMORY_DEVICE = 1 };

/* A symmetric CSR graph.  With index64 = 0 the arrays use the width's types:
 * offsets int32 (standard) / int64 (big), neighbours int32, weights
 * uint32 / uint64; device arrays in these types are used in place, without a
 * copy, and must stay valid and unmodified during the call.  With index64 = 1
 * offsets and neighbours are the int64 arrays of the reference's input files
 * (src/graph.cpp:47-122); the library narrows and validates them on the GPU
 * with the reference's rules and messages.  index64 = 2 means int64 offsets
 * with int32 neighbours (the packed multi-graph layout).  NULL weights mean unit weights
 * (the reference's file input always has unit weights,
 * src/graph.cpp:117-118). */
typedef struct gp_graph {
    int64_t n;
    int64_t m;
    int32_t width;
    int32_t memory;
    int32_t index64;
    int32_t reserved;
    const void* offsets;
    const void* neighbors;
    const void* edge_weights;
    const void* vertex_weights;
} gp_graph;

/* Partition options; gp_options_default() gives the production values of
 * app/partition_main.cu:37-82. */
typedef struct gp_options {
    int32_t parts;               /* 2..32 */
    int32_t cluster_size_factor; /* <= 0: max(64, ceil(512/parts)) */
    double imbalance;            /* >= 1.0, default 1.03 */
    uint32_t seed;
    int32_t verify;              /* strict checks, the reference's --verify */
    int32_t deterministic;       /* (gain, vertex id) ranking inside rebalance buckets */
    int32_t pack_isolated;       /* default 1 */
    int32_t max_levels;          /* default 24 */
    int32_t max_rounds;          /* refinement phases per level, default 32 */
    double stop_ratio;           /* default 0.90 */
    double growth_ratio;         /* refine a level when n >= ratio * last refined n; 2.0 */
    int32_t log;                 /* print the reference's key=value lines to stdout */
    int32_t reserved;
} gp_options;

typedef struct gp_report {
    int64_t n, m;
    uint64_t cut;                 /* final undirected cut (final_edge_cut=) */
    uint64_t capacity;            /* floor(ratio * W / k) */
    uint64_t total_edge_weight;   /* undirected */
    uint64_t part_weights[32];
    int32_t levels;               /* hierarchy levels incl. the input */
    int32_t reserved;
    int64_t coarsest_n;
    uint64_t initial_cut;         /* cut of the spectral partition on the coarsest level */
    double coarsen_seconds;
    double initial_seconds;
    double uncoarsen_seconds;
    double free_seconds;
    double algorithm_seconds;     /* the reference's algorithm_total_seconds scope */
    double prepare_seconds;       /* upload + narrowing + validation (outside the algorithm scope) */
} gp_report;

typedef struct gp_refine_stats {
    int32_t rounds;
    uint64_t proposals, accepted, initial_cut, final_cut, final_max_part_weight;
    int32_t admission_iterations, admission_fallbacks;
} gp_refine_stats;

typedef struct gp_ctx gp_ctx;
typedef struct gp_hierarchy gp_hierarchy;

void gp_options_default(gp_options* options);

/* Context on CUDA device `device`. */
gp_status gp_ctx_create(int device, gp_ctx** out);
void gp_ctx_destroy(gp_ctx* ctx);
/* Message of the last failure on this context ("" if none). */
const char* gp_ctx_error(const gp_ctx* ctx);

/* include/partition_capacity.hpp:12-23 (host only). */
gp_status gp_partition_capacity(uint64_t total, int parts, double ratio, uint64_t* out);

/* Full pipeline (replaces app/partition_main.cu:59-96: coarsen,
 * initial_partition_gpu, uncoarsen).  labels has n int32 entries, in host
 * memory when graph->memory is HOST, else in device memory.  The report's
 * algorithm_seconds covers the reference's algorithm_total_seconds scope:
 * from the uploaded, validated graph to device labels with scratch released. */
gp_status gp_partition(gp_ctx* ctx, const gp_graph* graph, const gp_options* options,
                       int32_t* labels, gp_report* report);

/* Packed multi-graph CSR.  `packed` holds several instances back to back:
 * offsets has n_total+1 entries and indexes the concatenated neighbour (and
 * weight) arrays, neighbour ids are local to their instance (0 <= id < the
 * instance's vertex count).  This partitions the instance of vertices
 * [vertex_begin, vertex_end) exactly as gp_partition would partition it on
 * its own; `labels` points at that instance's labels (vertex_end -
 * vertex_begin entries, host or device like the graph).  No counterpart in
 * the reference, which takes one graph per process run. */
gp_status gp_partition_range(gp_ctx* ctx, const gp_graph* packed, int64_t vertex_begin, int64_t vertex_end,
                             const gp_options* options, int32_t* labels, gp_report* report);

/* Device memory of the context's caching allocator: bytes in use, bytes
 * cached for reuse, and the peak in use (optionally reset to the current
 * value).  gp_ctx_trim returns the cached blocks to the driver. */
gp_status gp_ctx_memory(gp_ctx* ctx, uint64_t* live, uint64_t* cached, uint64_t* peak, int reset_peak);
gp_status gp_ctx_trim(gp_ctx* ctx);
/* Counters of the context's caching allocator since its creation: blocks
 * requested, blocks obtained from the driver (cudaMalloc), cached blocks
 * returned to the driver to make room, and host milliseconds spent in the
 * allocator.  A partition of a graph seen before normally needs no driver
 * allocation at all. */
gp_status gp_ctx_allocator_stats(gp_ctx* ctx, uint64_t* requests, uint64_t* driver_allocs, uint64_t* cache_frees,
                                 double* host_ms);

/* One SCLP aggregation (replaces gpart::aggregate, include/coarsen.hpp:88-92;
 * src/coarsen.cu:1661-1671).  map: n int32 (host).  cluster_size_factor and
 * pack_isolated are used as given. */
gp_status gp_aggregate(gp_ctx* ctx, const gp_graph* graph, int parts, uint32_t seed, int level,
                       int cluster_size_factor, int pack_isolated, int32_t* map,
                       int64_t* coarse_n, uint64_t* cluster_cap);

/* Contraction (replaces gpart::contract, include/coarsen.hpp:94-97;
 * src/coarsen.cu:1826-1831).  Host outputs: offsets (coarse_n+1), neighbours
 * and edge weights sized for at least graph->m entries, vertex weights
 * (coarse_n); rows come out sorted by target. */
gp_status gp_contract(gp_ctx* ctx, const gp_graph* graph, const int32_t* map, int64_t coarse_n,
                      int64_t* offsets, int32_t* neighbors, uint64_t* edge_weights,
                      uint64_t* vertex_weights, int64_t* coarse_m);

/* Coarsening to a host hierarchy (replaces gpart::coarsen,
 * include/coarsen.hpp:99-101; the export of app/coarsen_main.cu:13-79). */
gp_status gp_coarsen(gp_ctx* ctx, const gp_graph* graph, const gp_options* options,
                     gp_hierarchy** out);
int32_t gp_hierarchy_levels(const gp_hierarchy* h);
/* Copies level `level`; any output pointer may be NULL (then only sizes). */
gp_status gp_hierarchy_level(const gp_hierarchy* h, int level, int64_t* n, int64_t* m,
                             int64_t* offsets, int32_t* neighbors, uint64_t* edge_weights,
                             uint64_t* vertex_weights, int32_t* map_to_next);
/* The reference's write_hierarchy layout (include/hierarchy.hpp:42-126). */
gp_status gp_hierarchy_write(const gp_hierarchy* h, const char* path);
void gp_hierarchy_free(gp_hierarchy* h);

/* Spectral initial partition (replaces gpart::initial_partition_gpu,
 * include/initial_partition.hpp:9-12).  labels: n int32 (host). */
gp_status gp_initial_partition(gp_ctx* ctx, const gp_graph* graph, int parts, double ratio,
                               uint32_t seed, int32_t* labels);

/* gp_initial_partition with its diffusion vectors (same reference interface,
 * include/initial_partition.hpp:9-12; the trace replaces no reference
 * output).  For recursion depth d (0 = the root bisection) trace[d*n + v] is
 * the normalised FP32 value that ordered vertex v in its task's split
 * (src/initial_partition_gpu.cu:206-233), NaN when v was in no open task at
 * that depth.  *depths receives the number of depths of the task tree for
 * `parts`; trace (host, may be NULL to query) must hold trace_depths >= that
 * many rows of n floats. */
gp_status gp_initial_partition_trace(gp_ctx* ctx, const gp_graph* graph, int parts, double ratio, uint32_t seed,
                                     int32_t* labels, float* trace, int32_t trace_depths, int32_t* depths);

/* FP32 diffusion of one bisection task (src/initial_partition_gpu.cu:81-142):
 * vertices with labels[v] == group, seed ^ group, `steps` steps; x: n floats
 * (host), 0 outside the group. */
gp_status gp_diffusion(gp_ctx* ctx, const gp_graph* graph, const int32_t* labels, int group,
                       uint32_t seed, int steps, float* x);

/* Incremental bucketed refinement (replaces gpart::refine_partition,
 * include/refine.hpp:57-61).  labels: n int32 (host), refined in place. */
gp_status gp_refine(gp_ctx* ctx, const gp_graph* graph, int32_t* labels, int parts, double ratio,
                    int max_rounds, int deterministic, gp_refine_stats* stats);

/* GPU recount: exact directed cut and per-part loads (the semantics of
 * tools/verify_partition.py:22-65 and src/graph.cpp:192-212). */
gp_status gp_cut(gp_ctx* ctx, const gp_graph* graph, const int32_t* labels, int parts,
                 uint64_t* directed_cut, uint64_t* loads);

/* Partition analysis on the GPU: the per-part report of the reference's CPU
 * analyzer (replaces graph_untils/analyze_partition.cpp:425-499 over the
 * directed CSR entries; edge weights are the graph's integer weights, unit
 * when NULL, where the analyzer reads float values).  `labels` (n entries,
 * host or device like the graph) must lie in [0, parts), 1 <= parts <= 1024,
 * else GP_EINVAL.  per_part (parts entries) and summary may be NULL. */
typedef struct gp_part_stats {
    uint64_t vertices;             /* |V(pi)|: vertex count */
    uint64_t internal_edges;       /* entries with both ends in the part */
    uint64_t outgoing_cut_edges;   /* entries from the part to another */
    uint64_t incoming_cut_edges;   /* entries from another part into it */
    uint64_t weighted_internal;
    uint64_t weighted_outgoing;
    uint64_t weighted_incoming;
} gp_part_stats;

typedef struct gp_analysis {
    int32_t parts;
    int32_t reserved;
    uint64_t directed_edge_cut;          /* global cut |C(G,P)|, directed entries */
    uint64_t weighted_directed_edge_cut;
    uint64_t max_local_cut;              /* max over parts of outgoing + incoming */
    uint64_t weighted_max_local_cut;
    double avg_local_cut;
    double weighted_avg_local_cut;
    double vertex_avg;                   /* n / parts */
    uint64_t min_vertices, max_vertices;
    double vertex_imbalance;             /* max / avg */
    double vertex_max_deviation;         /* max |part - avg| / avg */
    double edge_set_avg;                 /* (m + directed cut) / parts */
    uint64_t min_edge_set, max_edge_set; /* internal + outgoing + incoming */
    double edge_set_imbalance;
    double edge_set_max_deviation;
} gp_analysis;

gp_status gp_analyze(gp_ctx* ctx, const gp_graph* graph, const int32_t* labels, int parts, gp_part_stats* per_part,
                     gp_analysis* summary);

/* Symmetrise and deduplicate a CSR (replaces graph_untils/csr_symmetrize.cpp:
 * 277-538, the reference's preprocessing of directed or asymmetric inputs):
 * every entry (v, u) with u != v stands for the undirected edge {u, v}; self
 * loops are dropped; the output holds both directions of every distinct edge,
 * rows ascending by neighbour -- the same offsets and indices the reference
 * writes.  Edge and vertex weights of the input are ignored (the output is
 * unweighted, as the reference's).  offsets_out: n + 1 int64; neighbors_out:
 * `capacity` entries of neighbor_bytes (4 = int32, 8 = int64 as in the
 * reference's files); both in host memory when graph->memory is HOST, else
 * device memory.  At most 2 * m entries are needed; when `capacity` is
 * smaller than the output, nothing is written, info still reports the sizes
 * and GP_EINVAL is returned. */
typedef struct gp_symmetrize_info {
    int64_t self_loops_removed;
    int64_t unique_undirected_edges;
    int64_t output_directed_edges;   /* entries of the symmetric CSR */
} gp_symmetrize_info;

gp_status gp_symmetrize(gp_ctx* ctx, const gp_graph* graph, int64_t* offsets_out, void* neighbors_out,
                        int32_t neighbor_bytes, int64_t capacity, gp_symmetrize_info* info);

/* R-MAT graph generated on the GPU: 2^scale vertices, edge_factor * 2^scale
 * pairs with quadrant probabilities (a, b, c, 1 - a - b - c), vertex ids
 * relabelled by a seeded permutation, then symmetrised like gp_symmetrize.
 * The pairs and the permutation are drawn exactly as the package's host
 * generator draws them (horkxg_b200/graphs.py rmat(), the graphs both bench
 * arms read), so the CSR is identical to that generator's files.  No
 * counterpart in the reference, whose RMAT inputs come from its tools'
 * external files; this makes the largest configured inputs (RMAT-26) without
 * the host.  Output as in gp_symmetrize, in host or device memory per
 * `memory` (GP_MEMORY_HOST / GP_MEMORY_DEVICE). */
gp_status gp_generate_rmat(gp_ctx* ctx, int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                           int32_t memory, int64_t* offsets_out, void* neighbors_out, int32_t neighbor_bytes,
                           int64_t capacity, gp_symmetrize_info* info);

/* Kernel launches issued by this context so far (all of them are the
 * library's own sm_100a kernels). */
uint64_t gp_launch_count(const gp_ctx* ctx);
/* Host waits on the context's stream so far (device-to-host round trips). */
uint64_t gp_sync_count(const gp_ctx* ctx);
/* How the host thread waits for the context's stream: 0 (default) polls,
 * which gives the lowest latency per round trip; 1 sleeps until the work is
 * done, which frees the core for other host threads when many contexts run
 * at once (the server's slots). */
gp_status gp_ctx_set_sync_mode(gp_ctx* ctx, int blocking);
/* Number of contexts expected to run at once on the device (default 1).
 * The context's grid-stride kernels then take at most about 1/share of the
 * device's block slots, so that kernels of other contexts run beside them;
 * results do not depend on it.  The server sets it to its slot count. */
gp_status gp_ctx_set_device_share(gp_ctx* ctx, int share);
/* Small coarsest graphs (at most 4096 vertices, 2,097,152 edges and rows of
 * at most 4096 edges) run the spectral diffusion in one thread-block cluster
 * instead of a cooperative grid; both compute the same values.  enable = 0 keeps the
 * grid kernel for every graph (default 1). */
gp_status gp_ctx_set_small_diffusion(gp_ctx* ctx, int enable);

/* Hubs (vertices of more than 2048 edges) aggregate their neighbours'
 * clusters in hash tables.  on_chip = 1 (default) keeps the table of every hub
 * of up to about 9,400 edges in one CTA's shared memory, on levels whose
 * total edge weight fits 32 bits; 0 keeps every table in global memory.  Both
 * give the same hierarchy. */
gp_status gp_ctx_set_hub_tables(gp_ctx* ctx, int on_chip);

/* The rebalance loop of the default (non-deterministic) refinement
 * (src/refine_incremental.cuh:303-330, one host round trip per iteration in
 * the reference) as a CUDA graph: the iteration's kernels form the body of a
 * conditional WHILE node, and a one-warp kernel after them ends the loop on
 * the device (no mover, no part above capacity, or 2k + 4 iterations); one
 * round trip per rebalance reads the summed counters.  mode 0 (default)
 * drives the same kernels from the host; 1 builds a level's graph once that
 * level's host loop has run 8 iterations (building costs about as much as ten
 * round trips); 2 uses the graph from a level's first rebalance.  Measured on
 * one B200 the graph saves host round trips but not consistently time: RMAT-20
 * partitions ran 3-8% faster, RMAT-24 within run-to-run noise, graphs of
 * 10^4-10^5 vertices 4-6% slower (their rebalances end after one or two
 * iterations, so building the graph does not pay).  The deterministic mode
 * and profiling always use the host loop. */
gp_status gp_ctx_set_graph_loops(gp_ctx* ctx, int mode);

/* Spectral initial partition that allocates no device memory.
 *
 * For callers that cannot call cudaMalloc: a process whose device memory is
 * owned by another allocator (a framework pool that accounts for every byte;
 * a raw cudaMalloc would bypass its budget and can fail or fragment it), or a
 * latency-bound caller that cannot afford cudaMalloc's implicit
 * synchronisation.  This entry point has no counterpart in the reference;
 * it computes the same labels as gp_initial_partition.
 *
 * The caller passes the graph in device memory in the width's own types
 * (index64 = 0; at most 65536 vertices -- larger graphs are rejected with
 * GP_EINVAL), `labels` as a device array of n int32 entries, and the stream
 * to run on (NULL = the legacy default stream).  All scratch lives in a 4 MiB
 * array compiled into the library, which every GPU that loads the library
 * holds until the process exits.  The first call on a device looks the
 * array's device address up (cudaGetSymbolAddress); make that first call
 * before any stream capture.  Every call shares the one array, so calls that
 * overlap on the GPU (concurrent streams or threads) race and must be
 * serialised by the caller.  On failure a message is written to `message`
 * (if not NULL, at most message_capacity bytes including the terminator). */
gp_status gp_initial_partition_static(const gp_graph* graph, int parts, double ratio, uint32_t seed,
                                      int32_t* labels, void* stream, char* message,
                                      uint64_t message_capacity);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events with the library's. */
void* gp_ctx_stream(const gp_ctx* ctx);

/* Per-kernel CUDA-event timing on the context stream (off by default).
 * Enabling (or disabling) clears the table. */
gp_status gp_profile_enable(gp_ctx* ctx, int on);
/* Writes one line per kernel: "<name> <launches> <milliseconds> <algorithmic
 * bytes>" (bytes are recorded for the kernels whose traffic model is known,
 * else 0). */
gp_status gp_profile_dump(gp_ctx* ctx, char* buffer, uint64_t capacity);

/* ------------------------------------------------------------------------
 * Serving and batching (no counterpart in the reference).
 *
 * A server owns `slots` contexts on one device, each with its own stream,
 * memory pool and host worker thread.  Submitted requests wait in a FIFO
 * queue and are admitted in arrival order whenever a slot is idle and the
 * projected device footprint (gp_footprint_bytes) of the running requests
 * plus the next one fits in `memory_budget`; their work overlaps on the
 * device.  Each request runs the same pipeline as gp_partition, so its result
 * does not depend on the other requests (bit-identical when
 * options.deterministic is set).  The graph arrays and `labels` of a request
 * must stay valid until gp_server_wait returns for it.
 * ---------------------------------------------------------------------- */
typedef struct gp_server gp_server;

typedef struct gp_request_info {
    int32_t status;
    int32_t slot;                 /* slot that ran the request */
    double queued_seconds;        /* submit -> admitted */
    double service_seconds;       /* admitted -> labels written */
    double latency_seconds;       /* submit -> labels written */
    uint64_t footprint_bytes;     /* projection used for admission */
    char message[192];            /* failure message, "" on success */
} gp_request_info;

/* Projected peak device bytes of one partition (an upper bound of the
 * library's own allocations; caller-owned device input is not counted). */
uint64_t gp_footprint_bytes(int64_t n, int64_t m, int32_t parts, int32_t width, int32_t index64_host);

gp_status gp_server_create(int device, int32_t slots, uint64_t memory_budget, gp_server** out);
/* Waits for every admitted and queued request, then releases the slots. */
void gp_server_destroy(gp_server* server);
const char* gp_server_error(const gp_server* server);
/* Queue one graph; GP_ENOMEM if its projection alone exceeds the budget. */
gp_status gp_server_submit(gp_server* server, const gp_graph* graph, const gp_options* options, int32_t* labels,
                           uint64_t* ticket);
/* Queue one instance of a packed CSR (see gp_partition_range). */
gp_status gp_server_submit_range(gp_server* server, const gp_graph* packed, int64_t vertex_begin,
                                 int64_t vertex_end, const gp_options* options, int32_t* labels, uint64_t* ticket);
gp_status gp_server_poll(gp_server* server, uint64_t ticket, int32_t* done);
/* Blocks until the request is done, returns its status and releases the
 * ticket. */
gp_status gp_server_wait(gp_server* server, uint64_t ticket, gp_report* report, gp_request_info* info);

/* Partitions every instance of a packed CSR (vertex_offsets: count+1 host
 * entries, instance i = vertices [vertex_offsets[i], vertex_offsets[i+1]))
 * on the server's slots, largest instances first.  options, reports and
 * statuses have `count` entries (options NULL = defaults; reports/statuses
 * may be NULL); labels has n_total entries.  Returns the first failing
 * instance's status (details in gp_server_error). */
gp_status gp_partition_batch(gp_server* server, const gp_graph* packed, int32_t count,
                             const int64_t* vertex_offsets, const gp_options* options, int32_t* labels,
                             gp_report* reports, int32_t* statuses);

#ifdef __cplusplus
}
#endif
#endif
