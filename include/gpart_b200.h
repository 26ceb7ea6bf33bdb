/*
 * gpart_b200 — C ABI of the B200-native multilevel k-way graph partitioner.
 *
 * Every entry point takes plain pointers and sizes; no C++ or framework types
 * cross this boundary and no exception escapes it.  Host buffers belong to the
 * caller.  Each function returns a gp_status; on failure gp_last_error()
 * returns a thread-local message.
 *
 * Reference interfaces replaced (Acc-GPart, paths inside its source tree):
 *   gp_partition            the pipeline that app/partition_main.cu:47-137 drives:
 *                           load → partition_capacity → coarsen
 *                           (include/coarsen.hpp:111) → initial_partition_metis
 *                           (include/initial_partition.hpp:6) → uncoarsen
 *                           (include/uncoarsen.hpp:19) → labels
 *   gp_partition_device     the same pipeline on caller-owned device buffers
 *                           (the reference's resident DeviceWeightedGraph path,
 *                           include/graph.hpp:148-171)
 *   gp_refine               refine_partition (include/refine.hpp:84-88)
 *   gp_read_csr_int64       load_weighted_graph (include/graph.hpp:173, src/graph.cpp:47)
 *   gp_write_csr_int64      the on-disk int64 CSR format that loader reads
 *   gp_partition_capacity   partition_capacity (include/partition_capacity.hpp:14)
 *   gp_verify               gpart_verify_csr (tools/verify_csr.cpp:37-110), extended
 *                           with vertex/edge weights and a caller-chosen epsilon
 *   gp_edge_cut             host_cut (src/graph.cpp:184)
 */
#ifndef GPART_B200_H
#define GPART_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gp_status {
    GP_OK = 0,
    GP_INVALID_ARGUMENT = 1,    /* malformed CSR, k outside 2..128, bad epsilon ...   */
    GP_CAPACITY_INFEASIBLE = 2, /* floor(total*eps/k) cannot hold the total weight    */
    GP_OUT_OF_MEMORY = 3,       /* device or host allocation failed                   */
    GP_DEVICE_TIMEOUT = 4,      /* a bounded device wait gave up                      */
    GP_INTERNAL = 5,            /* an algorithm invariant failed (reference would throw) */
    GP_CUDA_ERROR = 6,          /* a CUDA runtime call failed                         */
    GP_NO_DEVICE = 7,           /* no usable CUDA device / extension not loaded       */
    GP_IO_ERROR = 8             /* file could not be opened, read or written          */
} gp_status;

/* A graph in CSR form. offsets[n+1], neighbors[m] (int32), vertex_weights[n]
 * and edge_weights[m] (uint32).  A NULL weight array means unit weights,
 * exactly like the reference's implicit unit edge weights
 * (include/detail/edge_weight.hpp:8).  The graph must be symmetric with equal
 * reverse weights and strictly positive vertex weights. */
typedef struct gp_csr {
    int64_t n;
    int64_t m;
    const int32_t* offsets;
    const int32_t* neighbors;
    const uint32_t* vertex_weights;
    const uint32_t* edge_weights;
} gp_csr;

/* Per-call statistics (all times in seconds, measured with CUDA events on
 * the context stream where noted). */
typedef struct gp_stats {
    uint64_t edge_cut;            /* final undirected cut                            */
    uint64_t max_part_weight;     /* heaviest part                                   */
    uint64_t capacity;            /* floor(total*eps/k)                              */
    uint64_t initial_cut;         /* cut of the METIS partition of the coarsest graph */
    int32_t levels;               /* graphs in the hierarchy (input included)        */
    int32_t coarsest_vertices;
    double coarsen_seconds;       /* device time of coarsening                       */
    double initial_seconds;       /* METIS step, including its copies                */
    double uncoarsen_seconds;     /* projection + refinement                         */
    double algorithm_seconds;     /* input resident → labels resident                */
    double h2d_seconds;           /* host → device copy of the input (gp_partition)  */
    double d2h_seconds;           /* device → host copy of the labels (gp_partition) */
    uint64_t kernel_launches;     /* kernels this library launched during the call   */
    uint64_t algorithmic_bytes;   /* compulsory HBM traffic model of the V-cycle     */
    uint64_t device_peak_bytes;   /* most device memory the call held at once in the
                                     context's arenas (its measured footprint)       */
    uint32_t hierarchy_reused;    /* 1: a server request reused a kept hierarchy      */
    uint32_t reserved;
} gp_stats;

/* Flags for gp_partition / gp_partition_device. */
#define GP_FLAG_VERIFY           0x1u /* the reference's --verify invariants, on host copies */
#define GP_FLAG_KEEP_HIERARCHY   0x2u /* keep host copies of every level for gp_level_*     */
#define GP_FLAG_NO_SEED_MATCHING 0x4u /* GPART_HEM_COARSEN=0 (app/partition_main.cu:57)    */
#define GP_FLAG_QUIET            0x8u /* no per-level key=value log lines on stdout        */
#define GP_FLAG_COARSEN_ONLY     0x10u /* stop after coarsening (levels kept, no labels)   */
#define GP_FLAG_REQUIRE_BALANCED 0x20u /* gp_refine: reject an over-capacity start
                                          (RefineOptions::allow_initial_imbalance = false) */

typedef struct gp_context gp_context;

/* One context per host thread; contexts are independent of each other.  The
 * context owns a device arena and a CUDA stream on `device`. */
gp_status gp_context_create(int device, gp_context** out);
void gp_context_destroy(gp_context* ctx);
const char* gp_last_error(void);
const char* gp_version(void);

/* Coarsening knobs of the reference CLI's environment variables
 * (app/partition_main.cu:55-87): "seed_matching" (GPART_HEM_COARSEN),
 * "capacity_safe_fast_path" (GPART_REGRET_FORCE_FULL), "cluster_size_factor"
 * (GPART_COARSE_BETA, 0 = default rule), "progressive_fine_factor"
 * (GPART_FINE_FACTOR), "progressive_capacity_growth" (GPART_CAPACITY_GROWTH),
 * "heavy_edge_degree_limit" (GPART_HEM_DEGREE_LIMIT).  Also "arena_chunk_mb"
 * (1..2^24, default 256): the smallest block the context's grow-only device
 * arenas request from cudaMalloc at a time. */
gp_status gp_set_option(gp_context* ctx, const char* name, int64_t value);

/* Partition a host CSR.  Copies the graph to the device, runs the V-cycle,
 * copies int32 labels (length n, values in [0,k)) back to labels_out. */
gp_status gp_partition(gp_context* ctx, const gp_csr* graph, int32_t k,
                       double epsilon, uint32_t seed, uint32_t flags,
                       int32_t* labels_out, gp_stats* stats);

/* Same, with every pointer of `graph` and labels_out in device memory of the
 * context's device.  `stream` is a cudaStream_t (NULL: the context stream);
 * the call returns after the labels are written. */
gp_status gp_partition_device(gp_context* ctx, const gp_csr* graph, int32_t k,
                              double epsilon, uint32_t seed, uint32_t flags,
                              int32_t* labels_out_device, void* stream,
                              gp_stats* stats);

/* What one gp_refine call did: the RefineStats fields of the reference
 * (include/refine.hpp:28-53) that describe its moves. */
typedef struct gp_refine_stats {
    int32_t rounds;               /* label-propagation rounds run                     */
    int32_t admission_iterations; /* capacity-repair iterations                       */
    int32_t checkpoint_updates;   /* rounds that improved the best cut                */
    int32_t reserved;
    uint64_t proposals;           /* label-propagation movers, summed over rounds     */
    uint64_t accepted;            /* vertices moved: propagation, repair, exchange    */
    uint64_t initial_cut, final_cut, final_max_part_weight, capacity;
    uint64_t lp_cut_gain, lp_cut_loss;             /* cut change of propagation batches */
    uint64_t rebalance_cut_gain, rebalance_cut_loss;/* cut change of repair batches   */
    uint64_t group_cut_gain, group_accepted;        /* capacity exchange batches      */
    double seconds;               /* device time of the refinement                    */
    uint64_t kernel_launches;
} gp_refine_stats;

/* refine_partition (include/refine.hpp:84-88, src/refine.cu:470-481): refines
 * the host labelling `labels` (n int32 in [0,k), overwritten with the result)
 * of the host graph with one level of the pipeline's refinement — capacity
 * repair of an over-capacity start, up to max_rounds (0..64; the pipeline
 * uses 32) label-propagation rounds with priority filtering and exact
 * updates, then on graphs of at most 65,536 vertices up to exchange_rounds
 * (0..8; the pipeline uses 2) capacity-exchange batches.  Capacity repair
 * orders donors and receiver tickets deterministically (the reference orders
 * them by atomic arrival).  Flags: GP_FLAG_VERIFY, GP_FLAG_QUIET,
 * GP_FLAG_REQUIRE_BALANCED.  A start whose repair cannot restore capacity
 * returns GP_CAPACITY_INFEASIBLE and leaves `labels` unchanged. */
gp_status gp_refine(gp_context* ctx, const gp_csr* graph, int32_t k, double epsilon,
                    int32_t max_rounds, int32_t exchange_rounds, uint32_t flags,
                    int32_t* labels, gp_refine_stats* stats);

/* Cut and part loads of a labelling of a device-resident graph
 * (refine_cut_kernel + accumulate_part_weights_kernel, src/refine.cu:63-126).
 * graph pointers, labels (n int32 in [0,k)), cut_out (1 uint64) and
 * loads_out (k uint64) are device memory; cut_out receives the directed
 * cut / 2.  Ordered on `stream` (NULL: the context stream); returns after the
 * results are written.  Per-block partial sums live in the context arena.
 * Labels outside [0,k), neighbours outside [0,n) and offsets outside [0,m]
 * are skipped, never dereferenced, and make the call return
 * GP_INVALID_ARGUMENT. */
gp_status gp_evaluate_device(gp_context* ctx, const gp_csr* graph, const int32_t* labels,
                             int32_t k, uint64_t* cut_out, uint64_t* loads_out,
                             void* stream);

/* Allocation-free twin of gp_evaluate_device, with no counterpart in the
 * reference.  For callers that cannot let a library allocate device memory:
 * a framework whose caching allocator owns the device-memory budget, or a
 * serving loop that must not call cudaMalloc/cudaFree (which can synchronise
 * the device) once it is running.  It calls no cudaMalloc, cudaFree or other
 * allocating routine and needs no context: the per-block partial sums live
 * in one fixed file-scope device array of 592 x 130 uint64 (616 KB) that every
 * GPU loading this library holds until the process exits.  k is limited to
 * 1..128 (the array's capacity); larger k returns GP_INVALID_ARGUMENT.
 * Runs on the current device and `stream` (NULL: the legacy default stream)
 * and returns without waiting for the results, so it cannot report bad
 * device data as a status: labels outside [0,k), neighbours outside [0,n) and
 * offsets outside [0,m] are skipped, never dereferenced, and *cut_out then
 * receives UINT64_MAX (no real cut reaches it).  The first call on each
 * device looks up the array's device address (cudaGetSymbolAddress) and
 * caches it; make that first call before any stream capture.  The cache
 * assumes the device's primary context for the life of the process (no
 * cudaDeviceReset, no other driver-API context current).  All calls on a
 * device share the one array and it keeps the last call's contents: calls
 * whose work overlaps on the GPU (different streams, or different host
 * threads) race on it and must be serialised by the caller. */
gp_status gp_evaluate_device_static(const gp_csr* graph, const int32_t* labels,
                                    int32_t k, uint64_t* cut_out,
                                    uint64_t* loads_out, void* stream);

/* ---- many graphs on one GPU ---- */

/* One partition request of a batch or a server.  `graph` is a host CSR
 * (for a server request naming a resident graph it is ignored); labels_out
 * is a host buffer of n int32.  The library fills stats, status and the two
 * times: queue_seconds (submit -> start, servers only) and run_seconds
 * (start -> labels in labels_out). */
typedef struct gp_request {
    gp_csr graph;
    int32_t k;
    double epsilon;
    uint32_t seed;
    uint32_t flags;
    int32_t* labels_out;
    gp_stats stats;
    gp_status status;
    double queue_seconds;
    double run_seconds;
} gp_request;

/* Partition `count` independent graphs of any sizes on the context's GPU,
 * up to `concurrency` at a time (1..64; each in-flight graph has its own
 * stream and device arena, kept by the context for later batches), largest
 * first.  No counterpart in the reference, which partitions one graph per
 * process (app/partition_main.cu); the batched form of that path.  Every
 * result is identical to gp_partition of the same request alone.  Returns
 * GP_OK when every request succeeded, else the status of the first failed
 * request (per-request status in requests[i].status). */
gp_status gp_partition_batch(gp_context* ctx, gp_request* requests, int32_t count, int32_t concurrency);

/* The batched form over several GPUs of this node (graph-level placement,
 * no collective: each graph runs wholly on one device and its labels are
 * copied to its host buffer).  Graphs are placed by gp_plan_placement over
 * `devices` (device ordinals); on each device up to `concurrency` graphs run
 * at a time, largest first.  Every result is identical to gp_partition of
 * the same request alone.  Status as gp_partition_batch. */
gp_status gp_partition_batch_devices(gp_context* ctx, const int32_t* devices, int32_t device_count,
                                     gp_request* requests, int32_t count, int32_t concurrency);

/* Longest-processing-time placement of `count` work items on `devices`
 * devices: items in decreasing work (ties: lower index first), each to the
 * device with the least work placed so far (ties: lower device).  Writes
 * device_of[count] (0..devices-1) and, if non-NULL, device_work[devices].
 * Deterministic, so every process of a job computes the same plan.  The
 * batched form uses work = 4(n+1) + 8m (+4m with edge weights) bytes, one
 * CSR sweep with its neighbour gathers.  Needs no device. */
gp_status gp_plan_placement(const uint64_t* work, int32_t count, int32_t devices, int32_t* device_of,
                            uint64_t* device_work);

/* A partition server: `workers` threads, each with its own context on
 * `device`, take requests as they arrive.  A request is admitted when its
 * estimated device footprint fits in what is left of hbm_budget_bytes
 * (0: no limit) among the requests running; smaller requests may pass a
 * waiting larger one, and an idle device always admits the next request.
 * The estimate of a request on a resident graph that has run before is that
 * graph's measured footprint (the largest device_peak_bytes of its requests,
 * less the k-wide affinity cache) plus the cache of the request's k and an
 * eighth more; otherwise a static estimate from n, m and k.  Graphs added
 * with gp_server_add_graph stay resident on the device and are partitioned
 * without an upload.  With a budget, a worker whose device arenas hold more
 * than budget/workers after a request releases them.  No counterpart in the
 * reference. */
typedef struct gp_server gp_server;
gp_status gp_server_create(int device, int32_t workers, uint64_t hbm_budget_bytes, gp_server** out);
/* The same server over several GPUs: `workers_per_device` workers on each of
 * `devices`, an HBM budget per device, resident graphs copied to every
 * device; a request runs on the first device with a free worker whose budget
 * admits it (graph-level placement; no collective). */
gp_status gp_server_create_devices(const int32_t* devices, int32_t device_count, int32_t workers_per_device,
                                   uint64_t hbm_budget_bytes, gp_server** out);
/* Uploads a host CSR once (to every device of the server); requests name it
 * by *graph_id. */
gp_status gp_server_add_graph(gp_server* server, const gp_csr* graph, int32_t* graph_id);
/* The admission estimate, in bytes, of a request of part count k on a
 * resident graph. */
gp_status gp_server_footprint(gp_server* server, int32_t graph_id, int32_t k, uint64_t* bytes);
/* Keeps the coarsened hierarchies of resident graphs on the device, up to
 * bytes_per_device on each device of the server (0: none, the default).  A
 * hierarchy depends on the graph, k, the seed and GP_FLAG_NO_SEED_MATCHING,
 * not on epsilon, so a later request with the same four skips coarsening
 * (stats.hierarchy_reused = 1) and yields exactly the labels a fresh call
 * would.  Least recently used hierarchies not in use by a request are
 * dropped beyond the budget, which is separate from hbm_budget_bytes.  Call
 * once, before the first request. */
gp_status gp_server_keep_hierarchies(gp_server* server, uint64_t bytes_per_device);
/* Device bytes the kept hierarchies hold, summed over the devices. */
gp_status gp_server_kept_bytes(gp_server* server, uint64_t* bytes);
/* Queues a request (graph_id -1: request->graph is a host CSR).  The request
 * and its buffers must stay valid until gp_server_wait returns for it. */
gp_status gp_server_submit(gp_server* server, gp_request* request, int32_t graph_id, uint64_t* ticket);
/* Waits up to timeout_seconds (< 0: no limit) for a request; returns
 * GP_DEVICE_TIMEOUT if it is still running, else GP_OK with the request's
 * own status in request->status. */
gp_status gp_server_wait(gp_server* server, uint64_t ticket, double timeout_seconds);
/* Finishes every queued request, then stops the workers. */
void gp_server_destroy(gp_server* server);

/* Kernel timing for measurement: between begin and end, every launch of a
 * kernel whose name contains `kernel_substring` is bracketed by CUDA events
 * on the stream it runs on; end returns the launch count, the summed device
 * time in milliseconds and the summed algorithmic bytes of those launches
 * (compulsory HBM traffic, reported by the kernels that model it; 0 for the
 * others).  Profiling is per host thread. */
gp_status gp_profile_begin(gp_context* ctx, const char* kernel_substring);
gp_status gp_profile_end(gp_context* ctx, uint64_t* launches, double* total_ms,
                         double* algorithmic_bytes);

/* Thread-mapping thresholds (gp_set_option names in brackets).  They decide
 * which kernel and how many threads handle a row, never a value, so a
 * partition does not depend on them.  They replace fixed thresholds of the
 * reference (src/coarsen.cu:288-291, incremental.cuh:8, src/coarsen.cu:1513):
 *   medium_degree     [8, 256]    coarsening rows up to this: a warp and a shared hash
 *   large_narrow      [256, 2048] coarsening rows up to this: the smaller shared table
 *   build_short       [8, 2048]   cache-build rows up to this: 8 lanes per row
 *   rebuild_divisor   [1, 1e5]    cache rebuilt when moved entries exceed (n k w + 8 m) / this
 *   on_demand_degree  [0, 32]     no cache on levels whose maximum degree is at most this
 *   refine_heavy_small / _mid / _large [64, 8192]  refinement rows longer than this go to the
 *                     block-per-2048-entry-chunk kernels, on levels of at most 65,536
 *                     vertices / at most 2^20 / larger (defaults 256 / 512 / 2048) */
typedef struct gp_tuning {
    int32_t medium_degree, large_narrow, build_short, rebuild_divisor, on_demand_degree;
    double default_ms;  /* best partition time with the thresholds the call started from */
    double tuned_ms;    /* best partition time with the thresholds chosen */
    int32_t trials;     /* partitions timed */
    int32_t refine_heavy_small, refine_heavy_mid, refine_heavy_large;
} gp_tuning;

/* Autotuner: partitions `graph` (host memory; uploaded once) `repeats` times
 * per candidate setting, one threshold at a time over a fixed candidate
 * list, keeping a value when it is at least 1% faster (best of the repeats,
 * CUDA-event algorithm time).  Every trial's labels must equal those of the
 * starting thresholds (GP_INTERNAL otherwise).  The chosen thresholds stay
 * set on `ctx` and are reported in `out`. */
gp_status gp_autotune(gp_context* ctx, const gp_csr* graph, int32_t k, double epsilon,
                      uint32_t seed, int32_t repeats, gp_tuning* out);

/* load_weighted_graph + make_device_weighted (src/graph.cpp:47-116,
 * 205-218): the reference's int64 indptr/indices files read straight into
 * device memory owned by the context.  Each file is read in chunks of 8 Mi
 * values into two pinned buffers, so that the read of one chunk overlaps the
 * copy and the device-side narrowing to int32 of the previous one.  The
 * checks and messages are load_weighted_graph's.  The graph (unit weights)
 * stays on the device until the next load or gp_context_destroy; n and m
 * are returned. */
gp_status gp_load_csr_int64(gp_context* ctx, const char* indptr_path,
                            const char* indices_path, int64_t* n, int64_t* m);
/* gp_partition of the graph of the last gp_load_csr_int64 (the upload is
 * already done); labels_out is host memory of n entries. */
gp_status gp_partition_loaded(gp_context* ctx, int32_t k, double epsilon,
                              uint32_t seed, uint32_t flags, int32_t* labels_out,
                              gp_stats* stats);

/* Hierarchy of the last call made with GP_FLAG_KEEP_HIERARCHY.  Level 0 is
 * the input.  gp_level_copy fills any non-NULL array; `map` (length n of the
 * level) maps this level's vertices to the next level and is absent for the
 * last level.  metadata[4] = {maximum_degree bound, has_heavy_rows,
 * incident_weight_bound, 0}. */
gp_status gp_level_count(gp_context* ctx, int32_t* levels);
gp_status gp_level_size(gp_context* ctx, int32_t level, int64_t* n, int64_t* m);
gp_status gp_level_copy(gp_context* ctx, int32_t level, int32_t* offsets,
                        int32_t* neighbors, uint32_t* edge_weights,
                        uint32_t* vertex_weights, int32_t* map,
                        uint64_t* metadata);
/* METIS labels of the coarsest graph from the last call. */
gp_status gp_initial_labels(gp_context* ctx, int32_t* labels, int64_t capacity);

/* ---- host utilities (no device needed) ---- */

/* floor(total*eps/k) in long double, with the reference's feasibility check. */
gp_status gp_partition_capacity(uint64_t total, int32_t k, double epsilon,
                                uint64_t* capacity);

/* Read the reference's on-disk format: int64 indptr[n+1], int64 indices[m].
 * Narrows to int32 with the same range checks.  Call with NULL outputs to
 * get n and m, then again with buffers of that size. */
gp_status gp_read_csr_int64(const char* indptr_path, const char* indices_path,
                            int64_t* n, int64_t* m, int32_t* offsets,
                            int32_t* neighbors);
gp_status gp_write_csr_int64(const char* indptr_path, const char* indices_path,
                             const gp_csr* graph);

/* One level of a hierarchy for gp_write_hierarchy: its CSR (NULL weights
 * are unit weights) and, for every level but the last, `map`: the level's
 * vertices (length graph.n) to the next level's. */
typedef struct gp_level {
    gp_csr graph;
    const int32_t* map;
} gp_level;

/* write_hierarchy (include/hierarchy.hpp:38-123): the Jet-compatible int32
 * file of a hierarchy.  Layout, all int32: the level count, then per level
 * i: n, m, offsets[n+1], neighbors[m], edge weights[m], vertex weights[n]
 * and, for i > 0, the map of level i-1 (n_{i-1} entries, each < n_i).  The
 * file is written to path + ".tmp" and renamed into place; on any error the
 * temporary is removed and the reference's message is set
 * (GP_INVALID_ARGUMENT for a value outside int32 or an invalid map entry,
 * GP_IO_ERROR for the file). */
gp_status gp_write_hierarchy(const gp_level* levels, int32_t count, const char* path);
/* The hierarchy kept by the last GP_FLAG_KEEP_HIERARCHY call of `ctx`,
 * written as gp_write_hierarchy does. */
gp_status gp_write_kept_hierarchy(gp_context* ctx, const char* path);

/* Exact undirected cut of `labels` (directed sum / 2; odd sum is an error). */
gp_status gp_edge_cut(const gp_csr* graph, const int32_t* labels, uint64_t* cut);

/* Independent verifier: cut, part loads (vertex weights), capacity
 * floor(total*eps/k) and whether every load fits.  Writes one JSON line of at
 * most json_capacity bytes.  Returns GP_OK even when capacity is violated;
 * check *capacity_ok. */
gp_status gp_verify(const gp_csr* graph, const int32_t* labels, int32_t k,
                    double epsilon, int32_t check_symmetry, uint64_t* cut,
                    uint64_t* loads /* k entries or NULL */,
                    int32_t* capacity_ok, char* json, size_t json_capacity);

/* ---- seeded synthetic inputs (counter-based, identical on every host) ---- */

/* Generators write into caller buffers; call with NULL arrays first to learn
 * n and m.  Weight arrays may be NULL. */
gp_status gp_generate_grid2d(int32_t width, int32_t height, int64_t* n, int64_t* m,
                             int32_t* offsets, int32_t* neighbors);
/* 3D 7-point mesh, id = x + X*(y + Y*z).  With weighted != 0 vertex weights
 * are uniform in [1,4] and edge weights uniform in [1,16], keyed by the
 * unordered endpoint pair so the CSR stays symmetric. */
gp_status gp_generate_mesh3d(int32_t x, int32_t y, int32_t z, int32_t weighted,
                             uint64_t seed, int64_t* n, int64_t* m,
                             int32_t* offsets, int32_t* neighbors,
                             uint32_t* vertex_weights, uint32_t* edge_weights);
/* R-MAT: edge_factor * 2^scale samples with probabilities (a,b,c,1-a-b-c),
 * symmetrised, self loops and duplicates removed, rows sorted.  The graph is
 * cached per (scale, edge_factor, a, b, c, seed) inside the library so the
 * two-phase call generates once. */
gp_status gp_generate_rmat(int32_t scale, int32_t edge_factor, double a,
                           double b, double c, uint64_t seed, int64_t* n,
                           int64_t* m, int32_t* offsets, int32_t* neighbors);
/* Uniform random weights in [lo,hi] keyed by (seed, vertex) and by
 * (seed, min(u,v), max(u,v)) for edges, so reverse edges agree. */
gp_status gp_generate_weights(const gp_csr* graph, uint64_t seed, uint32_t vw_lo,
                              uint32_t vw_hi, uint32_t ew_lo, uint32_t ew_hi,
                              uint32_t* vertex_weights, uint32_t* edge_weights);

#ifdef __cplusplus
}
#endif
#endif /* GPART_B200_H */
