/*
 * louvain_b200.h -- C ABI of the B200 Louvain engine.
 *
 * Plain C types only (no CUDA or torch types): pointers, sizes, status
 * codes.  Every entry point returns an lv_status and never exits the
 * process; lv_last_error() gives the message of the calling thread's last
 * failure.
 *
 * Reference interfaces replaced (upicine/louvain-community-detection):
 *   parseGraph            utils.cu:168-229   -> lv_graph_load_mtx
 *   initHostGraph         utils.cu:13-28     -> lv_graph_from_edges / _csr
 *   initDevGraph+copyToDevice+initCommAggr+setInitComm
 *                         utils.cu:66-108    -> lv_engine_load
 *   modularityOptimization modularity.cu:438-520 / modularity.cuh:6
 *                                            -> lv_phase_move
 *   aggregation           aggregation.cu:387-462 / aggregation.cuh:6
 *                                            -> lv_phase_aggregate
 *   main's phase loop     main.cu:43-48      -> lv_run / lv_run_device
 *   computeModularity     modularity.cu:428-436 -> lv_modularity_fp64
 *   printCommunities      utils.cu:270-293   -> lv_get_assignment
 *   deleteDevGraph/deleteAggrData/deleteHostGraph utils.cu:30-64
 *                                            -> lv_engine_destroy,
 *                                               lv_graph_destroy
 *
 * Identifiers are 32-bit unsigned (as the reference's `unsigned int`),
 * weights FP32, CSR offsets 64-bit so graphs with more than 2^32 stored
 * entries fit.
 */
#ifndef LOUVAIN_B200_H
#define LOUVAIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LV_ABI_VERSION 2

typedef enum lv_status {
    LV_OK = 0,
    LV_ERR_ARG = 1,        /* invalid argument                              */
    LV_ERR_IO = 2,         /* file could not be opened (utils.cu:171-174)   */
    LV_ERR_PARSE = 3,      /* malformed Matrix Market input                 */
    LV_ERR_NOMEM = 4,      /* host or device allocation failed              */
    LV_ERR_CUDA = 5,       /* CUDA runtime error                            */
    LV_ERR_STATE = 6,      /* call out of order (e.g. no graph loaded)      */
    LV_ERR_LIMIT = 7,      /* size beyond a documented limit                */
    LV_ERR_TIMEOUT = 8     /* a bounded device wait gave up                 */
} lv_status;

/* Move decision rule (the two reference implementations differ here).
 * LV_RULE_PY:   move iff max_gain > 0                 (louvian.py:148-151)
 * LV_RULE_CUDA: move iff max_gain - e_own/m > 0       (modularity.cu:182,
 *                                                      278, 374)          */
typedef enum lv_rule { LV_RULE_PY = 0, LV_RULE_CUDA = 1 } lv_rule;

/* Arithmetic of the move gains (modularity.cu:149-152 and
 * louvian.py:135-138 evaluate the same expression).
 * LV_GAIN_FP32: FP32, operation by operation, as the reference CUDA program
 *               (the default).
 * LV_GAIN_FP64: FP64, operation by operation, as louvian.py.  With every
 *               weight sum exact in FP32 (integer weights, sums below 2^24)
 *               the runs equal louvian.py's; with large m (above ~1e7) the
 *               two modes can break near-ties differently.                */
typedef enum lv_gain { LV_GAIN_FP32 = 0, LV_GAIN_FP64 = 1 } lv_gain;

typedef struct lv_config {
    int device;             /* CUDA device ordinal                          */
    lv_rule rule;           /* decision rule, default LV_RULE_PY            */
    uint32_t max_passes;    /* cap on passes per level (0 = 100000)         */
    uint32_t max_levels;    /* cap on levels (0 = no cap)                   */
    int use_graphs;         /* capture each level's pass in a CUDA graph
                               and replay it (default 1)                    */
    void *stream;           /* cudaStream_t to run on; NULL = own stream    */
    lv_gain gain;           /* gain arithmetic, default LV_GAIN_FP32        */
    int level_kernel;       /* 1: run a single graph's pass loop as one
                               persistent cooperative kernel per level; 0
                               (default): per-kernel launches, in a level
                               graph or from the host as use_graphs says    */
    int contract_sort;      /* 1: contract a single graph by sorting the
                               entries by (new row, new column) and summing
                               runs (rows then ordered by column); 0
                               (default): hash merge per community        */
    int apply_launch;       /* 1: apply each bucket's moves in a launch of
                               its own after the bucket's proposals; 0
                               (default): every bucket step applies its own
                               moves into a second copy of the community
                               state (same results, one launch less per
                               bucket)                                      */
    int modularity_full;    /* 1: every pass's modularity from a sweep over
                               all entries; 0 (default): on levels of at
                               least 2^23 entries, after a pass that moved
                               under a quarter of the entries, the next
                               pass's sweep visits only the rows of the
                               vertices it moved.  That update assumes every
                               edge is stored in both of its rows with the
                               same weight, as the reference's reader and
                               every graph built here store it; set 1 for a
                               caller's CSR that is not symmetric          */
} lv_config;

/* Per-level record (the reference prints none of this; -v here adds it). */
typedef struct lv_level_info {
    uint32_t n_vertices;    /* V of the level                               */
    uint64_t n_entries;     /* E of the level (stored adjacency entries)    */
    uint32_t passes;        /* move passes run                              */
    uint32_t moved;         /* 1 if the level's first pass gained >= g      */
    double q_start;         /* Q of the singleton partition                 */
    double q_end;           /* Q after the last pass                        */
    float move_ms;          /* device time of the move phase (incl. set-up) */
    float aggregate_ms;     /* device time of the contraction (0 if none)   */
    float prepare_ms;       /* part of move_ms: degree classes, row sums,
                               initial modularity                           */
} lv_level_info;

typedef struct lv_result {
    double modularity;      /* Q the reference prints (modularity.cu:504)   */
    uint32_t n_vertices;    /* input vertex count                           */
    uint32_t n_communities; /* communities in the final assignment          */
    uint32_t n_levels;      /* phases run                                   */
    uint64_t edges_processed; /* sum over passes of that pass's E           */
    float alg_ms;           /* device time of the phase loop (main.cu:56)   */
    float copy_ms;          /* device time of upload + set-up (main.cu:19-35)*/
} lv_result;

typedef struct lv_graph lv_graph;   /* host CSR, owned by the library      */
typedef struct lv_engine lv_engine; /* device state, owned by the library  */

/* ---- status ---------------------------------------------------------- */
const char *lv_status_string(lv_status s);
const char *lv_last_error(void);
int lv_abi_version(void);
void lv_config_default(lv_config *cfg);

/* ---- host graphs ------------------------------------------------------ */
/* Matrix Market reader with the reference's semantics (utils.cu:132-229):
 * '%' lines before the size header are skipped; the header is
 * `rows cols nnz` and V = cols; indices are 1-based unless any entry line
 * holds a 0; |weight| is used, 1.0 when a line has none (a missing weight
 * repeats the previous line's); every off-diagonal entry is stored in both
 * rows, a diagonal entry once, rows in file order.  Unlike the reference,
 * malformed lines, truncated files and out-of-range indices are errors
 * (LV_ERR_PARSE) instead of undefined behaviour.                          */
lv_status lv_graph_load_mtx(const char *path, lv_graph **out);

/* Same CSR construction from an edge list (the lines of an MTX file). */
lv_status lv_graph_from_edges(uint32_t n_vertices, uint64_t n_edges,
                              const uint32_t *src, const uint32_t *dst,
                              const float *weights, lv_graph **out);

/* Adopts a ready CSR (copied): offsets[n+1], cols[E], weights[E]. */
lv_status lv_graph_from_csr(uint32_t n_vertices, const uint64_t *offsets,
                            const uint32_t *cols, const float *weights,
                            lv_graph **out);

/* Read-only views of a host graph (valid until lv_graph_destroy). */
lv_status lv_graph_view(const lv_graph *g, uint32_t *n_vertices,
                        uint64_t *n_entries, const uint64_t **offsets,
                        const uint32_t **cols, const float **weights,
                        uint32_t *max_degree);
void lv_graph_destroy(lv_graph *g);

/* Binary CSR files (no counterpart in the reference): this library's own
 * format ("LVBCSR01", n, max degree, nnz, offsets, cols, weights;
 * little-endian), so a parsed graph reloads without the text parse
 * (the CLI's --cache keeps one beside the .mtx).  Loading checks that the
 * file is a consistent CSR.                                               */
lv_status lv_graph_save(const lv_graph *g, const char *path);
lv_status lv_graph_load(const char *path, lv_graph **out);

/* ---- engine ----------------------------------------------------------- */
lv_status lv_engine_create(const lv_config *cfg, lv_engine **out);
void lv_engine_destroy(lv_engine *e);

/* Uploads a host graph and resets the state (every vertex its own
 * community, assignment = identity): initDevGraph + copyToDevice +
 * initCommAggr + setInitComm (utils.cu:66-108).                          */
lv_status lv_engine_load(lv_engine *e, const lv_graph *g);

/* Same from a CSR already in device memory (caller keeps ownership and
 * must keep it alive and unchanged until the next load or destroy).      */
lv_status lv_engine_load_device(lv_engine *e, uint32_t n_vertices,
                                uint64_t n_entries, const uint64_t *d_offsets,
                                const uint32_t *d_cols, const float *d_weights);

/* The reference's CSR construction (parseGraph, utils.cu:168-229) built on
 * the device from edge lines: every row keeps file order, an off-diagonal
 * line (i, j, w) is stored in rows i and j, i == j once, weights |w| (1
 * without a weight array).  The rows come from a stable device sort of the
 * directed entries by row.  Indices 0-based, < n_vertices (else
 * LV_ERR_PARSE); at most 2^31 - 1 lines.
 * lv_engine_load_edges: host edge lines -> device -> CSR -> engine (as
 * lv_engine_load).  lv_engine_load_mtx: the Matrix Market reader of
 * lv_graph_load_mtx (parallel host parse), then the device build.
 * lv_csr_from_edges_device: device in, device out on `stream`; d_cols and
 * d_weights_out need room for 2 * n_edges entries, d_offsets for
 * n_vertices + 1; *n_entries receives the entry count; scratch is
 * allocated and freed on the stream.                                      */
lv_status lv_engine_load_edges(lv_engine *e, uint32_t n_vertices, uint64_t n_edges,
                               const uint32_t *src, const uint32_t *dst,
                               const float *weights);
lv_status lv_engine_load_mtx(lv_engine *e, const char *path);
lv_status lv_csr_from_edges_device(uint32_t n_vertices, uint64_t n_edges,
                                   const uint32_t *d_src, const uint32_t *d_dst,
                                   const float *d_weights, uint64_t *d_offsets,
                                   uint32_t *d_cols, float *d_weights_out,
                                   uint64_t *n_entries, void *stream);

/* One phase of local moving on the current level (modularityOptimization,
 * modularity.cu:438-520).  *more = 1 when the first pass gained at least
 * min_gain (the caller should aggregate and call again), 0 when the run
 * is over; *q = the modularity the reference would print on return 0
 * (Q before the failing pass), or Q after the last pass on return 1.
 * Like the reference, on *more = 0 the failing pass's moves are dropped
 * from the assignment.                                                   */
lv_status lv_phase_move(lv_engine *e, float min_gain, int *more, double *q);

/* Contracts the current level's communities into the next level's graph
 * (aggregation, aggregation.cu:387-462).                                 */
lv_status lv_phase_aggregate(lv_engine *e);

/* Whole run (main.cu:43-48) on a host graph: upload, phases, contraction,
 * final assignment left on the device (lv_get_assignment reads it).      */
lv_status lv_run(lv_engine *e, const lv_graph *g, float min_gain,
                 lv_result *res);

/* Whole run with inputs and output in device memory: d_assignment
 * receives n_vertices community ids; nothing crosses PCIe except a few
 * scalars per level.                                                      */
lv_status lv_run_device(lv_engine *e, uint32_t n_vertices, uint64_t n_entries,
                        const uint64_t *d_offsets, const uint32_t *d_cols,
                        const float *d_weights, float min_gain,
                        uint32_t *d_assignment, lv_result *res);

/* Final (or current) community of every input vertex -> host buffer.  */
lv_status lv_get_assignment(lv_engine *e, uint32_t *out, size_t n);

/* The community listing of printCommunities (utils.cu:270-293) grouped on
 * the device and copied to the host once: out[0..C] the offsets of every
 * community's members, out[C+1 .. C+1+n) the input vertices community by
 * community, ascending within each (a stable device sort by community).
 * *n_communities receives C; with out NULL only C is returned (the buffer
 * needs C + 1 + n entries).                                                */
lv_status lv_get_communities(lv_engine *e, uint32_t *out, size_t cap,
                             uint32_t *n_communities);

/* Per-level records of the last run; *count receives how many exist.    */
lv_status lv_get_levels(lv_engine *e, lv_level_info *out, uint32_t cap,
                        uint32_t *count);

/* Current level's sizes.                                                */
lv_status lv_get_level_size(lv_engine *e, uint32_t *n_vertices,
                            uint64_t *n_entries);

/* Current level state -> host buffers (each NULL or n_vertices long):
 * community of every vertex, community sizes, weighted degrees.  For
 * parity tests and debugging.                                            */
lv_status lv_get_level_state(lv_engine *e, uint32_t *comm, uint32_t *comm_size,
                             float *weighted_degree);

/* Current level CSR -> host buffers (offsets n+1, cols/weights E).       */
lv_status lv_get_level_csr(lv_engine *e, uint64_t *offsets, uint32_t *cols,
                           float *weights);

/* Overwrites the current level's communities (n_vertices ids < n) and
 * recomputes sizes and totals, so contraction can be checked on a given
 * partition.                                                             */
lv_status lv_set_level_comm(lv_engine *e, const uint32_t *comm);

/* FP64 modularity of an arbitrary partition of the CURRENT level graph,
 * computed on the device:  sum intra w / 2m - sum a_c^2 / 4m^2.          */
lv_status lv_modularity_fp64(lv_engine *e, const uint32_t *partition,
                             double *q);

/* Degree bucket (0 = degree 0, else 1..7 for (0,4] ... (319,inf)) of every
 * vertex of the current level, as the move phase groups them
 * (modularity.cu:5-18,439).                                              */
lv_status lv_get_buckets(lv_engine *e, uint8_t *bucket_of, size_t n);

/* ---- batched form (no counterpart in the reference, which runs one graph
 * per process: main.cu:5-70) --------------------------------------------
 * Runs the reference's whole phase loop on many graphs at once: they are
 * packed as one block-diagonal union (vertex ids offset per graph) and every
 * kernel serves all of them; each graph keeps its own m, modularity, stop
 * rule and levels, so its result equals a run of that graph alone
 * (lv_run).  A graph whose phase ends is finalised and leaves the union.
 *
 * lv_batch_run_device: the union CSR is in device memory; graph g owns the
 * vertices [graph_offsets[g], graph_offsets[g+1]) (host array, n_graphs+1
 * entries) and its rows may only name its own vertices.  d_assignment
 * (n_vertices) receives every vertex's community id local to its graph;
 * modularity (host, n_graphs) each graph's final Q; levels (host,
 * n_graphs, may be NULL) its number of phases.                            */
lv_status lv_batch_run_device(lv_engine *e, uint32_t n_graphs,
                              const uint64_t *graph_offsets, uint32_t n_vertices,
                              uint64_t n_entries, const uint64_t *d_offsets,
                              const uint32_t *d_cols, const float *d_weights,
                              float min_gain, uint32_t *d_assignment,
                              double *modularity, uint32_t *levels,
                              lv_result *res);

/* Same from host graphs (packed and uploaded by the call); assignment
 * (host) receives the local ids of graph 0's vertices, then graph 1's...  */
lv_status lv_batch_run(lv_engine *e, uint32_t n_graphs,
                       const lv_graph *const *graphs, float min_gain,
                       uint32_t *assignment, double *modularity,
                       uint32_t *levels, lv_result *res);

/* ---- served form (no counterpart in the reference) ----------------------
 * Continuous batching of graph requests on one device.  lv_serve_submit
 * queues a graph by reference and returns at once (thread-safe beside the
 * other calls); the graph must stay alive and unchanged until
 * lv_serve_poll has returned its result.  A request goes to the first lane
 * whose size bound holds its entries; a lane is one union of resident
 * graphs with its own engine, stream and share of the device budget.  A
 * lane's step admits its queued graphs that fit (first come first served,
 * while slots and budget last), appends them to its union at the level
 * boundary and runs one level for every resident graph (the batched form's
 * level); graphs whose run ends are finalised, copied out and leave,
 * freeing their slot and memory for the next admissions.  Separate lanes
 * keep small graphs from waiting on the levels of large ones, and with
 * `background` set every lane is stepped by its own worker thread, so the
 * lanes run concurrently on the device.  Every graph keeps its own m,
 * modularity, stop rule and levels, so its result equals lv_run on it
 * alone.  Times are milliseconds on the server's clock (from creation).
 * After an error other than LV_ERR_ARG / LV_ERR_LIMIT the server should be
 * destroyed.                                                               */
typedef struct lv_server lv_server;

typedef struct {
  float min_gain;
  uint64_t budget_bytes;         /* device memory for all lanes */
  uint32_t max_graphs;           /* resident graphs per lane (0: 4096) */
  uint32_t n_lanes;              /* 1..4 */
  uint64_t lane_max_entries[4];  /* lane i takes requests with at most this
                                    many entries (ascending; the last lane
                                    takes the rest) */
  float lane_share[4];           /* share of the budget per lane */
  int background;                /* step the lanes on worker threads */
  uint32_t lane_solo;            /* bit i set: lane i runs its requests one
                                    at a time through the single-graph path
                                    (lv_run on the lane's engine and stream)
                                    instead of a union, so a large graph is
                                    never paced by others' levels, and solo
                                    lanes overlap on the device            */
} lv_serve_config;

/* 4 background lanes: unions of graphs with <= 2^18 entries (10% of the
 * budget) and <= 2^22 (30%), and two solo lanes for larger graphs (30%
 * each); budget 8 GiB; min_gain 1e-6.  Lanes with the same bound form a
 * group: a request goes to the group's lane with the fewest entries
 * resident or queued.  A union lane holds a fifth of its budget for
 * per-vertex state at 192 B a vertex and the rest for adjacency at 40 B an
 * entry; a solo lane admits a graph whose sizes fit those capacities and
 * allocates for it when it runs.                                           */
void lv_serve_config_default(lv_serve_config *c);

typedef struct {
  uint64_t ticket;
  double modularity;
  uint32_t n_vertices;
  uint32_t n_communities;
  uint32_t levels;
  uint32_t lane;
  double submit_ms; /* lv_serve_submit */
  double admit_ms;  /* joined a union */
  double done_ms;   /* result copied out */
} lv_serve_result;

typedef struct {
  uint32_t queued, resident, finished, slot_cap, n_lanes;
  uint64_t resident_vertices, resident_entries; /* input sizes, resident graphs */
  uint64_t cap_vertices, cap_entries, budget_bytes;
  uint64_t steps, admitted, completed;
} lv_serve_stats;

lv_status lv_serve_create(const lv_config *cfg, const lv_serve_config *scfg,
                          lv_server **out);
lv_status lv_serve_submit(lv_server *s, const lv_graph *g, uint64_t *ticket);
/* Without background workers: one step of every lane.  With them: nothing
 * to do.  resident / queued (may be NULL): graphs resident and waiting.    */
lv_status lv_serve_step(lv_server *s, uint32_t *resident, uint32_t *queued);
/* Blocks (background mode) until a result is ready, nothing is queued or
 * resident, or timeout_ms passes; *idle (may be NULL) = 1 when nothing is
 * queued, resident or waiting to be polled.                                */
lv_status lv_serve_wait(lv_server *s, uint32_t timeout_ms, int *idle);
/* Pops the oldest finished request: *got = 1 and its result (assignment:
 * n_vertices local community ids, may be NULL; cap its capacity), or
 * *got = 0 when none is finished.                                          */
lv_status lv_serve_poll(lv_server *s, lv_serve_result *res,
                        uint32_t *assignment, size_t cap, int *got);
lv_status lv_serve_get_stats(lv_server *s, lv_serve_stats *out);
/* A lane's engine, for lv_set_profiling / lv_get_kernel_stats only (owned
 * by the server: never load, run or destroy it).                           */
lv_status lv_serve_engine(lv_server *s, uint32_t lane, lv_engine **out);
void lv_serve_destroy(lv_server *s);

/* ---- autotuning (no counterpart in the reference) -----------------------
 * Every degree bucket (1..7) can run on any move kernel variant whose
 * shape holds its degrees; all variants give the same proposals, so the
 * choice changes speed only.  Variants: G-lane groups with one entry per
 * lane (LV_KERNEL_LANES4/8/16/32: degree <= G), a warp per vertex with a
 * 128- or 512-slot shared table (LV_KERNEL_WARP128: <= 84, WARP512: <= 319)
 * and a block per vertex with a 4096-slot table (LV_KERNEL_BLOCK: <= 2048).
 * lv_autotune times every fitting variant of every non-empty bucket on the
 * loaded graph's current level (proposals only; the state is unchanged)
 * and keeps the fastest; the engine uses its tuning until changed.        */
enum {
  LV_KERNEL_LANES4 = 0,
  LV_KERNEL_LANES8 = 1,
  LV_KERNEL_LANES16 = 2,
  LV_KERNEL_LANES32 = 3,
  LV_KERNEL_WARP128 = 4,
  LV_KERNEL_WARP512 = 5,
  LV_KERNEL_BLOCK = 6
};
typedef struct lv_tuning {
  uint8_t bucket_kernel[8]; /* [b] for buckets b = 1..7; [0] unused       */
  float bucket_ms[8];       /* lv_autotune: time per launch of the choice */
} lv_tuning;

/* reps: timed launches per variant (0: 5). */
lv_status lv_autotune(lv_engine *e, uint32_t reps, lv_tuning *out);
lv_status lv_set_tuning(lv_engine *e, const lv_tuning *t);
lv_status lv_get_tuning(lv_engine *e, lv_tuning *t);

/* ---- kernel timing (no counterpart in the reference, whose only timers
 * are main.cu:19-56's two regions) --------------------------------------
 * With profiling on, every launch group is bracketed by CUDA events on the
 * engine's stream and its device time accumulated with its algorithmic
 * HBM bytes (reads + writes the algorithm needs, counted from the level's
 * V, E and bucket sizes).                                                */
typedef struct lv_kernel_stat {
    char name[32];          /* move_b1..move_b7, apply, modularity,
                               level_init, contract                        */
    uint64_t launches;      /* launch groups timed                          */
    double total_ms;        /* summed device time                           */
    double bytes;           /* summed algorithmic bytes                     */
} lv_kernel_stat;

lv_status lv_set_profiling(lv_engine *e, int on);
lv_status lv_get_kernel_stats(lv_engine *e, lv_kernel_stat *out, uint32_t cap,
                              uint32_t *count);
lv_status lv_reset_kernel_stats(lv_engine *e);

/* Kernels this library has launched in the process so far (all engines). */
lv_status lv_get_launch_count(uint64_t *count);

/* Times the library has made the host wait for a stream (all engines): a
 * single graph's level costs the class counts of its set-up, the level
 * graph's result and the contraction's class sizes (plus one for hubs and
 * one for the largest communities' tables when a level has them).        */
lv_status lv_get_sync_count(uint64_t *count);

/* ---- fault injection, for tests (no counterpart in the reference, which
 * exits on any CUDA error, utils.cuh:95-100) -------------------------------
 * From this call on, the nth device allocation the library makes (n >= 1)
 * fails as if the device were out of memory: the entry point that needed
 * it returns LV_ERR_NOMEM and the engine stays usable (the next run
 * allocates again).  n = 0 switches the injection off.  Process-wide.      */
lv_status lv_debug_fail_device_alloc(uint64_t n);

/* ---- modularity without allocation (no counterpart in the reference) ----
 * The FP64 modularity of lv_modularity_fp64 for a graph and partition that
 * the caller keeps in device memory, for callers that must not allocate on
 * the call path: latency-bound serving loops that cannot stall in the
 * allocator (or on the device-wide synchronisation of a cudaFree), and
 * processes whose device memory belongs to another allocator (a caching
 * allocator, a budget carved out at start-up).  It allocates nothing: its
 * scratch is a fixed array in the library's device memory (8 MiB per device
 * that loads the library, held until the process exits).
 *   n_vertices <= 1048576 (else LV_ERR_LIMIT); d_cols and d_weights must
 *   not be NULL when n_vertices > 0 (else LV_ERR_ARG); partition ids must be
 *   < n_vertices (else LV_ERR_ARG, and *d_q is set to NaN); otherwise *d_q
 *   receives Q, and *q_host too when q_host is not NULL.  Runs on `stream`
 *   (a cudaStream_t, NULL = legacy default stream) and returns after the
 *   stream has finished the work.
 * Every call shares the one array (cleared at the start of each call), so
 * calls that overlap on the GPU race.  The first call on a device looks up
 * the array's address with that device current: make it before any stream
 * capture begins.                                                         */
lv_status lv_modularity_noalloc(uint32_t n_vertices, const uint64_t *d_offsets,
                                const uint32_t *d_cols, const float *d_weights,
                                const uint32_t *d_partition, double *d_q,
                                double *q_host, void *stream);

#ifdef __cplusplus
}
#endif
#endif
