/*
 * louvain_oracle.h -- CPU restatement of the reference Louvain path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA engine, its
 * C ABI, the CLI) links, loads or calls this library.  It is used by the
 * tests as the checker, by __graft_entry__.smoke() as the checker, and by
 * bench.py as the timed CPU baseline (the reference's CPU path restated).
 *
 * It restates two reference implementations of the same algorithm:
 *   - louvian.py (the reference's CPU prototype), in FP64, with its exact
 *     summation orders, so that per-pass modularity values match it bit for
 *     bit (ORC_PREC_FP64 + ORC_ROWS_FIRST_SEEN);
 *   - the engine's FP32 gain arithmetic (ORC_PREC_FP32 + ORC_ROWS_SORTED),
 *     which follows modularity.cu:149-152 for the gain expression, so that
 *     partitions produced on the GPU can be compared exactly.
 * Parity is pinned against golden vectors generated by running louvian.py
 * itself (tests/golden/make_golden.py).
 */
#ifndef LOUVAIN_ORACLE_H
#define LOUVAIN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Move decision rule.
 * ORC_RULE_CUDA: move iff  max_gain - e_own/m > 0   (modularity.cu:182,278,374)
 * ORC_RULE_PY:   move iff  max_gain > 0              (louvian.py:148-151)   */
enum { ORC_RULE_CUDA = 0, ORC_RULE_PY = 1 };

/* Arithmetic.
 * ORC_PREC_FP64: every quantity in double, louvian.py's summation orders.
 * ORC_PREC_FP32: FP32 gains as modularity.cu:149-152; sums of FP32 inputs
 *                accumulated in FP64 and rounded once to FP32.           */
enum { ORC_PREC_FP64 = 0, ORC_PREC_FP32 = 1 };

/* Row order of a contracted graph.
 * ORC_ROWS_FIRST_SEEN: neighbour communities in order of first occurrence
 *                      (louvian.py:193-202).
 * ORC_ROWS_SORTED:     ascending new community id (canonical form).      */
enum { ORC_ROWS_FIRST_SEEN = 0, ORC_ROWS_SORTED = 1 };

enum {
    ORC_OK = 0,
    ORC_ERR_IO = 2,
    ORC_ERR_PARSE = 3,
    ORC_ERR_NOMEM = 5,
    ORC_ERR_ARG = 1
};

typedef struct {
    uint32_t n_vertices;   /* V at the start of the level            */
    uint64_t n_entries;    /* E (stored adjacency entries)           */
    uint32_t passes;       /* move passes run in the level           */
    uint32_t moved;        /* 1 if the level's first pass gained     */
    double q_start;        /* modularity of the singleton partition  */
    double q_end;          /* modularity after the last pass         */
} orc_level_stat;

/* Matrix Market reader with utils.cu:132-229 semantics.
 * as_float != 0 parses weights as FP32 and takes |w| (utils.cu:294-295);
 * as_float == 0 parses them as FP64 without abs (louvian.py:23-28).
 * Arrays are malloc'd; release with orc_free.                            */
int orc_read_mtx(const char *path, int as_float, uint32_t *n, uint64_t *nnz,
                 uint64_t **off, uint32_t **col, double **w, uint32_t *max_deg,
                 char *err, int errlen);
void orc_free(void *p);

/* Degree bucket of every vertex: 0 for degree 0 (never moves), else the
 * index 1..7 of (0,4],(4,8],(8,16],(16,32],(32,84],(84,319],(319,inf)
 * (modularity.cu:439, louvian.py:76).                                    */
void orc_buckets(uint32_t n, const uint64_t *off, uint8_t *bucket_of);

/* One level's move phase (modularity.cu:438-520, louvian.py:75-99).
 * comm_out receives the community of every vertex after the last pass.
 * q_trace (optional) receives Q after every pass.  Returns 1 when the
 * first pass gained at least `threshold` (the algorithm continues), 0 when
 * it ends; *q_report receives the value the reference prints at the end.
 * A negative return is an error.                                          */
int orc_move_phase(uint32_t n, const uint64_t *off, const uint32_t *col,
                   const double *w, double threshold, int rule, int prec,
                   uint32_t max_passes, uint32_t *comm_out, double *q_trace,
                   uint32_t max_trace, uint32_t *passes, double *q_start,
                   double *q_end);

/* Contraction (aggregation.cu:387-462, louvian.py:204-215).  comm holds one
 * community id < n per vertex.  new_off has room for n+1, new_col/new_w for
 * nnz entries, new_id for n.  Returns the new vertex count in *new_n and
 * the new entry count in *new_nnz.                                        */
int orc_contract(uint32_t n, const uint64_t *off, const uint32_t *col,
                 const double *w, const uint32_t *comm, int row_order,
                 int prec, uint32_t *new_n, uint64_t *new_nnz,
                 uint64_t *new_off, uint32_t *new_col, double *new_w,
                 uint32_t *new_id);

/* Whole run (main.cu:43-48): phases and contractions until a phase's first
 * pass gains less than `threshold`.  assignment[v] is the final community
 * of every input vertex (ids dense, ascending by first community id).
 * *q_final is the modularity the reference reports.                      */
int orc_louvain(uint32_t n, const uint64_t *off, const uint32_t *col,
                const double *w, double threshold, int rule, int prec,
                int row_order, uint32_t max_passes, uint32_t max_levels,
                uint32_t *assignment, double *q_final, orc_level_stat *stats,
                uint32_t max_stats, uint32_t *n_levels);

/* Host threads of the move decisions and the intra-weight sum (default 1:
 * the sequential restatement, every sum in louvian.py's order).  Each
 * bucket is one Jacobi step, so the decisions do not depend on the thread
 * count; with several threads the intra weight is summed per vertex range
 * and the ranges added in order (equal to the sequential sum whenever the
 * sums are exact, as with integer weights).                               */
void orc_set_threads(int t);
int orc_get_threads(void);

/* FP64 modularity of an arbitrary partition (part[v] < n):
 * Q = sum_v sum_{u in N(v), part(u)=part(v)} w / 2m - sum_c a_c^2 / 4m^2.  */
double orc_modularity(uint32_t n, const uint64_t *off, const uint32_t *col,
                      const double *w, const uint32_t *part);

#ifdef __cplusplus
}
#endif
#endif
