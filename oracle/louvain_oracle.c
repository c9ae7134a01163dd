/*
 * louvain_oracle.c -- CPU restatement of the reference Louvain path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg use it; the product never does.
 *
 * Reference anchors (file:line within upicine/louvain-community-detection):
 *   MTX reader ............ utils.cu:132-229 (parseGraphSize,
 *                           isZeroStartingIndex, parseGraph)
 *   weighted degree / m ... modularity.cu:27-49,457-458; louvian.py:49-56
 *   buckets ............... modularity.cu:5-18,439; louvian.py:76,84-86
 *   isLowerIdx ............ modularity.cu:85-93; louvian.py:115-118
 *   gain / argmax ......... modularity.cu:143-187,333-379;
 *                           louvian.py:120-151
 *   apply + comm totals ... modularity.cu:382-398,495-498;
 *                           louvian.py:64-73
 *   modularity ............ modularity.cu:400-436; louvian.py:101-113
 *   pass / stop rule ...... modularity.cu:466-519; louvian.py:83-99
 *   contraction ........... aggregation.cu:21-45,387-462;
 *                           louvian.py:163-215
 *   level loop ............ main.cu:43-48; louvian.py:228-232
 *
 * Summation orders in ORC_PREC_FP64 follow louvian.py exactly, including
 * CPython 3.12's compensated (Neumaier) builtin sum() at louvian.py:53 and
 * louvian.py:111, so per-pass Q values equal louvian.py's bit for bit.
 */
#include "louvain_oracle.h"

#include <errno.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NBUCKETS 7
static const uint64_t kBucketHi[NBUCKETS + 1] = {0, 4, 8, 16, 32, 84, 319,
                                                 UINT64_MAX};

void orc_free(void *p) { free(p); }

/* Host threads for the move decisions and the intra-weight sum (1: the
 * plain sequential restatement). */
static int g_threads = 1;
void orc_set_threads(int t) { g_threads = t < 1 ? 1 : (t > 256 ? 256 : t); }
int orc_get_threads(void) { return g_threads; }

static void set_err(char *err, int errlen, const char *msg, long line) {
    if (!err || errlen <= 0) return;
    if (line >= 0)
        snprintf(err, (size_t)errlen, "%s (line %ld)", msg, line);
    else
        snprintf(err, (size_t)errlen, "%s", msg);
}

/* ------------------------------------------------------------------ */
/* Matrix Market reader (utils.cu:132-229).                            */
/* ------------------------------------------------------------------ */

/* Splits one line into at most 4 whitespace separated tokens. */
static int split_tokens(char *s, char **tok, int maxtok) {
    int nt = 0;
    while (*s) {
        while (*s == ' ' || *s == '\t' || *s == '\r') s++;
        if (!*s) break;
        if (nt < maxtok) tok[nt] = s;
        nt++;
        while (*s && *s != ' ' && *s != '\t' && *s != '\r') s++;
        if (*s) *s++ = '\0';
    }
    return nt;
}

static int parse_u64(const char *t, uint64_t *out) {
    if (!t || !*t || *t == '-') return 0;
    char *end = NULL;
    errno = 0;
    unsigned long long v = strtoull(t, &end, 10);
    if (errno || end == t || *end) return 0;
    *out = (uint64_t)v;
    return 1;
}

int orc_read_mtx(const char *path, int as_float, uint32_t *n_out,
                 uint64_t *nnz_out, uint64_t **off_out, uint32_t **col_out,
                 double **w_out, uint32_t *max_deg_out, char *err,
                 int errlen) {
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_err(err, errlen, "Error opening file", -1);
        return ORC_ERR_IO;
    }
    fseek(f, 0, SEEK_END);
    long fsz = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *buf = (char *)malloc((size_t)fsz + 1);
    if (!buf) {
        fclose(f);
        return ORC_ERR_NOMEM;
    }
    size_t got = fread(buf, 1, (size_t)fsz, f);
    fclose(f);
    buf[got] = '\0';

    char *p = buf;
    long lineno = 0;
    char *line = NULL;
    /* Header: skip lines beginning with '%' (utils.cu:137-139). */
    for (;;) {
        if (!*p) {
            free(buf);
            set_err(err, errlen, "missing size header", lineno);
            return ORC_ERR_PARSE;
        }
        line = p;
        char *nl = strchr(p, '\n');
        if (nl) {
            *nl = '\0';
            p = nl + 1;
        } else {
            p += strlen(p);
        }
        lineno++;
        if (line[0] != '%') break;
    }
    char *tok[4];
    int nt = split_tokens(line, tok, 4);
    uint64_t rows, cols, nnz;
    if (nt < 3 || !parse_u64(tok[0], &rows) || !parse_u64(tok[1], &cols) ||
        !parse_u64(tok[2], &nnz) || cols > 0xFFFFFFFEull ||
        nnz > 0xFFFFFFFFull) {
        free(buf);
        set_err(err, errlen, "bad size header", lineno);
        return ORC_ERR_PARSE;
    }
    (void)rows; /* utils.cu:142 overwrites rows with cols */
    uint32_t n = (uint32_t)cols;

    uint32_t *v1s = (uint32_t *)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    uint32_t *v2s = (uint32_t *)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    double *ws = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
    if (!v1s || !v2s || !ws) {
        free(buf); free(v1s); free(v2s); free(ws);
        return ORC_ERR_NOMEM;
    }
    /* Weight carries over from the previous line when a line has none
     * (the stream extraction at utils.cu:294 leaves `weight` untouched);
     * it starts at 1.0 (utils.cu:289).  louvian.py:27 uses 1.0 unless the
     * line has exactly three fields. */
    double wprev = 1.0;
    int zero_based = 0;
    for (uint64_t i = 0; i < nnz; i++) {
        if (!*p) {
            free(buf); free(v1s); free(v2s); free(ws);
            set_err(err, errlen, "fewer entry lines than the header's nnz",
                    lineno + 1);
            return ORC_ERR_PARSE;
        }
        line = p;
        char *nl = strchr(p, '\n');
        if (nl) {
            *nl = '\0';
            p = nl + 1;
        } else {
            p += strlen(p);
        }
        lineno++;
        nt = split_tokens(line, tok, 4);
        uint64_t a, b;
        if (nt < 2 || !parse_u64(tok[0], &a) || !parse_u64(tok[1], &b)) {
            free(buf); free(v1s); free(v2s); free(ws);
            set_err(err, errlen, "bad entry line", lineno);
            return ORC_ERR_PARSE;
        }
        if (a > 0xFFFFFFFFull || b > 0xFFFFFFFFull) {
            free(buf); free(v1s); free(v2s); free(ws);
            set_err(err, errlen, "vertex index out of range", lineno);
            return ORC_ERR_PARSE;
        }
        double wt;
        if (as_float) {
            if (nt >= 3) {
                char *end = NULL;
                float fw = strtof(tok[2], &end);
                if (end == tok[2]) {
                    free(buf); free(v1s); free(v2s); free(ws);
                    set_err(err, errlen, "bad weight", lineno);
                    return ORC_ERR_PARSE;
                }
                wprev = (double)fabsf(fw); /* utils.cu:295 */
            }
            wt = wprev;
        } else {
            if (nt == 3) {
                char *end = NULL;
                wt = strtod(tok[2], &end);
                if (end == tok[2]) {
                    free(buf); free(v1s); free(v2s); free(ws);
                    set_err(err, errlen, "bad weight", lineno);
                    return ORC_ERR_PARSE;
                }
            } else {
                wt = 1.0;
            }
        }
        if (a == 0 || b == 0) zero_based = 1; /* utils.cu:143-166 */
        v1s[i] = (uint32_t)a;
        v2s[i] = (uint32_t)b;
        ws[i] = wt;
    }
    free(buf);

    uint64_t *deg = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    if (!deg) {
        free(v1s); free(v2s); free(ws);
        return ORC_ERR_NOMEM;
    }
    for (uint64_t i = 0; i < nnz; i++) {
        uint32_t a = v1s[i], b = v2s[i];
        if (!zero_based) { a--; b--; } /* utils.cu:297-300 */
        if (a >= n || b >= n) {
            free(v1s); free(v2s); free(ws); free(deg);
            set_err(err, errlen, "vertex index exceeds the header's size",
                    -1);
            return ORC_ERR_PARSE;
        }
        v1s[i] = a;
        v2s[i] = b;
        if (a != b) {
            deg[a + 1]++;
            deg[b + 1]++;
        } else {
            deg[a + 1]++;
        }
    }
    uint64_t *off = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)n + 1));
    if (!off) {
        free(v1s); free(v2s); free(ws); free(deg);
        return ORC_ERR_NOMEM;
    }
    off[0] = 0;
    uint32_t max_deg = 0;
    for (uint32_t i = 1; i <= n; i++) { /* utils.cu:214-218 */
        off[i] = off[i - 1] + deg[i];
        if (deg[i] > max_deg) max_deg = (uint32_t)deg[i];
    }
    uint64_t E = off[n];
    uint32_t *col = (uint32_t *)malloc(sizeof(uint32_t) * (E ? E : 1));
    double *w = (double *)malloc(sizeof(double) * (E ? E : 1));
    if (!col || !w) {
        free(v1s); free(v2s); free(ws); free(deg); free(off); free(col);
        free(w);
        return ORC_ERR_NOMEM;
    }
    /* Row cursors: entries land in each row in file order (utils.cu:200-227). */
    for (uint32_t i = 0; i < n; i++) deg[i] = off[i];
    for (uint64_t i = 0; i < nnz; i++) {
        uint32_t a = v1s[i], b = v2s[i];
        if (a != b) {
            col[deg[a]] = b; w[deg[a]++] = ws[i];
            col[deg[b]] = a; w[deg[b]++] = ws[i];
        } else {
            col[deg[a]] = a; w[deg[a]++] = ws[i];
        }
    }
    free(v1s); free(v2s); free(ws); free(deg);
    *n_out = n;
    *nnz_out = E;
    *off_out = off;
    *col_out = col;
    *w_out = w;
    if (max_deg_out) *max_deg_out = max_deg;
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* Buckets                                                             */
/* ------------------------------------------------------------------ */

static int bucket_of_degree(uint64_t d) {
    if (d == 0) return 0;
    for (int b = 1; b <= NBUCKETS; b++)
        if (d <= kBucketHi[b]) return b;
    return NBUCKETS;
}

void orc_buckets(uint32_t n, const uint64_t *off, uint8_t *bucket_of) {
    for (uint32_t v = 0; v < n; v++)
        bucket_of[v] = (uint8_t)bucket_of_degree(off[v + 1] - off[v]);
}

/* ------------------------------------------------------------------ */
/* Summation helpers                                                   */
/* ------------------------------------------------------------------ */

/* CPython 3.12 builtin sum() over floats: Neumaier compensation, the
 * compensation added once at the end when it is non-zero and finite. */
typedef struct { double f, c; } neu_sum;
static inline void neu_add(neu_sum *s, double x) {
    double t = s->f + x;
    if (fabs(s->f) >= fabs(x))
        s->c += (s->f - t) + x;
    else
        s->c += (x - t) + s->f;
    s->f = t;
}
static inline double neu_result(const neu_sum *s) {
    double r = s->f;
    if (s->c != 0.0 && isfinite(s->c)) r += s->c;
    return r;
}

/* ------------------------------------------------------------------ */
/* Move phase                                                          */
/* ------------------------------------------------------------------ */

typedef struct {
    uint32_t n;
    const uint64_t *off;
    const uint32_t *col;
    const double *w;
    int prec;
    double *k;        /* weighted degree (FP32 values in FP32 mode)     */
    double m;         /* sum k / 2 (FP64)                                */
    float m32;        /* FP32 copy used by FP32 gains                    */
    uint32_t *comm;
    uint32_t *comm_sz;
    double *a;        /* community totals                                */
    uint32_t *new_comm;
    double *acc;      /* per-community scratch, all zero between uses    */
    uint32_t *touched;
} mstate;

static double intra_range(const mstate *s, uint32_t v0, uint32_t v1) {
    double intra = 0.0;
    for (uint32_t v = v0; v < v1; v++) {
        uint32_t cv = s->comm[v];
        for (uint64_t j = s->off[v]; j < s->off[v + 1]; j++)
            if (s->comm[s->col[j]] == cv) intra += s->w[j];
    }
    return intra;
}

typedef struct {
    const mstate *s;
    uint32_t v0, v1;
    double out;
} intra_job;

static void *intra_worker(void *arg) {
    intra_job *j = (intra_job *)arg;
    j->out = intra_range(j->s, j->v0, j->v1);
    return NULL;
}

/* Intra-community weight: in vertex order on one thread (louvian.py's
 * order); with several threads, per-range partial sums added in range
 * order (equal whenever the sums are exact, e.g. integer weights). */
static double intra_weight(const mstate *s) {
    const int T = g_threads;
    if (T <= 1 || s->n < 65536) return intra_range(s, 0, s->n);
    pthread_t th[256];
    intra_job jobs[256];
    for (int t = 0; t < T; t++) {
        jobs[t].s = s;
        jobs[t].v0 = (uint32_t)((uint64_t)s->n * t / T);
        jobs[t].v1 = (uint32_t)((uint64_t)s->n * (t + 1) / T);
        if (pthread_create(&th[t], NULL, intra_worker, &jobs[t]) != 0) {
            jobs[t].out = intra_range(s, jobs[t].v0, jobs[t].v1);
            th[t] = 0;
        }
    }
    double intra = 0.0;
    for (int t = 0; t < T; t++) {
        if (th[t]) pthread_join(th[t], NULL);
        intra += jobs[t].out;
    }
    return intra;
}

static double state_modularity(const mstate *s) {
    /* louvian.py:101-113 (FP64 mode): sum of squares with builtin sum()
     * over communities in ascending order, intra weight in plain order. */
    double intra = intra_weight(s);
    double asq;
    if (s->prec == ORC_PREC_FP64) {
        neu_sum ns = {0.0, 0.0};
        for (uint32_t c = 0; c < s->n; c++) neu_add(&ns, s->a[c] * s->a[c]);
        asq = neu_result(&ns);
        return (intra / (2 * s->m)) - (asq / (4 * (s->m * s->m)));
    }
    asq = 0.0;
    for (uint32_t c = 0; c < s->n; c++) asq += s->a[c] * s->a[c];
    return (intra / (2.0 * s->m)) - (asq / (4.0 * s->m * s->m));
}

static inline int is_lower_idx(const mstate *s, uint32_t cv, uint32_t ce) {
    /* modularity.cu:85-93, louvian.py:115-118 */
    if (s->comm_sz[cv] == 1 && s->comm_sz[ce] == 1) return ce < cv;
    return 1;
}

static void decide(mstate *s, uint32_t v, int rule, double *acc_s, uint32_t *touched) {
    const uint64_t b = s->off[v], e_end = s->off[v + 1];
    const uint32_t cv = s->comm[v];
    uint32_t nt = 0;
    /* neighbour-community sums (louvian.py:122-124) */
    for (uint64_t j = b; j < e_end; j++) {
        uint32_t c = s->comm[s->col[j]];
        if (acc_s[c] == 0.0 && nt < (uint32_t)(e_end - b)) {
            /* track every community once; zero weights re-track harmlessly */
            touched[nt++] = c;
        }
        acc_s[c] += s->w[j];
    }
    uint32_t target = cv;
    if (s->prec == ORC_PREC_FP64) {
        double max_gain = -INFINITY;
        uint32_t max_comm = UINT32_MAX;
        double e_own = 0.0;
        const double kv = s->k[v], m = s->m;
        for (uint64_t j = b; j < e_end; j++) {
            uint32_t e = s->col[j];
            uint32_t ce = s->comm[e];
            if (ce == cv && e != v) e_own += s->w[j];
            if (!is_lower_idx(s, cv, ce)) continue;
            double gain = (acc_s[ce] / m) +
                          (kv * ((s->a[cv] - kv) - s->a[ce]) / (2 * (m * m)));
            if (gain > max_gain || (gain == max_gain && ce < max_comm)) {
                max_gain = gain;
                max_comm = ce;
            }
        }
        int move = (rule == ORC_RULE_PY) ? (max_gain > 0)
                                         : (max_gain - (e_own / m) > 0);
        if (move) target = max_comm;
    } else {
        float max_gain = -INFINITY;
        uint32_t max_comm = UINT32_MAX;
        double e_own64 = 0.0;
        const float kv = (float)s->k[v], m = s->m32;
        const float den = 2.0f * m * m;
        const float aown = (float)s->a[cv];
        for (uint64_t j = b; j < e_end; j++) {
            uint32_t e = s->col[j];
            uint32_t ce = s->comm[e];
            if (ce == cv && e != v) e_own64 += s->w[j];
            if (!is_lower_idx(s, cv, ce)) continue;
            float ec = (float)acc_s[ce];
            float ac = (float)s->a[ce];
            volatile float t1 = ec / m;
            volatile float t2 = (aown - kv) - ac;
            volatile float t3 = kv * t2;
            volatile float t4 = t3 / den;
            float gain = t1 + t4;
            if (gain > max_gain || (gain == max_gain && ce < max_comm)) {
                max_gain = gain;
                max_comm = ce;
            }
        }
        int move;
        if (rule == ORC_RULE_PY) {
            move = max_gain > 0.0f;
        } else {
            volatile float eo = (float)e_own64 / m;
            move = (max_gain - eo) > 0.0f;
        }
        if (move) target = max_comm;
    }
    for (uint32_t i = 0; i < nt; i++) acc_s[touched[i]] = 0.0;
    /* acc entries that summed to exactly zero without being tracked twice
     * are already zero, so the scratch is clean again. */
    s->new_comm[v] = target;
}

typedef struct {
    mstate *s;
    const uint32_t *vset;
    uint32_t i0, i1;
    int rule;
    double *acc;
    uint32_t *touched;
} decide_job;

static void *decide_worker(void *arg) {
    decide_job *j = (decide_job *)arg;
    for (uint32_t i = j->i0; i < j->i1; i++) decide(j->s, j->vset[i], j->rule, j->acc, j->touched);
    return NULL;
}

/* Every vertex of a bucket decides against the same state (one Jacobi
 * step, modularity.cu:466-499), so the decisions split over threads; each
 * thread has its own scratch and every decision is the sequential one. */
static void decide_bucket(mstate *s, const uint32_t *vset, uint32_t cnt, int rule,
                          double **acc_t, uint32_t **touched_t, int T) {
    if (T <= 1 || cnt < 4096) {
        for (uint32_t i = 0; i < cnt; i++) decide(s, vset[i], rule, acc_t[0], touched_t[0]);
        return;
    }
    pthread_t th[256];
    decide_job jobs[256];
    for (int t = 0; t < T; t++) {
        jobs[t].s = s;
        jobs[t].vset = vset;
        jobs[t].i0 = (uint32_t)((uint64_t)cnt * t / T);
        jobs[t].i1 = (uint32_t)((uint64_t)cnt * (t + 1) / T);
        jobs[t].rule = rule;
        jobs[t].acc = acc_t[t];
        jobs[t].touched = touched_t[t];
        if (pthread_create(&th[t], NULL, decide_worker, &jobs[t]) != 0) {
            decide_worker(&jobs[t]);
            th[t] = 0;
        }
    }
    for (int t = 0; t < T; t++)
        if (th[t]) pthread_join(th[t], NULL);
}

static void recompute_totals(mstate *s) {
    /* louvian.py:70-73 / modularity.cu:497-498 */
    for (uint32_t c = 0; c < s->n; c++) s->a[c] = 0.0;
    for (uint32_t v = 0; v < s->n; v++) s->a[s->comm[v]] += s->k[v];
}

int orc_move_phase(uint32_t n, const uint64_t *off, const uint32_t *col,
                   const double *w, double threshold, int rule, int prec,
                   uint32_t max_passes, uint32_t *comm_out, double *q_trace,
                   uint32_t max_trace, uint32_t *passes_out, double *q_start,
                   double *q_end) {
    mstate s;
    memset(&s, 0, sizeof(s));
    s.n = n; s.off = off; s.col = col; s.w = w; s.prec = prec;
    size_t nn = n ? n : 1;
    s.k = (double *)malloc(sizeof(double) * nn);
    s.comm = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s.comm_sz = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s.a = (double *)malloc(sizeof(double) * nn);
    s.new_comm = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s.acc = (double *)calloc(nn, sizeof(double));
    uint64_t maxdeg = 0;
    for (uint32_t v = 0; v < n; v++)
        if (off[v + 1] - off[v] > maxdeg) maxdeg = off[v + 1] - off[v];
    s.touched = (uint32_t *)malloc(sizeof(uint32_t) * (maxdeg ? maxdeg : 1));
    uint32_t *vset = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    uint8_t *bk = (uint8_t *)malloc(nn);
    if (!s.k || !s.comm || !s.comm_sz || !s.a || !s.new_comm || !s.acc ||
        !s.touched || !vset || !bk) {
        free(s.k); free(s.comm); free(s.comm_sz); free(s.a); free(s.new_comm);
        free(s.acc); free(s.touched); free(vset); free(bk);
        return -ORC_ERR_NOMEM;
    }
    /* decision scratch per thread (thread 0 uses the state's own) */
    int T = g_threads;
    double *acc_t[256];
    uint32_t *touched_t[256];
    acc_t[0] = s.acc;
    touched_t[0] = s.touched;
    for (int t = 1; t < T; t++) {
        acc_t[t] = (double *)calloc(nn, sizeof(double));
        touched_t[t] = (uint32_t *)malloc(sizeof(uint32_t) * (maxdeg ? maxdeg : 1));
        if (!acc_t[t] || !touched_t[t]) { /* fall back to fewer threads */
            free(acc_t[t]);
            free(touched_t[t]);
            T = t;
            break;
        }
    }
    /* weighted degree and m (louvian.py:49-56, modularity.cu:27-49,457) */
    double all_w = 0.0;
    for (uint32_t v = 0; v < n; v++) {
        if (prec == ORC_PREC_FP64) {
            neu_sum ns = {0.0, 0.0};
            for (uint64_t j = off[v]; j < off[v + 1]; j++) neu_add(&ns, w[j]);
            s.k[v] = neu_result(&ns);
        } else {
            double acc = 0.0;
            for (uint64_t j = off[v]; j < off[v + 1]; j++) acc += w[j];
            s.k[v] = (double)(float)acc;
        }
        all_w += s.k[v];
    }
    s.m = all_w / 2;
    s.m32 = (float)s.m;
    for (uint32_t v = 0; v < n; v++) {
        s.comm[v] = v;
        s.comm_sz[v] = 1;
        s.a[v] = s.k[v];
    }
    orc_buckets(n, off, bk);

    uint32_t passes = 0;
    int ret = 1;
    double act, old;
    if (!(s.m > 0.0)) {
        /* No edge weight: modularity is undefined; nothing can move. */
        for (uint32_t v = 0; v < n; v++) comm_out[v] = v;
        if (passes_out) *passes_out = 0;
        if (q_start) *q_start = 0.0;
        if (q_end) *q_end = 0.0;
        free(s.k); free(s.comm); free(s.comm_sz); free(s.a); free(s.new_comm);
        free(s.acc); free(s.touched); free(vset); free(bk);
        for (int t = 1; t < T; t++) { free(acc_t[t]); free(touched_t[t]); }
        return 0;
    }
    act = state_modularity(&s);
    if (q_start) *q_start = act;
    int first = 1;
    do {
        for (int b = 1; b <= NBUCKETS; b++) {
            uint32_t cnt = 0;
            for (uint32_t v = 0; v < n; v++)
                if (bk[v] == b) vset[cnt++] = v;
            if (!cnt) continue;
            decide_bucket(&s, vset, cnt, rule, acc_t, touched_t, T);
            for (uint32_t i = 0; i < cnt; i++) { /* louvian.py:64-68 */
                uint32_t v = vset[i];
                s.comm_sz[s.new_comm[v]]++;
                s.comm_sz[s.comm[v]]--;
                s.comm[v] = s.new_comm[v];
            }
            recompute_totals(&s);
        }
        old = act;
        act = state_modularity(&s);
        if (q_trace && passes < max_trace) q_trace[passes] = act;
        passes++;
        if (first && act - old < threshold) ret = 0;
        first = 0;
    } while (act - old >= threshold && passes < max_passes);

    memcpy(comm_out, s.comm, sizeof(uint32_t) * n);
    if (passes_out) *passes_out = passes;
    if (q_end) *q_end = act;
    free(s.k); free(s.comm); free(s.comm_sz); free(s.a); free(s.new_comm);
    free(s.acc); free(s.touched); free(vset); free(bk);
    for (int t = 1; t < T; t++) { free(acc_t[t]); free(touched_t[t]); }
    return ret;
}

/* ------------------------------------------------------------------ */
/* Contraction                                                         */
/* ------------------------------------------------------------------ */

static int cmp_u32(const void *x, const void *y) {
    uint32_t a = *(const uint32_t *)x, b = *(const uint32_t *)y;
    return (a > b) - (a < b);
}

int orc_contract(uint32_t n, const uint64_t *off, const uint32_t *col,
                 const double *w, const uint32_t *comm, int row_order,
                 int prec, uint32_t *new_n_out, uint64_t *new_nnz_out,
                 uint64_t *new_off, uint32_t *new_col, double *new_w,
                 uint32_t *new_id) {
    size_t nn = n ? n : 1;
    uint32_t *sz = (uint32_t *)calloc(nn, sizeof(uint32_t));
    uint32_t *mstart = (uint32_t *)calloc(nn + 1, sizeof(uint32_t));
    uint32_t *members = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    double *acc = (double *)calloc(nn, sizeof(double));
    uint8_t *seen = (uint8_t *)calloc(nn, 1);
    uint32_t *order = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    if (!sz || !mstart || !members || !acc || !seen || !order) {
        free(sz); free(mstart); free(members); free(acc); free(seen);
        free(order);
        return ORC_ERR_NOMEM;
    }
    for (uint32_t v = 0; v < n; v++) {
        if (comm[v] >= n) {
            free(sz); free(mstart); free(members); free(acc); free(seen);
            free(order);
            return ORC_ERR_ARG;
        }
        sz[comm[v]]++;
    }
    /* Renumber non-empty communities in ascending old id
     * (aggregation.cu:390-393, louvian.py:178-187). */
    uint32_t nc = 0;
    for (uint32_t c = 0; c < n; c++) new_id[c] = sz[c] ? nc++ : 0;
    /* Members of each new community in ascending vertex id
     * (louvian.py:189-191). */
    for (uint32_t v = 0; v < n; v++) mstart[new_id[comm[v]] + 1]++;
    for (uint32_t c = 0; c < nc; c++) mstart[c + 1] += mstart[c];
    {
        uint32_t *cur = (uint32_t *)malloc(sizeof(uint32_t) * (nc ? nc : 1));
        if (!cur) {
            free(sz); free(mstart); free(members); free(acc); free(seen);
            free(order);
            return ORC_ERR_NOMEM;
        }
        for (uint32_t c = 0; c < nc; c++) cur[c] = mstart[c];
        for (uint32_t v = 0; v < n; v++) members[cur[new_id[comm[v]]]++] = v;
        free(cur);
    }
    uint64_t pos = 0;
    new_off[0] = 0;
    for (uint32_t c = 0; c < nc; c++) {
        uint32_t no = 0;
        for (uint32_t i = mstart[c]; i < mstart[c + 1]; i++) {
            uint32_t v = members[i];
            for (uint64_t j = off[v]; j < off[v + 1]; j++) {
                uint32_t t = new_id[comm[col[j]]];
                if (!seen[t]) {
                    seen[t] = 1;
                    order[no++] = t;
                }
                acc[t] += w[j];
            }
        }
        if (row_order == ORC_ROWS_SORTED)
            qsort(order, no, sizeof(uint32_t), cmp_u32);
        for (uint32_t i = 0; i < no; i++) {
            uint32_t t = order[i];
            new_col[pos] = t;
            new_w[pos] = (prec == ORC_PREC_FP32) ? (double)(float)acc[t]
                                                 : acc[t];
            pos++;
            acc[t] = 0.0;
            seen[t] = 0;
        }
        new_off[c + 1] = pos;
    }
    *new_n_out = nc;
    *new_nnz_out = pos;
    free(sz); free(mstart); free(members); free(acc); free(seen); free(order);
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* Whole run                                                           */
/* ------------------------------------------------------------------ */

int orc_louvain(uint32_t n, const uint64_t *off, const uint32_t *col,
                const double *w, double threshold, int rule, int prec,
                int row_order, uint32_t max_passes, uint32_t max_levels,
                uint32_t *assignment, double *q_final, orc_level_stat *stats,
                uint32_t max_stats, uint32_t *n_levels) {
    size_t nn = n ? n : 1;
    uint64_t E = off[n];
    uint32_t cn = n;
    uint64_t *coff = (uint64_t *)malloc(sizeof(uint64_t) * (nn + 1));
    uint32_t *ccol = (uint32_t *)malloc(sizeof(uint32_t) * (E ? E : 1));
    double *cw = (double *)malloc(sizeof(double) * (E ? E : 1));
    uint64_t *noff = (uint64_t *)malloc(sizeof(uint64_t) * (nn + 1));
    uint32_t *ncol = (uint32_t *)malloc(sizeof(uint32_t) * (E ? E : 1));
    double *nw = (double *)malloc(sizeof(double) * (E ? E : 1));
    uint32_t *comm = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    uint32_t *nid = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    if (!coff || !ccol || !cw || !noff || !ncol || !nw || !comm || !nid) {
        free(coff); free(ccol); free(cw); free(noff); free(ncol); free(nw);
        free(comm); free(nid);
        return ORC_ERR_NOMEM;
    }
    memcpy(coff, off, sizeof(uint64_t) * (n + 1));
    memcpy(ccol, col, sizeof(uint32_t) * E);
    for (uint64_t j = 0; j < E; j++)
        cw[j] = (prec == ORC_PREC_FP32) ? (double)(float)w[j] : w[j];
    for (uint32_t v = 0; v < n; v++) assignment[v] = v; /* utils.cu:67 */
    uint32_t lev = 0;
    double qf = 0.0;
    for (;;) {
        uint32_t passes = 0;
        double qs = 0.0, qe = 0.0;
        int r = orc_move_phase(cn, coff, ccol, cw, threshold, rule, prec,
                               max_passes, comm, NULL, 0, &passes, &qs, &qe);
        if (r < 0) {
            free(coff); free(ccol); free(cw); free(noff); free(ncol); free(nw);
            free(comm); free(nid);
            return -r;
        }
        if (stats && lev < max_stats) {
            stats[lev].n_vertices = cn;
            stats[lev].n_entries = coff[cn];
            stats[lev].passes = passes;
            stats[lev].moved = (uint32_t)r;
            stats[lev].q_start = qs;
            stats[lev].q_end = qe;
        }
        lev++;
        if (!r) { /* modularity.cu:503-506: print Q_old and stop */
            qf = qs;
            break;
        }
        /* graphVertToComm (modularity.cu:51-56,515-517) */
        for (uint32_t v = 0; v < n; v++) assignment[v] = comm[assignment[v]];
        uint32_t nn2 = 0;
        uint64_t ne2 = 0;
        int rc = orc_contract(cn, coff, ccol, cw, comm, row_order, prec, &nn2,
                              &ne2, noff, ncol, nw, nid);
        if (rc) {
            free(coff); free(ccol); free(cw); free(noff); free(ncol); free(nw);
            free(comm); free(nid);
            return rc;
        }
        /* graphVertToNewComm (aggregation.cu:380-385) */
        for (uint32_t v = 0; v < n; v++) assignment[v] = nid[assignment[v]];
        uint64_t *t0 = coff; coff = noff; noff = t0;
        uint32_t *t1 = ccol; ccol = ncol; ncol = t1;
        double *t2 = cw; cw = nw; nw = t2;
        qf = qe;
        /* A level that merged nothing would repeat forever (only possible
         * with threshold <= 0, where the reference never terminates). */
        if (nn2 == cn) break;
        cn = nn2;
        if (max_levels && lev >= max_levels) break;
    }
    if (q_final) *q_final = qf;
    if (n_levels) *n_levels = lev;
    free(coff); free(ccol); free(cw); free(noff); free(ncol); free(nw);
    free(comm); free(nid);
    return ORC_OK;
}

double orc_modularity(uint32_t n, const uint64_t *off, const uint32_t *col,
                      const double *w, const uint32_t *part) {
    size_t nn = n ? n : 1;
    double *a = (double *)calloc(nn, sizeof(double));
    if (!a) return NAN;
    double total = 0.0, intra = 0.0;
    for (uint32_t v = 0; v < n; v++) {
        double k = 0.0;
        for (uint64_t j = off[v]; j < off[v + 1]; j++) {
            k += w[j];
            if (part[col[j]] == part[v]) intra += w[j];
        }
        a[part[v]] += k;
        total += k;
    }
    double m = total / 2.0;
    double asq = 0.0;
    for (uint32_t c = 0; c < n; c++) asq += a[c] * a[c];
    free(a);
    if (!(m > 0.0)) return 0.0;
    return intra / (2.0 * m) - asq / (4.0 * m * m);
}
