/*
 * CPU oracle for the Gotoh scoring path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is a plain-C restatement of the reference package's NumPy oracle
 * (src/gpusw/reference.py:38-125, `_score_codes`). It exists to check the CUDA engine
 * (tests, the smoke check and the CPU-baseline leg of the benchmark); the product never
 * calls it. Arithmetic is scalar int64 exactly like the reference:
 *
 *   rows i = reference residues (m), columns j = query residues (n),
 *   s(i,j) = SUB[r[i-1] * ns + q[j-1]]                       (reference.py:71-72, :92)
 *   F(i,j) = max(H(i-1,j) + go, F(i-1,j) + ge)                (reference.py:84-87)
 *   E(i,j) = max(H(i,j-1) + go, E(i,j-1) + ge)                (reference.py:88-91)
 *   H(i,j) = max(H(i-1,j-1) + s, E, F), clamped at 0 in local  (reference.py:92-98)
 *   boundaries H(0,j), H(i,0) per mode / free-end flags        (reference.py:58-78)
 *   result: local best; global corner; semiglobal max(corner, endcol if free_q,
 *   endrow if free_r), then max(.,0) if both are free          (reference.py:114-125)
 *   empty sequences                                            (reference.py:48-54)
 *
 * The pair loop is spread over POSIX threads; each pair is scored independently.
 *
 * oracle_locate adds the best-cell coordinates the engine's gpusw_locate_pairs returns (the
 * reference is score-only; its examples re-align on the CPU to find coordinates,
 * examples/legacy_16s_gpu_align.py:280-292): the same recurrence, local or anchored at the
 * start (global boundaries), keeping the maximum of H over all cells and the first cell that
 * holds it in row-major order (reference row, then query column).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_NEG (-(INT64_C(1) << 30))

enum { MODE_LOCAL = 0, MODE_GLOBAL = 1, MODE_SEMI = 2 };

typedef struct {
    const int32_t *sub;
    int ns, mode, go, ge, free_q, free_r;
} oracle_scheme;

static int64_t ladder(int go, int ge, int64_t k) { return (int64_t)go + (k - 1) * (int64_t)ge; }

/* One (query, reference) pair; hp/f are caller scratch of n+1 int64 each. */
static int64_t score_one(const uint8_t *q, int64_t n, const uint8_t *r, int64_t m,
                         const oracle_scheme *s, int64_t *hp, int64_t *f) {
    const int local = s->mode == MODE_LOCAL, global = s->mode == MODE_GLOBAL;
    const int semi = s->mode == MODE_SEMI;
    const int64_t go = s->go, ge = s->ge;
    if (n == 0 || m == 0) {
        if (local || (n == 0 && m == 0)) return 0;
        if (n == 0) return (semi && s->free_q) ? 0 : ladder(s->go, s->ge, m);
        return (semi && s->free_r) ? 0 : ladder(s->go, s->ge, n);
    }
    hp[0] = 0;
    for (int64_t j = 1; j <= n; ++j) {
        if (local) hp[j] = 0;
        else if (global) hp[j] = ladder(s->go, s->ge, j);
        else hp[j] = s->free_r ? 0 : ladder(s->go, s->ge, j);
        f[j] = ORACLE_NEG;
    }
    f[0] = ORACLE_NEG;
    int64_t best = 0, endcol = ORACLE_NEG;
    for (int64_t i = 1; i <= m; ++i) {
        const int32_t *subrow = s->sub + (int64_t)r[i - 1] * s->ns;
        int64_t hleft;
        if (local) hleft = 0;
        else if (global) hleft = ladder(s->go, s->ge, i);
        else hleft = s->free_q ? 0 : ladder(s->go, s->ge, i);
        int64_t diag = hp[0];
        hp[0] = hleft;
        int64_t eleft = ORACLE_NEG;
        /* the same cell update in both branches; local mode clamps at 0 and keeps the
         * running maximum, the others read their result from the last row and column */
        if (local) {
            for (int64_t j = 1; j <= n; ++j) {
                int64_t fj = hp[j] + go, fe = f[j] + ge;
                fj = fe > fj ? fe : fj;
                int64_t ej = hleft + go, ee = eleft + ge;
                ej = ee > ej ? ee : ej;
                int64_t h = diag + (int64_t)subrow[q[j - 1]];
                h = ej > h ? ej : h;
                h = fj > h ? fj : h;
                h = h < 0 ? 0 : h;
                best = h > best ? h : best;
                diag = hp[j];
                hp[j] = h;
                f[j] = fj;
                hleft = h;
                eleft = ej;
            }
        } else {
            for (int64_t j = 1; j <= n; ++j) {
                int64_t fj = hp[j] + go, fe = f[j] + ge;
                fj = fe > fj ? fe : fj;
                int64_t ej = hleft + go, ee = eleft + ge;
                ej = ee > ej ? ee : ej;
                int64_t h = diag + (int64_t)subrow[q[j - 1]];
                h = ej > h ? ej : h;
                h = fj > h ? fj : h;
                diag = hp[j];
                hp[j] = h;
                f[j] = fj;
                hleft = h;
                eleft = ej;
            }
            if (hp[n] > endcol) endcol = hp[n];           /* H(i, n), last query column */
        }
    }
    if (local) return best;
    const int64_t corner = hp[n];                          /* H(m, n) */
    if (global) return corner;
    int64_t endrow = ORACLE_NEG;                           /* max_j H(m, j), last ref row */
    for (int64_t j = 1; j <= n; ++j) endrow = hp[j] > endrow ? hp[j] : endrow;
    int64_t res = corner;
    if (s->free_q && endcol > res) res = endcol;
    if (s->free_r && endrow > res) res = endrow;
    if (s->free_q && s->free_r && res < 0) res = 0;
    return res;
}

int64_t oracle_score(const uint8_t *q, int64_t n, const uint8_t *r, int64_t m,
                     const int32_t *sub, int ns, int mode, int go, int ge, int free_q,
                     int free_r) {
    oracle_scheme s = {sub, ns, mode, go, ge, free_q, free_r};
    int64_t *buf = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(n + 1));
    if (!buf) return INT64_MIN;
    int64_t v = score_one(q, n, r, m, &s, buf, buf + n + 1);
    free(buf);
    return v;
}

typedef struct {
    const uint8_t *qcodes, *rcodes;
    const int32_t *qoff, *roff, *qi, *rj;
    int64_t npairs;
    int64_t ncols;              /* > 0: cross product, pair k = (qi[k / ncols], k % ncols) */
    const oracle_scheme *s;
    int64_t *out;
    int64_t next;               /* shared work counter */
    pthread_mutex_t lock;
    int64_t maxq;
    int failed;
} job_t;

static void *worker(void *arg) {
    job_t *job = (job_t *)arg;
    int64_t *buf = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(job->maxq + 1));
    if (!buf) { job->failed = 1; return NULL; }
    for (;;) {
        pthread_mutex_lock(&job->lock);
        int64_t k0 = job->next;
        job->next += 64;
        pthread_mutex_unlock(&job->lock);
        if (k0 >= job->npairs) break;
        int64_t k1 = k0 + 64 < job->npairs ? k0 + 64 : job->npairs;
        for (int64_t k = k0; k < k1; ++k) {
            int64_t a, b;
            if (job->ncols > 0) { a = job->qi[k / job->ncols]; b = k % job->ncols; }
            else { a = job->qi[k]; b = job->rj[k]; }
            const uint8_t *q = job->qcodes + job->qoff[a];
            const uint8_t *r = job->rcodes + job->roff[b];
            job->out[k] = score_one(q, job->qoff[a + 1] - job->qoff[a], r,
                                    job->roff[b + 1] - job->roff[b], job->s, buf,
                                    buf + job->maxq + 1);
        }
    }
    free(buf);
    return NULL;
}

static int run_job(job_t *job, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t tid[256];
    pthread_mutex_init(&job->lock, NULL);
    int started = 0;
    for (int t = 0; t < nthreads; ++t)
        if (pthread_create(&tid[t], NULL, worker, job) == 0) ++started;
    if (started == 0) worker(job);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    pthread_mutex_destroy(&job->lock);
    return job->failed ? -1 : 0;
}

static int64_t max_len(const int32_t *off, const int32_t *idx, int64_t n, int64_t all) {
    int64_t mx = 0;
    if (idx) {
        for (int64_t k = 0; k < n; ++k) { int64_t l = off[idx[k] + 1] - off[idx[k]]; if (l > mx) mx = l; }
    } else {
        for (int64_t k = 0; k < all; ++k) { int64_t l = off[k + 1] - off[k]; if (l > mx) mx = l; }
    }
    return mx;
}

/* out[k] = score(query qi[k], reference rj[k]). Returns 0 on success. */
int oracle_score_pairs(const uint8_t *qcodes, const int32_t *qoff, const uint8_t *rcodes,
                       const int32_t *roff, const int32_t *qi, const int32_t *rj,
                       int64_t npairs, const int32_t *sub, int ns, int mode, int go, int ge,
                       int free_q, int free_r, int nthreads, int64_t *out) {
    oracle_scheme s = {sub, ns, mode, go, ge, free_q, free_r};
    job_t job;
    memset(&job, 0, sizeof(job));
    job.qcodes = qcodes; job.rcodes = rcodes; job.qoff = qoff; job.roff = roff;
    job.qi = qi; job.rj = rj; job.npairs = npairs; job.ncols = 0; job.s = &s; job.out = out;
    job.maxq = max_len(qoff, qi, npairs, 0);
    return run_job(&job, nthreads);
}

/* out[a * nr + b] = score(query qlist[a], reference b) for a < nq, b < nr. */
int oracle_score_cross(const uint8_t *qcodes, const int32_t *qoff, const int32_t *qlist,
                       int64_t nq, const uint8_t *rcodes, const int32_t *roff, int64_t nr,
                       const int32_t *sub, int ns, int mode, int go, int ge, int free_q,
                       int free_r, int nthreads, int64_t *out) {
    oracle_scheme s = {sub, ns, mode, go, ge, free_q, free_r};
    job_t job;
    memset(&job, 0, sizeof(job));
    job.qcodes = qcodes; job.rcodes = rcodes; job.qoff = qoff; job.roff = roff;
    job.qi = qlist; job.rj = NULL; job.npairs = nq * nr; job.ncols = nr; job.s = &s;
    job.out = out;
    job.maxq = max_len(qoff, qlist, nq, 0);
    if (nr == 0) return 0;
    return run_job(&job, nthreads);
}

/* out[0] = max of H over all cells; out[1], out[2] = 0-based reference row and query column
 * of the first cell (row-major) holding it, or -1, -1 when no cell scores above 0 in local
 * mode. anchored = 0: local; anchored = 1: global boundaries (both sequences start at their
 * first residue), the end anywhere. Returns 0, or -1 when out of memory. */
int oracle_locate(const uint8_t *q, int64_t n, const uint8_t *r, int64_t m, const int32_t *sub,
                  int ns, int go, int ge, int anchored, int64_t *out) {
    out[0] = 0; out[1] = -1; out[2] = -1;
    if (n == 0 || m == 0) return 0;
    int64_t *hp = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(n + 1));
    if (!hp) return -1;
    int64_t *f = hp + n + 1;
    hp[0] = 0;
    for (int64_t j = 1; j <= n; ++j) { hp[j] = anchored ? ladder(go, ge, j) : 0; f[j] = ORACLE_NEG; }
    int64_t best = anchored ? ORACLE_NEG : 0, bi = -1, bj = -1;
    for (int64_t i = 1; i <= m; ++i) {
        const int32_t *subrow = sub + (int64_t)r[i - 1] * ns;
        int64_t hleft = anchored ? ladder(go, ge, i) : 0, diag = hp[0], eleft = ORACLE_NEG;
        hp[0] = hleft;
        for (int64_t j = 1; j <= n; ++j) {
            int64_t fj = hp[j] + go, fe = f[j] + ge;
            if (fe > fj) fj = fe;
            int64_t ej = hleft + go, ee = eleft + ge;
            if (ee > ej) ej = ee;
            int64_t h = diag + (int64_t)subrow[q[j - 1]];
            if (ej > h) h = ej;
            if (fj > h) h = fj;
            if (!anchored && h < 0) h = 0;
            if (h > best) { best = h; bi = i - 1; bj = j - 1; }
            diag = hp[j]; hp[j] = h; f[j] = fj; hleft = h; eleft = ej;
        }
    }
    free(hp);
    out[0] = best; out[1] = bi; out[2] = bj;
    return 0;
}
