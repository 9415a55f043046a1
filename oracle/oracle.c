/*
 * Oracle of the B200 numerical phase -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of PaStiX 6.4's numerical factorization and solve on a
 * given block symbolic structure, used by the tests, the smoke check and the
 * CPU baseline of bench.py as the checker.  The product (libpastix_b200.so)
 * never links or calls it.
 *
 * Followed reference code (file:line within the PaStiX tree):
 *   fill-in            kernels/cpucblk_zinit.c:395-487 (cpucblk_zfillin_fr)
 *   POTRF panel        kernels/core_zpotrfsp.c:68-190, :220, :334
 *   GETRF panel        kernels/core_zgetrfsp.c:65-200, :217-275, :305-330, :355-395
 *   SYTRF panel        kernels/core_zsytrfsp.c:66-220, :234-275, :432-460, :487-540,
 *                      DL^T workspace kernels/core_zscalo.c:171
 *   off-diagonal TRSM  kernels/core_ztrsmsp.c:149-200, :356
 *   update GEMM        kernels/core_zgemmsp.c:404-474 (core_zgemmsp_2d2d)
 *   dependencies       kernels/cpucblk_zmpi_coeftab.c:543-614 (ctrbcnt), dynamic
 *                      scheduler sopalin/sequential_zpotrf.c:195-294
 *   solve              kernels/solve_ztrsmsp.c:76-160 (blok trsm / gemm),
 *                      :302 (forward), :468 (backward), :664 (diag)
 *   static pivot       criterion = eps * ||A||_F, sopalin/pastix_task_sopalin.c:464-495
 * Parity status: no reference output vectors exist for this path; the
 * oracle is pinned by the reference's own known-answer checks (backward
 * error thresholds of example/simple.c:140 and test/z_bcsc_tests.c:179-186,
 * zero static pivots on SPD matrices) and by the uniqueness of the LL^T,
 * LDL^T and LU-without-pivoting factors of a given ordering (LAPACK on the
 * dense permuted matrix), see tests/test_oracle.py.
 *
 * BLAS: plain loops by default; ora_load_blas() binds cblas_dgemm /
 * cblas_sgemm from an OpenBLAS shared object (the reference's kernels call
 * CBLAS at the same places) for the timed CPU baseline.
 */
#include <dlfcn.h>
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int64_t n, cblknbr, bloknbr;
    const int64_t *cb_fcol, *cb_lcol, *cb_fblok; /* cb_fblok has cblknbr + 1 entries */
    const int64_t *bk_frow, *bk_lrow, *bk_fcblk;
} ora_symbol_t;

typedef void (*gemm_d_t)(int, int, int, int, int, int, double, const double *, int, const double *, int, double,
                         double *, int);
typedef void (*gemm_s_t)(int, int, int, int, int, int, float, const float *, int, const float *, int, float, float *,
                         int);
static struct {
    gemm_d_t dgemm;
    gemm_s_t sgemm;
    void (*set_threads)(int);
} ora_blas;

/* Bind cblas_{d,s}gemm from a BLAS library; returns 0 on success. */
int ora_load_blas(const char *path) {
    void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return -1;
    ora_blas.dgemm = (gemm_d_t)dlsym(h, "cblas_dgemm");
    ora_blas.sgemm = (gemm_s_t)dlsym(h, "cblas_sgemm");
    ora_blas.set_threads = (void (*)(int))dlsym(h, "openblas_set_num_threads");
    if (ora_blas.set_threads) ora_blas.set_threads(1); /* BLAS threads forced to 1 (common/api.c:1179) */
    return (ora_blas.dgemm && ora_blas.sgemm) ? 0 : -2;
}
void ora_unload_blas(void) { memset(&ora_blas, 0, sizeof(ora_blas)); }

/* 2D layout offsets: coefind[b] for every blok, returns the total size */
int64_t ora_layout(const ora_symbol_t *s, int64_t *coefind) {
    int64_t off = 0;
    for (int64_t k = 0; k < s->cblknbr; k++) {
        int64_t nc = s->cb_lcol[k] - s->cb_fcol[k] + 1;
        for (int64_t b = s->cb_fblok[k]; b < s->cb_fblok[k + 1]; b++) {
            coefind[b] = off;
            off += (s->bk_lrow[b] - s->bk_frow[b] + 1) * nc;
        }
    }
    return off;
}

static int64_t ora_cblk_of(const ora_symbol_t *s, int64_t col) {
    int64_t lo = 0, hi = s->cblknbr - 1;
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) / 2;
        if (s->cb_fcol[mid] <= col) lo = mid; else hi = mid - 1;
    }
    return lo;
}

/* position of entry (r, c), r >= c, in the 2D layout; -1 when outside */
static int64_t ora_position(const ora_symbol_t *s, const int64_t *coefind, int64_t r, int64_t c) {
    int64_t k = ora_cblk_of(s, c);
    int64_t lo = s->cb_fblok[k], hi = s->cb_fblok[k + 1] - 1;
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) / 2;
        if (s->bk_frow[mid] <= r) lo = mid; else hi = mid - 1;
    }
    if (r < s->bk_frow[lo] || r > s->bk_lrow[lo]) return -1;
    int64_t ld = s->bk_lrow[lo] - s->bk_frow[lo] + 1;
    return coefind[lo] + (r - s->bk_frow[lo]) + (c - s->cb_fcol[k]) * ld;
}

#define T double
#define SFX d
#define IS_DOUBLE 1
#include "oracle_core.inc"
#undef T
#undef SFX
#undef IS_DOUBLE
#define T float
#define SFX s
#define IS_DOUBLE 0
#include "oracle_core.inc"
#undef T
#undef SFX
#undef IS_DOUBLE

int ora_fill_d(const ora_symbol_t *s, const int64_t *coefind, int fact, const int64_t *colptr, const int64_t *rowind,
               const double *val, double *L, double *U) {
    return ora_d_fill(s, coefind, fact, colptr, rowind, val, L, U);
}
int ora_fill_s(const ora_symbol_t *s, const int64_t *coefind, int fact, const int64_t *colptr, const int64_t *rowind,
               const double *val, float *L, float *U) {
    return ora_s_fill(s, coefind, fact, colptr, rowind, val, L, U);
}

/* ---------------- factorization: dynamic scheduler over cblks ---------------- */
typedef struct {
    const ora_symbol_t *s;
    const int64_t *coefind;
    int fact, single;
    double crit;
    void *L, *U;
    int64_t maxoff;             /* max off-diagonal coefficients of a cblk (DL^T workspace) */
    atomic_int_fast64_t *ctrb;  /* contributions still to receive */
    pthread_mutex_t *locks;     /* per facing cblk */
    pthread_mutex_t qmu;
    pthread_cond_t qcv;
    int64_t *queue, qhead, qtail, done;
    atomic_int_fast64_t npiv;
} ora_sched_t;

static void ora_do_cblk(ora_sched_t *S, int64_t k, void *work) {
    const ora_symbol_t *s = S->s;
    int64_t fb = s->cb_fblok[k], lb = s->cb_fblok[k + 1];
    int64_t np;
    if (S->single) np = ora_s_panel(s, S->coefind, S->fact, S->crit, k, (float *)S->L, (float *)S->U, (float *)work);
    else np = ora_d_panel(s, S->coefind, S->fact, S->crit, k, (double *)S->L, (double *)S->U, (double *)work);
    if (np) atomic_fetch_add(&S->npiv, np);
    int64_t boff = fb + 1 < lb ? S->coefind[fb + 1] : 0;
    for (int64_t b = fb + 1; b < lb; b++) {
        int64_t f = s->bk_fcblk[b];
        pthread_mutex_lock(&S->locks[f]);
        if (S->single) {
            float *L = (float *)S->L, *U = (float *)S->U;
            if (S->fact == 0) ora_s_update(s, S->coefind, k, b, L, L, 0, L, 0);
            else if (S->fact == 1) ora_s_update(s, S->coefind, k, b, L, (float *)work, boff, L, 0);
            else {
                ora_s_update(s, S->coefind, k, b, L, U, 0, L, 0);
                if (b + 1 < lb) ora_s_update(s, S->coefind, k, b, U, L, 0, U, 1);
            }
        } else {
            double *L = (double *)S->L, *U = (double *)S->U;
            if (S->fact == 0) ora_d_update(s, S->coefind, k, b, L, L, 0, L, 0);
            else if (S->fact == 1) ora_d_update(s, S->coefind, k, b, L, (double *)work, boff, L, 0);
            else {
                ora_d_update(s, S->coefind, k, b, L, U, 0, L, 0);
                if (b + 1 < lb) ora_d_update(s, S->coefind, k, b, U, L, 0, U, 1);
            }
        }
        pthread_mutex_unlock(&S->locks[f]);
        if (atomic_fetch_sub(&S->ctrb[f], 1) == 1) {
            pthread_mutex_lock(&S->qmu);
            S->queue[S->qtail++] = f;
            pthread_cond_signal(&S->qcv);
            pthread_mutex_unlock(&S->qmu);
        }
    }
}

static void *ora_worker(void *arg) {
    ora_sched_t *S = (ora_sched_t *)arg;
    size_t es = S->single ? sizeof(float) : sizeof(double);
    void *work = malloc((size_t)(S->maxoff > 0 ? S->maxoff : 1) * es);
    for (;;) {
        pthread_mutex_lock(&S->qmu);
        while (S->qhead == S->qtail && S->done < S->s->cblknbr) pthread_cond_wait(&S->qcv, &S->qmu);
        if (S->done >= S->s->cblknbr) {
            pthread_mutex_unlock(&S->qmu);
            break;
        }
        int64_t k = S->queue[S->qhead++];
        pthread_mutex_unlock(&S->qmu);
        ora_do_cblk(S, k, work);
        pthread_mutex_lock(&S->qmu);
        S->done++;
        if (S->done >= S->s->cblknbr) pthread_cond_broadcast(&S->qcv);
        pthread_mutex_unlock(&S->qmu);
    }
    free(work);
    return NULL;
}

/* Factorize in place; fact: 0 POTRF, 1 SYTRF, 2 GETRF.  single: float panels.
 * Returns the number of static pivots. */
int64_t ora_factor(const ora_symbol_t *s, const int64_t *coefind, int fact, int single, double crit, void *L, void *U,
                   int nthreads) {
    ora_sched_t S;
    memset(&S, 0, sizeof(S));
    S.s = s; S.coefind = coefind; S.fact = fact; S.single = single; S.crit = crit; S.L = L; S.U = U;
    S.ctrb = calloc((size_t)s->cblknbr, sizeof(*S.ctrb));
    S.locks = malloc((size_t)s->cblknbr * sizeof(pthread_mutex_t));
    S.queue = malloc((size_t)s->cblknbr * sizeof(int64_t));
    for (int64_t k = 0; k < s->cblknbr; k++) {
        pthread_mutex_init(&S.locks[k], NULL);
        int64_t nc = s->cb_lcol[k] - s->cb_fcol[k] + 1, off = 0;
        for (int64_t b = s->cb_fblok[k] + 1; b < s->cb_fblok[k + 1]; b++) {
            atomic_fetch_add(&S.ctrb[s->bk_fcblk[b]], 1);
            off += (s->bk_lrow[b] - s->bk_frow[b] + 1) * nc;
        }
        if (off > S.maxoff) S.maxoff = off;
    }
    for (int64_t k = 0; k < s->cblknbr; k++)
        if (atomic_load(&S.ctrb[k]) == 0) S.queue[S.qtail++] = k;
    pthread_mutex_init(&S.qmu, NULL);
    pthread_cond_init(&S.qcv, NULL);
    if (nthreads < 1) nthreads = 1;
    if (nthreads == 1) {
        ora_worker(&S);
    } else {
        pthread_t *th = malloc((size_t)nthreads * sizeof(pthread_t));
        for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, ora_worker, &S);
        for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
        free(th);
    }
    int64_t np = atomic_load(&S.npiv);
    for (int64_t k = 0; k < s->cblknbr; k++) pthread_mutex_destroy(&S.locks[k]);
    free((void *)S.ctrb);
    free(S.locks);
    free(S.queue);
    return np;
}

/* Copy 2D-layout panels into the one-panel-per-cblk layout of the product
 * (column major, ld = stride, blok b at row offset rowoff[b]) for comparison. */
void ora_to_panels(const ora_symbol_t *s, const int64_t *coefind, const int64_t *cb_coef, const int64_t *cb_stride,
                   const int64_t *bk_rowoff, int single, const void *src, void *dst) {
    for (int64_t k = 0; k < s->cblknbr; k++) {
        int64_t nc = s->cb_lcol[k] - s->cb_fcol[k] + 1, st = cb_stride[k];
        for (int64_t b = s->cb_fblok[k]; b < s->cb_fblok[k + 1]; b++) {
            int64_t m = s->bk_lrow[b] - s->bk_frow[b] + 1;
            for (int64_t c = 0; c < nc; c++)
                for (int64_t i = 0; i < m; i++) {
                    int64_t from = coefind[b] + i + c * m, to = cb_coef[k] + bk_rowoff[b] + i + c * st;
                    if (single) ((float *)dst)[to] = ((const float *)src)[from];
                    else ((double *)dst)[to] = ((const double *)src)[from];
                }
        }
    }
}

/* ---------------- solve (double; float factors go through oracle.py casts) ---------------- */
/* forward: L y = b, blok by blok (solve_cblk_ztrsmsp_forward) */
static void ora_fwd(const ora_symbol_t *s, const int64_t *coefind, const double *L, int unit, int64_t nrhs, double *B,
                    int64_t ldb) {
    for (int64_t k = 0; k < s->cblknbr; k++) {
        int64_t fc = s->cb_fcol[k], nc = s->cb_lcol[k] - fc + 1;
        int64_t fb = s->cb_fblok[k];
        const double *D = L + coefind[fb];
        for (int64_t j = 0; j < nrhs; j++) {
            double *y = B + fc + j * ldb;
            for (int64_t c = 0; c < nc; c++) {
                if (!unit) y[c] /= D[c + c * nc];
                for (int64_t i = c + 1; i < nc; i++) y[i] -= D[i + c * nc] * y[c];
            }
        }
        for (int64_t b = fb + 1; b < s->cb_fblok[k + 1]; b++) {
            int64_t m = s->bk_lrow[b] - s->bk_frow[b] + 1;
            const double *P = L + coefind[b];
            for (int64_t j = 0; j < nrhs; j++) {
                const double *y = B + fc + j * ldb;
                double *t = B + s->bk_frow[b] + j * ldb;
                for (int64_t c = 0; c < nc; c++)
                    for (int64_t i = 0; i < m; i++) t[i] -= P[i + c * m] * y[c];
            }
        }
    }
}

/* backward: P^T x = y, cblks in reverse order; diagonal solve, then the
 * off-diagonal bloks of the cblks facing it are applied (browtab walk,
 * solve_cblk_ztrsmsp_backward) -- written here as the equivalent gather over
 * the cblk's own off-diagonal bloks before its diagonal solve. */
static void ora_bwd(const ora_symbol_t *s, const int64_t *coefind, const double *P, int unit, int64_t nrhs, double *B,
                    int64_t ldb) {
    for (int64_t k = s->cblknbr - 1; k >= 0; k--) {
        int64_t fc = s->cb_fcol[k], nc = s->cb_lcol[k] - fc + 1;
        int64_t fb = s->cb_fblok[k];
        for (int64_t b = fb + 1; b < s->cb_fblok[k + 1]; b++) {
            int64_t m = s->bk_lrow[b] - s->bk_frow[b] + 1;
            const double *Q = P + coefind[b];
            for (int64_t j = 0; j < nrhs; j++) {
                double *x = B + fc + j * ldb;
                const double *t = B + s->bk_frow[b] + j * ldb;
                for (int64_t c = 0; c < nc; c++) {
                    double acc = 0;
                    for (int64_t i = 0; i < m; i++) acc += Q[i + c * m] * t[i];
                    x[c] -= acc;
                }
            }
        }
        const double *D = P + coefind[fb];
        for (int64_t j = 0; j < nrhs; j++) {
            double *x = B + fc + j * ldb;
            for (int64_t c = nc - 1; c >= 0; c--) {
                for (int64_t i = c + 1; i < nc; i++) x[c] -= D[i + c * nc] * x[i];
                if (!unit) x[c] /= D[c + c * nc];
            }
        }
    }
}

/* Solve A X = B on permuted vectors with FP64 factors (trans: A^T X = B). */
void ora_solve(const ora_symbol_t *s, const int64_t *coefind, int fact, const double *L, const double *U, int trans,
               int64_t nrhs, double *B, int64_t ldb) {
    if (fact == 0) {
        ora_fwd(s, coefind, L, 0, nrhs, B, ldb);
        ora_bwd(s, coefind, L, 0, nrhs, B, ldb);
    } else if (fact == 1) {
        ora_fwd(s, coefind, L, 1, nrhs, B, ldb);
        for (int64_t k = 0; k < s->cblknbr; k++) {  /* solve_cblk_zdiag */
            int64_t fc = s->cb_fcol[k], nc = s->cb_lcol[k] - fc + 1;
            const double *D = L + coefind[s->cb_fblok[k]];
            for (int64_t j = 0; j < nrhs; j++)
                for (int64_t c = 0; c < nc; c++) B[fc + c + j * ldb] /= D[c + c * nc];
        }
        ora_bwd(s, coefind, L, 1, nrhs, B, ldb);
    } else if (!trans) {
        ora_fwd(s, coefind, L, 1, nrhs, B, ldb);
        ora_bwd(s, coefind, U, 0, nrhs, B, ldb);
    } else {
        ora_fwd(s, coefind, U, 0, nrhs, B, ldb);
        ora_bwd(s, coefind, L, 1, nrhs, B, ldb);
    }
}
