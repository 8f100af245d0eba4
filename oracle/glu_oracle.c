/*
 * Test infrastructure only -- the oracle, never shipped or measured.
 *
 * Plain-C restatement of the reference's numeric path, sequential, for sizes
 * that finish in seconds.  Pinned against the reference's own CPU code
 * compiled from the reference tree (oracle/_ref/libglu_ref.so): pattern,
 * levels and predictLU values bit-exact, solve bit-exact on the same factors.
 *
 *  orc_factor_f32/f64 -- src/numeric.cu:10-103 (RL) and :204-345 (RL_onecol_*)
 *      executed column by column in level order: scale the L part by the
 *      pivot (numeric.cu:36-47), scatter it into a dense scratch column
 *      (numeric.cu:44), and for every column j of U-row k subtract
 *      scratch[i] * A(k,j) from every A(i,j), i > k, of column j
 *      (numeric.cu:58-89); the product is rounded before the subtraction as
 *      atomicAdd(&A, -tmp*s) does.  GESP (numeric.cu:139-140): a pivot with
 *      |d| < pert is replaced by +pert, only in columns with an L part.
 *  orc_pert -- numeric.cu:490-506.
 *  orc_solve_f32 -- src/symbolic.cc:200-251.
 *  orc_leveling -- src/symbolic.cc:106-151.
 *  orc_fill_in -- src/symbolic.cc:11-53.
 */
#define _GNU_SOURCE /* pthread_barrier_t, sysconf */
#include "glu_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* The targets j of U-row k are independent (each touches only column j), so
 * for rows with many targets they are split over a team of threads; every
 * entry still receives its updates one pivot k at a time, in the same order,
 * so the result does not depend on the thread count.  Rows are ascending in
 * every column: A(k,j) is found by binary search and the update starts right
 * after it, skipping the rows <= k that numeric.cu:58-89 scans without
 * changing them. */
#define FACTOR_UPDATE(T)                                                                      \
    static void update_targets_##T(const struct fctx_##T *c, uint32_t k, int64_t e0,         \
                                   int64_t e1) {                                              \
        for (int64_t e = e0; e < e1; ++e) {                                                   \
            uint32_t j = c->cidx[e];                                                          \
            uint32_t lo = c->cptr[j], hi = c->cptr[j + 1];                                    \
            while (lo < hi) {                                                                 \
                uint32_t mid = lo + (hi - lo) / 2;                                            \
                if (c->ridx[mid] < k) lo = mid + 1; else hi = mid;                            \
            }                                                                                 \
            T s = 0;                                                                          \
            uint32_t p = lo;                                                                  \
            if (p < c->cptr[j + 1] && c->ridx[p] == k) s = c->val[p++];                       \
            for (; p < c->cptr[j + 1]; ++p) {                                                 \
                T prod = c->tmp[c->ridx[p]] * s;                                              \
                c->val[p] = c->val[p] + (-prod);                                              \
            }                                                                                 \
        }                                                                                     \
    }

#define FACTOR_CTX(T)                                                                         \
    struct fctx_##T {                                                                         \
        uint32_t n;                                                                           \
        const uint32_t *cptr, *ridx, *diag, *rptr, *cidx, *rdiag;                             \
        int32_t num_lev;                                                                      \
        const int32_t *level_ptr, *level_idx;                                                 \
        T *val, *tmp, pert;                                                                   \
        int nthreads;                                                                         \
        pthread_barrier_t bar;                                                                \
    };

/* Pivot k's own work: GESP, L(:,k) /= d, scatter into the scratch column. */
#define FACTOR_PIVOT(T, FABS)                                                                 \
    static int pivot_##T(struct fctx_##T *c, uint32_t k) {                                    \
        uint32_t dk = c->diag[k], l0 = dk + 1, l1 = c->cptr[k + 1];                           \
        if (l1 == l0) return 0;                                                               \
        if (c->pert > 0 && FABS(c->val[dk]) < c->pert) c->val[dk] = c->pert;                  \
        for (uint32_t p = l0; p < l1; ++p) {                                                  \
            c->val[p] /= c->val[dk];                                                          \
            c->tmp[c->ridx[p]] = c->val[p];                                                   \
        }                                                                                     \
        return 1;                                                                             \
    }                                                                                         \
    static void clear_##T(struct fctx_##T *c, uint32_t k) {                                   \
        for (uint32_t p = c->diag[k] + 1; p < c->cptr[k + 1]; ++p) c->tmp[c->ridx[p]] = 0;   \
    }

#define WIDE_ROW 64 /* targets from which a row is split over the team */

/* Worker w of the team: all workers walk the same pivot sequence; worker 0
 * does the per-pivot serial work and the narrow rows alone, wide rows are
 * split between two barriers. */
#define FACTOR_WORKER(T)                                                                      \
    struct warg_##T { struct fctx_##T *c; int w; };                                           \
    static void *worker_##T(void *arg) {                                                      \
        struct fctx_##T *c = ((struct warg_##T *)arg)->c;                                     \
        const int w = ((struct warg_##T *)arg)->w, nt = c->nthreads;                          \
        for (int32_t lv = 0; lv < c->num_lev; ++lv) {                                         \
            for (int32_t q = c->level_ptr[lv]; q < c->level_ptr[lv + 1]; ++q) {               \
                uint32_t k = (uint32_t)c->level_idx[q];                                       \
                if (c->diag[k] + 1 == c->cptr[k + 1]) continue;                               \
                const int64_t e0 = (int64_t)c->rdiag[k] + 1, e1 = (int64_t)c->rptr[k + 1];    \
                if (e1 - e0 < WIDE_ROW || nt == 1) {                                          \
                    if (w == 0) {                                                             \
                        pivot_##T(c, k);                                                      \
                        update_targets_##T(c, k, e0, e1);                                     \
                        clear_##T(c, k);                                                      \
                    }                                                                         \
                    continue;                                                                 \
                }                                                                             \
                if (w == 0) pivot_##T(c, k);                                                  \
                pthread_barrier_wait(&c->bar);                                                \
                const int64_t len = e1 - e0;                                                  \
                update_targets_##T(c, k, e0 + len * w / nt, e0 + len * (w + 1) / nt);          \
                pthread_barrier_wait(&c->bar);                                                \
                if (w == 0) clear_##T(c, k);                                                  \
            }                                                                                 \
        }                                                                                     \
        return NULL;                                                                          \
    }

#define FACTOR_DEF(T, FABS, NAME)                                                             \
    FACTOR_CTX(T)                                                                             \
    FACTOR_UPDATE(T)                                                                          \
    FACTOR_PIVOT(T, FABS)                                                                     \
    FACTOR_WORKER(T)                                                                          \
    void NAME(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,   \
              const uint32_t *rptr, const uint32_t *cidx, const uint32_t *rdiag,              \
              int32_t num_lev, const int32_t *level_ptr, const int32_t *level_idx, T *val,    \
              T pert) {                                                                       \
        struct fctx_##T c = {n, cptr, ridx, diag, rptr, cidx, rdiag, num_lev, level_ptr,      \
                             level_idx, val, NULL, pert, oracle_threads()};                   \
        c.tmp = (T *)calloc(n ? n : 1, sizeof(T));                                            \
        pthread_t th[64];                                                                     \
        struct warg_##T args[64];                                                             \
        int started = 1;                                                                      \
        pthread_barrier_init(&c.bar, NULL, (unsigned)c.nthreads);                             \
        for (int w = 1; w < c.nthreads; ++w) {                                                \
            args[w].c = &c;                                                                   \
            args[w].w = w;                                                                    \
            if (pthread_create(&th[w], NULL, worker_##T, &args[w]) != 0) abort();             \
            ++started;                                                                        \
        }                                                                                     \
        args[0].c = &c;                                                                       \
        args[0].w = 0;                                                                        \
        worker_##T(&args[0]);                                                                 \
        for (int w = 1; w < started; ++w) pthread_join(th[w], NULL);                          \
        pthread_barrier_destroy(&c.bar);                                                      \
        free(c.tmp);                                                                          \
    }

/* Threads of the factorization team: GLU_ORACLE_THREADS, else the online
 * processors, at most 64. */
static int oracle_threads(void) {
    const char *e = getenv("GLU_ORACLE_THREADS");
    long v = e ? strtol(e, NULL, 10) : sysconf(_SC_NPROCESSORS_ONLN);
    if (v < 1) v = 1;
    if (v > 64) v = 64;
    return (int)v;
}

typedef float f32_t;
typedef double f64_t;
FACTOR_DEF(f32_t, fabsf, orc_factor_f32)
FACTOR_DEF(f64_t, fabs, orc_factor_f64)

float orc_pert(uint32_t n, const uint32_t *cptr, const float *val) {
    float norm = 0;
    for (uint32_t i = 0; i < n; ++i) {
        float t = 0;
        for (uint32_t p = cptr[i]; p < cptr[i + 1]; ++p) t += fabsf(val[p]);
        if (norm < t) norm = t;
    }
    return 3.45e-4f * norm;
}

void orc_solve_f32(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                   const float *val, const uint32_t *col_perm, const uint32_t *row_perm_inv,
                   const int32_t *pivot, const double *col_scale_perm, const double *row_scale,
                   int mc64, const float *rhs, float *x) {
    float *b = (float *)malloc(sizeof(float) * (n ? n : 1));
    for (uint32_t j = 0; j < n; ++j) {
        uint32_t p = (uint32_t)pivot[j];
        b[j] = mc64 ? (float)(rhs[col_perm[p]] * col_scale_perm[p]) : rhs[col_perm[p]];
    }
    for (uint32_t j = 0; j < n; ++j)
        for (uint32_t p = diag[j] + 1; p < cptr[j + 1]; ++p) b[ridx[p]] -= val[p] * b[j];
    for (int64_t jj = (int64_t)n - 1; jj >= 0; --jj) {
        b[jj] /= val[diag[jj]];
        for (uint32_t p = cptr[jj]; p < diag[jj]; ++p) b[ridx[p]] -= val[p] * b[jj];
    }
    for (uint32_t j = 0; j < n; ++j)
        x[j] = mc64 ? (float)(b[row_perm_inv[j]] * row_scale[j]) : b[row_perm_inv[j]];
    free(b);
}

#define SWEEPS_BODY(T)                                                                         \
    if (!trans) {                                                                              \
        for (uint32_t j = 0; j < n; ++j)                                                       \
            for (uint32_t p = diag[j] + 1; p < cptr[j + 1]; ++p) y[ridx[p]] -= val[p] * y[j]; \
        for (int64_t j = (int64_t)n - 1; j >= 0; --j) {                                        \
            y[j] /= val[diag[j]];                                                              \
            for (uint32_t p = cptr[j]; p < diag[j]; ++p) y[ridx[p]] -= val[p] * y[j];         \
        }                                                                                      \
    } else {                                                                                   \
        for (uint32_t j = 0; j < n; ++j) {                                                     \
            T acc = y[j];                                                                      \
            for (uint32_t p = cptr[j]; p < diag[j]; ++p) acc -= val[p] * y[ridx[p]];          \
            y[j] = acc / val[diag[j]];                                                         \
        }                                                                                      \
        for (int64_t j = (int64_t)n - 1; j >= 0; --j) {                                        \
            T acc = y[j];                                                                      \
            for (uint32_t p = diag[j] + 1; p < cptr[j + 1]; ++p) acc -= val[p] * y[ridx[p]];  \
            y[j] = acc;                                                                        \
        }                                                                                      \
    }

void orc_sweeps_f32(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                    const float *val, float *y, int trans) {
    SWEEPS_BODY(float)
}

void orc_sweeps_f64(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                    const double *val, double *y, int trans) {
    SWEEPS_BODY(double)
}

int32_t orc_leveling(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                     const uint32_t *rptr, const uint32_t *cidx, const uint32_t *rdiag,
                     int32_t *level_ptr, int32_t *level_idx) {
    int32_t *lev = (int32_t *)malloc(sizeof(int32_t) * (n ? n : 1));
    int32_t *size = (int32_t *)calloc(n + 1, sizeof(int32_t));
    int32_t num_lev = 0;
    for (uint32_t i = 0; i < n; ++i) {
        int32_t mx = -1;
        for (uint32_t p = cptr[i]; p < diag[i]; ++p) {
            uint32_t c = ridx[p];
            if (diag[c] + 1 != cptr[c + 1] && lev[c] > mx) mx = lev[c];
        }
        for (uint32_t e = rptr[i]; e < rdiag[i]; ++e)
            if (lev[cidx[e]] > mx) mx = lev[cidx[e]];
        lev[i] = mx + 1;
        size[lev[i]]++;
        if (lev[i] + 1 > num_lev) num_lev = lev[i] + 1;
    }
    level_ptr[0] = 0;
    for (int32_t l = 0; l < num_lev; ++l) level_ptr[l + 1] = level_ptr[l] + size[l];
    for (int32_t l = 0; l < num_lev; ++l) size[l] = level_ptr[l];
    for (uint32_t i = 0; i < n; ++i) level_idx[size[lev[i]]++] = (int32_t)i;
    free(lev);
    free(size);
    return num_lev;
}

static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}

uint32_t orc_fill_in(uint32_t n, const uint32_t *ap, const uint32_t *ai, uint32_t cap,
                     uint32_t *sym_c_ptr, uint32_t *sym_r_idx, uint32_t *l_col_ptr) {
    uint32_t *col = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1));
    uint32_t *tmp = (uint32_t *)malloc(sizeof(uint32_t) * (2 * n + 2));
    uint32_t nnz = 0;
    sym_c_ptr[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t len = ap[i + 1] - ap[i];
        memcpy(col, ai + ap[i], sizeof(uint32_t) * len);
        qsort(col, len, sizeof(uint32_t), cmp_u32);
        /* merge L patterns of the columns met in ascending order (symbolic.cc:22-37) */
        for (uint32_t j = 0; j < len; ++j) {
            uint32_t k = col[j];
            if (k >= i) break;
            const uint32_t *h = sym_r_idx + l_col_ptr[k], *e = sym_r_idx + sym_c_ptr[k + 1];
            uint32_t a = 0, t = 0;
            while (h < e || a < len) {
                if (a >= len || (h < e && *h < col[a]))
                    tmp[t++] = *h++;
                else if (h >= e || col[a] < *h)
                    tmp[t++] = col[a++];
                else {
                    tmp[t++] = *h++;
                    ++a;
                }
            }
            memcpy(col, tmp, sizeof(uint32_t) * t);
            len = t;
        }
        /* structural diagonal (symbolic.cc:39-43) */
        uint32_t d = 0;
        while (d < len && col[d] < i) ++d;
        if (d == len || col[d] != i) {
            memmove(col + d + 1, col + d, sizeof(uint32_t) * (len - d));
            col[d] = i;
            ++len;
        }
        if (nnz + len > cap) {
            free(col);
            free(tmp);
            return 0;
        }
        l_col_ptr[i] = nnz + d;
        memcpy(sym_r_idx + nnz, col, sizeof(uint32_t) * len);
        nnz += len;
        sym_c_ptr[i + 1] = nnz;
    }
    free(col);
    free(tmp);
    return nnz;
}
