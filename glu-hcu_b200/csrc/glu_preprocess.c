/* NICSLU preprocessing for the drop-in surface (see include/glu_preprocess.h). */
#include "glu_preprocess.h"

#include <stdlib.h>
#include <string.h>

#include "nicslu.h"

struct glu_pre_s {
    SNicsLU s;
    int created;
    uint32_t n, nnz;
    double *ax;
    uint32_t *ai, *ap;
    uint32_t *pos;
    double *scale;
};

static void release(struct glu_pre_s *p) {
    if (!p) return;
    if (p->created) NicsLU_Destroy(&p->s);
    free(p->ax);
    free(p->ai);
    free(p->ap);
    free(p->pos);
    free(p->scale);
    free(p);
}

int glu_pre_analyze(uint32_t n, uint32_t nnz, const double *ax, const uint32_t *ai,
                    const uint32_t *ap, glu_pre_t *out) {
    struct glu_pre_s *p;
    int ret;
    uint32_t i, c, q, k;
    if (!out || !ax || !ai || !ap) return NICSLU_ARGUMENT_ERROR;
    *out = NULL;
    if (n == 0 || nnz == 0) return NICSLU_MATRIX_INVALID;
    p = (struct glu_pre_s *)calloc(1, sizeof(*p));
    if (!p) return NICSLU_MEMORY_OVERFLOW;
    NicsLU_Initialize(&p->s);
    p->created = 1;
    /* NicsLU_CreateMatrix copies its inputs (nicslu_matrix.c:44-46) */
    ret = NicsLU_CreateMatrix(&p->s, n, nnz, (double *)ax, (uint32_t *)ai, (uint32_t *)ap);
    if (ret != NICS_OK) goto fail;
    p->s.cfgi[0] = 1; /* column (CSC) mode, as GLU configures it */
    p->s.cfgf[1] = 0;
    ret = NicsLU_Analyze(&p->s);
    if (ret != NICS_OK) goto fail;

    p->n = n;
    p->nnz = nnz;
    p->ax = (double *)malloc(sizeof(double) * nnz);
    p->ai = (uint32_t *)malloc(sizeof(uint32_t) * nnz);
    p->ap = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1));
    p->pos = (uint32_t *)malloc(sizeof(uint32_t) * nnz);
    p->scale = (double *)malloc(sizeof(double) * nnz);
    if (!p->ax || !p->ai || !p->ap || !p->pos || !p->scale) {
        ret = NICSLU_MEMORY_OVERFLOW;
        goto fail;
    }
    /* identity pivots, then the permuted copy: new column i holds NICSLU's
       major index row_perm[i] with its (already permuted) minor indices */
    for (i = 0; i < n; ++i) {
        p->s.pivot[i] = (int__t)i;
        p->s.pivot_inv[i] = (int__t)i;
    }
    p->ap[0] = 0;
    k = 0;
    for (i = 0; i < n; ++i) {
        c = p->s.row_perm[i];
        for (q = p->s.ap[c]; q < p->s.ap[c + 1]; ++q) {
            p->ax[k] = p->s.ax[q];
            p->ai[k] = p->s.ai[q];
            p->pos[q] = k;
            /* MC64 scaling as applied in place by NicsLU_Analyze:
               ax[q] *= row_scale[c] * col_scale_perm[ai[q]] */
            p->scale[q] = p->s.cfgi[1] ? p->s.row_scale[c] * p->s.col_scale_perm[p->s.ai[q]] : 1.0;
            ++k;
        }
        p->ap[i + 1] = k;
    }
    *out = p;
    return 0;
fail:
    release(p);
    return ret;
}

uint32_t glu_pre_n(glu_pre_t p) { return p ? p->n : 0; }
uint32_t glu_pre_nnz(glu_pre_t p) { return p ? p->nnz : 0; }

void glu_pre_matrix(glu_pre_t p, double *ax, uint32_t *ai, uint32_t *ap) {
    if (ax) memcpy(ax, p->ax, sizeof(double) * p->nnz);
    if (ai) memcpy(ai, p->ai, sizeof(uint32_t) * p->nnz);
    if (ap) memcpy(ap, p->ap, sizeof(uint32_t) * (p->n + 1));
}

void glu_pre_transform(glu_pre_t p, uint32_t *col_perm, uint32_t *row_perm_inv, int32_t *pivot,
                       double *col_scale_perm, double *row_scale, int *mc64_scale) {
    uint32_t n = p->n;
    if (col_perm) memcpy(col_perm, p->s.col_perm, sizeof(uint32_t) * n);
    if (row_perm_inv) memcpy(row_perm_inv, p->s.row_perm_inv, sizeof(uint32_t) * n);
    if (pivot) memcpy(pivot, p->s.pivot, sizeof(int32_t) * n);
    if (col_scale_perm) memcpy(col_scale_perm, p->s.col_scale_perm, sizeof(double) * n);
    if (row_scale) memcpy(row_scale, p->s.row_scale, sizeof(double) * n);
    if (mc64_scale) *mc64_scale = (int)p->s.cfgi[1];
}

void glu_pre_source_map(glu_pre_t p, uint32_t *pos, double *scale) {
    if (pos) memcpy(pos, p->pos, sizeof(uint32_t) * p->nnz);
    if (scale) memcpy(scale, p->scale, sizeof(double) * p->nnz);
}

void glu_pre_destroy(glu_pre_t p) { release(p); }

int NicsLU_ReadTripletColumnToSparse(char *file, uint__t *n, uint__t *nnz, real__t **ax, uint__t **ai,
                                     uint__t **ap);

int glu_pre_read_mtx(const char *file, uint32_t *n, uint32_t *nnz, double **ax, uint32_t **ai,
                     uint32_t **ap) {
    if (!file || !n || !nnz || !ax || !ai || !ap) return NICSLU_ARGUMENT_ERROR;
    *ax = NULL;
    *ai = NULL;
    *ap = NULL;
    return NicsLU_ReadTripletColumnToSparse((char *)file, n, nnz, ax, ai, ap);
}

void glu_pre_free(void *ptr) { free(ptr); }
