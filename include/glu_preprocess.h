/*
 * glu_preprocess.h -- NICSLU static pivoting, scaling and ordering.
 *
 * Plain C wrapper around the third-party NICSLU library that the reference
 * bundles (src/nicslu, LGPL-2.1), linked unmodified.  It runs the same
 * sequence as the reference's preprocess_from_arrays
 * (src/preprocess/preprocess_arrays.c:18-98): NicsLU_Initialize,
 * NicsLU_CreateMatrix, column mode (cfgi[0]=1), cfgf[1]=0, NicsLU_Analyze
 * (MC64 matching + scaling, AMD ordering), then dumps the permuted, scaled
 * CSC matrix with identity pivots as my_DumpA does
 * (src/preprocess/preprocess.c:8-79).
 *
 * In addition it returns, for every entry q of the input matrix, its position
 * in the dumped matrix and the FP64 factor that NICSLU's MC64 scaling applied
 * to it (nicslu_mc64scale.c:8-46), so that new values of the same pattern can
 * be placed without re-running NICSLU:  dumped_ax[pos[q]] == ax[q] * scale[q]
 * bit for bit.
 */
#ifndef GLU_PREPROCESS_H
#define GLU_PREPROCESS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct glu_pre_s *glu_pre_t;

/* Returns 0 or a NICSLU error code (nicslu.h:11-28), e.g. -5 for a
 * structurally singular matrix, -7 for an invalid one, -8 for duplicates. */
int glu_pre_analyze(uint32_t n, uint32_t nnz, const double *ax, const uint32_t *ai,
                    const uint32_t *ap, glu_pre_t *out);
uint32_t glu_pre_n(glu_pre_t p);
uint32_t glu_pre_nnz(glu_pre_t p);
/* The preprocessed CSC matrix (ax[nnz], ai[nnz], ap[n+1]). */
void glu_pre_matrix(glu_pre_t p, double *ax, uint32_t *ai, uint32_t *ap);
/* SNicsLU col_perm, row_perm_inv, pivot, col_scale_perm, row_scale, cfgi[1]:
 * the arrays Symbolic_Matrix::solve reads (src/symbolic.cc:207-213). */
void glu_pre_transform(glu_pre_t p, uint32_t *col_perm, uint32_t *row_perm_inv, int32_t *pivot,
                       double *col_scale_perm, double *row_scale, int *mc64_scale);
/* Position in the preprocessed matrix and scale factor of every input entry. */
void glu_pre_source_map(glu_pre_t p, uint32_t *pos, double *scale);
void glu_pre_destroy(glu_pre_t p);

/* Reads a Matrix Market file with NICSLU's reader (triplets stored column by
 * column, as lu_cmd requires, src/nicslu/util/nicslu_readfile.c:98-228) into
 * malloc'd CSC arrays; free them with glu_pre_free.  Returns 0 or the NICSLU
 * error code (-4 cannot open, -7 invalid). */
int glu_pre_read_mtx(const char *file, uint32_t *n, uint32_t *nnz, double **ax, uint32_t **ai,
                     uint32_t **ap);
void glu_pre_free(void *ptr);

#ifdef __cplusplus
}
#endif

#endif /* GLU_PREPROCESS_H */
