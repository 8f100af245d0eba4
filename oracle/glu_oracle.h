/* Test infrastructure only: plain-C restatement of the reference's numeric
 * path (see glu_oracle.c).  All arrays are the Symbolic_Matrix arrays of
 * include/symbolic.h in the reference. */
#ifndef GLU_ORACLE_H
#define GLU_ORACLE_H
#include <stdint.h>

/* Right-looking column factorization in level order, FP32 / FP64.
 * pert > 0 enables the GESP replacement |d| < pert -> d = pert. */
void orc_factor_f32(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                    const uint32_t *rptr, const uint32_t *cidx, const uint32_t *rdiag,
                    int32_t num_lev, const int32_t *level_ptr, const int32_t *level_idx, float *val,
                    float pert);
void orc_factor_f64(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                    const uint32_t *rptr, const uint32_t *cidx, const uint32_t *rdiag,
                    int32_t num_lev, const int32_t *level_ptr, const int32_t *level_idx, double *val,
                    double pert);
/* pert of LUonDevice: 3.45e-4 * max column sum of |val| in FP32. */
float orc_pert(uint32_t n, const uint32_t *cptr, const float *val);
/* Symbolic_Matrix::solve: permute/scale, L sweep, U sweep, permute/scale. */
void orc_solve_f32(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                   const float *val, const uint32_t *col_perm, const uint32_t *row_perm_inv,
                   const int32_t *pivot, const double *col_scale_perm, const double *row_scale,
                   int mc64, const float *rhs, float *x);
/* Plain triangular sweeps on the permuted system (y overwritten).
 * trans = 0: L then U;  trans = 1: U^T then L^T.  FP64 versions take FP64 values. */
void orc_sweeps_f32(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                    const float *val, float *y, int trans);
void orc_sweeps_f64(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                    const double *val, double *y, int trans);
/* Symbolic_Matrix::leveling; returns num_lev, fills level_ptr[num_lev+1], level_idx[n]. */
int32_t orc_leveling(uint32_t n, const uint32_t *cptr, const uint32_t *ridx, const uint32_t *diag,
                     const uint32_t *rptr, const uint32_t *cidx, const uint32_t *rdiag,
                     int32_t *level_ptr, int32_t *level_idx);
/* Symbolic_Matrix::fill_in by sorted-list merging; returns nnz or 0 if cap is exceeded. */
uint32_t orc_fill_in(uint32_t n, const uint32_t *ap, const uint32_t *ai, uint32_t cap,
                     uint32_t *sym_c_ptr, uint32_t *sym_r_idx, uint32_t *l_col_ptr);
#endif
