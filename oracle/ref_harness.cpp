// Test infrastructure only: a C-ABI driver around the reference's own CPU code
// (the bundled NICSLU library, the reference preprocessing wrapper and
// Symbolic_Matrix from src/symbolic.cc), compiled from the reference tree by
// oracle/Makefile into oracle/_ref/.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it; the product never does.
//
// Call sequences follow the reference:
//   ref_analyze   -> src/preprocess/preprocess_arrays.c:18-98 (NicsLU_Initialize,
//                    NicsLU_CreateMatrix, cfgi[0]=1, cfgf[1]=0, NicsLU_Analyze,
//                    my_DumpA).  preprocess_arrays.c itself does not compile
//                    (it passes 7 arguments to the 6-parameter
//                    NicsLU_CreateMatrix), so the sequence is restated here.
//   ref_symbolic  -> src/lu_cmd.cpp:90-108 / src/glu_binding.cpp:105-109
//                    (fill_in, csr, predictLU, leveling).
//   ref_solve     -> src/symbolic.cc:200-251 (Symbolic_Matrix::solve).
//   ref_nicslu_*  -> src/nicslu/demo/demop_time.c (multi-threaded NICSLU
//                    factor / refactor / solve), the CPU baseline.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <vector>

#include "nicslu.h"
#include "preprocess.h"
#include "symbolic.h"

namespace {
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};
// A stream in the bad state skips all formatting, so the reference's progress
// messages never reach the locale machinery of the statically linked C++
// runtime (which is not set up when this library is loaded from Python).
std::ostream &null_stream() {
    static NullBuf buf;
    static std::ostream os(&buf);
    os.setstate(std::ios::badbit);
    return os;
}
}  // namespace

struct RefCtx {
    SNicsLU *nicslu = nullptr;
    bool analyzed = false;
    unsigned n = 0;
    unsigned nnzA = 0;
    double *ax = nullptr;
    unsigned *ai = nullptr;
    unsigned *ap = nullptr;
    Symbolic_Matrix *sym = nullptr;
};

extern "C" {

RefCtx *ref_create(void) { return new RefCtx(); }

void ref_destroy(RefCtx *c) {
    if (!c) return;
    delete c->sym;
    if (c->nicslu) {
        if (c->analyzed) NicsLU_Destroy(c->nicslu);
        free(c->nicslu);
    }
    free(c->ax);
    free(c->ai);
    free(c->ap);
    delete c;
}

// NICSLU preprocessing of an n x n CSC matrix; returns 0 or the NICSLU error.
int ref_analyze(RefCtx *c, unsigned n, unsigned nnz, const double *ax,
                const unsigned *ai, const unsigned *ap) {
    c->nicslu = static_cast<SNicsLU *>(malloc(sizeof(SNicsLU)));
    NicsLU_Initialize(c->nicslu);
    // NicsLU_CreateMatrix copies its inputs (nicslu_matrix.c:44-46).
    int ret = NicsLU_CreateMatrix(c->nicslu, n, nnz, const_cast<double *>(ax),
                                  const_cast<unsigned *>(ai), const_cast<unsigned *>(ap));
    c->analyzed = true;
    if (ret != NICS_OK) return ret;
    c->nicslu->cfgi[0] = 1;
    c->nicslu->cfgf[1] = 0;
    ret = NicsLU_Analyze(c->nicslu);
    if (ret != NICS_OK) return ret;
    ret = my_DumpA(c->nicslu, &c->ax, &c->ai, &c->ap);
    if (ret != 0) return ret;
    c->n = c->nicslu->n;
    c->nnzA = c->nicslu->nnz;
    return 0;
}

unsigned ref_n(RefCtx *c) { return c->n; }
unsigned ref_nnzA(RefCtx *c) { return c->nnzA; }

void ref_get_dumped(RefCtx *c, double *ax, unsigned *ai, unsigned *ap) {
    memcpy(ax, c->ax, sizeof(double) * c->nnzA);
    memcpy(ai, c->ai, sizeof(unsigned) * c->nnzA);
    memcpy(ap, c->ap, sizeof(unsigned) * (c->n + 1));
}

void ref_get_perm(RefCtx *c, unsigned *row_perm, unsigned *row_perm_inv,
                  unsigned *col_perm, unsigned *col_perm_inv, double *row_scale,
                  double *col_scale_perm, int *pivot, int *pivot_inv,
                  unsigned *mc64_flag) {
    SNicsLU *s = c->nicslu;
    unsigned n = c->n;
    memcpy(row_perm, s->row_perm, sizeof(unsigned) * n);
    memcpy(row_perm_inv, s->row_perm_inv, sizeof(unsigned) * n);
    memcpy(col_perm, s->col_perm, sizeof(unsigned) * n);
    memcpy(col_perm_inv, s->col_perm_inv, sizeof(unsigned) * n);
    memcpy(row_scale, s->row_scale, sizeof(double) * n);
    memcpy(col_scale_perm, s->col_scale_perm, sizeof(double) * n);
    memcpy(pivot, s->pivot, sizeof(int) * n);
    memcpy(pivot_inv, s->pivot_inv, sizeof(int) * n);
    *mc64_flag = s->cfgi[1];
}

// Load an already-preprocessed CSC (for symbolic-only checks without NICSLU).
void ref_set_csc(RefCtx *c, unsigned n, unsigned nnz, const double *ax,
                 const unsigned *ai, const unsigned *ap) {
    c->n = n;
    c->nnzA = nnz;
    c->ax = static_cast<double *>(malloc(sizeof(double) * (nnz ? nnz : 1)));
    c->ai = static_cast<unsigned *>(malloc(sizeof(unsigned) * (nnz ? nnz : 1)));
    c->ap = static_cast<unsigned *>(malloc(sizeof(unsigned) * (n + 1)));
    memcpy(c->ax, ax, sizeof(double) * nnz);
    memcpy(c->ai, ai, sizeof(unsigned) * nnz);
    memcpy(c->ap, ap, sizeof(unsigned) * (n + 1));
}

// The reference symbolic phase on the dumped (or loaded) CSC.
int ref_symbolic(RefCtx *c) {
    delete c->sym;
    c->sym = new Symbolic_Matrix(c->n, null_stream(), null_stream());
    c->sym->fill_in(c->ai, c->ap);
    c->sym->csr();
    c->sym->predictLU(c->ai, c->ap, c->ax);
    c->sym->leveling();
    return 0;
}

unsigned ref_lu_nnz(RefCtx *c) { return c->sym->nnz; }
int ref_num_lev(RefCtx *c) { return c->sym->num_lev; }

void ref_get_symbolic(RefCtx *c, unsigned *sym_c_ptr, unsigned *sym_r_idx,
                      unsigned *l_col_ptr, unsigned *csr_r_ptr, unsigned *csr_c_idx,
                      unsigned *csr_diag_ptr, float *val, int *level_ptr,
                      int *level_idx) {
    Symbolic_Matrix *s = c->sym;
    unsigned n = s->n, nnz = s->nnz;
    memcpy(sym_c_ptr, s->sym_c_ptr.data(), sizeof(unsigned) * (n + 1));
    memcpy(sym_r_idx, s->sym_r_idx.data(), sizeof(unsigned) * nnz);
    memcpy(l_col_ptr, s->l_col_ptr.data(), sizeof(unsigned) * n);
    memcpy(csr_r_ptr, s->csr_r_ptr.data(), sizeof(unsigned) * (n + 1));
    memcpy(csr_c_idx, s->csr_c_idx.data(), sizeof(unsigned) * nnz);
    memcpy(csr_diag_ptr, s->csr_diag_ptr.data(), sizeof(unsigned) * n);
    memcpy(val, s->val.data(), sizeof(float) * nnz);
    memcpy(level_ptr, s->level_ptr.data(), sizeof(int) * (s->num_lev + 1));
    memcpy(level_idx, s->level_idx.data(), sizeof(int) * n);
}

// Symbolic_Matrix::solve with the given factor values (needs ref_analyze).
void ref_solve(RefCtx *c, const float *luval, const float *rhs, float *x) {
    Symbolic_Matrix *s = c->sym;
    std::vector<float> saved(s->val);
    memcpy(s->val.data(), luval, sizeof(float) * s->nnz);
    std::vector<float> b(rhs, rhs + s->n);
    std::vector<float> out = s->solve(c->nicslu, b);
    memcpy(x, out.data(), sizeof(float) * s->n);
    s->val.swap(saved);
}

// Load a Symbolic_Matrix from arrays (pattern, CSR, values, levels) without
// running the reference's symbolic phase, e.g. to time LUonDevice on a
// pattern whose reference fill_in would take minutes.  The arrays must be the
// ones the reference's symbolic phase produces (the product's symbolic phase
// produces them bit for bit).
void ref_load_pattern(RefCtx *c, unsigned n, unsigned nnz, const unsigned *sym_c_ptr,
                      const unsigned *sym_r_idx, const unsigned *l_col_ptr, const unsigned *csr_r_ptr,
                      const unsigned *csr_c_idx, const unsigned *csr_diag_ptr, const float *val,
                      int num_lev, const int *level_ptr, const int *level_idx) {
    delete c->sym;
    c->n = n;
    Symbolic_Matrix *s = new Symbolic_Matrix(n, null_stream(), null_stream());
    s->nnz = nnz;
    s->num_lev = num_lev;
    s->sym_c_ptr.assign(sym_c_ptr, sym_c_ptr + n + 1);
    s->sym_r_idx.assign(sym_r_idx, sym_r_idx + nnz);
    s->l_col_ptr.assign(l_col_ptr, l_col_ptr + n);
    s->csr_r_ptr.assign(csr_r_ptr, csr_r_ptr + n + 1);
    s->csr_c_idx.assign(csr_c_idx, csr_c_idx + nnz);
    s->csr_diag_ptr.assign(csr_diag_ptr, csr_diag_ptr + n);
    s->val.assign(val, val + nnz);
    s->level_ptr.assign(level_ptr, level_ptr + num_lev + 1);
    s->level_idx.assign(level_idx, level_idx + n);
    c->sym = s;
}

// Replace the factor values held by the Symbolic_Matrix (used by the GPU
// reference driver, which factors them in place).
void ref_set_val(RefCtx *c, const float *val) {
    memcpy(c->sym->val.data(), val, sizeof(float) * c->sym->nnz);
}
void ref_get_val(RefCtx *c, float *val) {
    memcpy(val, c->sym->val.data(), sizeof(float) * c->sym->nnz);
}
Symbolic_Matrix *ref_symbolic_matrix(RefCtx *c) { return c->sym; }

// ---------------------------------------------------------------------------
// NICSLU CPU baseline (src/nicslu/demo/demop_time.c sequence, with the thread
// count passed explicitly; column mode as GLU configures it).
struct RefNics {
    SNicsLU *s;
    unsigned n;
};

void *ref_nicslu_create(unsigned n, unsigned nnz, const double *ax, const unsigned *ai,
                        const unsigned *ap, unsigned threads, double *t_analyze_factor,
                        int *status) {
    RefNics *h = new RefNics();
    h->n = n;
    h->s = static_cast<SNicsLU *>(malloc(sizeof(SNicsLU)));
    NicsLU_Initialize(h->s);
    int ret = NicsLU_CreateMatrix(h->s, n, nnz, const_cast<double *>(ax),
                                  const_cast<unsigned *>(ai), const_cast<unsigned *>(ap));
    if (ret == NICS_OK) {
        h->s->cfgi[0] = 1;
        ret = NicsLU_Analyze(h->s);
    }
    t_analyze_factor[0] = h->s->stat[0];
    if (ret == NICS_OK && threads > 1) {
        NicsLU_CreateScheduler(h->s);
        ret = NicsLU_CreateThreads(h->s, threads, 1);
        if (ret == NICS_OK) ret = NicsLU_Factorize_MT(h->s);
    } else if (ret == NICS_OK) {
        ret = NicsLU_Factorize(h->s);
    }
    t_analyze_factor[1] = h->s->stat[1];
    *status = ret;
    return h;
}

unsigned ref_nicslu_threads(void *hp) {
    RefNics *h = static_cast<RefNics *>(hp);
    return h->s->cfgi[5];
}

int ref_nicslu_refactor(void *hp, const double *ax, unsigned threads, double *t) {
    RefNics *h = static_cast<RefNics *>(hp);
    int ret = threads > 1 ? NicsLU_ReFactorize_MT(h->s, const_cast<double *>(ax))
                          : NicsLU_ReFactorize(h->s, const_cast<double *>(ax));
    *t = h->s->stat[2];
    return ret;
}

int ref_nicslu_solve(void *hp, double *rhs_inout, double *t) {
    RefNics *h = static_cast<RefNics *>(hp);
    int ret = NicsLU_Solve(h->s, rhs_inout);
    *t = h->s->stat[3];
    return ret;
}

int ref_nicslu_refine(void *hp, double *x, const double *b, double eps, unsigned maxiter) {
    RefNics *h = static_cast<RefNics *>(hp);
    return NicsLU_Refine(h->s, x, const_cast<double *>(b), eps, maxiter);
}

size_t ref_nicslu_lu_nnz(void *hp) { return static_cast<RefNics *>(hp)->s->lu_nnz; }

void ref_nicslu_destroy(void *hp) {
    RefNics *h = static_cast<RefNics *>(hp);
    NicsLU_Destroy(h->s);
    free(h->s);
    delete h;
}

}  // extern "C"
