/*
 * glu_b200.h -- C ABI of the B200 GLU sparse LU engine.
 *
 * Plain C: opaque handles, plain pointers and sizes, status codes, no
 * exceptions across the boundary and no CUDA or torch types (a stream is passed
 * as a void* holding a cudaStream_t; NULL is the legacy default stream).
 *
 * The reference's numeric path is one C++ call,
 *     void LUonDevice(Symbolic_Matrix&, ostream& out, ostream& err, bool PERTURB)
 * (include/numeric.h:6, src/numeric.cu:347-639), fed by Symbolic_Matrix's
 * fill_in / csr / predictLU / leveling (src/symbolic.cc:11-151) and followed by
 * the CPU solve Symbolic_Matrix::solve (src/symbolic.cc:200-251).  The entry
 * points below replace those calls one for one; a header-only C++ shim in
 * glu_luondevice.hpp re-provides LUonDevice on top of them.
 *
 * Numerics: factors and the plain solves are FP32 as in the reference
 * (include/type.h:3); glu_solve_refined adds FP64 residuals on the original
 * matrix and an FP64 solution update.
 *
 * Threading: handles are independent; a handle must not be used by two threads
 * at once.  The last error message is thread-local.
 */
#ifndef GLU_B200_H
#define GLU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GLU_OK = 0,
    GLU_ERR_ARG = -1,           /* invalid argument or inconsistent arrays      */
    GLU_ERR_CUDA = -2,          /* a CUDA runtime call failed                   */
    GLU_ERR_NOMEM = -3,         /* host or device allocation failed             */
    GLU_ERR_SINGULAR = -4,      /* zero or non-finite pivot met                 */
    GLU_ERR_TIMEOUT = -5,       /* a bounded device-side wait ran out           */
    GLU_ERR_STATE = -6,         /* call out of order (e.g. solve before factor) */
    GLU_ERR_NOT_CONVERGED = -7, /* refinement stopped above its tolerance       */
    GLU_ERR_NO_DEVICE = -8,     /* no CUDA device                               */
    GLU_ERR_UNSUPPORTED = -9    /* size or mode outside what the build handles  */
} glu_status;

typedef enum { GLU_HOST = 0, GLU_DEVICE = 1 } glu_memory;

typedef struct glu_symbolic_s *glu_symbolic_t;
typedef struct glu_handle_s *glu_handle_t;
typedef void *glu_stream;

/* Message of the last failing call on this thread ("" if none). */
const char *glu_last_error(void);
/* Library version string. */
const char *glu_version(void);

/* ---------------------------------------------------------------- symbolic --
 * Fill pattern of L+U, its CSR transpose and the slot map that places A's
 * values into the pattern.  Replaces Symbolic_Matrix::fill_in / csr /
 * predictLU (src/symbolic.cc:11-103); the arrays are identical to the
 * reference's.  A is the preprocessed n x n CSC matrix (ap[n+1], ai[nnz_a]),
 * the output of preprocess()/my_DumpA (src/preprocess/preprocess.c:8-79).
 */
glu_status glu_symbolic_analyze(uint32_t n, uint32_t nnz_a, const uint32_t *ap,
                                const uint32_t *ai, glu_symbolic_t *out);
glu_status glu_symbolic_sizes(glu_symbolic_t s, uint32_t *n, uint32_t *nnz_lu);
/* Copies out sym_c_ptr[n+1], sym_r_idx[nnz], l_col_ptr[n], csr_r_ptr[n+1],
 * csr_c_idx[nnz], csr_diag_ptr[n] (include/symbolic.h:15-21).  NULL skips. */
glu_status glu_symbolic_export(glu_symbolic_t s, uint32_t *sym_c_ptr, uint32_t *sym_r_idx,
                               uint32_t *l_col_ptr, uint32_t *csr_r_ptr,
                               uint32_t *csr_c_idx, uint32_t *csr_diag_ptr);
/* LU position of every entry of A (a_slot[nnz_a]). */
glu_status glu_symbolic_slots(glu_symbolic_t s, uint32_t *a_slot);
/* predictLU (src/symbolic.cc:82-103): FP32 LU values from A's FP64 values. */
glu_status glu_predict_lu(glu_symbolic_t s, const double *ax, float *val);
void glu_symbolic_destroy(glu_symbolic_t s);

/* ------------------------------------------------------------------ handle --
 * A device-resident pattern with `batch` value sets of the same pattern.
 * Creation uploads the pattern, builds the level sets on the GPU (replacing
 * Symbolic_Matrix::leveling, src/symbolic.cc:106-151, bit-exact) and plans the
 * factorization schedule.  Replaces the allocation and copy-in half of
 * LUonDevice (src/numeric.cu:435-488), done once per pattern instead of once
 * per call.
 */
glu_status glu_create(glu_symbolic_t s, int device, uint32_t batch, glu_handle_t *out);
/* Same from raw Symbolic_Matrix arrays (for the LUonDevice shim). */
glu_status glu_create_from_pattern(int device, uint32_t n, uint32_t nnz,
                                   const uint32_t *sym_c_ptr, const uint32_t *sym_r_idx,
                                   const uint32_t *l_col_ptr, const uint32_t *csr_r_ptr,
                                   const uint32_t *csr_c_idx, const uint32_t *csr_diag_ptr,
                                   uint32_t batch, glu_handle_t *out);
void glu_destroy(glu_handle_t h);

/* Level sets built on the GPU: num_lev, level_ptr[num_lev+1], level_idx[n]
 * (Symbolic_Matrix::num_lev / level_ptr / level_idx).  NULL arrays skip. */
glu_status glu_levels(glu_handle_t h, int32_t *num_lev, int32_t *level_ptr, int32_t *level_idx);

/* Permutations and scalings applied by the solves, with the meaning they have
 * in Symbolic_Matrix::solve (src/symbolic.cc:207-247): col_perm = SNicsLU
 * col_perm, row_perm_inv = SNicsLU row_perm_inv, pivot = SNicsLU pivot,
 * col_scale_perm / row_scale = SNicsLU col_scale_perm / row_scale, mc64_scale =
 * SNicsLU cfgi[1].  Without this call the solves work on the preprocessed
 * system itself (identity permutations, no scaling). */
glu_status glu_set_transform(glu_handle_t h, const uint32_t *col_perm, const uint32_t *row_perm_inv,
                             const int32_t *pivot, const double *col_scale_perm,
                             const double *row_scale, int mc64_scale);

/* The original (unpreprocessed) matrix A0 in CSC (src_ap[n+1], src_ai[nnz_src])
 * and, for each of its entries, the LU slot and the FP64 factor that maps it
 * into the preprocessed, scaled system: LU[src_slot[q]] = (float)(ax0[q] *
 * src_scale[q]).  Enables glu_load_source_values (refactorization with new
 * values) and glu_solve_refined (FP64 residuals on A0). */
glu_status glu_set_source(glu_handle_t h, uint32_t nnz_src, const uint32_t *src_ap,
                          const uint32_t *src_ai, const uint32_t *src_slot,
                          const double *src_scale);

/* ------------------------------------------------------------------ values --
 * Value sets [first, first+count) of the batch, each nnz_lu FP32 values in the
 * layout of Symbolic_Matrix::val, contiguous one set after another. */
glu_status glu_load_lu_values(glu_handle_t h, uint32_t first, uint32_t count, const float *val,
                              glu_memory where, glu_stream stream);
glu_status glu_store_lu_values(glu_handle_t h, uint32_t first, uint32_t count, float *val,
                               glu_memory where, glu_stream stream);
/* New values of A0 (nnz_src FP64 each, one set after another) placed into the
 * LU layout on the GPU; they are kept for the FP64 residuals of refinement. */
glu_status glu_load_source_values(glu_handle_t h, uint32_t first, uint32_t count,
                                  const double *ax0, glu_memory where, glu_stream stream);

/* --------------------------------------------------------------- factorize --
 * In-place FP32 LU (no pivoting) of value sets [first, first+count): the
 * level-scheduled right-looking column algorithm of RL / RL_onecol_*
 * (src/numeric.cu:10-345).  perturb != 0 is the GESP mode of RL_perturb
 * (numeric.cu:105-202, 490-506): pert = 3.45e-4 * ||A||_1 (FP32, of each value
 * set) and a pivot with |d| < pert is replaced by +pert.  Without perturbation
 * a zero or non-finite pivot returns GLU_ERR_SINGULAR (after the whole batch
 * is factored); the reference has no such check. */
glu_status glu_factor(glu_handle_t h, uint32_t first, uint32_t count, int perturb,
                      glu_stream stream);

/* ------------------------------------------------------------------- solve --
 * FP32 solve of A x = b with value set `inst` for nrhs right-hand sides
 * (b and x: nrhs x n, one right-hand side after another).  Same arithmetic
 * sequence as Symbolic_Matrix::solve (src/symbolic.cc:200-251): permute and
 * scale b, unit-L sweep, U sweep, permute and scale back.  x may alias b. */
glu_status glu_solve(glu_handle_t h, uint32_t inst, uint32_t nrhs, const float *b, float *x,
                     glu_memory where, glu_stream stream);
/* glu_solve for callers that cannot allocate device memory.  No counterpart in
 * the reference.  glu_solve allocates its working vectors on first use; some
 * hosts may not call cudaMalloc while they run: a simulator whose device
 * memory is owned and pooled by a framework (a second allocator would fight
 * it for memory), or a real-time loop that must not stall in the allocator.
 * This variant takes the working vectors from a fixed array of about 8 MiB
 * that the library keeps in the memory of every GPU that loads it, for the
 * life of the process, and calls no allocating routine.  b and x are device
 * pointers (nrhs x n FP32), the handle must be factored.  Limits: n * nrhs <=
 * 1,048,576 and a dense trailing block of order <= 262,080; larger problems
 * return GLU_ERR_UNSUPPORTED before touching the GPU.  The first call on a
 * device looks up that array's device address (once per device), so make the
 * first call before any stream capture.  Like glu_solve, the call waits for
 * its stream to finish before it returns (it reads the solve's status).  All
 * calls share the one array and it keeps the last call's contents: calls that
 * overlap on the GPU (other streams, other handles, other host threads) race
 * and must be serialized by the caller. */
glu_status glu_solve_noalloc(glu_handle_t h, uint32_t inst, uint32_t nrhs, const float *b, float *x,
                             glu_stream stream);
/* FP32 solve of A^T x = b with the same factors (U^T then L^T sweeps). */
glu_status glu_solve_transposed(glu_handle_t h, uint32_t inst, uint32_t nrhs, const float *b,
                                float *x, glu_memory where, glu_stream stream);

typedef struct {
    uint32_t iterations;     /* refinement steps taken (max over the systems)   */
    double residual;         /* max over systems of ||b - A0 x||_2 / ||b||_2    */
    double residual_inf;     /* max over systems of ||b - A0 x||_inf / ||b||_inf */
} glu_refine_stats;

/* Mixed-precision iterative refinement for value sets [first, first+count),
 * nrhs right-hand sides each (b, x: count x nrhs x n FP64): x = solve(b), then
 * repeat r = b - A0 x (FP64 SpMV on the original matrix), x += solve(r) until
 * ||r||_2 / ||b||_2 <= tol or maxit steps.  transposed != 0 solves A0^T x = b.
 * Needs glu_set_source and glu_load_source_values.  Returns
 * GLU_ERR_NOT_CONVERGED (with x and stats filled) when tol is not met. */
glu_status glu_solve_refined(glu_handle_t h, uint32_t first, uint32_t count, uint32_t nrhs,
                             const double *b, double *x, double tol, uint32_t maxit,
                             int transposed, glu_memory where, glu_refine_stats *stats,
                             glu_stream stream);

/* -------------------------------------------------- many systems at once --
 * Independent systems of different patterns and sizes (one handle each),
 * factored or solved together: every system's kernels go to streams[i %
 * nstreams] (nstreams 0: the legacy default stream) and the host waits once
 * per call (factorization) or once per refinement step (solve) for all of
 * them, instead of once per system.  No counterpart in the reference.
 * glu_factor_many factors every value set of each handle.
 * glu_solve_refined_many: system i solves its nrhs[i] right-hand sides per
 * value set, b[i] / x[i] laid out as in glu_solve_refined; refinement steps of
 * all systems run in lockstep, a system stops when its own residual meets
 * tol.  stats (nullable) receives one record per system.  The first failing
 * system's status is returned, its index in the message. */
glu_status glu_factor_many(uint32_t count, const glu_handle_t *handles, int perturb, const glu_stream *streams,
                           uint32_t nstreams);
glu_status glu_solve_refined_many(uint32_t count, const glu_handle_t *handles, const uint32_t *nrhs,
                                  const double *const *b, double *const *x, double tol, uint32_t maxit,
                                  glu_memory where, glu_refine_stats *stats, const glu_stream *streams,
                                  uint32_t nstreams);

/* ------------------------------------------------------------------- stats --*/
typedef struct {
    uint32_t n;
    uint32_t nnz_lu;
    uint32_t batch;
    int32_t num_lev;           /* levels of the reference level schedule          */
    uint32_t wide_levels;      /* levels run as their own launch                  */
    uint32_t chain_segments;   /* runs of narrow levels run by the cluster kernel */
    uint32_t dense_tail;       /* order of the trailing block factored densely    */
    double factor_flops;       /* sum_k |L_k| + 2 |L_k||U_k|                      */
    uint64_t factor_launches;  /* kernel launches of the last glu_factor call     */
    float last_factor_ms;      /* device time of the last glu_factor call         */
    float pert;                /* perturbation of the last GESP factorization     */
    uint32_t supernodes;       /* supernodes of the sparse part (0: column path)   */
    uint32_t sn_levels;        /* levels of the supernodal schedule               */
    double sn_update_flops;    /* supernode updates: sum 2 m w nt                  */
    double sn_update_bytes;    /* their algorithmic bytes: L21, U12 read once, the
                                  m x nt outputs read and written (+ positions)   */
    double sn_panel_bytes;     /* supernode panels: L21, U12 read and written      */
    uint32_t sn_sweep_levels;  /* levels of the supernodal L and U solve sweeps    */
    double dense_update_bytes; /* last glu_factor call, dense trailing updates:
                                  C read and written once per launch plus one
                                  FP32 read of the panels' L21 and U12          */
    double dense_update_flops; /* and their flops, 2 K per updated entry        */
    uint64_t solve_launches;   /* kernel launches of the last solve call (glu_solve,
                                  glu_solve_transposed, glu_solve_refined)       */
    uint32_t couple_columns;   /* sparse columns whose update of the dense trailing
                                  block is deferred to tensor-core products after
                                  the sparse part (tuning.defer_tail)           */
    uint32_t couple_groups;    /* those products (up to 128 columns each)        */
} glu_stats;
glu_status glu_get_stats(glu_handle_t h, glu_stats *stats);

/* Per-kernel device times of glu_factor, for profiling.  After
 * glu_profile_enable(h, 1) every later glu_factor brackets each launch with
 * CUDA events on its stream; glu_kernel_times returns, per kernel kind, the
 * summed milliseconds and launch counts of the last glu_factor call (arrays
 * of GLU_KERNEL_KINDS entries; see glu_kernel_kind_name).  Off by default:
 * the events add a little time between launches. */
#define GLU_KERNEL_KINDS 16
glu_status glu_profile_enable(glu_handle_t h, int on);
glu_status glu_kernel_times(glu_handle_t h, float *ms, uint32_t *launches);
const char *glu_kernel_kind_name(int kind);

/* FP32 fused multiply-add throughput of a device in TFLOP/s (a short
 * microbenchmark, about a second), the compute bound of the factorization's
 * roofline.  No counterpart in the reference. */
glu_status glu_measure_fp32_peak(int device, double *tflops);

/* Device-side waits of the handle's kernels (the dense-tail solve's block
 * flags, the tensor-core update's pipeline barriers) give up after `polls`
 * polls: the kernel sets a status flag, finishes without further waiting, and
 * the call returns GLU_ERR_TIMEOUT with the handle still usable.  0 restores
 * the default (2^24 polls, a few seconds).  The reference has no bounded
 * waits: a stuck kernel blocks its per-level cudaDeviceSynchronize
 * (src/numeric.cu:615-616) forever. */
glu_status glu_set_wait_limit(glu_handle_t h, uint32_t polls);

/* Failure injection for tests of the error paths; no counterpart in the
 * reference.  Nothing here faults or hangs a GPU: the failures are made on
 * the host or are a flag that nothing sets, met by a bounded wait.
 *   GLU_INJECT_ALLOC_FAILURES: the next `value` device allocations of the
 *     library fail as out of memory (process-wide; h may be NULL).
 *   GLU_INJECT_UNSET_SOLVE_FLAG: in the next solve of h, the dense-tail
 *     sweeps start their block tickets at 1, so no block sets the first
 *     block's completion flag and every block that needs it waits until the
 *     wait limit; the call returns GLU_ERR_TIMEOUT (value ignored). */
typedef enum { GLU_INJECT_ALLOC_FAILURES = 1, GLU_INJECT_UNSET_SOLVE_FLAG = 2 } glu_inject;
glu_status glu_debug_inject(glu_handle_t h, int what, uint32_t value);

/* Schedule knobs (the autotuner's search space).  Applies to later calls. */
typedef struct {
    uint32_t wide_work;        /* a level with more update work runs alone       */
    uint32_t chain_cluster;    /* CTAs of the cluster running narrow-level runs  */
    uint32_t group_lanes;      /* lanes per (column, update-target) pair: 4..32  */
    uint32_t dense_tail_min;   /* smallest dense trailing block (above n: none)  */
    uint32_t dense_tail_max;   /* largest trailing block factored in a buffer    */
    uint32_t solve_thin;       /* solve levels with at most this many columns run
                                  in the cluster kernel                          */
    uint32_t solve_cluster;    /* CTAs of that cluster (1..16)                   */
    uint32_t sn_width;         /* widest supernode of the sparse factorization
                                  (1..64); 0 factors column by column            */
    uint32_t sn_small;         /* 1: supernodes with few rows and targets run one
                                  per warp, grouped into blocks; 0: a block each */
    uint32_t dense_lookahead;  /* dense trailing blocks at least this wide factor
                                  the next panel during the current update
                                  (0: never)                                     */
    uint32_t dense_tc_min;     /* dense trailing blocks at least this wide update
                                  on the tensor cores (tcgen05, FP32 accuracy by
                                  a three-part BF16 split), each update region
                                  whose area over the value sets reaches
                                  min(dense_tc_min^2, two 128 x 128 tiles per
                                  SM); 0: FP32 FMA always                      */
    uint32_t dense_rate;       /* dense-block throughput (GFLOP/s) the split cost
                                  model assumes; 0: built in (FMA or tensor-core
                                  rate, whichever the block would use)           */
    uint32_t sn_sweep_fused;   /* 0 (default): one launch per supernodal solve
                                  sweep level (a second one for the groups of
                                  small supernodes of a wide level, or only
                                  that one where the level has nothing else);
                                  1: each sweep is one launch in
                                  which a supernode waits (bounded) for the ones
                                  that update it (slower on the patterns
                                  measured: the ticket and the waits cost more
                                  than the level launches)                      */
    uint32_t batch_tile;       /* value sets one supernode-update block applies
                                  its tile to (its metadata and target positions
                                  computed once); 0: chosen from the grid size */
    uint32_t defer_tail;       /* > 0: when the dense trailing block updates on
                                  the tensor cores, sparse supernodes whose update
                                  of it is large leave that update out, and the
                                  block takes it afterwards as tensor-core
                                  products of up to 128 of their columns each, as
                                  many as a cost model finds worth it, with a
                                  product costed at (the block's area) /
                                  defer_tail scattered entry updates (1: the
                                  built-in estimate; larger values defer more);
                                  0: every supernode scatters its own update    */
    uint32_t dense_group;      /* panels per look-ahead group of the dense trailing
                                  block (2..4): panel j of a group first takes the
                                  updates of panels 0..j-1 on its row and column,
                                  and the rest of the block then one update of
                                  K = 64 x group (fewer reads and writes of it) */
} glu_tuning;
glu_status glu_get_tuning(glu_handle_t h, glu_tuning *t);
glu_status glu_set_tuning(glu_handle_t h, const glu_tuning *t);

#ifdef __cplusplus
}
#endif

#endif /* GLU_B200_H */
