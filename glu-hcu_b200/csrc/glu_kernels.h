// Kernel launchers of libglu_b200 (implemented in the .cu files).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "glu_common.cuh"

namespace glu {

// ------------------------------------------------------------ sparse factor --
constexpr uint32_t kItemUnroll = 4;       // elements per lane per work item
constexpr uint32_t kMaxItemBlocks = 148 * 16;
constexpr uint32_t kChainThreads = 1024;

// One level of the sparse schedule: its active columns are sched_cols[s0, s1),
// processed by groups of G lanes, with atomics when atomic != 0.
struct LevelInfo {
    uint32_t s0, s1, G, atomic;
};

struct FactorPlanDev {
    const uint32_t *sched_cols;  // active columns, level by level
    const uint32_t *item_off;    // work-item prefix over sched_cols (per level G)
    const LevelInfo *levels;     // per sparse level
};

cudaError_t launch_factor_level(const DevPattern &P, const FactorPlanDev &F, float *val,
                                uint64_t stride, uint32_t count, const float *pert_z,
                                const LevelInfo &cur, const LevelInfo *prev, uint32_t items,
                                cudaStream_t st);
cudaError_t launch_scale_level(const DevPattern &P, const FactorPlanDev &F, float *val,
                               uint64_t stride, uint32_t count, const float *pert_z,
                               const LevelInfo &lv, cudaStream_t st);
// The cluster kernel itself (for occupancy queries).
const void *chain_kernel_ptr();
cudaError_t launch_factor_chain(const DevPattern &P, const FactorPlanDev &F, float *val,
                                uint64_t stride, uint32_t count, const float *pert_z, uint32_t l0,
                                uint32_t l1, uint32_t cluster, cudaStream_t st);

// ------------------------------------------------------- supernodal factor --
constexpr uint32_t kSnMaxWidth = 64;       // widest supernode
constexpr uint32_t kSnPanelThreads = 128;  // threads of a panel block (rows or targets per block)

constexpr uint32_t kSnSmallWidth = 16;         // small supernode: width <= this, few off-diagonal rows/entries
constexpr uint32_t kSnSmallFlag = 0x80000000u;  // block-map entry of a group of small supernodes
constexpr uint32_t kSnDiagSmallPerBlock = 8;    // narrow diagonal blocks per block of the diagonal launches (a warp each)

// Supernodes in level order: their records, the block maps of the panel and
// update launches, the target metadata and the update's position table
// (nullable) with its offset per supernode.
struct SnPlanDev {
    const uint4 *meta;        // per supernode: {first column, width, L21 rows m, targets nt}
    const uint2 *dmap;        // per diagonal-block block: {supernode, 0} or {first of dsmall, kSnSmallFlag | count}
    const uint32_t *dsmall;   // supernodes of width 2..kSnSmallWidth of the diagonal launches, eight to a block
    const uint2 *pmap;        // per panel block: {supernode, part} or {first of psmall, kSnSmallFlag | count}
    const uint2 *umap;        // per update block: {supernode, tile} or {first of usmall, kSnSmallFlag | count}
    const uint32_t *psmall;   // small supernodes of the panel launches, four to a block
    const uint32_t *usmall;   // small supernodes of the update launches, eight to a block
    const uint32_t *tgt_off;  // [count + 1] prefix of the targets
    const uint4 *tgt;         // per target: {CSC position of row l, rows present (0: none), extra rows, 0}
    const uint32_t *pos;      // CSC positions of the update outputs, or nullptr
    const uint64_t *pos_off;  // [count]
    // When the dense tail [t, n) is complete and factored in place, row i >= t
    // of tail column j sits at tail_start[j - t] + (i - t): the update computes
    // those positions instead of searching for them (tail_full != 0).
    const uint32_t *tail_start = nullptr;
    uint32_t t = 0;
    uint32_t tail_full = 0;
    // Per supernode (level order), when any defers its update of the dense
    // tail: {first L21 row, first target} of the deferred corner (rows and
    // targets in the tail); updates there are skipped.  {m, nt} for the
    // others.  nullptr: none deferred.
    const uint2 *cut = nullptr;
};

// Blocks [b0, b0 + blocks) of one level's diagonal-block, panel or update
// map.  diag runs before panel, panel before update.
cudaError_t launch_sn_diag(const DevPattern &P, const SnPlanDev &S, float *val, uint64_t stride, uint32_t count,
                           const float *pert_z, uint32_t b0, uint32_t blocks, cudaStream_t st);
cudaError_t launch_sn_panel(const DevPattern &P, const SnPlanDev &S, float *val, uint64_t stride, uint32_t count,
                            const float *pert_z, uint32_t b0, uint32_t blocks, uint32_t max_width, cudaStream_t st);
cudaError_t launch_sn_update(const DevPattern &P, const SnPlanDev &S, float *val, uint64_t stride, uint32_t count,
                             uint32_t b0, uint32_t blocks, uint32_t atomic, uint32_t batch_tile, cudaStream_t st);
// Setup, once per pattern: the target metadata (S.meta, S.tgt_off set), then
// the position table (S.tgt set).
cudaError_t launch_sn_targets(const DevPattern &P, const SnPlanDev &S, uint32_t nsn, uint4 *tgt, cudaStream_t st);
cudaError_t launch_sn_positions(const DevPattern &P, const SnPlanDev &S, uint32_t nsn, uint32_t *pos,
                                cudaStream_t st);

// ------------------------------------------------------------- dense tail --
// The trailing m x m block [t, n) x [t, n) is fully dense; element (i, j) of it
// is val[doff[j] + i] (column-major, one base offset per column).
constexpr int kDenseNB = 64;        // panel width
constexpr int kPanelRows = 128;     // rows (or columns) per panel block
constexpr int kGemmTile = 128;      // trailing-update tile

cudaError_t launch_dense_panel(float *val, uint64_t stride, uint32_t count, const uint32_t *doff,
                               uint32_t m, uint32_t k0, uint32_t kb, const float *pert_z,
                               float *diag_scratch, uint32_t last_has_l, uint32_t num_sms, cudaStream_t st);
// Launches one panel step makes: 2 when its blocks over all value sets fill
// several waves (the diagonal blocks factored once in a launch of their own).
uint32_t dense_panel_launches(uint32_t count, uint32_t m, uint32_t k0, uint32_t kb, uint32_t num_sms);
// Part of the trailing update after the panels [k0, k0 + kb) (kb <=
// kDenseGroupMax x kDenseNB): rows [r_lo, r_hi) and columns [c_lo, c_hi) of the trailing block
// (relative to k0 + kb); writeback != 0 also stores the factored diagonal
// block of the panel at wb_k0 from diag_scratch.
struct DenseRegion {
    uint32_t r_lo, r_hi, c_lo, c_hi, writeback, wb_k0;
};
cudaError_t launch_dense_update(float *val, uint64_t stride, uint32_t count, const uint32_t *doff,
                                uint32_t m, uint32_t k0, uint32_t kb, const float *diag_scratch,
                                DenseRegion reg, cudaStream_t st);
// The same update on the tensor cores (glu_dense_tc.cu): the panels' L21 rows
// and U12 columns are first packed as three BF16 parts (pack[z][i][768], one
// row per trailing row or column, part p at 256 p; panel j of a look-ahead
// group in slots 64 j .. 64 j + 63), then tiles of the region are computed by
// tcgen05 from TMA loads of the packs (K up to 256).  dense_tc_tensor_map
// describes a pack buffer of `batch` value sets for the loads.
constexpr uint32_t kDensePackRow = 768;  // BF16 values (three parts of 256 slots)
constexpr uint32_t kDenseGroupMax = 4;   // panels of a look-ahead group (K = 64 x 4)
constexpr uint32_t kTcTile = 128;  // update tile of the tensor-core kernel (M = N)
cudaError_t dense_tc_tensor_map(uint16_t *pack, uint32_t m, uint32_t batch, CUtensorMap *map);
cudaError_t launch_dense_pack(const float *val, uint64_t stride, uint32_t count, const uint32_t *doff, uint32_t m,
                              uint32_t k0, uint32_t kb, uint32_t slot0, uint16_t *packA, uint16_t *packB,
                              cudaStream_t st);
cudaError_t launch_dense_update_tc(const CUtensorMap &mapA, const CUtensorMap &mapB, float *val, uint64_t stride,
                                   uint32_t count, const uint32_t *doff, uint32_t m, uint32_t k0, uint32_t kb,
                                   const float *diag_scratch, DenseRegion reg, uint32_t *status,
                                   uint32_t spin_limit, uint32_t num_sms, uint32_t *tile_counter, cudaStream_t st);
// The deferred coupling of the sparse part into the trailing block: sparse
// columns whose update of the block is large skip it in the supernodal
// updates (their supernode's cut), and after the sparse part the block takes
// A22 -= L(tail, K) U(K, tail) for the deferred columns K, in groups of up to
// 128 (slots slot0 .. slot0 + ncols - 1 of all deferred columns).
// couple_pack writes one group's operands into the packs: for slot g and
// 128-wide tail block b, lstart[g][b] .. lstart[g][b + 1] are the CSC
// positions of column k_g's rows in tail rows [128 b, 128 b + 128), and
// ustart[g][b] .. ustart[g][b + 1] the CSR positions of row k_g's entries in
// tail columns [128 b, 128 b + 128) (nblk + 1 entries per slot, nblk = the
// tail's 128-blocks).  couple_update_tc is the tensor-core update of the whole
// block from those packs.
cudaError_t launch_couple_pack(const DevPattern &P, const float *val, uint64_t stride, uint32_t count, uint32_t t,
                               uint32_t m, uint32_t ncols, uint32_t slot0, const uint32_t *lstart,
                               const uint32_t *ustart, uint16_t *packA, uint16_t *packB, cudaStream_t st);
cudaError_t launch_couple_update_tc(const CUtensorMap &mapA, const CUtensorMap &mapB, float *val, uint64_t stride,
                                    uint32_t count, const uint32_t *doff, uint32_t m, uint32_t ncols,
                                    uint32_t *status, uint32_t spin_limit, uint32_t num_sms, uint32_t *tile_counter,
                                    cudaStream_t st);
// A trailing block that is dense but not completely filled is factored in a
// separate m x m column-major buffer: gather copies the block's pattern
// entries of the CSC values into the (zeroed) buffer, scatter copies the
// factored entries back.  Entries outside the pattern stay exactly zero
// through the factorization.  tail_start[j] = CSC position of the first row
// >= t in column t + j.
cudaError_t launch_dense_gather(const DevPattern &P, const float *val, uint64_t stride, uint32_t count,
                                uint32_t t, uint32_t m, const uint32_t *tail_start, float *dbuf,
                                cudaStream_t st);
cudaError_t launch_dense_scatter(const DevPattern &P, float *val, uint64_t stride, uint32_t count,
                                 uint32_t t, uint32_t m, const uint32_t *tail_start, const float *dbuf,
                                 cudaStream_t st);

// -------------------------------------------------------------- utilities --
// pert[z] = 3.45e-4 * max_col sum |val| (FP32, column order), numeric.cu:490-506.
cudaError_t launch_pert(const DevPattern &P, const float *val, uint64_t stride, uint32_t count,
                        float *colsum_scratch, float *pert_z, cudaStream_t st);
// ORs DEV_ZERO_PIVOT / DEV_NONFINITE_PIVOT into *status for bad pivots.
cudaError_t launch_check_pivots(const DevPattern &P, const float *val, uint64_t stride,
                                uint32_t count, uint32_t *status, cudaStream_t st);
// LU values from source values: val[p] = src[p] < 0 ? 0 : (float)(ax[src[p]] * scale[src[p]]).
cudaError_t launch_gather_values(const int64_t *lu_src, const double *ax, uint64_t ax_stride,
                                 const double *scale, uint32_t nnz, float *val, uint64_t stride,
                                 uint32_t count, cudaStream_t st);

// ------------------------------------------------------------------ levels --
// Level sets (symbolic.cc:106-151) built on the device; scratch must hold
// level_scratch_bytes(n) bytes.
size_t level_scratch_bytes(uint32_t n);
cudaError_t build_levels(const DevPattern &P, void *scratch, int32_t *level_of, int32_t *level_ptr,
                         int32_t *level_idx, int32_t *num_lev_dev, uint32_t *status,
                         cudaStream_t st);

// ------------------------------------------------------------------ solves --
// Level schedule of one sparse sweep over the columns [0, t): the columns
// level by level (cols, lptr on the device) and the launches that run them.
// A step is one level with its own launch (kind 0, columns [c0, c1) of cols)
// or a run of thin levels [l0, l1) inside one thread-block cluster (kind 1).
// Every sweep is in scatter form: once x_j is final, its column (L, U: CSC)
// or row (U^T, L^T: CSR) is subtracted from the other unknowns.  Work items
// are (j, chunk of kSweepChunk entries); item_off is their prefix over cols.
struct SweepStep {
    uint32_t kind, l0, l1, s0, s1;  // levels [l0, l1), columns cols[s0, s1)
};
struct SweepPlan {
    const uint32_t *cols = nullptr;
    const uint32_t *lptr = nullptr;
    const uint32_t *item_off = nullptr;
    const SweepStep *steps = nullptr;  // host array
    uint32_t nsteps = 0;
    uint32_t nlev = 0;
};
enum SweepMode : int { SWEEP_L = 0, SWEEP_U = 1, SWEEP_UT = 2, SWEEP_LT = 3 };
constexpr uint32_t kSweepChunk = 128;

// Supernodal L or U sweep (used when the factor is supernodal): per block of
// the sweep (levels one after another) its supernode and part, per supernode
// (sweep order) its record {first column, width, L: first L21 position,
// L: L21 rows}; the host-side levels.  A level's blocks are its supernodes'
// parts first, then its groups of small supernodes.
struct SnSweepLevel {
    uint32_t b0, blocks;  // first block, blocks
    uint32_t big;         // blocks [b0, b0 + big) are supernode parts, the rest small groups
};
// Blocks of small-supernode groups from which a per-level sweep gives them a
// launch of their own: a warp-per-supernode kernel that keeps four (L) or
// five (U) blocks per SM resident, against the full kernel's two (L) or four
// (U).  The thresholds are where the waves saved on 148 SMs outweigh one more
// chained launch; below them the level stays one launch.
constexpr uint32_t kSnSweepSplitL = 592;
constexpr uint32_t kSnSweepSplitU = 2048;
// Launches of one level of a per-level sweep: {full kernel, small-group kernel}.
inline uint2 sn_sweep_level_launches(const SnSweepLevel &lv, bool upper) {
    const uint32_t small = lv.blocks - lv.big;
    if (lv.blocks == 0) return {0u, 0u};
    if (lv.big == 0) return {0u, 1u};
    if (small >= (upper ? kSnSweepSplitU : kSnSweepSplitL)) return {1u, 1u};
    return {1u, 0u};
}
struct SnSweepPlan {
    const uint2 *map = nullptr;     // {supernode, part} or {first of small[], kSnSmallFlag | count}
    const uint4 *meta = nullptr;
    const uint32_t *small = nullptr;  // small supernodes, grouped eight to a block
    const SnSweepLevel *levels = nullptr;  // host array
    uint32_t nlev = 0;
    // One launch for the whole sweep (fused != 0): blocks take tickets in map
    // order (levels ascending), block k waits until done[q] == indeg[q] for
    // the supernodes q = wait_idx[wait_off[k] ..] it solves, and after its
    // scatter adds one to done[q] for q = rel_idx[rel_off[k] ..], the
    // supernodes whose unknowns it updated.
    uint32_t fused = 0;
    uint32_t nblocks = 0, ns = 0;
    const uint32_t *wait_off = nullptr, *wait_idx = nullptr, *rel_off = nullptr, *rel_idx = nullptr;
    const uint32_t *indeg = nullptr;
};
constexpr uint32_t kSnSweepRows = 256;    // L21 rows per block of the L sweep
constexpr uint32_t kSnSweepAbove = 1024;  // U entries per block of the U sweep

// Value sets solved together: set z uses the factors at val + z * vstride
// (dense tail at dval + z * dstride) and the right-hand sides
// [z * nrhs, (z + 1) * nrhs) of the vectors (contiguous, n each).
struct SolveBatch {
    uint32_t count = 1;
    uint64_t vstride = 0;
    uint64_t dstride = 0;
    const float *dinv = nullptr;  // inverses of the dense tail's diagonal blocks of the first set
    uint32_t *sweep_done = nullptr;  // count x (supernodes) counters of the fused sweeps (null: per level)
};
// Inverses of the 64 x 64 diagonal blocks of the dense tail's L and U, per
// value set: dinv[z][b][0: L, 1: U][64 x 64] (row-major), from the factors.
cudaError_t launch_dense_diag_inv(const float *dval, uint64_t dstride, uint32_t count, const uint32_t *doff,
                                  uint32_t m, float *dinv, cudaStream_t st);

struct SolvePlanDev {
    uint32_t t;                     // first column of the dense tail (n if none)
    uint32_t m;                     // order of the dense tail
    const uint32_t *doff;           // dense tail column offsets (into the dense view)
    const uint32_t *tail_start;     // CSC position of the first row >= t of each tail column
    const uint32_t *tail_row_start; // CSR position of the first column >= t of each tail row
    SweepPlan sweep[4];             // L, U, U^T, L^T
    SnSweepPlan sn[2];              // supernodal L and U sweeps (nlev == 0: column sweeps)
    uint32_t cluster;               // CTAs of the thin-level cluster kernel
    uint32_t spin_limit;            // polls of a device-side wait before it gives up
    uint32_t ticket_base;           // first block ticket of the dense sweeps (0; 1 leaves the first
                                    // block's flag unset: a diagnostic of the bounded waits)
};

// Supernodal sweep over the columns [0, t) (forward L, or backward U), then
// y[0, t) = xo[0, t).
cudaError_t run_sn_sweep(const DevPattern &P, const SnSweepPlan &W, bool upper, uint32_t t, const float *val,
                         float *y, float *xo, uint32_t nrhs, const SolveBatch &B, uint32_t *done, uint32_t *ticket,
                         uint32_t *status, uint32_t spin_limit, cudaStream_t st);

// Transform in: y[j] = rhs[col_perm[piv[j]]] * (mc64 ? col_scale_perm[piv[j]] : 1)
// (symbolic.cc:215-223); out: x[j] = y[row_perm_inv[j]] * (mc64 ? row_scale[j] : 1)
// (symbolic.cc:242-247).  Transposed solves use the mirrored maps.
struct TransformDev {
    const uint32_t *in_idx;     // source index of each permuted entry
    const double *in_scale;     // scale of each permuted entry (nullable)
    const uint32_t *out_idx;
    const double *out_scale;
    const uint32_t *tin_idx;    // transposed: in
    const double *tin_scale;
    const uint32_t *tout_idx;   // transposed: out
    const double *tout_scale;
};

constexpr uint32_t kSolveChainThreads = 512;
// FP32 triangular solves on y (nrhs vectors of n per value set, one after
// another, B.count value sets), in place.  val: CSC factor values; dval: base
// of the dense tail view.  xo: scratch of y's size (finished values of the
// dividing sweeps); counters / ticket: scratch of the dense tail sweeps
// (B.count * (m / 64 + 1) flags, B.count tickets).
cudaError_t solve_lower_unit(const DevPattern &P, const SolvePlanDev &S, const float *val,
                             const float *dval, float *y, float *xo, uint32_t nrhs, uint32_t *counters,
                             uint32_t *ticket, uint32_t *status, const SolveBatch &B, cudaStream_t st);
cudaError_t solve_upper(const DevPattern &P, const SolvePlanDev &S, const float *val,
                        const float *dval, float *y, float *xo, uint32_t nrhs, uint32_t *counters,
                        uint32_t *ticket, uint32_t *status, const SolveBatch &B, cudaStream_t st);
// Transposed: U^T z = y (forward), then L^T w = z (backward).
cudaError_t solve_upper_trans(const DevPattern &P, const SolvePlanDev &S, const float *val,
                              const float *dval, float *y, float *xo, uint32_t nrhs, uint32_t *counters,
                              uint32_t *ticket, uint32_t *status, const SolveBatch &B, cudaStream_t st);
cudaError_t solve_lower_unit_trans(const DevPattern &P, const SolvePlanDev &S, const float *val,
                                   const float *dval, float *y, float *xo, uint32_t nrhs, uint32_t *counters,
                                   uint32_t *ticket, uint32_t *status, const SolveBatch &B, cudaStream_t st);

// Permute/scale kernels of the solve transforms.
cudaError_t launch_transform_f32(const uint32_t *idx, const double *scale, const float *in,
                                 float *out, uint32_t n, uint32_t nrhs, cudaStream_t st);
cudaError_t launch_transform_f64_to_f32(const uint32_t *idx, const double *scale, const double *in,
                                        float *out, uint32_t n, uint32_t nrhs, cudaStream_t st);
cudaError_t launch_transform_f32_to_f64_add(const uint32_t *idx, const double *scale,
                                            const float *in, double *x, uint32_t n, uint32_t nrhs,
                                            int accumulate, cudaStream_t st);

// FP64 residual r = b - A0 x (or A0^T) per right-hand side, with per-vector
// sums of squares and max-abs accumulated into norms[2*v + {0,1}].  nvec
// vectors; vector v uses the A0 values ax0 + (v / nrhs_per_set) * ax0_stride.
cudaError_t launch_residual(const uint32_t *a_rptr, const uint32_t *a_cidx, const uint32_t *a_vmap,
                            const double *ax0, uint32_t n, const double *b, const double *x,
                            double *r, uint32_t nvec, uint32_t nrhs_per_set, uint64_t ax0_stride,
                            double *norms, cudaStream_t st);
cudaError_t launch_norms(const double *v, uint32_t n, uint32_t nvec, double *norms,
                         cudaStream_t st);

}  // namespace glu
