// Triangular solves with the factors, on the device.
//
// The reference solves on the CPU in FP32 (Symbolic_Matrix::solve,
// src/symbolic.cc:200-251): permute/scale b, unit-L column sweep (:226-229),
// U column sweep with the diagonal divide (:232-239), permute/scale back.
// Here the same sweeps run on the GPU:
//
//  * sparse columns (in front of the dense trailing block) are processed level
//    by level, with level sets of each sweep's own dependency graph computed
//    once per pattern: a level with many columns gets its own launch (one warp
//    per column); a run of thin levels executes inside one thread-block
//    cluster that steps from level to level with hardware cluster barriers.
//    L and U sweeps scatter (x_i -= L(i,j) x_j with atomics), the transposed
//    sweeps gather (dot products, no atomics);
//  * the dense trailing block is solved by row blocks of 64: a block adds the
//    contribution of every finished earlier block (one 64 x 64 tile each,
//    staged in shared memory) and then solves its diagonal tile; blocks are
//    claimed in order through a ticket and wait (bounded) on per-block flags;
//  * the coupling between the two (U entries of tail columns in sparse rows)
//    is one parallel scatter or gather over the tail columns.
#include <cooperative_groups.h>

#include <algorithm>

#include "glu_common.cuh"
#include "glu_kernels.h"

namespace cg = cooperative_groups;

namespace glu {


// ------------------------------------------------------------ sparse sweeps --
// Every sweep is in scatter form: once x_j is final, the entries of its
//   SWEEP_L : CSC column j below the diagonal   (x_j = y_j)
//   SWEEP_U : CSC column j above the diagonal   (x_j = y_j / U(j,j))
//   SWEEP_UT: CSR row j right of the diagonal    (x_j = y_j / U(j,j))
//   SWEEP_LT: CSR row j left of the diagonal     (x_j = y_j)
// are subtracted: y_target -= entry * x_j.  A long column or row is split into
// items of kSweepChunk entries that run in parallel; every item of j reads
// the same y_j (nothing writes y_j while its level runs) and the dividing
// sweeps store the finished x_j to xo (item 0 of j).
template <int kMode>
__device__ __forceinline__ void sweep_item(const DevPattern &P, const float *__restrict__ val, float *y, float *xo,
                                           uint32_t nrhs, const uint32_t *__restrict__ cols,
                                           const uint32_t *__restrict__ item_off, uint32_t s0, uint32_t s1,
                                           uint32_t it, uint32_t lane) {
    constexpr bool kDiv = (kMode == SWEEP_U || kMode == SWEEP_UT);
    constexpr bool kRow = (kMode == SWEEP_UT || kMode == SWEEP_LT);
    const uint32_t s = upper_slot(item_off, s0, s1, it);
    const uint32_t j = cols[s];
    const uint32_t rem = it - item_off[s];
    uint32_t p0, p1;
    if (kMode == SWEEP_L) {
        p0 = P.diag[j] + 1;
        p1 = P.cptr[j + 1];
    } else if (kMode == SWEEP_U) {
        p0 = P.cptr[j];
        p1 = P.diag[j];
    } else if (kMode == SWEEP_UT) {
        p0 = P.rdiag[j] + 1;
        p1 = P.rptr[j + 1];
    } else {
        p0 = P.rptr[j];
        p1 = P.rdiag[j];
    }
    const uint32_t e0 = p0 + rem * kSweepChunk;
    const uint32_t e1 = min(e0 + kSweepChunk, p1);
    const uint32_t n = P.n;
    const float d = kDiv ? val[P.diag[j]] : 1.0f;
    for (uint32_t r = 0; r < nrhs; ++r) {
        float *yr = y + size_t(r) * n;
        float xj = __ldcg(yr + j);
        if (kDiv) {
            xj = xj / d;
            if (rem == 0 && lane == 0) xo[size_t(r) * n + j] = xj;
        }
        if (xj == 0.0f) continue;
        for (uint32_t e = e0 + lane; e < e1; e += 32) {
            const uint32_t tgt = kRow ? P.cidx[e] : P.ridx[e];
            const float v = kRow ? val[P.cpos[e]] : val[e];
            atomicAdd(yr + tgt, -__fmul_rn(v, xj));
        }
    }
}

// One level, own launch: warps over the items of cols[s0, s1).
template <int kMode>
__global__ void __launch_bounds__(256) k_sweep_level(DevPattern P, const float *__restrict__ val, float *y, float *xo,
                                                     uint32_t nrhs, const uint32_t *__restrict__ cols,
                                                     const uint32_t *__restrict__ item_off, uint32_t s0,
                                                     uint32_t s1, uint64_t vstride, uint64_t ystride) {
    val += blockIdx.z * vstride;  // value set blockIdx.z, its right-hand sides
    y += blockIdx.z * ystride;
    xo += blockIdx.z * ystride;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    const uint32_t it0 = item_off[s0], it1 = item_off[s1];
    for (uint32_t it = it0 + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < it1; it += nw)
        sweep_item<kMode>(P, val, y, xo, nrhs, cols, item_off, s0, s1, it, lane);
}

// A run of thin levels [l0, l1) inside one cluster; cluster barrier between
// levels; values of y written by other blocks are read through L2.
template <int kMode>
__global__ void __launch_bounds__(kSolveChainThreads) k_sweep_chain(DevPattern P, const float *__restrict__ val,
                                                                    float *y, float *xo, uint32_t nrhs,
                                                                    const uint32_t *__restrict__ cols,
                                                                    const uint32_t *__restrict__ lptr,
                                                                    const uint32_t *__restrict__ item_off,
                                                                    uint32_t l0, uint32_t l1, uint64_t vstride,
                                                                    uint64_t ystride) {
    val += blockIdx.z * vstride;  // value set blockIdx.z, its right-hand sides
    y += blockIdx.z * ystride;
    xo += blockIdx.z * ystride;
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t nblk = cluster.num_blocks();
    const uint32_t rank = cluster.block_rank();
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    const uint32_t w0 = rank * wpb + (threadIdx.x >> 5), nw = nblk * wpb;
    for (uint32_t l = l0; l < l1; ++l) {
        const uint32_t s0 = lptr[l], s1 = lptr[l + 1];
        const uint32_t it0 = item_off[s0], it1 = item_off[s1];
        for (uint32_t it = it0 + w0; it < it1; it += nw) sweep_item<kMode>(P, val, y, xo, nrhs, cols, item_off, s0, s1, it, lane);
        cluster.sync();
    }
}

// Coupling of the dense tail with the sparse unknowns, one warp per tail
// column / row j (x_j final): y_i -= U(i,j) x_j for the U entries of tail
// column j in rows i < t (kRow = false, before the sparse U sweep), or
// y_c -= L(j,c) x_j for the L entries of tail row j in columns c < t
// (kRow = true, before the sparse L^T sweep).
template <bool kRow>
__global__ void __launch_bounds__(256) k_tail_coupling(DevPattern P, uint32_t t, uint32_t m,
                                                       const uint32_t *__restrict__ tail_start,
                                                       const float *__restrict__ val, float *y, uint32_t nrhs,
                                                       uint64_t vstride, uint64_t ystride) {
    val += blockIdx.z * vstride;  // value set blockIdx.z, its right-hand sides
    y += blockIdx.z * ystride;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t jj = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (jj >= m) return;
    const uint32_t j = t + jj, n = P.n;
    const uint32_t p0 = kRow ? P.rptr[j] : P.cptr[j], p1 = tail_start[jj];
    for (uint32_t r = 0; r < nrhs; ++r) {
        float *yr = y + size_t(r) * n;
        const float xj = yr[j];
        if (xj == 0.0f) continue;
        for (uint32_t p = p0 + lane; p < p1; p += 32) {
            const uint32_t tgt = kRow ? P.cidx[p] : P.ridx[p];
            const float v = kRow ? val[P.cpos[p]] : val[p];
            atomicAdd(yr + tgt, -__fmul_rn(v, xj));
        }
    }
}

// y[j] = xo[j] for the sparse unknowns j < t (after a dividing sweep).
__global__ void k_copy_sparse(const float *__restrict__ xo, float *y, uint32_t t, uint32_t n) {
    const size_t off = size_t(blockIdx.y) * n;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < t; j += gridDim.x * blockDim.x) y[off + j] = xo[off + j];
}

template <int kMode>
static cudaError_t run_sweep(const DevPattern &P, const SolvePlanDev &S, const float *val, float *y, float *xo,
                             uint32_t nrhs, const SolveBatch &B, cudaStream_t st) {
    const SweepPlan &sw = S.sweep[kMode];
    const uint64_t ystride = uint64_t(nrhs) * P.n;
    // blocks per value set of a wide level: about eight per SM in all
    const uint32_t wide_blocks = std::max<uint32_t>(1u, (148u * 8u + B.count - 1) / B.count);
    for (uint32_t i = 0; i < sw.nsteps; ++i) {
        const SweepStep &s = sw.steps[i];
        if (s.kind == 0) {
            k_sweep_level<kMode><<<dim3(wide_blocks, 1, B.count), 256, 0, st>>>(
                P, val, y, xo, nrhs, sw.cols, sw.item_off, s.s0, s.s1, B.vstride, ystride);
        } else {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(S.cluster, 1, B.count);
            cfg.blockDim = dim3(kSolveChainThreads, 1, 1);
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = S.cluster;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            cudaError_t e = cudaLaunchKernelEx(&cfg, k_sweep_chain<kMode>, P, val, y, xo, nrhs, sw.cols, sw.lptr,
                                               sw.item_off, s.l0, s.l1, B.vstride, ystride);
            if (e != cudaSuccess) return e;
        }
    }
    if ((kMode == SWEEP_U || kMode == SWEEP_UT) && S.t > 0) {
        uint32_t bx = (S.t + 255) / 256;
        if (bx > 1024) bx = 1024;
        k_copy_sparse<<<dim3(bx, nrhs * B.count, 1), 256, 0, st>>>(xo, y, S.t, P.n);
    }
    return cudaGetLastError();
}

// --------------------------------------------------------- dense tail sweeps --
// Solve T x = y on the dense block (rows [t, t+m) of y), where
//   kMode 0: T = L   (unit lower,      T(i,c) = val[doff[c] + i])
//   kMode 1: T = U   (upper,           T(i,c) = val[doff[c] + i])
//   kMode 2: T = U^T (lower,           T(i,c) = val[doff[i] + c])
//   kMode 3: T = L^T (unit upper,      T(i,c) = val[doff[i] + c])
// Row blocks of 64 are claimed in solve order (ascending for lower, descending
// for upper), interleaved over the value sets; flags[b] = 1 once block b of
// a set is solved.  The diagonal block's
// solve is a product with its inverse (dinv, computed once per factorization
// by k_dense_diag_inv), so the step between two blocks of the chain is a
// parallel 64 x 64 mat-vec instead of 64 dependent substitution steps.
constexpr int kRB = 64;
constexpr int kRHSChunk = 4;

// Inverses of the 64 x 64 diagonal blocks of the dense tail: blockIdx.y = 0
// the unit lower L_bb, 1 the upper U_bb; dinv[z][b][which] row-major.  Thread
// j computes column j by substitution (rows past the tail's end are the
// identity).  blockIdx.z selects the value set.
__global__ void __launch_bounds__(kRB) k_dense_diag_inv(const float *__restrict__ val, uint64_t dstride,
                                                         const uint32_t *__restrict__ doff, uint32_t m,
                                                         float *__restrict__ dinv) {
    __shared__ float T[kRB][kRB + 1];
    __shared__ float X[kRB][kRB + 1];
    const uint32_t b = blockIdx.x, which = blockIdx.y, j = threadIdx.x;
    const uint32_t nb = (m + kRB - 1) / kRB;
    val += blockIdx.z * dstride;
    const uint32_t rb0 = b * kRB, rows = min(uint32_t(kRB), m - rb0);
    for (uint32_t e = j; e < uint32_t(kRB * kRB); e += kRB) {
        const uint32_t c = e / kRB, i = e % kRB;
        T[i][c] = (i < rows && c < rows) ? val[doff[rb0 + c] + rb0 + i] : (i == c ? 1.0f : 0.0f);
    }
    __syncthreads();
    if (which == 0) {  // unit lower: X(:, j) = L^-1 e_j
        for (uint32_t i = 0; i < uint32_t(kRB); ++i) X[i][j] = i == j ? 1.0f : 0.0f;
        for (uint32_t i = j + 1; i < uint32_t(kRB); ++i) {
            float acc = 0.0f;
            for (uint32_t k = j; k < i; ++k) acc = fmaf(T[i][k], X[k][j], acc);
            X[i][j] = -acc;
        }
    } else {  // upper: X(:, j) = U^-1 e_j
        for (uint32_t i = 0; i < uint32_t(kRB); ++i) X[i][j] = 0.0f;
        X[j][j] = 1.0f / T[j][j];
        for (uint32_t i = j; i-- > 0;) {
            float acc = 0.0f;
            for (uint32_t k = i + 1; k <= j; ++k) acc = fmaf(T[i][k], X[k][j], acc);
            X[i][j] = -acc / T[i][i];
        }
    }
    float *out = dinv + ((size_t(blockIdx.z) * nb + b) * 2 + which) * kRB * kRB;
    for (uint32_t i = 0; i < uint32_t(kRB); ++i) out[i * kRB + j] = X[i][j];
}

template <int kMode>
__global__ void __launch_bounds__(256, 4) k_dense_trsv(const float *__restrict__ val, const uint32_t *__restrict__ doff,
                                                    uint32_t t, uint32_t m, float *y, uint32_t n, uint32_t nrhs,
                                                    uint32_t *flags, uint32_t *ticket, uint32_t *status,
                                                    uint32_t spin_limit, uint32_t ticket_base, uint64_t dstride,
                                                    uint64_t ystride, const float *__restrict__ dinv) {
    constexpr bool kLower = (kMode == 0 || kMode == 2);
    constexpr bool kTrans = (kMode >= 2);
    constexpr int kWhich = (kMode == 0 || kMode == 3) ? 0 : 1;  // inverse of L or of U
    __shared__ float tile[kRB][kRB + 1];
    __shared__ float xs[kRB][kRHSChunk];
    __shared__ float part[4][kRB][kRHSChunk];
    __shared__ uint32_t s_blk;
    const uint32_t tid = threadIdx.x;
    const uint32_t nb = (m + kRB - 1) / kRB;
    // One ticket counter for the launch, handed out block-row-major over the
    // value sets (ticket = block * count + set): every set's chain advances
    // at once, and a block waits only on blocks of smaller tickets, which
    // are running or done.
    if (tid == 0) s_blk = atomicAdd(ticket, 1u) + ticket_base;
    __syncthreads();
    const uint32_t count = gridDim.z, tg = s_blk;
    if (tg >= nb * count) return;
    const uint32_t z = tg % count, tk = tg / count;
    val += z * dstride;
    y += z * ystride;
    flags += size_t(z) * nb;
    const uint32_t b = kLower ? tk : nb - 1 - tk;
    const uint32_t rb0 = b * kRB, rb1 = min(rb0 + kRB, m);
    const uint32_t rows = rb1 - rb0;
    auto T = [&](uint32_t i, uint32_t c) -> float {
        return kTrans ? val[doff[i] + c] : val[doff[c] + i];
    };
    constexpr int kTilePer = kRB * kRB / 256;
    const float *inv = dinv + ((size_t(z) * nb + b) * 2 + kWhich) * kRB * kRB;  // row-major
    // tile T(rb0.., block s in solve order): independent of x
    auto load_tile = [&](uint32_t s, float (&tv)[kTilePer]) {
        const uint32_t c = kLower ? s : nb - 1 - s;
        const uint32_t cb0 = c * kRB, cb1 = min(cb0 + kRB, m);
#pragma unroll
        for (int qq = 0; qq < kTilePer; ++qq) {
            const uint32_t e = tid + qq * 256, a = e / kRB, bb = e % kRB;  // coalesced along bb
            const uint32_t i = kTrans ? a : bb, cc = kTrans ? bb : a;
            tv[qq] = (rb0 + i < rb1 && cb0 + cc < cb1) ? T(rb0 + i, cb0 + cc) : 0.0f;
        }
    };
    for (uint32_t rc0 = 0; rc0 < nrhs; rc0 += kRHSChunk) {
        const uint32_t nr = min(uint32_t(kRHSChunk), nrhs - rc0);
        const uint32_t row = tid & (kRB - 1), q = tid / kRB;  // 4 quarters of 16 columns
        float acc[kRHSChunk] = {0.f, 0.f, 0.f, 0.f};
        // contributions of the finished blocks, in solve order; the next
        // block's tile is in flight while this one waits and computes
        float tv[kTilePer], tn[kTilePer];
        if (tk > 0) load_tile(0, tv);
        for (uint32_t s = 0; s < tk; ++s) {
            const uint32_t c = kLower ? s : nb - 1 - s;
            const uint32_t cb0 = c * kRB, cb1 = min(cb0 + kRB, m);
            if (s + 1 < tk) load_tile(s + 1, tn);
            if (kTrans) {  // transposed: through shared memory, loads coalesced along the rows
#pragma unroll
                for (int qq = 0; qq < kTilePer; ++qq) {
                    const uint32_t e = tid + qq * 256, a = e / kRB, bb = e % kRB;
                    tile[a][bb] = tv[qq];
                }
            }
            if (tid == 0) wait_count(flags + c, 1u, status, spin_limit);
            __syncthreads();
            for (uint32_t e = tid; e < kRB * kRHSChunk; e += 256) {
                uint32_t cc = e / kRHSChunk, r = e % kRHSChunk;
                float v = 0.0f;
                if (cb0 + cc < cb1 && r < nr) v = __ldcg(y + size_t(rc0 + r) * n + t + cb0 + cc);
                xs[cc][r] = v;
            }
            __syncthreads();
            if (kTrans) {
#pragma unroll 4
                for (uint32_t cc = q * 16; cc < q * 16 + 16; ++cc) {
                    float tv2 = tile[row][cc];
#pragma unroll
                    for (int r = 0; r < kRHSChunk; ++r) acc[r] = fmaf(tv2, xs[cc][r], acc[r]);
                }
            } else {  // thread (row, q) holds T(row, q + 4 j), j < 16: multiplied in registers
#pragma unroll
                for (int qq = 0; qq < kTilePer; ++qq) {
                    const uint32_t cc = q + 4 * qq;
#pragma unroll
                    for (int r = 0; r < kRHSChunk; ++r) acc[r] = fmaf(tv[qq], xs[cc][r], acc[r]);
                }
            }
            __syncthreads();
#pragma unroll
            for (int qq = 0; qq < kTilePer; ++qq) tv[qq] = tn[qq];
        }
#pragma unroll
        for (int r = 0; r < kRHSChunk; ++r) part[q][row][r] = acc[r];
        // r = y - (contributions) for the block's rows, then x = T_bb^-1 r
#pragma unroll
        for (int qq = 0; qq < kTilePer; ++qq) {
            const uint32_t e = tid + qq * 256, a = e / kRB, bb = e % kRB;  // inverse element (a, bb)
            const float dv = __ldg(inv + e);
            if (kTrans)
                tile[bb][a] = dv;
            else
                tile[a][bb] = dv;
        }
        __syncthreads();
        if (tid < kRB * kRHSChunk) {
            const uint32_t i = tid % kRB, r = tid / kRB;
            float v = 0.0f;
            if (i < rows && r < nr)
                v = __ldcg(y + size_t(rc0 + r) * n + t + rb0 + i) -
                    (part[0][i][r] + part[1][i][r] + part[2][i][r] + part[3][i][r]);
            xs[i][r] = v;
        }
        __syncthreads();
        {
            float acc2[kRHSChunk] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
            for (uint32_t cc = q * 16; cc < q * 16 + 16; ++cc) {
                const float tv = tile[row][cc];
#pragma unroll
                for (int r = 0; r < kRHSChunk; ++r) acc2[r] = fmaf(tv, xs[cc][r], acc2[r]);
            }
#pragma unroll
            for (int r = 0; r < kRHSChunk; ++r) part[q][row][r] = acc2[r];
        }
        __syncthreads();
        if (tid < kRB * kRHSChunk) {
            const uint32_t i = tid % kRB, r = tid / kRB;
            if (i < rows && r < nr)
                __stcg(y + size_t(rc0 + r) * n + t + rb0 + i,
                       (part[0][i][r] + part[1][i][r]) + (part[2][i][r] + part[3][i][r]));
        }
        __syncthreads();
    }
    if (tid == 0) {
        __threadfence();
        st_release_gpu(flags + b, 1u);
    }
}

cudaError_t launch_dense_diag_inv(const float *dval, uint64_t dstride, uint32_t count, const uint32_t *doff,
                                  uint32_t m, float *dinv, cudaStream_t st) {
    if (m == 0) return cudaSuccess;
    k_dense_diag_inv<<<dim3((m + kRB - 1) / kRB, 2, count), kRB, 0, st>>>(dval, dstride, doff, m, dinv);
    return cudaGetLastError();
}

template <int kMode>
static cudaError_t dense_sweep(const SolvePlanDev &S, const float *dval, float *y, uint32_t n,
                               uint32_t nrhs, uint32_t *flags, uint32_t *ticket, uint32_t *status,
                               const SolveBatch &B, cudaStream_t st) {
    if (S.m == 0) return cudaSuccess;
    uint32_t nb = (S.m + kRB - 1) / kRB;
    cudaError_t e = cudaMemsetAsync(flags, 0, sizeof(uint32_t) * nb * B.count, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ticket, 0, sizeof(uint32_t) * B.count, st);
    if (e != cudaSuccess) return e;
    k_dense_trsv<kMode><<<dim3(nb, 1, B.count), 256, 0, st>>>(dval, S.doff, S.t, S.m, y, n, nrhs, flags, ticket,
                                                              status, S.spin_limit, S.ticket_base, B.dstride,
                                                              uint64_t(nrhs) * n, B.dinv);
    return cudaGetLastError();
}

static cudaError_t tail_coupling(const DevPattern &P, const SolvePlanDev &S, const float *val, float *y,
                                 uint32_t nrhs, bool rows, const SolveBatch &B, cudaStream_t st) {
    if (S.m == 0 || S.t == 0) return cudaSuccess;
    const dim3 grid((S.m + 7) / 8, 1, B.count);
    const uint64_t ystride = uint64_t(nrhs) * P.n;
    if (rows)
        k_tail_coupling<true><<<grid, 256, 0, st>>>(P, S.t, S.m, S.tail_row_start, val, y, nrhs, B.vstride, ystride);
    else
        k_tail_coupling<false><<<grid, 256, 0, st>>>(P, S.t, S.m, S.tail_start, val, y, nrhs, B.vstride, ystride);
    return cudaGetLastError();
}

cudaError_t solve_lower_unit(const DevPattern &P, const SolvePlanDev &S, const float *val,
                             const float *dval, float *y, float *xo, uint32_t nrhs, uint32_t *counters,
                             uint32_t *ticket, uint32_t *status, const SolveBatch &B, cudaStream_t st) {
    cudaError_t e = S.sn[0].nlev ? run_sn_sweep(P, S.sn[0], false, S.t, val, y, xo, nrhs, B, B.sweep_done, ticket,
                                                status, S.spin_limit, st)
                                 : run_sweep<SWEEP_L>(P, S, val, y, xo, nrhs, B, st);
    if (e != cudaSuccess) return e;
    return dense_sweep<0>(S, dval, y, P.n, nrhs, counters, ticket, status, B, st);
}

cudaError_t solve_upper(const DevPattern &P, const SolvePlanDev &S, const float *val,
                        const float *dval, float *y, float *xo, uint32_t nrhs, uint32_t *counters,
                        uint32_t *ticket, uint32_t *status, const SolveBatch &B, cudaStream_t st) {
    cudaError_t e = dense_sweep<1>(S, dval, y, P.n, nrhs, counters, ticket, status, B, st);
    if (e == cudaSuccess) e = tail_coupling(P, S, val, y, nrhs, false, B, st);
    if (e == cudaSuccess)
        e = S.sn[1].nlev ? run_sn_sweep(P, S.sn[1], true, S.t, val, y, xo, nrhs, B, B.sweep_done, ticket, status,
                                        S.spin_limit, st)
                         : run_sweep<SWEEP_U>(P, S, val, y, xo, nrhs, B, st);
    return e;
}

cudaError_t solve_upper_trans(const DevPattern &P, const SolvePlanDev &S, const float *val,
                              const float *dval, float *y, float *xo, uint32_t nrhs, uint32_t *counters,
                              uint32_t *ticket, uint32_t *status, const SolveBatch &B, cudaStream_t st) {
    cudaError_t e = run_sweep<SWEEP_UT>(P, S, val, y, xo, nrhs, B, st);
    if (e == cudaSuccess) e = dense_sweep<2>(S, dval, y, P.n, nrhs, counters, ticket, status, B, st);
    return e;
}

cudaError_t solve_lower_unit_trans(const DevPattern &P, const SolvePlanDev &S, const float *val,
                                   const float *dval, float *y, float *xo, uint32_t nrhs, uint32_t *counters,
                                   uint32_t *ticket, uint32_t *status, const SolveBatch &B, cudaStream_t st) {
    cudaError_t e = dense_sweep<3>(S, dval, y, P.n, nrhs, counters, ticket, status, B, st);
    if (e == cudaSuccess) e = tail_coupling(P, S, val, y, nrhs, true, B, st);
    if (e == cudaSuccess) e = run_sweep<SWEEP_LT>(P, S, val, y, xo, nrhs, B, st);
    return e;
}

// --------------------------------------------------------------- transforms --
__global__ void k_transform_f32(const uint32_t *__restrict__ idx, const double *__restrict__ scale,
                                const float *__restrict__ in, float *__restrict__ out, uint32_t n) {
    const size_t off = size_t(blockIdx.y) * n;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        float v = in[off + idx[j]];
        // float * double evaluated in double, stored as float (symbolic.cc:219,244)
        out[off + j] = scale ? static_cast<float>(static_cast<double>(v) * scale[j]) : v;
    }
}

__global__ void k_transform_f64_to_f32(const uint32_t *__restrict__ idx, const double *__restrict__ scale,
                                       const double *__restrict__ in, float *__restrict__ out, uint32_t n) {
    const size_t off = size_t(blockIdx.y) * n;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double v = in[off + idx[j]];
        out[off + j] = static_cast<float>(scale ? v * scale[j] : v);
    }
}

__global__ void k_transform_f32_to_f64(const uint32_t *__restrict__ idx, const double *__restrict__ scale,
                                       const float *__restrict__ in, double *__restrict__ x, uint32_t n,
                                       int accumulate) {
    const size_t off = size_t(blockIdx.y) * n;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double v = static_cast<double>(in[off + idx[j]]);
        if (scale) v *= scale[j];
        x[off + j] = accumulate ? x[off + j] + v : v;
    }
}

static inline dim3 tgrid(uint32_t n, uint32_t nrhs) {
    uint32_t bx = (n + 255) / 256;
    if (bx > 1024) bx = 1024;
    return dim3(bx, nrhs, 1);
}

cudaError_t launch_transform_f32(const uint32_t *idx, const double *scale, const float *in,
                                 float *out, uint32_t n, uint32_t nrhs, cudaStream_t st) {
    k_transform_f32<<<tgrid(n, nrhs), 256, 0, st>>>(idx, scale, in, out, n);
    return cudaGetLastError();
}
cudaError_t launch_transform_f64_to_f32(const uint32_t *idx, const double *scale, const double *in,
                                        float *out, uint32_t n, uint32_t nrhs, cudaStream_t st) {
    k_transform_f64_to_f32<<<tgrid(n, nrhs), 256, 0, st>>>(idx, scale, in, out, n);
    return cudaGetLastError();
}
cudaError_t launch_transform_f32_to_f64_add(const uint32_t *idx, const double *scale,
                                            const float *in, double *x, uint32_t n, uint32_t nrhs,
                                            int accumulate, cudaStream_t st) {
    k_transform_f32_to_f64<<<tgrid(n, nrhs), 256, 0, st>>>(idx, scale, in, x, n, accumulate);
    return cudaGetLastError();
}

// ---------------------------------------------------------- FP64 residuals --
// r = b - A0 x with A0 in CSR form (a_rptr/a_cidx; a_vmap gives the CSC
// position of each CSR entry in ax0), one warp per row, deterministic order.
// norms[2v] += sum r^2, norms[2v+1] = max |r| for right-hand side v.
__global__ void __launch_bounds__(256) k_residual(const uint32_t *__restrict__ rptr, const uint32_t *__restrict__ cidx,
                                                  const uint32_t *__restrict__ vmap, const double *__restrict__ ax0,
                                                  uint32_t n, const double *__restrict__ b,
                                                  const double *__restrict__ x, double *__restrict__ r,
                                                  double *norms, uint32_t nrhs_per_set, uint64_t ax0_stride) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t v = blockIdx.y;
    const size_t off = size_t(v) * n;
    ax0 += (v / nrhs_per_set) * ax0_stride;  // the value set of vector v
    double ss = 0.0, mx = 0.0;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) / 32; row < n;
         row += gridDim.x * blockDim.x / 32) {
        double acc = 0.0;
        for (uint32_t e = rptr[row] + lane; e < rptr[row + 1]; e += 32)
            acc = fma(ax0[vmap[e]], x[off + cidx[e]], acc);
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        double rv = b[off + row] - acc;
        if (lane == 0) {
            r[off + row] = rv;
            ss += rv * rv;
            mx = fmax(mx, fabs(rv));
        }
    }
    if (lane == 0) {
        atomicAdd(norms + 2 * v, ss);
        // non-negative doubles order like their bit patterns
        atomicMax(reinterpret_cast<unsigned long long *>(norms + 2 * v + 1),
                  static_cast<unsigned long long>(__double_as_longlong(mx)));
    }
}

cudaError_t launch_residual(const uint32_t *a_rptr, const uint32_t *a_cidx, const uint32_t *a_vmap,
                            const double *ax0, uint32_t n, const double *b, const double *x,
                            double *r, uint32_t nvec, uint32_t nrhs_per_set, uint64_t ax0_stride,
                            double *norms, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(norms, 0, sizeof(double) * 2 * nvec, st);
    if (e != cudaSuccess) return e;
    uint32_t blocks = (n + 7) / 8;
    // about eight blocks per SM in all
    const uint32_t cap = std::max<uint32_t>(1u, (148u * 8u + nvec - 1) / nvec);
    if (blocks > cap) blocks = cap;
    k_residual<<<dim3(blocks, nvec, 1), 256, 0, st>>>(a_rptr, a_cidx, a_vmap, ax0, n, b, x, r, norms,
                                                      std::max<uint32_t>(nrhs_per_set, 1u), ax0_stride);
    return cudaGetLastError();
}

__global__ void k_norms(const double *__restrict__ v, uint32_t n, double *norms) {
    const size_t off = size_t(blockIdx.y) * n;
    double ss = 0.0, mx = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double a = v[off + i];
        ss += a * a;
        mx = fmax(mx, fabs(a));
    }
    for (int o = 16; o > 0; o >>= 1) {
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(norms + 2 * blockIdx.y, ss);
        atomicMax(reinterpret_cast<unsigned long long *>(norms + 2 * blockIdx.y + 1),
                  static_cast<unsigned long long>(__double_as_longlong(mx)));
    }
}

cudaError_t launch_norms(const double *v, uint32_t n, uint32_t nvec, double *norms,
                         cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(norms, 0, sizeof(double) * 2 * nvec, st);
    if (e != cudaSuccess) return e;
    uint32_t blocks = (n + 255) / 256;
    if (blocks > 256) blocks = 256;
    k_norms<<<dim3(blocks, nvec, 1), 256, 0, st>>>(v, n, norms);
    return cudaGetLastError();
}

}  // namespace glu
