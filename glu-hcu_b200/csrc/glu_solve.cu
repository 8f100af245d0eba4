// Triangular solves with the factors, on the device.
//
// The reference solves on the CPU in FP32 (Symbolic_Matrix::solve,
// src/symbolic.cc:200-251): permute/scale b, unit-L column sweep (:226-229),
// U column sweep with the diagonal divide (:232-239), permute/scale back.
// Here the same sweeps run on the GPU:
//
//  * sparse columns (in front of the dense trailing block) are processed
//    sync-free: one warp per column, claimed in dependency order through an
//    atomic ticket, waits (bounded) until every column it depends on has
//    finished, then scatters its updates (L, U: atomics plus a per-row
//    completion counter) or gathers them (L^T, U^T: dot products behind
//    per-column done flags);
//  * the dense trailing block is solved by row blocks of 64: a block adds the
//    contribution of every finished earlier block (one 64 x 64 tile each,
//    staged in shared memory) and then solves its diagonal tile; blocks are
//    claimed in order through a ticket and wait (bounded) on per-block flags.
//
// Every wait gives up after kSpinLimit polls and sets DEV_TIMEOUT, so a
// broken dependency can never hang the device.
#include "glu_common.cuh"
#include "glu_kernels.h"

namespace glu {

// Bounded wait until *cnt reaches target.  Returns false on timeout.
__device__ __forceinline__ bool wait_count(const uint32_t *cnt, uint32_t target, uint32_t *status) {
    uint32_t spins = 0;
    while (ld_acquire_gpu(cnt) < target) {
        if (++spins > kSpinLimit) {
            atomicOr(status, DEV_TIMEOUT);
            return false;
        }
        if ((spins & 1023u) == 0 && (ld_acquire_gpu(status) & DEV_TIMEOUT)) return false;
        __nanosleep(64);
    }
    return true;
}

// ------------------------------------------------------------ sparse sweeps --
// Forward unit-L sweep over columns [0, t) in scatter form: x_i -= L(i,j) x_j.
// need[i] = number of columns c < min(i, t) with L(i,c) != 0.
__global__ void __launch_bounds__(256) k_sparse_lower(DevPattern P, uint32_t t, const float *__restrict__ val,
                                                      float *y, uint32_t nrhs, const uint32_t *need,
                                                      uint32_t *cnt, uint32_t *ticket, uint32_t *status) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t j = 0;
    if (lane == 0) j = atomicAdd(ticket, 1u);
    j = __shfl_sync(0xffffffffu, j, 0);
    if (j >= t) return;
    if (lane == 0) wait_count(cnt + j, need[j], status);
    __syncwarp();
    const uint32_t n = P.n;
    const uint32_t l0 = P.diag[j] + 1, l1 = P.cptr[j + 1];
    for (uint32_t r = 0; r < nrhs; ++r) {
        float xj = __ldcg(y + size_t(r) * n + j);
        if (xj == 0.0f) continue;
        for (uint32_t p = l0 + lane; p < l1; p += 32)
            atomicAdd(y + size_t(r) * n + P.ridx[p], -__fmul_rn(val[p], xj));
    }
    __threadfence();
    for (uint32_t p = l0 + lane; p < l1; p += 32) atomicAdd(cnt + P.ridx[p], 1u);
}

// Backward U sweep in scatter form, columns claimed from n-1 down.  Columns of
// the dense tail ([t, n)) are already solved: they only scatter their U rows
// that lie above t.  need[r] = number of columns c > r with U(r,c) != 0.
__global__ void __launch_bounds__(256) k_sparse_upper(DevPattern P, uint32_t t, const uint32_t *__restrict__ doff,
                                                      const float *__restrict__ val, float *y, uint32_t nrhs,
                                                      const uint32_t *need, uint32_t *cnt, uint32_t *ticket,
                                                      uint32_t *status) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t tk = 0;
    if (lane == 0) tk = atomicAdd(ticket, 1u);
    tk = __shfl_sync(0xffffffffu, tk, 0);
    const uint32_t n = P.n;
    if (tk >= n) return;
    const uint32_t j = n - 1 - tk;
    const uint32_t u0 = P.cptr[j];
    uint32_t u1;
    if (j >= t) {
        u1 = doff[j - t];  // rows < t of a tail column
    } else {
        u1 = P.diag[j];
        if (lane == 0) wait_count(cnt + j, need[j], status);
        __syncwarp();
        const float d = val[P.diag[j]];
        for (uint32_t r = lane; r < nrhs; r += 32) {
            float *pj = y + size_t(r) * n + j;
            __stcg(pj, __ldcg(pj) / d);
        }
        __syncwarp();
        __threadfence_block();
    }
    for (uint32_t r = 0; r < nrhs; ++r) {
        float xj = __ldcg(y + size_t(r) * n + j);
        if (xj == 0.0f) continue;
        for (uint32_t p = u0 + lane; p < u1; p += 32)
            atomicAdd(y + size_t(r) * n + P.ridx[p], -__fmul_rn(val[p], xj));
    }
    __threadfence();
    for (uint32_t p = u0 + lane; p < u1; p += 32) atomicAdd(cnt + P.ridx[p], 1u);
}

// Forward U^T sweep over columns [0, t) in gather form:
// z_j = (y_j - sum_{i<j} U(i,j) z_i) / U(j,j).  done[i] = 1 when z_i is final.
// For tail columns (j >= t) only the part over rows i < t is subtracted here.
__global__ void __launch_bounds__(256) k_sparse_upper_trans(DevPattern P, uint32_t t, const uint32_t *__restrict__ doff,
                                                            const float *__restrict__ val, float *y,
                                                            uint32_t nrhs, uint32_t *done, uint32_t *ticket,
                                                            uint32_t *status) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t j = 0;
    if (lane == 0) j = atomicAdd(ticket, 1u);
    j = __shfl_sync(0xffffffffu, j, 0);
    const uint32_t n = P.n;
    if (j >= n) return;
    const uint32_t u0 = P.cptr[j];
    const uint32_t u1 = (j >= t) ? doff[j - t] : P.diag[j];
    for (uint32_t p = u0 + lane; p < u1; p += 32) wait_count(done + P.ridx[p], 1u, status);
    __syncwarp();
    for (uint32_t r = 0; r < nrhs; ++r) {
        float acc = 0.0f;
        for (uint32_t p = u0 + lane; p < u1; p += 32)
            acc = fmaf(val[p], __ldcg(y + size_t(r) * n + P.ridx[p]), acc);
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            float *pj = y + size_t(r) * n + j;
            float v = __ldcg(pj) - acc;
            if (j < t) v = v / val[P.diag[j]];
            __stcg(pj, v);
        }
    }
    __syncwarp();
    if (lane == 0 && j < t) {
        __threadfence();
        st_release_gpu(done + j, 1u);
    }
}

// Backward L^T sweep over columns [0, t) in gather form (tail already done):
// w_j = z_j - sum_{i>j} L(i,j) w_i, columns claimed from t-1 down.
__global__ void __launch_bounds__(256) k_sparse_lower_trans(DevPattern P, uint32_t t, const float *__restrict__ val,
                                                            float *y, uint32_t nrhs, uint32_t *done,
                                                            uint32_t *ticket, uint32_t *status) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t tk = 0;
    if (lane == 0) tk = atomicAdd(ticket, 1u);
    tk = __shfl_sync(0xffffffffu, tk, 0);
    if (tk >= t) return;
    const uint32_t j = t - 1 - tk;
    const uint32_t n = P.n;
    const uint32_t l0 = P.diag[j] + 1, l1 = P.cptr[j + 1];
    for (uint32_t p = l0 + lane; p < l1; p += 32) {
        uint32_t i = P.ridx[p];
        if (i < t) wait_count(done + i, 1u, status);
    }
    __syncwarp();
    for (uint32_t r = 0; r < nrhs; ++r) {
        float acc = 0.0f;
        for (uint32_t p = l0 + lane; p < l1; p += 32)
            acc = fmaf(val[p], __ldcg(y + size_t(r) * n + P.ridx[p]), acc);
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            float *pj = y + size_t(r) * n + j;
            __stcg(pj, __ldcg(pj) - acc);
        }
    }
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        st_release_gpu(done + j, 1u);
    }
}

// --------------------------------------------------------- dense tail sweeps --
// Solve T x = y on the dense block (rows [t, t+m) of y), where
//   kMode 0: T = L   (unit lower,      T(i,c) = val[doff[c] + i])
//   kMode 1: T = U   (upper,           T(i,c) = val[doff[c] + i])
//   kMode 2: T = U^T (lower,           T(i,c) = val[doff[i] + c])
//   kMode 3: T = L^T (unit upper,      T(i,c) = val[doff[i] + c])
// Row blocks of 64 are claimed in solve order (ascending for lower, descending
// for upper); flags[b] = 1 once block b is solved.
constexpr int kRB = 64;
constexpr int kRHSChunk = 4;

template <int kMode>
__global__ void __launch_bounds__(256) k_dense_trsv(const float *__restrict__ val, const uint32_t *__restrict__ doff,
                                                    uint32_t t, uint32_t m, float *y, uint32_t n, uint32_t nrhs,
                                                    uint32_t *flags, uint32_t *ticket, uint32_t *status) {
    constexpr bool kLower = (kMode == 0 || kMode == 2);
    constexpr bool kTrans = (kMode >= 2);
    constexpr bool kUnit = (kMode == 0 || kMode == 3);
    __shared__ float tile[kRB][kRB + 1];
    __shared__ float xs[kRB][kRHSChunk];
    __shared__ float part[4][kRB][kRHSChunk];
    __shared__ uint32_t s_blk;
    const uint32_t tid = threadIdx.x;
    const uint32_t nb = (m + kRB - 1) / kRB;
    if (tid == 0) s_blk = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t tk = s_blk;
    if (tk >= nb) return;
    const uint32_t b = kLower ? tk : nb - 1 - tk;
    const uint32_t rb0 = b * kRB, rb1 = min(rb0 + kRB, m);
    const uint32_t rows = rb1 - rb0;
    auto T = [&](uint32_t i, uint32_t c) -> float {
        return kTrans ? val[doff[i] + c] : val[doff[c] + i];
    };
    for (uint32_t rc0 = 0; rc0 < nrhs; rc0 += kRHSChunk) {
        const uint32_t nr = min(uint32_t(kRHSChunk), nrhs - rc0);
        const uint32_t row = tid & (kRB - 1), q = tid / kRB;  // 4 quarters of 16 columns
        float acc[kRHSChunk] = {0.f, 0.f, 0.f, 0.f};
        // contributions of the finished blocks, in solve order
        for (uint32_t s = 0; s < tk; ++s) {
            const uint32_t c = kLower ? s : nb - 1 - s;
            const uint32_t cb0 = c * kRB, cb1 = min(cb0 + kRB, m);
            if (tid == 0) wait_count(flags + c, 1u, status);
            __syncthreads();
            // stage tile T(rb0.., cb0..) and x(cb0..)
            for (uint32_t e = tid; e < kRB * kRB; e += 256) {
                uint32_t a = e / kRB, bb = e % kRB;  // coalesced along bb
                uint32_t i, cc;
                if (kTrans) { i = a; cc = bb; } else { cc = a; i = bb; }
                float v = 0.0f;
                if (rb0 + i < rb1 && cb0 + cc < cb1) v = T(rb0 + i, cb0 + cc);
                tile[i][cc] = v;
            }
            for (uint32_t e = tid; e < kRB * kRHSChunk; e += 256) {
                uint32_t cc = e / kRHSChunk, r = e % kRHSChunk;
                float v = 0.0f;
                if (cb0 + cc < cb1 && r < nr) v = __ldcg(y + size_t(rc0 + r) * n + t + cb0 + cc);
                xs[cc][r] = v;
            }
            __syncthreads();
#pragma unroll 4
            for (uint32_t cc = q * 16; cc < q * 16 + 16; ++cc) {
                float tv = tile[row][cc];
#pragma unroll
                for (int r = 0; r < kRHSChunk; ++r) acc[r] = fmaf(tv, xs[cc][r], acc[r]);
            }
            __syncthreads();
        }
#pragma unroll
        for (int r = 0; r < kRHSChunk; ++r) part[q][row][r] = acc[r];
        // diagonal tile
        for (uint32_t e = tid; e < kRB * kRB; e += 256) {
            uint32_t a = e / kRB, bb = e % kRB;
            uint32_t i, cc;
            if (kTrans) { i = a; cc = bb; } else { cc = a; i = bb; }
            float v = 0.0f;
            if (rb0 + i < rb1 && rb0 + cc < rb1) v = T(rb0 + i, rb0 + cc);
            tile[i][cc] = v;
        }
        __syncthreads();
        // one warp per right-hand side solves the diagonal tile
        const uint32_t w = tid >> 5, lane = tid & 31;
        if (w < nr) {
            const uint32_t r = w;
            float v0 = 0.f, v1 = 0.f;  // rows lane and lane+32
            if (lane < rows) v0 = __ldcg(y + size_t(rc0 + r) * n + t + rb0 + lane) -
                                  (part[0][lane][r] + part[1][lane][r] + part[2][lane][r] + part[3][lane][r]);
            if (lane + 32 < rows) v1 = __ldcg(y + size_t(rc0 + r) * n + t + rb0 + lane + 32) -
                                       (part[0][lane + 32][r] + part[1][lane + 32][r] + part[2][lane + 32][r] +
                                        part[3][lane + 32][r]);
            for (uint32_t s = 0; s < rows; ++s) {
                const uint32_t c = kLower ? s : rows - 1 - s;
                float xc = __shfl_sync(0xffffffffu, c < 32 ? v0 : v1, c & 31);
                if (!kUnit) xc = xc / tile[c][c];
                if (lane == (c & 31)) {
                    if (c < 32) v0 = xc; else v1 = xc;
                }
                // update the rows still to solve
                uint32_t i0 = lane, i1 = lane + 32;
                bool pend0 = kLower ? (i0 > c) : (i0 < c);
                bool pend1 = kLower ? (i1 > c) : (i1 < c);
                if (pend0 && i0 < rows) v0 -= tile[i0][c] * xc;
                if (pend1 && i1 < rows) v1 -= tile[i1][c] * xc;
            }
            if (lane < rows) __stcg(y + size_t(rc0 + r) * n + t + rb0 + lane, v0);
            if (lane + 32 < rows) __stcg(y + size_t(rc0 + r) * n + t + rb0 + lane + 32, v1);
        }
        __syncthreads();
    }
    if (tid == 0) {
        __threadfence();
        st_release_gpu(flags + b, 1u);
    }
}

template <int kMode>
static cudaError_t dense_sweep(const SolvePlanDev &S, const float *val, float *y, uint32_t n,
                               uint32_t nrhs, uint32_t *flags, uint32_t *ticket, uint32_t *status,
                               cudaStream_t st) {
    if (S.m == 0) return cudaSuccess;
    uint32_t nb = (S.m + kRB - 1) / kRB;
    cudaError_t e = cudaMemsetAsync(flags, 0, sizeof(uint32_t) * nb, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ticket, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_dense_trsv<kMode><<<nb, 256, 0, st>>>(val, S.doff, S.t, S.m, y, n, nrhs, flags, ticket, status);
    return cudaGetLastError();
}

static cudaError_t reset(uint32_t *counters, uint32_t n, uint32_t *ticket, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(uint32_t) * n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ticket, 0, sizeof(uint32_t), st);
    return e;
}

static inline uint32_t warp_blocks(uint32_t warps) { return (warps + 7) / 8; }

cudaError_t solve_lower_unit(const DevPattern &P, const SolvePlanDev &S, const float *val,
                             float *y, uint32_t nrhs, uint32_t *counters, uint32_t *ticket,
                             uint32_t *status, cudaStream_t st) {
    cudaError_t e;
    if (S.t > 0) {
        if ((e = reset(counters, P.n, ticket, st)) != cudaSuccess) return e;
        k_sparse_lower<<<warp_blocks(S.t), 256, 0, st>>>(P, S.t, val, y, nrhs, S.l_indeg, counters,
                                                         ticket, status);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return dense_sweep<0>(S, val, y, P.n, nrhs, counters, ticket, status, st);
}

cudaError_t solve_upper(const DevPattern &P, const SolvePlanDev &S, const float *val, float *y,
                        uint32_t nrhs, uint32_t *counters, uint32_t *ticket, uint32_t *status,
                        cudaStream_t st) {
    cudaError_t e = dense_sweep<1>(S, val, y, P.n, nrhs, counters, ticket, status, st);
    if (e != cudaSuccess) return e;
    if (S.t > 0) {
        if ((e = reset(counters, P.n, ticket, st)) != cudaSuccess) return e;
        k_sparse_upper<<<warp_blocks(P.n), 256, 0, st>>>(P, S.t, S.doff, val, y, nrhs, S.u_indeg,
                                                         counters, ticket, status);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t solve_upper_trans(const DevPattern &P, const SolvePlanDev &S, const float *val,
                              float *y, uint32_t nrhs, uint32_t *counters, uint32_t *ticket,
                              uint32_t *status, cudaStream_t st) {
    cudaError_t e;
    if (S.t > 0) {
        if ((e = reset(counters, P.n, ticket, st)) != cudaSuccess) return e;
        k_sparse_upper_trans<<<warp_blocks(P.n), 256, 0, st>>>(P, S.t, S.doff, val, y, nrhs,
                                                               counters, ticket, status);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return dense_sweep<2>(S, val, y, P.n, nrhs, counters, ticket, status, st);
}

cudaError_t solve_lower_unit_trans(const DevPattern &P, const SolvePlanDev &S, const float *val,
                                   float *y, uint32_t nrhs, uint32_t *counters, uint32_t *ticket,
                                   uint32_t *status, cudaStream_t st) {
    cudaError_t e = dense_sweep<3>(S, val, y, P.n, nrhs, counters, ticket, status, st);
    if (e != cudaSuccess) return e;
    if (S.t > 0) {
        if ((e = reset(counters, P.n, ticket, st)) != cudaSuccess) return e;
        k_sparse_lower_trans<<<warp_blocks(S.t), 256, 0, st>>>(P, S.t, val, y, nrhs, counters,
                                                               ticket, status);
        e = cudaGetLastError();
    }
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
                                                  double *norms) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t v = blockIdx.y;
    const size_t off = size_t(v) * n;
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
                            double *r, uint32_t nrhs, double *norms, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(norms, 0, sizeof(double) * 2 * nrhs, st);
    if (e != cudaSuccess) return e;
    uint32_t blocks = (n + 7) / 8;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_residual<<<dim3(blocks, nrhs, 1), 256, 0, st>>>(a_rptr, a_cidx, a_vmap, ax0, n, b, x, r, norms);
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
