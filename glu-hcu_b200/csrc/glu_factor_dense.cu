// Dense trailing block of the numeric factorization, factored in place.
//
// The circuit and grid matrices this engine targets end in a trailing block
// [t, n) x [t, n) in which every entry is in the L+U pattern.  In the CSC
// layout the rows t..n-1 of each such column are its last m = n - t entries,
// so the block is a column-major matrix with one base offset per column
// (element (i, j) at val[doff[j] + i]) and can be factored where it lies,
// without a copy.  The right-looking column algorithm of the reference
// (src/numeric.cu:10-345) applied to this block is the unpivoted dense LU; it
// is computed here blocked (panel width kDenseNB):
//   1. panel:  A11 = L11 U11 (every block factors the small diagonal block in
//              registers), L21 = A21 U11^-1, U12 = L11^-1 A12;
//   2. update: A22 -= L21 U12 (register-tiled FP32).
// Each entry receives the same operations as in the column algorithm (FP32,
// different summation order; L21 entries are multiplied by the pivot's
// correctly rounded reciprocal instead of divided by the pivot).  GESP
// perturbation (numeric.cu:139-140) is applied to every pivot whose column
// has an L part.
#include "glu_common.cuh"
#include "glu_kernels.h"
#include "glu_tri.cuh"

namespace glu {

// Panel step (kb <= kDenseNB columns at k0).  Every block factors the
// diagonal block itself (tri_diag_lu, 256 threads); block 0 stores it to
// diag_scratch (the update kernel writes it back, so no block here overwrites
// an entry another block may still read); blocks [1, 1 + nL) then solve 128
// rows of L21 (x U11 = a), the rest 128 columns of U12 (L11 x = a), one per
// thread, chunked (tri_rows_solve).  The rows or columns are copied to shared
// memory asynchronously while the diagonal block is factored.  blockIdx.z
// selects the value set.  With from_scratch set, block b of the launch is
// block b + 1 of the step and takes the diagonal block already factored into
// diag_scratch by a launch of block 0 alone (the same code, so the same
// values) instead of factoring it again: for many value sets the redundant
// factorizations would outweigh the row solves.
constexpr int kPW = kPanelRows + 1;  // leading dimension of the panel work tile
constexpr size_t kPanelSmem =
    sizeof(float) * (size_t(kDenseNB) * kPW + size_t(kDenseNB) * kTriML + 2 * kTriMax) + sizeof(uint32_t) * kDenseNB;
static_assert(kDenseNB == kTriMax, "panel width is the triangular block width");
static_assert(2 * kPanelRows == kTriThreads, "128 rows per panel block");

__global__ void __launch_bounds__(kTriThreads) k_dense_panel(float *val_base, uint64_t stride,
                                                             const uint32_t *__restrict__ doff, uint32_t m,
                                                             uint32_t k0, uint32_t kb, const float *pert_z,
                                                             float *diag_scratch, uint32_t last_has_l, uint32_t nL,
                                                             uint32_t from_scratch) {
    extern __shared__ float4 psm4[];
    float *sW = reinterpret_cast<float *>(psm4);  // [k][thread]: rows of L21 or columns of U12
    float *sM = sW + kDenseNB * kPW;               // U11 (row-major, pivot reciprocals in the padding) or L11^T
    float(*urow)[kTriMax] = reinterpret_cast<float(*)[kTriMax]>(sM + kDenseNB * kTriML);
    uint32_t *sCol = reinterpret_cast<uint32_t *>(sM + kDenseNB * kTriML + 2 * kTriMax);
    float *val = val_base + blockIdx.z * stride;
    const float pert = pert_z ? pert_z[blockIdx.z] : 0.0f;
    const uint32_t tid = threadIdx.x, b = blockIdx.x + from_scratch;
    const uint32_t r0 = k0 + kb;
    if (tid < kb) sCol[tid] = doff[k0 + tid] + k0;
    // this block's rows (columns) of the panel, in flight during the LU
    if (b >= 1 && b <= nL) {
        const uint32_t rb = r0 + (b - 1) * kPanelRows;
        for (uint32_t e = tid; e < kb * kPanelRows; e += kTriThreads) {
            const uint32_t c = e / kPanelRows, t = e - c * kPanelRows;
            if (rb + t < m) tri_async_copy(sW + c * kPW + t, val + doff[k0 + c] + rb + t);
        }
    } else if (b > nL) {
        const uint32_t j0 = r0 + (b - 1 - nL) * kPanelRows;
        const uint32_t ncol = min(uint32_t(kPanelRows), m - j0);
        for (uint32_t e = tid; e < ncol * kb; e += kTriThreads) {
            const uint32_t cc = e / kb, rr = e - cc * kb;
            tri_async_copy(sW + rr * kPW + cc, val + doff[j0 + cc] + k0 + rr);
        }
    }
    tri_async_commit();
    __syncthreads();
    // the diagonal block
    const uint32_t row = tid >> 2, q = tid & 3;
    float a[kTriChunk];
    if (from_scratch) {
        const float *ds = diag_scratch + size_t(blockIdx.z) * kDenseNB * kDenseNB;
#pragma unroll
        for (int jj = 0; jj < kTriChunk; ++jj) {
            const uint32_t cc = q * kTriChunk + jj;
            a[jj] = (row < kb && cc < kb) ? ld_cg(ds + cc * kDenseNB + row) : 0.0f;
        }
    } else {
#pragma unroll
        for (int jj = 0; jj < kTriChunk; ++jj) {
            const uint32_t cc = q * kTriChunk + jj;
            a[jj] = (row < kb && cc < kb) ? ld_cg(val + sCol[cc] + row) : 0.0f;
        }
        // a pivot is perturbed only when its column has an L part
        tri_diag_lu(a, kb, (r0 < m) || last_has_l, pert, urow);
    }
    if (b == 0) {
        float *ds = diag_scratch + size_t(blockIdx.z) * kDenseNB * kDenseNB;
#pragma unroll
        for (int jj = 0; jj < kTriChunk; ++jj) {
            const uint32_t cc = q * kTriChunk + jj;
            if (row < kb && cc < kb) ds[cc * kDenseNB + row] = a[jj];
        }
        tri_async_wait();
        return;
    }
    const bool lrows = b <= nL;
#pragma unroll
    for (int jj = 0; jj < kTriChunk; ++jj) {
        const uint32_t cc = q * kTriChunk + jj;
        if (lrows)
            sM[row * kTriML + cc] = a[jj];  // M = U11 (row-major)
        else
            sM[cc * kTriML + row] = a[jj];  // M = L11^T
    }
    if (lrows) {
        __syncthreads();
        if (tid < kb) sM[tid * kTriML + kTriMax] = 1.0f / sM[tid * kTriML + tid];
    }
    tri_async_wait();
    __syncthreads();
    if (tid < kPanelRows) {
        if (lrows)
            tri_rows_solve<true>(sW, kPW, tid, sM, kb);
        else
            tri_rows_solve<false>(sW, kPW, tid, sM, kb);
    }
    __syncthreads();
    if (lrows) {
        const uint32_t rb = r0 + (b - 1) * kPanelRows;
        for (uint32_t e = tid; e < kb * kPanelRows; e += kTriThreads) {
            const uint32_t c = e / kPanelRows, t = e - c * kPanelRows;
            if (rb + t < m) st_cg(val + doff[k0 + c] + rb + t, sW[c * kPW + t]);
        }
    } else {
        const uint32_t j0 = r0 + (b - 1 - nL) * kPanelRows;
        const uint32_t ncol = min(uint32_t(kPanelRows), m - j0);
        for (uint32_t e = tid; e < ncol * kb; e += kTriThreads) {
            const uint32_t cc = e / kb, rr = e - cc * kb;
            st_cg(val + doff[j0 + cc] + k0 + rr, sW[rr * kPW + cc]);
        }
    }
}

// Trailing update A22 -= L21 U12 on a TB x TB tile per block (256 threads as a
// 16 x 16 grid, RM x RM outputs each, K = kb <= 64 staged once in shared
// memory).  TB = 128 for large trailing blocks, 64 when 128-wide tiles would
// leave SMs idle.  Block (0,0) first writes the factored diagonal block back
// from diag_scratch.
template <int TB>
struct UpdateTile {
    static constexpr int RM = TB / 16;
    static constexpr int LDB = TB + 4;
    static constexpr int LDC = TB + 1;
    static constexpr size_t AB = (size_t(kDenseNB) * TB + size_t(kDenseNB) * LDB) * 4;
    static constexpr size_t C = size_t(TB) * LDC * 4;
    static constexpr size_t Smem = AB > C ? AB : C;
};

template <int TB>
__global__ void __launch_bounds__(256, 2) k_dense_update(float *val_base, uint64_t stride,
                                                         const uint32_t *__restrict__ doff,
                                                         uint32_t m, uint32_t k0, uint32_t kb,
                                                         const float *diag_scratch, DenseRegion reg) {
    constexpr int RM = UpdateTile<TB>::RM;
    constexpr int LDB = UpdateTile<TB>::LDB;
    constexpr int LDC = UpdateTile<TB>::LDC;
    extern __shared__ float4 smem4[];
    float *smem = reinterpret_cast<float *>(smem4);
    float *sA = smem;                    // [k][row]
    float *sB = smem + kDenseNB * TB;    // [k][col], padded
    float *sC = smem;                    // [col][row], padded (reuses sA/sB)
    float *val = val_base + blockIdx.z * stride;
    const uint32_t tid = threadIdx.x;
    if (reg.writeback && blockIdx.x == 0 && blockIdx.y == 0) {
        // the factored diagonal block of the panel at wb_k0, kept in scratch
        // while that panel's blocks still read the original
        const float *ds = diag_scratch + size_t(blockIdx.z) * kDenseNB * kDenseNB;
        const uint32_t wk = reg.wb_k0, wb = min(uint32_t(kDenseNB), m - wk);
        for (uint32_t e = tid; e < wb * wb; e += blockDim.x) {
            uint32_t c = e / wb, r = e - c * wb;
            st_cg(val + doff[wk + c] + wk + r, ds[c * kDenseNB + r]);
        }
    }
    const uint32_t r0 = k0 + kb;
    if (r0 >= m) return;
    // tile of the trailing block: rows [rbase, rbase + TB) of [r_lo, r_hi),
    // columns [cbase, cbase + TB) of [c_lo, c_hi)
    const uint32_t rbase = reg.r_lo + blockIdx.x * TB, cbase = reg.c_lo + blockIdx.y * TB;
    const uint32_t rlim = reg.r_hi, mp = reg.c_hi;  // (mp: column limit)
    if (rbase >= rlim || cbase >= mp) return;
    const uint32_t tx = tid & 15, ty = tid >> 4;
    // C tile into registers (through shared memory for coalescing): every
    // entry then receives its updates one k at a time, in increasing k, as in
    // the column algorithm.  (Loops unrolled so that many loads are in flight.)
#pragma unroll 16
    for (uint32_t e = tid; e < uint32_t(TB) * TB; e += 256) {
        uint32_t col = e / TB, row = e - col * TB;
        float v = 0.0f;
        if (cbase + col < mp && rbase + row < rlim) v = ld_cg(val + doff[r0 + cbase + col] + r0 + rbase + row);
        sC[col * LDC + row] = v;
    }
    __syncthreads();
    float acc[RM][RM];
#pragma unroll
    for (int j = 0; j < RM; ++j)
#pragma unroll
        for (int i = 0; i < RM; ++i) acc[i][j] = sC[(tx * RM + j) * LDC + ty * RM + i];
    __syncthreads();
    // K = kb (one or two panels) in chunks of kDenseNB, in increasing k
    for (uint32_t kc = 0; kc < kb; kc += kDenseNB) {
        const uint32_t kn = min(uint32_t(kDenseNB), kb - kc);
        // stage L21 tile: sA[k][row]
#pragma unroll 16
        for (uint32_t e = tid; e < uint32_t(kDenseNB) * TB; e += 256) {
            uint32_t k = e / TB, row = e - k * TB;
            float v = 0.0f;
            if (k < kn && rbase + row < rlim) v = ld_cg(val + doff[k0 + kc + k] + r0 + rbase + row);
            sA[k * TB + row] = v;
        }
        // stage U12 tile: sB[k][col]; lanes run along k (contiguous in memory)
        {
            uint32_t lane = tid & 31, w = tid >> 5;
#pragma unroll 8
            for (uint32_t col = w; col < uint32_t(TB); col += 8) {
                bool cok = cbase + col < mp;
                const float *src = cok ? val + doff[r0 + cbase + col] + k0 + kc : nullptr;
#pragma unroll
                for (uint32_t h = 0; h < uint32_t(kDenseNB); h += 32) {
                    uint32_t k = h + lane;
                    float v = (cok && k < kn) ? ld_cg(src + k) : 0.0f;
                    sB[k * LDB + col] = v;
                }
            }
        }
        __syncthreads();
#pragma unroll 4
        for (uint32_t k = 0; k < kn; ++k) {
            float av[RM], bv[RM];
#pragma unroll
            for (int q = 0; q < RM; q += 4) {
                float4 a4 = *reinterpret_cast<const float4 *>(sA + k * TB + ty * RM + q);
                float4 b4 = *reinterpret_cast<const float4 *>(sB + k * LDB + tx * RM + q);
                av[q] = a4.x; av[q + 1] = a4.y; av[q + 2] = a4.z; av[q + 3] = a4.w;
                bv[q] = b4.x; bv[q + 1] = b4.y; bv[q + 2] = b4.z; bv[q + 3] = b4.w;
            }
#pragma unroll
            for (int i = 0; i < RM; ++i)
#pragma unroll
                for (int j = 0; j < RM; ++j) acc[i][j] = fmaf(-av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RM; ++j)
#pragma unroll
        for (int i = 0; i < RM; ++i) sC[(tx * RM + j) * LDC + ty * RM + i] = acc[i][j];
    __syncthreads();
#pragma unroll 4
    for (uint32_t e = tid; e < uint32_t(TB) * TB; e += 256) {
        uint32_t col = e / TB, row = e - col * TB;
        if (cbase + col < mp && rbase + row < rlim)
            st_cg(val + doff[r0 + cbase + col] + r0 + rbase + row, sC[col * LDC + row]);
    }
}

uint32_t dense_panel_launches(uint32_t count, uint32_t m, uint32_t k0, uint32_t kb, uint32_t num_sms) {
    const uint32_t nL = (m - (k0 + kb) + kPanelRows - 1) / kPanelRows;
    return (nL && uint64_t(count) * (1 + 2 * nL) > 4ull * num_sms) ? 2u : 1u;
}

cudaError_t launch_dense_panel(float *val, uint64_t stride, uint32_t count, const uint32_t *doff,
                               uint32_t m, uint32_t k0, uint32_t kb, const float *pert_z,
                               float *diag_scratch, uint32_t last_has_l, uint32_t num_sms, cudaStream_t st) {
    static PerDeviceOnce attr;
    cudaError_t e = attr.run([] {
        return cudaFuncSetAttribute(k_dense_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kPanelSmem));
    });
    if (e != cudaSuccess) return e;
    uint32_t rest = m - (k0 + kb);
    uint32_t nL = (rest + kPanelRows - 1) / kPanelRows;
    uint32_t nU = nL;
    // more blocks than a few waves: factor the diagonal blocks once, then the
    // rows and columns from them (one launch more, the LU not repeated per block)
    if (dense_panel_launches(count, m, k0, kb, num_sms) == 2) {
        k_dense_panel<<<dim3(1, 1, count), kTriThreads, kPanelSmem, st>>>(val, stride, doff, m, k0, kb, pert_z,
                                                                           diag_scratch, last_has_l, nL, 0);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        k_dense_panel<<<dim3(nL + nU, 1, count), kTriThreads, kPanelSmem, st>>>(val, stride, doff, m, k0, kb, pert_z,
                                                                                 diag_scratch, last_has_l, nL, 1);
        return cudaGetLastError();
    }
    dim3 grid(1 + nL + nU, 1, count);
    k_dense_panel<<<grid, kTriThreads, kPanelSmem, st>>>(val, stride, doff, m, k0, kb, pert_z, diag_scratch,
                                                          last_has_l, nL, 0);
    return cudaGetLastError();
}

cudaError_t launch_dense_update(float *val, uint64_t stride, uint32_t count, const uint32_t *doff,
                                uint32_t m, uint32_t k0, uint32_t kb, const float *diag_scratch,
                                DenseRegion reg, cudaStream_t st) {
    static PerDeviceOnce attr;
    cudaError_t e = attr.run([] {
        cudaError_t r = cudaFuncSetAttribute(k_dense_update<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(UpdateTile<128>::Smem));
        if (r == cudaSuccess)
            r = cudaFuncSetAttribute(k_dense_update<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(UpdateTile<64>::Smem));
        return r;
    });
    if (e != cudaSuccess) return e;
    const uint32_t rows = reg.r_hi > reg.r_lo ? reg.r_hi - reg.r_lo : 0;
    const uint32_t cols = reg.c_hi > reg.c_lo ? reg.c_hi - reg.c_lo : 0;
    if ((rows == 0 || cols == 0) && !reg.writeback) return cudaSuccess;
    const uint32_t r128 = (rows + 127) / 128, c128 = (cols + 127) / 128;
    if (uint64_t(r128) * c128 * count >= 2 * 148) {
        dim3 grid(r128, c128, count);
        k_dense_update<128><<<grid, 256, UpdateTile<128>::Smem, st>>>(val, stride, doff, m, k0, kb, diag_scratch, reg);
    } else {
        dim3 grid(std::max<uint32_t>((rows + 63) / 64, 1), std::max<uint32_t>((cols + 63) / 64, 1), count);
        k_dense_update<64><<<grid, 256, UpdateTile<64>::Smem, st>>>(val, stride, doff, m, k0, kb, diag_scratch, reg);
    }
    return cudaGetLastError();
}

// ------------------------------------------------ dense buffer gather/scatter --
// One warp per tail column; blockIdx.z selects the value set.
__global__ void __launch_bounds__(256) k_dense_gather(DevPattern P, const float *__restrict__ val_base,
                                                      uint64_t stride, uint32_t t, uint32_t m,
                                                      const uint32_t *__restrict__ tail_start, float *dbuf) {
    const float *val = val_base + blockIdx.z * stride;
    float *D = dbuf + size_t(blockIdx.z) * m * m;
    const uint32_t j = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (j >= m) return;
    float *col = D + size_t(j) * m;
    for (uint32_t p = tail_start[j] + lane; p < P.cptr[t + j + 1]; p += 32) col[P.ridx[p] - t] = val[p];
}

__global__ void __launch_bounds__(256) k_dense_scatter(DevPattern P, float *val_base, uint64_t stride,
                                                       uint32_t t, uint32_t m,
                                                       const uint32_t *__restrict__ tail_start,
                                                       const float *__restrict__ dbuf) {
    float *val = val_base + blockIdx.z * stride;
    const float *D = dbuf + size_t(blockIdx.z) * m * m;
    const uint32_t j = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (j >= m) return;
    const float *col = D + size_t(j) * m;
    for (uint32_t p = tail_start[j] + lane; p < P.cptr[t + j + 1]; p += 32) val[p] = col[P.ridx[p] - t];
}

cudaError_t launch_dense_gather(const DevPattern &P, const float *val, uint64_t stride, uint32_t count,
                                uint32_t t, uint32_t m, const uint32_t *tail_start, float *dbuf,
                                cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(dbuf, 0, sizeof(float) * size_t(m) * m * count, st);
    if (e != cudaSuccess) return e;
    k_dense_gather<<<dim3((m + 7) / 8, 1, count), 256, 0, st>>>(P, val, stride, t, m, tail_start, dbuf);
    return cudaGetLastError();
}

cudaError_t launch_dense_scatter(const DevPattern &P, float *val, uint64_t stride, uint32_t count,
                                 uint32_t t, uint32_t m, const uint32_t *tail_start, const float *dbuf,
                                 cudaStream_t st) {
    k_dense_scatter<<<dim3((m + 7) / 8, 1, count), 256, 0, st>>>(P, val, stride, t, m, tail_start, dbuf);
    return cudaGetLastError();
}

// --------------------------------------------------------------- utilities --
__global__ void k_colsum(DevPattern P, const float *val_base, uint64_t stride, float *colmax) {
    const float *val = val_base + blockIdx.z * stride;
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    float tmp = 0.0f;
    if (c < P.n) {
        // same order and precision as the reference's host loop (numeric.cu:495-502)
        for (uint32_t p = P.cptr[c]; p < P.cptr[c + 1]; ++p) tmp += fabsf(val[p]);
    }
    // block max, then one atomic (non-negative floats compare as integers)
    for (int o = 16; o > 0; o >>= 1) tmp = fmaxf(tmp, __shfl_xor_sync(0xffffffffu, tmp, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(colmax + blockIdx.z), __float_as_int(tmp));
}

__global__ void k_pert_finish(const float *colmax, float *pert_z, uint32_t count) {
    uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z < count) pert_z[z] = 3.45e-4f * colmax[z];
}

cudaError_t launch_pert(const DevPattern &P, const float *val, uint64_t stride, uint32_t count,
                        float *colsum_scratch, float *pert_z, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(colsum_scratch, 0, sizeof(float) * count, st);
    if (e != cudaSuccess) return e;
    k_colsum<<<dim3((P.n + 255) / 256, 1, count), 256, 0, st>>>(P, val, stride, colsum_scratch);
    k_pert_finish<<<(count + 255) / 256, 256, 0, st>>>(colsum_scratch, pert_z, count);
    return cudaGetLastError();
}

__global__ void k_check_pivots(DevPattern P, const float *val_base, uint64_t stride, uint32_t *status) {
    const float *val = val_base + blockIdx.z * stride;
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t flag = 0;
    if (c < P.n) {
        float d = val[P.diag[c]];
        if (d == 0.0f) flag |= DEV_ZERO_PIVOT;
        if (!isfinite(d)) flag |= DEV_NONFINITE_PIVOT;
    }
    flag = __reduce_or_sync(0xffffffffu, flag);
    if (flag && (threadIdx.x & 31) == 0) atomicOr(status, flag);
}

cudaError_t launch_check_pivots(const DevPattern &P, const float *val, uint64_t stride,
                                uint32_t count, uint32_t *status, cudaStream_t st) {
    k_check_pivots<<<dim3((P.n + 255) / 256, 1, count), 256, 0, st>>>(P, val, stride, status);
    return cudaGetLastError();
}

__global__ void k_gather_values(const int64_t *__restrict__ lu_src, const double *__restrict__ ax_base,
                                uint64_t ax_stride, const double *__restrict__ scale, uint32_t nnz,
                                float *val_base, uint64_t stride) {
    const double *ax = ax_base + blockIdx.z * ax_stride;
    float *val = val_base + blockIdx.z * stride;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x) {
        int64_t q = __ldg(lu_src + p);
        float v = 0.0f;
        if (q >= 0) {
            double a = ax[q];
            if (scale) a = a * __ldg(scale + q);
            v = static_cast<float>(a);
        }
        val[p] = v;
    }
}

cudaError_t launch_gather_values(const int64_t *lu_src, const double *ax, uint64_t ax_stride,
                                 const double *scale, uint32_t nnz, float *val, uint64_t stride,
                                 uint32_t count, cudaStream_t st) {
    uint32_t blocks = (nnz + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks == 0) blocks = 1;
    k_gather_values<<<dim3(blocks, 1, count), 256, 0, st>>>(lu_src, ax, ax_stride, scale, nnz, val, stride);
    return cudaGetLastError();
}

}  // namespace glu
