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
//              shared memory), L21 = A21 U11^-1, U12 = L11^-1 A12;
//   2. update: A22 -= L21 U12 (register-tiled FP32).
// Each entry receives the same operations as in the column algorithm (FP32,
// different summation order).  GESP perturbation (numeric.cu:139-140) is
// applied to every pivot whose column has an L part.
#include "glu_common.cuh"
#include "glu_kernels.h"

namespace glu {

// Factor the kb x kb diagonal block at (k0, k0) of the dense block in shared
// memory sF (column-major, leading dimension kDenseNB+1).  Step c: the pivot
// is fixed (GESP), every row i > c computes L(i,c) = A(i,c) / d once, then the
// block's threads update A(i,j), j > c, with a row split into halves between
// two threads.  Returns with sF holding L11 (unit, strictly lower) and U11.
__device__ __forceinline__ void factor_diag_block(const float *__restrict__ val,
                                                  const uint32_t *__restrict__ doff, uint32_t k0,
                                                  uint32_t kb, uint32_t m, float pert,
                                                  uint32_t last_has_l, float *sF, float *lcol) {
    constexpr int LD = kDenseNB + 1;
    const uint32_t tid = threadIdx.x;
    // load: consecutive threads take consecutive rows of a column
    for (uint32_t e = tid; e < kb * kb; e += blockDim.x) {
        uint32_t j = e / kb, i = e - j * kb;
        sF[j * LD + i] = ld_cg(val + doff[k0 + j] + k0 + i);
    }
    __syncthreads();
    const uint32_t row = tid >> 1, half = tid & 1;  // 64 rows x 2 halves
    for (uint32_t c = 0; c < kb; ++c) {
        // a pivot is perturbed only when its column has an L part
        const bool has_l = (k0 + c + 1 < m) || last_has_l;
        const float d = sF[c * LD + c];
        const float de = (has_l && pert > 0.0f && fabsf(d) < pert) ? pert : d;
        if (half == 0 && row > c && row < kb) {
            float l = sF[c * LD + row] / de;
            sF[c * LD + row] = l;
            lcol[row] = l;
        }
        // (a concurrent reader sees d or pert; both give the same de)
        if (tid == 0 && de != d) sF[c * LD + c] = de;
        __syncthreads();
        if (row > c && row < kb) {
            const float l = lcol[row];
            for (uint32_t j = c + 1 + half; j < kb; j += 2) sF[j * LD + row] -= l * sF[j * LD + c];
        }
        __syncthreads();
    }
}

// Panel step.  Block 0 stores the factored diagonal block to diag_scratch (the
// update kernel writes it back, so no block here overwrites an entry another
// block may still read); blocks [1, 1+nL) compute rows of L21, the rest
// columns of U12.  blockIdx.z selects the value set.
// Full-width panel step (kb == kDenseNB), register resident: the diagonal
// block is factored with every thread holding half a row (32 values) and the
// pivot rows broadcast through shared memory, one barrier per column; the
// L21 rows and U12 columns are then solved one per thread with the whole row
// or column in registers.  Loops over columns are unrolled so that every
// register index is static.
__device__ __forceinline__ void factor_diag_regs(const float *__restrict__ val, const uint32_t *__restrict__ doff,
                                                 uint32_t k0, uint32_t m, float pert, uint32_t last_has_l,
                                                 float *sF, float (*urow)[kDenseNB]) {
    constexpr int NB = kDenseNB;
    constexpr int LD = kDenseNB + 1;
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    const uint32_t row = tid >> 1, half = tid & 1;
    float a[32];
#pragma unroll
    for (int jj = 0; jj < 32; ++jj) a[jj] = ld_cg(val + doff[k0 + half * 32 + jj] + k0 + row);
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        const int hc = c >> 5, jc = c & 31;
        float *u = urow[c & 1];
        if (row == uint32_t(c)) {
            if (half == uint32_t(hc)) {
                // a pivot is perturbed only when its column has an L part
                const bool has_l = (k0 + c + 1 < m) || last_has_l;
                float d = a[jc];
                if (has_l && pert > 0.0f && fabsf(d) < pert) d = pert;
                a[jc] = d;
            }
#pragma unroll
            for (int jj = 0; jj < 32; ++jj)
                if (int(half) * 32 + jj >= c) u[half * 32 + jj] = a[jj];
        }
        __syncthreads();
        const float lsrc = __shfl_sync(0xffffffffu, a[jc], (lane & ~1u) | uint32_t(hc));
        if (row > uint32_t(c)) {
            const float l = lsrc / u[c];
            if (half == uint32_t(hc)) a[jc] = l;
#pragma unroll
            for (int jj = 0; jj < 32; ++jj)
                if (int(half) * 32 + jj > c) a[jj] = fmaf(-l, u[half * 32 + jj], a[jj]);
        }
    }
#pragma unroll
    for (int jj = 0; jj < 32; ++jj) sF[(half * 32 + jj) * LD + row] = a[jj];
    __syncthreads();
}

__global__ void __launch_bounds__(kPanelRows, 3) k_dense_panel_full(float *val_base, uint64_t stride,
                                                                    const uint32_t *__restrict__ doff, uint32_t m,
                                                                    uint32_t k0, const float *pert_z,
                                                                    float *diag_scratch, uint32_t last_has_l,
                                                                    uint32_t nL) {
    constexpr int NB = kDenseNB;
    constexpr int LD = kDenseNB + 1;
    __shared__ float sF[NB * LD];
    __shared__ float urow[2][NB];
    float *val = val_base + blockIdx.z * stride;
    const float pert = pert_z ? pert_z[blockIdx.z] : 0.0f;
    factor_diag_regs(val, doff, k0, m, pert, last_has_l, sF, urow);
    const uint32_t r0 = k0 + NB;
    const uint32_t tid = threadIdx.x;
    if (blockIdx.x == 0) {
        float *ds = diag_scratch + size_t(blockIdx.z) * NB * NB;
        for (uint32_t e = tid; e < NB * NB; e += blockDim.x) {
            uint32_t c = e / NB, r = e - c * NB;
            ds[c * NB + r] = sF[c * LD + r];
        }
        return;
    }
    float a[NB];
    if (blockIdx.x <= nL) {
        // row of L21: x U11 = a
        const uint32_t r = r0 + (blockIdx.x - 1) * kPanelRows + tid;
        if (r >= m) return;
#pragma unroll
        for (int c = 0; c < NB; ++c) a[c] = ld_cg(val + doff[k0 + c] + r);
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            const float l = a[c] / sF[c * LD + c];
            a[c] = l;
#pragma unroll
            for (int j = c + 1; j < NB; ++j) a[j] = fmaf(-l, sF[j * LD + c], a[j]);
        }
#pragma unroll
        for (int c = 0; c < NB; ++c) st_cg(val + doff[k0 + c] + r, a[c]);
    } else {
        // column of U12: L11 x = a
        const uint32_t j = r0 + (blockIdx.x - 1 - nL) * kPanelRows + tid;
        if (j >= m) return;
        float *col = val + doff[j] + k0;
#pragma unroll
        for (int r = 0; r < NB; ++r) a[r] = ld_cg(col + r);
#pragma unroll
        for (int r = 0; r < NB; ++r) {
            const float u = a[r];
#pragma unroll
            for (int i = r + 1; i < NB; ++i) a[i] = fmaf(-sF[r * LD + i], u, a[i]);
        }
#pragma unroll
        for (int r = 0; r < NB; ++r) st_cg(col + r, a[r]);
    }
}

constexpr int kPW = kPanelRows + 1;  // leading dimension of the panel work tile
constexpr size_t kPanelSmem = sizeof(float) * (size_t(kDenseNB) * (kDenseNB + 1) + kDenseNB + size_t(kDenseNB) * kPW);

__global__ void __launch_bounds__(kPanelRows) k_dense_panel(float *val_base, uint64_t stride,
                                                            const uint32_t *__restrict__ doff,
                                                            uint32_t m, uint32_t k0, uint32_t kb,
                                                            const float *pert_z, float *diag_scratch,
                                                            uint32_t last_has_l, uint32_t nL) {
    constexpr int NB = kDenseNB;
    constexpr int LD = kDenseNB + 1;
    extern __shared__ float4 psm4[];
    float *sF = reinterpret_cast<float *>(psm4);  // diagonal block, column-major
    float *lcol = sF + NB * LD;                   // multipliers of the current step
    float *sW = lcol + NB;                        // [k][thread]: rows of L21 or columns of U12
    float *val = val_base + blockIdx.z * stride;
    float pert = pert_z ? pert_z[blockIdx.z] : 0.0f;
    factor_diag_block(val, doff, k0, kb, m, pert, last_has_l, sF, lcol);
    const uint32_t r0 = k0 + kb;
    const uint32_t tid = threadIdx.x;
    if (blockIdx.x == 0) {
        float *ds = diag_scratch + size_t(blockIdx.z) * NB * NB;
        for (uint32_t e = tid; e < kb * kb; e += blockDim.x) {
            uint32_t c = e / kb, r = e - c * kb;
            ds[c * NB + r] = sF[c * LD + r];
        }
        return;
    }
    if (blockIdx.x <= nL) {
        // row of L21, one per thread: x U11 = a, in the thread's slot of sW
        const uint32_t r = r0 + (blockIdx.x - 1) * kPanelRows + tid;
        if (r >= m) return;
        float *w = sW + tid;
        for (uint32_t c = 0; c < kb; ++c) w[c * kPW] = ld_cg(val + doff[k0 + c] + r);
        for (uint32_t c = 0; c < kb; ++c) {
            const float l = w[c * kPW] / sF[c * LD + c];
            w[c * kPW] = l;
            for (uint32_t j = c + 1; j < kb; ++j) w[j * kPW] -= l * sF[j * LD + c];
        }
        for (uint32_t c = 0; c < kb; ++c) st_cg(val + doff[k0 + c] + r, w[c * kPW]);
    } else {
        // column of U12, one per thread: L11 x = a (loaded and stored with
        // consecutive threads on consecutive rows of one column)
        const uint32_t j0 = r0 + (blockIdx.x - 1 - nL) * kPanelRows;
        const uint32_t ncol = min(uint32_t(kPanelRows), m - j0);
        for (uint32_t e = tid; e < ncol * kb; e += blockDim.x) {
            uint32_t cc = e / kb, rr = e - cc * kb;
            sW[rr * kPW + cc] = ld_cg(val + doff[j0 + cc] + k0 + rr);
        }
        __syncthreads();
        if (tid < ncol) {
            float *w = sW + tid;
            for (uint32_t rr = 0; rr < kb; ++rr) {
                const float u = w[rr * kPW];
                for (uint32_t i = rr + 1; i < kb; ++i) w[i * kPW] -= sF[rr * LD + i] * u;
            }
        }
        __syncthreads();
        for (uint32_t e = tid; e < ncol * kb; e += blockDim.x) {
            uint32_t cc = e / kb, rr = e - cc * kb;
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

cudaError_t launch_dense_panel(float *val, uint64_t stride, uint32_t count, const uint32_t *doff,
                               uint32_t m, uint32_t k0, uint32_t kb, const float *pert_z,
                               float *diag_scratch, uint32_t last_has_l, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_dense_panel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(kPanelSmem));
        if (e != cudaSuccess) return e;
        attr = true;
    }
    uint32_t rest = m - (k0 + kb);
    uint32_t nL = (rest + kPanelRows - 1) / kPanelRows;
    uint32_t nU = nL;
    dim3 grid(1 + nL + nU, 1, count);
    if (kb == uint32_t(kDenseNB))
        k_dense_panel_full<<<grid, kPanelRows, 0, st>>>(val, stride, doff, m, k0, pert_z, diag_scratch, last_has_l, nL);
    else
        k_dense_panel<<<grid, kPanelRows, kPanelSmem, st>>>(val, stride, doff, m, k0, kb, pert_z, diag_scratch,
                                                            last_has_l, nL);
    return cudaGetLastError();
}

cudaError_t launch_dense_update(float *val, uint64_t stride, uint32_t count, const uint32_t *doff,
                                uint32_t m, uint32_t k0, uint32_t kb, const float *diag_scratch,
                                DenseRegion reg, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_dense_update<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(UpdateTile<128>::Smem));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_dense_update<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(UpdateTile<64>::Smem));
        if (e != cudaSuccess) return e;
        attr = true;
    }
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
