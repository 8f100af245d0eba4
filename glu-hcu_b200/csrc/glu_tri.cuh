// Small dense triangular kernels shared by the supernodal and the dense
// trailing-block factorization: the LU of a w x w diagonal block (w <= 64)
// and the triangular solves of the rows of L21 and the columns of U12 against
// it.  Both follow the right-looking column algorithm of the reference
// (src/numeric.cu:10-345): every entry receives its updates in increasing
// column order, then (L entries) its division by the pivot; products are
// fused multiply-adds.
//
// The code is written as short loops over 16-column chunks whose bodies are
// unrolled (register arrays need static indices): a fully unrolled 64-step
// form is tens of kilobytes of straight-line code that every block fetches
// once, and stalls on instruction fetch.
#pragma once

#include "glu_common.cuh"

namespace glu {

constexpr int kTriMax = 64;        // largest block width
constexpr int kTriChunk = 16;      // columns per unrolled chunk
constexpr int kTriThreads = 256;   // threads of the diagonal-block LU
constexpr int kTriML = kTriMax + 4;  // leading dimension of the operand matrix (16-byte rows)

#ifdef __CUDACC__

// LU of the w x w block (w <= 64) in registers.  256 threads: thread
// (row = tid / 4, quarter q = tid % 4) holds a[jj] = A(row, 16 q + jj); rows
// and columns >= w hold zeros.  Step c: the four threads of row c publish the
// row (pivot perturbed by GESP, numeric.cu:139-140, when its column has an L
// part: c < w - 1, or c = w - 1 and last_l), one barrier, then every row
// below computes L(row, c) = A(row, c) / U(c, c) and A(row, j) -= L(row, c)
// U(c, j) for j > c.  On return a holds L (strictly lower) and U.  urow:
// 2 x 64 floats of shared memory, 16-byte aligned.
__device__ __forceinline__ void tri_diag_lu(float (&a)[kTriChunk], uint32_t w, bool last_l, float pert,
                                            float (*urow)[kTriMax]) {
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    const uint32_t row = tid >> 2, q = tid & 3;
    const uint32_t warp_last_row = (tid >> 5) * 8 + 7;
    const uint32_t nq = (w + kTriChunk - 1) / kTriChunk;
    for (uint32_t cq = 0; cq < nq; ++cq) {
#pragma unroll
        for (int jc = 0; jc < kTriChunk; ++jc) {
            const uint32_t c = cq * kTriChunk + jc;
            if (c >= w) break;
            float *u = urow[c & 1];
            if (row == c) {
                if (q == cq) {
                    const bool has_l = c + 1 < w || last_l;
                    float p = a[jc];
                    if (has_l && pert > 0.0f && fabsf(p) < pert) p = pert;
                    a[jc] = p;
                }
                float4 *u4 = reinterpret_cast<float4 *>(u + q * kTriChunk);
#pragma unroll
                for (int v = 0; v < kTriChunk / 4; ++v)
                    u4[v] = make_float4(a[4 * v], a[4 * v + 1], a[4 * v + 2], a[4 * v + 3]);
            }
            __syncthreads();
            if (warp_last_row > c) {  // the warp has rows below the pivot
                const float lsrc = __shfl_sync(0xffffffffu, a[jc], (lane & ~3u) | cq);
                if (row > c && row < w) {
                    const float l = lsrc / u[c];
                    if (q == cq) a[jc] = l;
                    const float4 *u4 = reinterpret_cast<const float4 *>(u + q * kTriChunk);
#pragma unroll
                    for (int v = 0; v < kTriChunk / 4; ++v) {
                        const float4 uv = u4[v];
                        const float us[4] = {uv.x, uv.y, uv.z, uv.w};
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const uint32_t j = q * kTriChunk + 4 * v + e;
                            if (j > c) a[4 * v + e] = fmaf(-l, us[e], a[4 * v + e]);
                        }
                    }
                }
            }
        }
    }
}

// Solve within chunk cb of one row: x = the chunk's N <= 16 entries after the
// updates of the earlier chunks; for c = 16 cb + k < w in increasing order,
// x[k] *= 1 / M(c, c) (kDiv) and x[p] -= x[k] M(c, 16 cb + p) for p > k.
// M row-major in shared memory with leading dimension kTriML; with kDiv the
// row's padding holds the pivot's reciprocal, M[c * kTriML + kTriMax] = 1 /
// M(c, c) (correctly rounded), so that the solve's dependency chain is a
// multiply and a fused multiply-add per column instead of a division (one
// extra rounding of each L entry).
template <bool kDiv, int N>
__device__ __forceinline__ void tri_chunk_solve(float (&x)[N], const float *sM, uint32_t cb, uint32_t w) {
    static_assert(N <= kTriChunk, "one chunk");
    constexpr int NV = (N + 3) / 4;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const uint32_t c = cb * kTriChunk + k;
        if (c >= w) break;
        const float4 *m4 = reinterpret_cast<const float4 *>(sM + c * kTriML + cb * kTriChunk);
        float mr[4 * NV];
#pragma unroll
        for (int v = k / 4; v < NV; ++v) {
            const float4 t = m4[v];
            mr[4 * v] = t.x; mr[4 * v + 1] = t.y; mr[4 * v + 2] = t.z; mr[4 * v + 3] = t.w;
        }
        if (kDiv) x[k] = x[k] * sM[c * kTriML + kTriMax];
#pragma unroll
        for (int p = k + 1; p < N; ++p) x[p] = fmaf(-x[k], mr[p], x[p]);
    }
}

// y (chunk cj) -= x (solved chunk cb) times M(chunk cb rows, chunk cj columns),
// rows of M in increasing order.
__device__ __forceinline__ void tri_chunk_update(float (&y)[kTriChunk], const float (&x)[kTriChunk], const float *sM,
                                                 uint32_t cb, uint32_t cj, uint32_t w) {
#pragma unroll
    for (int k = 0; k < kTriChunk; ++k) {
        const uint32_t c = cb * kTriChunk + k;
        if (c >= w) break;
        const float4 *m4 = reinterpret_cast<const float4 *>(sM + c * kTriML + cj * kTriChunk);
#pragma unroll
        for (int v = 0; v < kTriChunk / 4; ++v) {
            const float4 t = m4[v];
            y[4 * v] = fmaf(-x[k], t.x, y[4 * v]);
            y[4 * v + 1] = fmaf(-x[k], t.y, y[4 * v + 1]);
            y[4 * v + 2] = fmaf(-x[k], t.z, y[4 * v + 2]);
            y[4 * v + 3] = fmaf(-x[k], t.w, y[4 * v + 3]);
        }
    }
}

// Solve x M = a for one row per thread (kDiv: M upper triangular; else
// unit upper triangular, which with M = L^T is the column solve L x = a),
// w <= 64.  The row lives in shared memory, entry c at sW[c * ldw + t];
// entries >= w are never stored back and never used as multipliers.
template <bool kDiv>
__device__ __forceinline__ void tri_rows_solve(float *sW, uint32_t ldw, uint32_t t, const float *sM, uint32_t w) {
    const uint32_t nch = (w + kTriChunk - 1) / kTriChunk;
    for (uint32_t cb = 0; cb < nch; ++cb) {
        float x[kTriChunk];
#pragma unroll
        for (int k = 0; k < kTriChunk; ++k) x[k] = sW[(cb * kTriChunk + k) * ldw + t];
        tri_chunk_solve<kDiv>(x, sM, cb, w);
#pragma unroll
        for (int k = 0; k < kTriChunk; ++k) sW[(cb * kTriChunk + k) * ldw + t] = x[k];
        for (uint32_t cj = cb + 1; cj < nch; ++cj) {
            float y[kTriChunk];
#pragma unroll
            for (int k = 0; k < kTriChunk; ++k) y[k] = sW[(cj * kTriChunk + k) * ldw + t];
            tri_chunk_update(y, x, sM, cb, cj, w);
#pragma unroll
            for (int k = 0; k < kTriChunk; ++k) sW[(cj * kTriChunk + k) * ldw + t] = y[k];
        }
    }
}

// Four-byte asynchronous copy global -> shared (completes at tri_async_wait).
__device__ __forceinline__ void tri_async_copy(float *dst, const float *src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void tri_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void tri_async_wait() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

#endif  // __CUDACC__

}  // namespace glu
