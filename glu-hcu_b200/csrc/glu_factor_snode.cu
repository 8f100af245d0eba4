// Supernodal form of the sparse factorization.
//
// The same right-looking column algorithm as the level kernels
// (src/numeric.cu:10-345), with runs of columns grouped.  A supernode is a run
// of columns [s, s+w), w <= kSnMaxWidth, whose lower parts are nested
// (Lpat(c) = {c+1} u Lpat(c+1)) and whose diagonal block is dense.  In the CSC
// layout every column c of it then holds the rows s..s+w-1 at consecutive
// positions (diag[c] - (c - s) onward) followed by the same m rows below the
// block, so the supernode is a dense (w + m) x w panel with one base offset
// per column, stored where it lies.  Column l = s + w - 1 is the last one; its
// U row lists the update targets j of the whole supernode, and in every target
// column the rows of the supernode present form a suffix k0..l (fill closure).
//
// Supernodes are leveled by the reference's column dependencies
// (symbolic.cc:106-151) contracted to supernodes.  Per level two launches:
//   panel:  A11 = L11 U11 (GESP pivots, numeric.cu:139-140), L21 = A21 U11^-1,
//           U12(:, j) = L11^-1 A12(:, j) for every target j;
//   update: A(rows of L21, j) -= L21 U12(:, j) for every target j, as 64 x 64
//           output tiles (FP32 FMA, K = w), scattered to the CSC positions of
//           column j found by search in its row list.
// Every entry receives the operations of the column algorithm in the same
// column order (fused multiply-add instead of multiply and subtract).  The
// panel blocks of a supernode each factor its diagonal block; the factored
// block goes to scratch and the update launch stores it.
#include "glu_common.cuh"
#include "glu_kernels.h"

namespace glu {

namespace {

constexpr int kLD = kSnMaxWidth + 1;  // leading dimension of the diagonal block in shared memory
constexpr int kTile = 64;             // update tile: 64 rows x 64 targets
constexpr int kTLd = kTile + 4;       // leading dimension of the update operand tiles

struct Sn {
    uint32_t s, w, l, m, nt;
};

__device__ __forceinline__ Sn sn_load(const DevPattern &P, const SnPlanDev &S, uint32_t i) {
    Sn d;
    d.s = S.sn_col[i];
    d.w = S.sn_w[i];
    d.l = d.s + d.w - 1;
    d.m = P.cptr[d.l + 1] - P.diag[d.l] - 1;
    d.nt = P.rptr[d.l + 1] - P.rdiag[d.l] - 1;
    return d;
}

// Number of rows of the supernode (ending at l, width w) present in target
// column j, whose row l sits at position pl: rows l, l-1, ... occupy
// pl, pl-1, ... while ridx[pl - i] == l - i.
__device__ __forceinline__ uint32_t seg_len(const DevPattern &P, uint32_t j, uint32_t pl, uint32_t l, uint32_t w) {
    uint32_t lo = 1, hi = min(w, pl - P.cptr[j] + 1);
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(P.ridx + pl - (mid - 1)) == l - (mid - 1))
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Factor the w x w diagonal block into sF (column-major, leading dimension
// kLD): unit L11 strictly below, U11 on and above the diagonal.  Pivot c is
// perturbed (GESP) when its column has an L part: c < w-1, or m > 0.
// 128 threads: thread = (row, half of the columns).
__device__ __forceinline__ void sn_factor_diag(const DevPattern &P, const float *__restrict__ val, const Sn &d,
                                               float pert, float *sF, float *lcol) {
    const uint32_t tid = threadIdx.x;
    const uint32_t w = d.w;
    for (uint32_t e = tid; e < w * w; e += blockDim.x) {
        const uint32_t cc = e / w, i = e - cc * w;
        sF[cc * kLD + i] = ld_cg(val + P.diag[d.s + cc] + i - cc);
    }
    __syncthreads();
    const uint32_t row = tid >> 1, half = tid & 1;
    for (uint32_t c = 0; c < w; ++c) {
        const bool has_l = (c + 1 < w) || d.m > 0;
        const float p = sF[c * kLD + c];
        const float de = (has_l && pert > 0.0f && fabsf(p) < pert) ? pert : p;
        if (half == 0 && row > c && row < w) {
            const float l = sF[c * kLD + row] / de;
            sF[c * kLD + row] = l;
            lcol[row] = l;
        }
        if (tid == 0 && de != p) sF[c * kLD + c] = de;
        __syncthreads();
        if (row > c && row < w) {
            const float l = lcol[row];
            for (uint32_t j = c + 1 + half; j < w; j += 2) sF[j * kLD + row] = fmaf(-l, sF[j * kLD + c], sF[j * kLD + row]);
        }
        __syncthreads();
    }
}

// Row r of L21: x U11 = a (a = row r of A21), W >= w columns in registers.
template <int W>
__device__ __forceinline__ void sn_l21_row(float *__restrict__ val, const uint32_t *sOff, uint32_t w, uint32_t r,
                                           const float *sF) {
    float a[W];
#pragma unroll
    for (int c = 0; c < W; ++c) a[c] = uint32_t(c) < w ? ld_cg(val + sOff[c] + r) : 0.0f;
#pragma unroll
    for (int c = 0; c < W; ++c) {
        if (uint32_t(c) < w) {
            const float l = a[c] / sF[c * kLD + c];
            a[c] = l;
#pragma unroll
            for (int j = c + 1; j < W; ++j) a[j] = fmaf(-l, sF[j * kLD + c], a[j]);
        }
    }
#pragma unroll
    for (int c = 0; c < W; ++c)
        if (uint32_t(c) < w) st_cg(val + sOff[c] + r, a[c]);
}

// Target column j of U12: L11 x = a over the supernode's rows present in
// column j (a suffix of length len; the rows above it are structural zeros).
template <int W>
__device__ __forceinline__ void sn_u12_col(float *__restrict__ val, uint32_t pl, uint32_t len, uint32_t w,
                                           const float *sF) {
    float a[W];
    const uint32_t z = w - len;  // first row present
#pragma unroll
    for (int k = 0; k < W; ++k) a[k] = (uint32_t(k) < w && uint32_t(k) >= z) ? ld_cg(val + pl - (w - 1 - k)) : 0.0f;
#pragma unroll
    for (int r = 0; r < W; ++r) {
        if (uint32_t(r) < w && uint32_t(r) >= z) {
            const float u = a[r];
#pragma unroll
            for (int i = r + 1; i < W; ++i) a[i] = fmaf(-sF[r * kLD + i], u, a[i]);  // a[i >= w] unused
        }
    }
#pragma unroll
    for (int k = 0; k < W; ++k)
        if (uint32_t(k) < w && uint32_t(k) >= z) st_cg(val + pl - (w - 1 - k), a[k]);
}

template <int W>
__device__ __forceinline__ void sn_panel_rows(const DevPattern &P, float *__restrict__ val, const Sn &d,
                                              uint32_t role, uint32_t q, const uint32_t *sOff, const float *sF) {
    const uint32_t tid = threadIdx.x;
    if (role == 1) {
        const uint32_t r = q * kSnPanelThreads + tid;
        if (r < d.m) sn_l21_row<W>(val, sOff, d.w, r, sF);
    } else {
        const uint32_t jt = q * kSnPanelThreads + tid;
        if (jt < d.nt) {
            const uint32_t e = P.rdiag[d.l] + 1 + jt;
            const uint32_t pl = P.cpos[e];
            const uint32_t len = seg_len(P, P.cidx[e], pl, d.l, d.w);
            sn_u12_col<W>(val, pl, len, d.w, sF);
        }
    }
}

}  // namespace

// Panel launch of one level: supernodes [i0, i1) of the level order, blocks
// S.pblk[i0] .. S.pblk[i1).  Per supernode of width w >= 2: block 0 stores the
// factored diagonal block to scratch, then ceil(m / T) blocks of L21 rows and
// ceil(nt / T) blocks of U12 columns (T = kSnPanelThreads).  Width 1: ceil(m / T)
// blocks scale the column.  blockIdx.z selects the value set.
__global__ void __launch_bounds__(kSnPanelThreads, 2) k_sn_panel(DevPattern P, SnPlanDev S, float *val_base,
                                                                 uint64_t stride, const float *pert_z,
                                                                 float *scr_base, uint64_t scr_stride,
                                                                 uint32_t i0, uint32_t i1) {
    __shared__ float sF[kSnMaxWidth * kLD];
    __shared__ float lcol[kSnMaxWidth];
    __shared__ uint32_t sOff[kSnMaxWidth];
    float *val = val_base + blockIdx.z * stride;
    const float pert = pert_z ? pert_z[blockIdx.z] : 0.0f;
    const uint32_t b = S.pblk[i0] + blockIdx.x;
    const uint32_t i = upper_slot(S.pblk, i0, i1, b);
    const Sn d = sn_load(P, S, i);
    const uint32_t tid = threadIdx.x;
    uint32_t t = b - S.pblk[i];
    if (d.w == 1) {
        // numeric.cu:133-143: pivot (perturbed when the column has an L part), L /= pivot
        const uint32_t dk = P.diag[d.s];
        const uint32_t r = t * kSnPanelThreads + tid;
        const float p = ld_cg(val + dk);
        const float de = (pert > 0.0f && fabsf(p) < pert) ? pert : p;  // m > 0 here
        if (r < d.m) st_cg(val + dk + 1 + r, ld_cg(val + dk + 1 + r) / de);
        // (a concurrent reader of the pivot sees p or pert; both give de)
        if (t == 0 && tid == 0 && de != p) st_cg(val + dk, de);
        return;
    }
    if (tid < d.w) sOff[tid] = P.diag[d.s + tid] + (d.l + 1 - (d.s + tid));
    sn_factor_diag(P, val, d, pert, sF, lcol);
    if (t == 0) {
        float *scr = scr_base + blockIdx.z * scr_stride + S.dscr[i];
        for (uint32_t e = tid; e < d.w * d.w; e += blockDim.x) {
            const uint32_t cc = e / d.w, r = e - cc * d.w;
            scr[e] = sF[cc * kLD + r];
        }
        return;
    }
    t -= 1;
    const uint32_t nLb = (d.m + kSnPanelThreads - 1) / kSnPanelThreads;
    const uint32_t role = t < nLb ? 1u : 2u;
    const uint32_t q = role == 1 ? t : t - nLb;
    if (d.w <= 2)
        sn_panel_rows<2>(P, val, d, role, q, sOff, sF);
    else if (d.w <= 4)
        sn_panel_rows<4>(P, val, d, role, q, sOff, sF);
    else if (d.w <= 8)
        sn_panel_rows<8>(P, val, d, role, q, sOff, sF);
    else if (d.w <= 16)
        sn_panel_rows<16>(P, val, d, role, q, sOff, sF);
    else if (d.w <= 32)
        sn_panel_rows<32>(P, val, d, role, q, sOff, sF);
    else
        sn_panel_rows<64>(P, val, d, role, q, sOff, sF);
}

// Update launch of one level: blocks S.ublk[i0] .. S.ublk[i1).  Per supernode
// of width >= 2, block 0 stores the factored diagonal block from scratch; the
// others are the 64 x 64 tiles of the update (row tiles fastest).  Levels with
// several supernodes accumulate with atomics (numeric.cu:82); a single
// supernode updates each entry from one thread: C is loaded, the K products
// are applied in column order, C is stored.
__global__ void __launch_bounds__(256) k_sn_update(DevPattern P, SnPlanDev S, float *val_base, uint64_t stride,
                                                   const float *scr_base, uint64_t scr_stride, uint32_t i0,
                                                   uint32_t i1, uint32_t atomic) {
    __shared__ __align__(16) float sL[kSnMaxWidth][kTLd];
    __shared__ __align__(16) float sU[kSnMaxWidth][kTLd];
    __shared__ uint32_t sOff[kSnMaxWidth];
    __shared__ uint32_t sPl[kTile], sLen[kTile], sEx[kTile];
    float *val = val_base + blockIdx.z * stride;
    const uint32_t b = S.ublk[i0] + blockIdx.x;
    const uint32_t i = upper_slot(S.ublk, i0, i1, b);
    const Sn d = sn_load(P, S, i);
    const uint32_t tid = threadIdx.x;
    uint32_t t = b - S.ublk[i];
    if (d.w >= 2) {
        if (t == 0) {
            const float *scr = scr_base + blockIdx.z * scr_stride + S.dscr[i];
            for (uint32_t e = tid; e < d.w * d.w; e += blockDim.x) {
                const uint32_t cc = e / d.w, r = e - cc * d.w;
                st_cg(val + P.diag[d.s + cc] + r - cc, scr[e]);
            }
            return;
        }
        t -= 1;
    }
    const uint32_t w = d.w;
    const uint32_t nrt = (d.m + kTile - 1) / kTile;
    const uint32_t r0 = (t % nrt) * kTile, c0 = (t / nrt) * kTile;
    if (tid < w) sOff[tid] = P.diag[d.s + tid] + (d.l + 1 - (d.s + tid)) + r0;
    if (tid < kTile) {
        const uint32_t jt = c0 + tid;
        uint32_t pl = 0, len = 0, ex = 0;
        if (jt < d.nt) {
            const uint32_t e = P.rdiag[d.l] + 1 + jt;
            const uint32_t j = P.cidx[e];
            pl = P.cpos[e];
            const uint32_t below = P.cptr[j + 1] - pl - 1;
            if (below >= d.m) {  // always, for a pattern closed under fill
                len = seg_len(P, j, pl, d.l, w);
                ex = below - d.m;  // rows of column j below l that are not in L21
            }
        }
        sPl[tid] = pl;
        sLen[tid] = len;
        sEx[tid] = ex;
    }
    __syncthreads();
    for (uint32_t e = tid; e < w * kTile; e += blockDim.x) {
        const uint32_t k = e / kTile, r = e - k * kTile;
        sL[k][r] = (r0 + r < d.m) ? ld_cg(val + sOff[k] + r) : 0.0f;
    }
    for (uint32_t e = tid; e < w * kTile; e += blockDim.x) {
        const uint32_t jt = e / w, k = e - jt * w;
        sU[k][jt] = (k + sLen[jt] >= w) ? ld_cg(val + sPl[jt] - (w - 1 - k)) : 0.0f;
    }
    const uint32_t tr = tid & 15, tc = tid >> 4;
    uint32_t rowid[4];
    const uint32_t lbase = P.diag[d.l] + 1;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const uint32_t r = r0 + tr * 4 + a;
        rowid[a] = r < d.m ? __ldg(P.ridx + lbase + r) : 0u;
    }
    __syncthreads();
    uint32_t pos[4][4];
    float acc[4][4];
#pragma unroll
    for (int bb = 0; bb < 4; ++bb) {
        const uint32_t jt = tc * 4 + bb;
        const bool tv = sLen[jt] != 0;
        const uint32_t pl = sPl[jt], ex = sEx[jt];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const uint32_t r = r0 + tr * 4 + a;
            uint32_t q = 0xffffffffu;
            float c = 0.0f;
            if (tv && r < d.m) {
                q = pl + 1 + r;
                if (ex) q = lower_bound_u32(P.ridx, q, q + ex + 1, rowid[a]);
                if (!atomic) c = ld_cg(val + q);
            }
            pos[a][bb] = q;
            acc[a][bb] = c;
        }
    }
    if (atomic) {
        for (uint32_t k = 0; k < w; ++k) {
            const float4 av = *reinterpret_cast<const float4 *>(&sL[k][tr * 4]);
            const float4 bv = *reinterpret_cast<const float4 *>(&sU[k][tc * 4]);
            const float ar[4] = {av.x, av.y, av.z, av.w}, br[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) acc[a][bb] = fmaf(ar[a], br[bb], acc[a][bb]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int bb = 0; bb < 4; ++bb)
                if (pos[a][bb] != 0xffffffffu) atomicAdd(val + pos[a][bb], -acc[a][bb]);
    } else {
        for (uint32_t k = 0; k < w; ++k) {
            const float4 av = *reinterpret_cast<const float4 *>(&sL[k][tr * 4]);
            const float4 bv = *reinterpret_cast<const float4 *>(&sU[k][tc * 4]);
            const float ar[4] = {av.x, av.y, av.z, av.w}, br[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) acc[a][bb] = fmaf(-ar[a], br[bb], acc[a][bb]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int bb = 0; bb < 4; ++bb)
                if (pos[a][bb] != 0xffffffffu) st_cg(val + pos[a][bb], acc[a][bb]);
    }
}

cudaError_t launch_sn_panel(const DevPattern &P, const SnPlanDev &S, float *val, uint64_t stride, uint32_t count,
                            const float *pert_z, float *scratch, uint64_t scr_stride, uint32_t i0, uint32_t i1,
                            uint32_t blocks, cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    k_sn_panel<<<dim3(blocks, 1, count), kSnPanelThreads, 0, st>>>(P, S, val, stride, pert_z, scratch, scr_stride,
                                                                   i0, i1);
    return cudaGetLastError();
}

cudaError_t launch_sn_update(const DevPattern &P, const SnPlanDev &S, float *val, uint64_t stride, uint32_t count,
                             const float *scratch, uint64_t scr_stride, uint32_t i0, uint32_t i1, uint32_t blocks,
                             uint32_t atomic, cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    k_sn_update<<<dim3(blocks, 1, count), 256, 0, st>>>(P, S, val, stride, scratch, scr_stride, i0, i1, atomic);
    return cudaGetLastError();
}

}  // namespace glu
