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
// (symbolic.cc:106-151) contracted to supernodes.  Per level three launches:
//   diag:   A11 = L11 U11 in place (GESP pivots, numeric.cu:139-140);
//   panel:  L21 = A21 U11^-1 (a row per thread), U12(:, j) = L11^-1 A12(:, j)
//           for every target j (a column per warp);
//   update: A(rows of L21, j) -= L21 U12(:, j) for every target j, as 64 x 64
//           output tiles (FP32 FMA, K = w), scattered to the CSC positions of
//           column j (a position table built once per pattern, or a search in
//           column j's row list).
// Every entry receives the operations of the column algorithm in the same
// column order (fused multiply-add instead of multiply and subtract; the L21
// rows of supernodes wider than one are multiplied by the pivot's correctly
// rounded reciprocal instead of divided by the pivot).
#include <algorithm>

#include "glu_common.cuh"
#include "glu_kernels.h"
#include "glu_tri.cuh"

namespace glu {

namespace {

constexpr int kLD = kSnMaxWidth + 1;  // leading dimension of the diagonal block in shared memory
constexpr int kSnPW = kSnPanelThreads + 1;  // leading dimension of the L21 rows in shared memory
// panel shared memory: the diagonal block (either layout), plus the rows of
// L21 in launches with a supernode wider than one chunk
constexpr size_t kSnPanelSmem = sizeof(float) * kSnMaxWidth * kTriML;
constexpr size_t kSnPanelSmemWide = kSnPanelSmem + sizeof(float) * kSnMaxWidth * kSnPW;
static_assert(kSnMaxWidth * kTriML >= kSnMaxWidth * kLD, "either layout fits");
static_assert(kSnMaxWidth == kTriMax, "supernode width is the triangular block width");
constexpr int kTile = 64;             // update tile: 64 rows x 64 targets
constexpr int kTLd = kTile + 4;       // leading dimension of the update operand tiles

struct Sn {
    uint32_t s, w, l, m, nt;
};

__device__ __forceinline__ Sn sn_load(const SnPlanDev &S, uint32_t i) {
    const uint4 r = S.meta[i];
    Sn d;
    d.s = r.x;
    d.w = r.y;
    d.l = d.s + d.w - 1;
    d.m = r.z;
    d.nt = r.w;
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

// Target column j of U12 by one warp: L11 x = a over the supernode's rows
// present in column j (a suffix from row z; the rows above it are structural
// zeros and stay untouched).  Lane k holds rows k and k + 32.
__device__ __forceinline__ void sn_u12_warp(float *__restrict__ val, const Sn &d, uint4 g, const float *sF,
                                            uint32_t lane) {
    const uint32_t pl = g.x;
    const uint32_t w = d.w;
    const uint32_t z = w - g.y;
    const uint32_t k0 = lane, k1 = lane + 32;
    const bool p0 = k0 < w && k0 >= z, p1 = k1 < w && k1 >= z;
    float a0 = p0 ? ld_cg(val + pl - (w - 1 - k0)) : 0.0f;
    float a1 = p1 ? ld_cg(val + pl - (w - 1 - k1)) : 0.0f;
    for (uint32_t r = z; r < w; ++r) {
        const float u = __shfl_sync(0xffffffffu, r < 32 ? a0 : a1, r & 31);
        if (k0 > r && k0 < w) a0 = fmaf(-sF[r * kLD + k0], u, a0);
        if (k1 > r && k1 < w) a1 = fmaf(-sF[r * kLD + k1], u, a1);
    }
    if (p0) st_cg(val + pl - (w - 1 - k0), a0);
    if (p1) st_cg(val + pl - (w - 1 - k1), a1);
}

constexpr uint32_t kFull = 0xffffffffu;

// Diagonal block of one narrow supernode (2 <= w <= kSnSmallWidth) by one
// warp: lane r holds row r; step c broadcasts row c by shuffles.  Same
// operations as tri_diag_lu: pivot c perturbed (GESP) when its column has an
// L part (c < w - 1, or m > 0); L(r,c) = A(r,c) / U(c,c), then A(r,j) -=
// L(r,c) U(c,j) for j > c.
__device__ __forceinline__ void sn_diag_small(const DevPattern &P, const SnPlanDev &S, float *__restrict__ val,
                                              uint32_t i, float pert, uint32_t lane) {
    constexpr int SW = int(kSnSmallWidth);
    const Sn d = sn_load(S, i);
    const uint32_t w = d.w;
    const bool rv = lane < w;
    const uint32_t bc = rv ? P.diag[d.s + lane] - lane : 0u;  // position of row s in column s + lane
    float a[SW];
#pragma unroll
    for (int c = 0; c < SW; ++c) {
        const uint32_t b = __shfl_sync(kFull, bc, c);
        a[c] = (rv && uint32_t(c) < w) ? ld_cg(val + b + lane) : 0.0f;
    }
#pragma unroll
    for (int c = 0; c < SW; ++c) {
        if (uint32_t(c) >= w) break;
        if (lane == uint32_t(c)) {
            const bool has_l = uint32_t(c) + 1 < w || d.m > 0;
            if (has_l && pert > 0.0f && fabsf(a[c]) < pert) a[c] = pert;
        }
        const float piv = __shfl_sync(kFull, a[c], c);
        const bool below = rv && lane > uint32_t(c);
        const float l = a[c] / piv;
#pragma unroll
        for (int j = c + 1; j < SW; ++j) {
            const float uj = __shfl_sync(kFull, a[j], c);
            if (below) a[j] = fmaf(-l, uj, a[j]);
        }
        if (below) a[c] = l;
    }
#pragma unroll
    for (int c = 0; c < SW; ++c) {
        const uint32_t b = __shfl_sync(kFull, bc, c);
        if (rv && uint32_t(c) < w) st_cg(val + b + lane, a[c]);
    }
}

// Row r of L21 for a supernode of width w <= N <= kTriChunk: x U11 = a in
// registers (U11 row-major in sM); a was loaded into xr beforehand.
template <int N>
__device__ __forceinline__ void sn_l21_chunk(float *__restrict__ val, const uint32_t *sOff, uint32_t w, uint32_t r,
                                             const float *sM, const float (&xr)[kTriChunk]) {
    float x[N];
#pragma unroll
    for (int c = 0; c < N; ++c) x[c] = xr[c];
    tri_chunk_solve<true>(x, sM, 0, w);
#pragma unroll
    for (int c = 0; c < N; ++c)
        if (uint32_t(c) < w) st_cg(val + sOff[c] + r, x[c]);
}

// Panel of one small supernode (w <= kSnSmallWidth, m <= 32, nt <= 32) by one
// warp: lane r solves L21 row r, lane j solves target column j of U12, with
// the factored diagonal block read in place (broadcast loads).
__device__ __forceinline__ void sn_panel_small(const DevPattern &P, const SnPlanDev &S, float *__restrict__ val,
                                               uint32_t i, float pert, uint32_t lane) {
    constexpr int SW = int(kSnSmallWidth);
    const Sn d = sn_load(S, i);
    const uint32_t w = d.w;
    if (w == 1) {
        // numeric.cu:133-143: pivot (perturbed when the column has an L part), L /= pivot
        const uint32_t dk = P.diag[d.s];
        const float p = ld_cg(val + dk);
        const float de = (pert > 0.0f && fabsf(p) < pert) ? pert : p;  // m > 0 here
        if (lane < d.m) st_cg(val + dk + 1 + lane, ld_cg(val + dk + 1 + lane) / de);
        if (lane == 0 && de != p) st_cg(val + dk, de);
        return;
    }
    const uint32_t dl = lane < w ? P.diag[d.s + lane] : 0u;  // position of the diagonal of column s+lane
    // row `lane` of L21: x U11 = a
    {
        const bool rv = lane < d.m;
        float a[SW];
#pragma unroll
        for (int c = 0; c < SW; ++c) {
            const uint32_t dc = __shfl_sync(kFull, dl, c);
            a[c] = (rv && uint32_t(c) < w) ? ld_cg(val + dc + (d.l + 1 - (d.s + c)) + lane) : 0.0f;
        }
#pragma unroll
        for (int c = 0; c < SW; ++c) {
            if (uint32_t(c) >= w) break;
            const float l = a[c] / ld_cg(val + __shfl_sync(kFull, dl, c));
            a[c] = l;
#pragma unroll
            for (int j = c + 1; j < SW; ++j) {
                const uint32_t dj = __shfl_sync(kFull, dl, j);
                if (uint32_t(j) < w) a[j] = fmaf(-l, ld_cg(val + dj - (j - c)), a[j]);
            }
        }
#pragma unroll
        for (int c = 0; c < SW; ++c) {
            const uint32_t dc = __shfl_sync(kFull, dl, c);  // every lane takes part in the shuffle
            if (rv && uint32_t(c) < w) st_cg(val + dc + (d.l + 1 - (d.s + c)) + lane, a[c]);
        }
    }
    // target column `lane` of U12: L11 x = a over the rows present
    {
        uint4 g = make_uint4(0u, 0u, 0u, 0u);
        if (lane < d.nt) g = S.tgt[S.tgt_off[i] + lane];
        const uint32_t z = w - g.y;  // g.y == 0: no target (z = w, nothing loaded or stored)
        float a[SW];
#pragma unroll
        for (int k = 0; k < SW; ++k) a[k] = (uint32_t(k) < w && uint32_t(k) >= z) ? ld_cg(val + g.x - (w - 1 - k)) : 0.0f;
#pragma unroll
        for (int r = 0; r < SW; ++r) {
            if (uint32_t(r) >= w) break;
            const uint32_t dr = __shfl_sync(kFull, dl, r);
            if (uint32_t(r) >= z) {
                const float u = a[r];
#pragma unroll
                for (int k = r + 1; k < SW; ++k)
                    if (uint32_t(k) < w) a[k] = fmaf(-ld_cg(val + dr + (k - r)), u, a[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < SW; ++k)
            if (uint32_t(k) < w && uint32_t(k) >= z) st_cg(val + g.x - (w - 1 - k), a[k]);
    }
}

// Update of one small supernode (w <= kSnSmallWidth, m * nt <= 256) by one
// warp, its m x nt outputs 32 at a time (same arithmetic as the tiles).
__device__ __forceinline__ void sn_update_small(const DevPattern &P, const SnPlanDev &S, float *__restrict__ val,
                                                uint32_t i, bool atomic, uint32_t lane) {
    constexpr int SW = int(kSnSmallWidth);
    const Sn d = sn_load(S, i);
    const uint32_t w = d.w, m = d.m, nout = d.m * d.nt;
    // L21 base of column s+lane: L21(r, c) at diag[s+c] + (l + 1 - (s+c)) + r
    const uint32_t bl = lane < w ? P.diag[d.s + lane] + (d.l + 1 - (d.s + lane)) : 0u;
    const uint32_t g0 = S.tgt_off[i];
    const uint32_t lbase = P.diag[d.l] + 1;
    for (uint32_t o0 = 0; o0 < nout; o0 += 32) {
        const uint32_t o = o0 + lane;
        const bool ov = o < nout;
        const uint32_t jt = ov ? o / m : 0u, r = ov ? o - jt * m : 0u;
        uint4 g = make_uint4(0u, 0u, 0u, 0u);
        if (ov) g = S.tgt[g0 + jt];
        const bool v = ov && g.y != 0;
        uint32_t q = g.x + 1 + r;
        if (v && g.z) {
            const uint32_t row = __ldg(P.ridx + lbase + r);
            if (S.pos)
                q = __ldg(S.pos + S.pos_off[i] + uint64_t(jt) * m + r);
            else if (S.tail_full && g.w >= S.t && row >= S.t)  // complete dense-tail column
                q = __ldg(S.tail_start + (g.w - S.t)) + (row - S.t);
            else
                q = lower_bound_u32(P.ridx, q, q + g.z + 1, row);
        }
        float acc = (v && !atomic) ? ld_cg(val + q) : 0.0f;
#pragma unroll
        for (int c = 0; c < SW; ++c) {
            if (uint32_t(c) >= w) break;
            const uint32_t bc = __shfl_sync(kFull, bl, c);
            if (v) {
                const float lv = ld_cg(val + bc + r);
                const float uv = (uint32_t(c) + g.y >= w) ? ld_cg(val + g.x - (w - 1 - c)) : 0.0f;
                acc = atomic ? fmaf(lv, uv, acc) : fmaf(-lv, uv, acc);
            }
        }
        if (v) {
            if (atomic)
                atomicAdd(val + q, -acc);
            else
                st_cg(val + q, acc);
        }
    }
}

}  // namespace

// Diagonal-block launch of one level: blocks [b0, b0 + gridDim.x) of the
// diagonal map, each one supernode wider than kSnSmallWidth (tri_diag_lu) or
// up to eight narrower ones (a warp each).  The diagonal block is factored in
// place: pivot c is perturbed (GESP, numeric.cu:139-140) when its column has
// an L part (c < w - 1, or m > 0); step c: L(i,c) = A(i,c) / U(c,c), then
// A(i,j) -= L(i,c) U(c,j) for j > c, as in the column algorithm.  blockIdx.z
// selects the value set.
__global__ void __launch_bounds__(kTriThreads, 1) k_sn_diag(DevPattern P, SnPlanDev S, float *val_base, uint64_t stride,
                                                            const float *pert_z, uint32_t b0) {
    __shared__ __align__(16) float urow[2][kTriMax];
    __shared__ uint32_t sBase[kSnMaxWidth];
    pdl_release();
    pdl_wait();  // the previous level's updates
    float *val = val_base + blockIdx.z * stride;
    const float pert = pert_z ? pert_z[blockIdx.z] : 0.0f;
    const uint2 bi = S.dmap[b0 + blockIdx.x];
    if (bi.y & kSnSmallFlag) {
        const uint32_t wi = threadIdx.x >> 5;
        if (wi < (bi.y & ~kSnSmallFlag)) sn_diag_small(P, S, val, S.dsmall[bi.x + wi], pert, threadIdx.x & 31);
        return;
    }
    const Sn d = sn_load(S, bi.x);
    const uint32_t tid = threadIdx.x, w = d.w;
    if (tid < w) sBase[tid] = P.diag[d.s + tid] - tid;  // position of row s in column s + tid
    __syncthreads();
    const uint32_t row = tid >> 2, q = tid & 3;
    float a[kTriChunk];
#pragma unroll
    for (int jj = 0; jj < kTriChunk; ++jj) {
        const uint32_t cc = q * kTriChunk + jj;
        a[jj] = (row < w && cc < w) ? ld_cg(val + sBase[cc] + row) : 0.0f;
    }
    tri_diag_lu(a, w, d.m > 0, pert, urow);
#pragma unroll
    for (int jj = 0; jj < kTriChunk; ++jj) {
        const uint32_t cc = q * kTriChunk + jj;
        if (row < w && cc < w) st_cg(val + sBase[cc] + row, a[jj]);
    }
}

// Panel launch of one level (after its diagonal blocks): blocks [b0, b0 +
// gridDim.x) of the panel map.  Per supernode: ceil(m / 128) blocks of L21 rows (one row per
// thread), then, for width >= 2, ceil(nt / 4) blocks of U12 target columns
// (one column per warp).  Width 1: the blocks scale the column by its pivot
// (numeric.cu:133-143).  blockIdx.z selects the value set.
__global__ void __launch_bounds__(kSnPanelThreads, 4) k_sn_panel(DevPattern P, SnPlanDev S, float *val_base,
                                                              uint64_t stride, const float *pert_z, uint32_t b0) {
    extern __shared__ float4 snp_sm4[];
    float *sF = reinterpret_cast<float *>(snp_sm4);  // L11 column-major (U12 blocks) or U11 row-major (L21 blocks)
    float *sW = sF + kSnMaxWidth * kTriML;           // rows of L21 when w > kTriChunk
    __shared__ uint32_t sOff[kSnMaxWidth];
    pdl_release();
    pdl_wait();  // this level's diagonal blocks
    float *val = val_base + blockIdx.z * stride;
    const float pert = pert_z ? pert_z[blockIdx.z] : 0.0f;
    const uint2 bi = S.pmap[b0 + blockIdx.x];
    if (bi.y & kSnSmallFlag) {  // small supernodes, one per warp
        const uint32_t wi = threadIdx.x >> 5;
        if (wi < (bi.y & ~kSnSmallFlag)) sn_panel_small(P, S, val, S.psmall[bi.x + wi], pert, threadIdx.x & 31);
        return;
    }
    const uint32_t i = bi.x, t = bi.y;
    const Sn d = sn_load(S, i);
    const uint32_t tid = threadIdx.x;
    if (d.w == 1) {
        const uint32_t dk = P.diag[d.s];
        const uint32_t r = t * kSnPanelThreads + tid;
        const float p = ld_cg(val + dk);
        const float de = (pert > 0.0f && fabsf(p) < pert) ? pert : p;  // m > 0 here
        if (r < d.m) st_cg(val + dk + 1 + r, ld_cg(val + dk + 1 + r) / de);
        // (a concurrent reader of the pivot sees p or pert; both give de)
        if (t == 0 && tid == 0 && de != p) st_cg(val + dk, de);
        return;
    }
    const uint32_t w = d.w;
    const uint32_t nLb = (d.m + kSnPanelThreads - 1) / kSnPanelThreads;
    const bool lrows = t < nLb;
    if (tid < w) sOff[tid] = P.diag[d.s + tid];
    __syncthreads();
    // This thread's row of A21 (w <= kTriChunk) does not depend on the
    // diagonal block: its loads are issued first.
    const uint32_t rr = t * kSnPanelThreads + tid;
    float xr[kTriChunk];
    if (lrows && w <= uint32_t(kTriChunk) && rr < d.m) {
#pragma unroll
        for (int c = 0; c < kTriChunk; ++c)
            xr[c] = uint32_t(c) < w ? ld_cg(val + sOff[c] + (d.l + 1 - (d.s + c)) + rr) : 0.0f;
    }
    // the factored diagonal block, eight independent loads in flight per thread:
    // L21 blocks keep U11 row-major (leading dimension kTriML), U12 blocks L11
    // column-major (leading dimension kLD)
    for (uint32_t e0 = 0; e0 < kSnMaxWidth * kSnMaxWidth; e0 += 8 * kSnPanelThreads) {
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t e = e0 + q * kSnPanelThreads + tid, cc = e >> 6, r = e & 63;
            v[q] = (cc < w && r < w) ? ld_cg(val + sOff[cc] + r - cc) : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t e = e0 + q * kSnPanelThreads + tid, cc = e >> 6, r = e & 63;
            if (cc < w && r < w) {
                if (lrows)
                    sF[r * kTriML + cc] = v[q];
                else
                    sF[cc * kLD + r] = v[q];
            }
        }
        if (e0 + 8 * kSnPanelThreads >= w * kSnMaxWidth) break;
    }
    __syncthreads();
    if (tid < w) {
        sOff[tid] += d.l + 1 - (d.s + tid);
        if (lrows) sF[tid * kTriML + kTriMax] = 1.0f / sF[tid * kTriML + tid];  // pivot reciprocals
    }
    __syncthreads();
    if (lrows) {
        // row r of L21: x U11 = a (a = row r of A21)
        const uint32_t r = t * kSnPanelThreads + tid;
        if (r >= d.m) return;
        if (w <= 2) {
            sn_l21_chunk<2>(val, sOff, w, r, sF, xr);
        } else if (w <= 4) {
            sn_l21_chunk<4>(val, sOff, w, r, sF, xr);
        } else if (w <= 8) {
            sn_l21_chunk<8>(val, sOff, w, r, sF, xr);
        } else if (w <= uint32_t(kTriChunk)) {
            sn_l21_chunk<kTriChunk>(val, sOff, w, r, sF, xr);
        } else {
            for (uint32_t c = 0; c < w; ++c) sW[c * kSnPW + tid] = ld_cg(val + sOff[c] + r);
            tri_rows_solve<true>(sW, kSnPW, tid, sF, w);
            for (uint32_t c = 0; c < w; ++c) st_cg(val + sOff[c] + r, sW[c * kSnPW + tid]);
        }
    } else {
        const uint32_t jt = (t - nLb) * (kSnPanelThreads / 32) + tid / 32;
        if (jt < d.nt) {
            const uint4 g = S.tgt[S.tgt_off[i] + jt];
            if (g.y != 0) sn_u12_warp(val, d, g, sF, tid & 31);
        }
    }
}

// Update launch of one level: blocks [b0, b0 + gridDim.x) of the update map,
// the 64 x 64 tiles of every supernode's update (row tiles fastest).  Levels with several
// supernodes accumulate with atomics (numeric.cu:82); a single supernode
// updates each entry from one thread: C is loaded, the K products are applied
// in column order, C is stored.  Target positions come from the precomputed
// table S.pos when present, else from a search in column j's rows.  A
// supernode whose update of the dense tail is deferred (S.cut) skips the
// entries of that corner; the update map holds none of its tiles that lie
// wholly inside it.
__global__ void __launch_bounds__(256, 5) k_sn_update(DevPattern P, SnPlanDev S, float *val_base, uint64_t stride,
                                                      uint32_t b0, uint32_t atomic, uint32_t count, uint32_t zpb) {
    __shared__ __align__(16) float sL[kSnMaxWidth][kTLd];
    __shared__ __align__(16) float sU[kSnMaxWidth][kTLd];
    __shared__ uint32_t sOff[kSnMaxWidth];
    __shared__ uint32_t sPl[kTile], sLen[kTile], sEx[kTile], sJ[kTile];
    // value sets [z0, z1) of this block: the tile's metadata and target
    // positions are the same for all of them and computed once
    const uint32_t z0 = blockIdx.z * zpb, z1 = min(z0 + zpb, count);
    pdl_release();
    const uint2 bi = S.umap[b0 + blockIdx.x];
    if (bi.y & kSnSmallFlag) {  // small supernodes, one per warp
        pdl_wait();  // this level's panels
        const uint32_t wi = threadIdx.x >> 5;
        if (wi < (bi.y & ~kSnSmallFlag))
            for (uint32_t z = z0; z < z1; ++z)
                sn_update_small(P, S, val_base + z * stride, S.usmall[bi.x + wi], atomic != 0, threadIdx.x & 31);
        return;
    }
    const uint32_t i = bi.x, t = bi.y;
    const Sn d = sn_load(S, i);
    const uint32_t tid = threadIdx.x;
    const uint32_t w = d.w;
    const uint32_t nrt = (d.m + kTile - 1) / kTile;
    const uint32_t r0 = (t % nrt) * kTile, c0 = (t / nrt) * kTile;
    const uint32_t tr = tid & 15, tc = tid >> 4;
    // Target positions from the table depend only on the tile: issued first,
    // in flight while the metadata and the operands are staged (a target that
    // cannot hold the rows has 0xffffffff in the table).
    uint32_t pos[4][4];
    if (S.pos) {
        const uint32_t *tab = S.pos + S.pos_off[i] + r0 + tr * 4;
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) {
            const uint32_t jt = tc * 4 + bb;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const uint32_t r = r0 + tr * 4 + a;
                pos[a][bb] = (c0 + jt < d.nt && r < d.m) ? __ldg(tab + uint64_t(c0 + jt) * d.m + a) : 0xffffffffu;
            }
        }
    }
    if (tid < w) sOff[tid] = P.diag[d.s + tid] + (d.l + 1 - (d.s + tid)) + r0;
    if (tid < kTile) {
        const uint32_t jt = c0 + tid;
        uint32_t pl = 0, len = 0, ex = 0, tj = 0;
        if (jt < d.nt) {
            const uint4 g = S.tgt[S.tgt_off[i] + jt];
            pl = g.x;
            len = g.y;
            ex = g.z;
            tj = g.w;
        }
        sPl[tid] = pl;
        sLen[tid] = len;
        sEx[tid] = ex;
        sJ[tid] = tj;
    }
    __syncthreads();
    if (!S.pos) {
        uint32_t rowid[4];
        const uint32_t lbase = P.diag[d.l] + 1;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const uint32_t r = r0 + tr * 4 + a;
            rowid[a] = r < d.m ? __ldg(P.ridx + lbase + r) : 0u;
        }
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) {
            const uint32_t jt = tc * 4 + bb;
            const bool tv = sLen[jt] != 0;
            const uint32_t pl = sPl[jt], ex = sEx[jt], tj = sJ[jt];
            // a complete dense-tail column: tail rows at fixed offsets
            const bool tcol = S.tail_full && tj >= S.t;
            const uint32_t ts = tcol ? __ldg(S.tail_start + (tj - S.t)) : 0u;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const uint32_t r = r0 + tr * 4 + a;
                uint32_t q = 0xffffffffu;
                if (tv && r < d.m) {
                    if (tcol && rowid[a] >= S.t) {
                        q = ts + (rowid[a] - S.t);
                    } else {
                        q = pl + 1 + r;
                        if (ex) q = lower_bound_u32(P.ridx, q, q + ex + 1, rowid[a]);
                    }
                }
                pos[a][bb] = q;
            }
        }
    }
    if (S.cut) {  // the deferred corner (tail rows x tail targets) is left out
        const uint2 cu = __ldg(S.cut + i);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int bb = 0; bb < 4; ++bb)
                if (r0 + tr * 4 + a >= cu.x && c0 + tc * 4 + bb >= cu.y) pos[a][bb] = 0xffffffffu;
    }
    // the metadata and positions above are plan data, read while this
    // level's panels finish; the values only after them
    pdl_wait();
    for (uint32_t z = z0; z < z1; ++z) {
    float *val = val_base + z * stride;
    if (z > z0) __syncthreads();  // the previous value set's operands are read
    for (uint32_t e = tid; e < w * kTile; e += blockDim.x) {
        const uint32_t k = e / kTile, r = e - k * kTile;
        sL[k][r] = (r0 + r < d.m) ? ld_cg(val + sOff[k] + r) : 0.0f;
    }
    for (uint32_t e = tid; e < w * kTile; e += blockDim.x) {
        const uint32_t jt = e / w, k = e - jt * w;
        sU[k][jt] = (k + sLen[jt] >= w) ? ld_cg(val + sPl[jt] - (w - 1 - k)) : 0.0f;
    }
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) acc[a][bb] = (!atomic && pos[a][bb] != 0xffffffffu) ? ld_cg(val + pos[a][bb]) : 0.0f;
    __syncthreads();
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
    }  // value sets
}

// Target metadata, one thread per (supernode, target) pair g (level order,
// S.tgt_off the prefix): {CSC position pl of the supernode's last row l in
// target column j, rows of the supernode present in column j (0: the column
// cannot hold the L21 rows), rows of column j below l that are not L21 rows,
// j}.
__global__ void __launch_bounds__(256) k_sn_targets(DevPattern P, SnPlanDev S, uint32_t nsn, uint4 *tgt) {
    const uint32_t total = S.tgt_off[nsn];
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        const uint32_t i = upper_slot(S.tgt_off, 0, nsn, g);
        const Sn d = sn_load(S, i);
        const uint32_t e = P.rdiag[d.l] + 1 + (g - S.tgt_off[i]);
        const uint32_t j = P.cidx[e];
        const uint32_t pl = P.cpos[e];
        const uint32_t below = P.cptr[j + 1] - pl - 1;
        uint4 o = make_uint4(pl, 0u, 0u, j);
        if (below >= d.m) {  // always, for a pattern closed under fill
            o.y = seg_len(P, j, pl, d.l, d.w);
            o.z = below - d.m;
        }
        tgt[g] = o;
    }
}

// Position table of the update scatter: for supernode i (level order) and its
// target jt, entry pos_off[i] + jt * m + r is the CSC position of L21 row r in
// column j (0xffffffff for a target that cannot hold the rows).  One warp per
// (supernode, target) pair.
__global__ void __launch_bounds__(256) k_sn_positions(DevPattern P, SnPlanDev S, uint32_t nsn, uint32_t *pos) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwarps = uint64_t(gridDim.x) * (blockDim.x / 32);
    const uint32_t total = S.tgt_off[nsn];
    for (uint64_t g = uint64_t(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32; g < total; g += nwarps) {
        const uint32_t i = upper_slot(S.tgt_off, 0, nsn, uint32_t(g));
        const uint32_t jt = uint32_t(g) - S.tgt_off[i];
        const Sn d = sn_load(S, i);
        const uint4 o = S.tgt[g];
        uint32_t *out = pos + S.pos_off[i] + uint64_t(jt) * d.m;
        const uint32_t lbase = P.diag[d.l] + 1;
        for (uint32_t r = lane; r < d.m; r += 32) {
            uint32_t q = 0xffffffffu;
            if (o.y != 0) {
                q = o.x + 1 + r;
                if (o.z) q = lower_bound_u32(P.ridx, q, q + o.z + 1, __ldg(P.ridx + lbase + r));
            }
            out[r] = q;
        }
    }
}

cudaError_t launch_sn_diag(const DevPattern &P, const SnPlanDev &S, float *val, uint64_t stride, uint32_t count,
                           const float *pert_z, uint32_t b0, uint32_t blocks, cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    return launch_chained(k_sn_diag, dim3(blocks, 1, count), dim3(kTriThreads), 0, st, P, S, val, stride, pert_z, b0);
}

cudaError_t launch_sn_panel(const DevPattern &P, const SnPlanDev &S, float *val, uint64_t stride, uint32_t count,
                            const float *pert_z, uint32_t b0, uint32_t blocks, uint32_t maxw, cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    static PerDeviceOnce attr;
    cudaError_t e = attr.run([] {
        return cudaFuncSetAttribute(k_sn_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSnPanelSmemWide));
    });
    if (e != cudaSuccess) return e;
    const size_t smem = maxw > uint32_t(kTriChunk) ? kSnPanelSmemWide : kSnPanelSmem;
    return launch_chained(k_sn_panel, dim3(blocks, 1, count), dim3(kSnPanelThreads), smem, st, P, S, val, stride, pert_z,
                          b0);
}

cudaError_t launch_sn_update(const DevPattern &P, const SnPlanDev &S, float *val, uint64_t stride, uint32_t count,
                             uint32_t b0, uint32_t blocks, uint32_t atomic, uint32_t batch_tile, cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    // several value sets per block once the grid has enough blocks without
    // them (or batch_tile of them when set)
    uint32_t zpb = 1;
    if (batch_tile)
        zpb = std::min(batch_tile, count);
    else
        while (zpb < 8 && zpb * 2 <= count && uint64_t(blocks) * ((count + zpb * 2 - 1) / (zpb * 2)) >= 4ull * 148 * 5)
            zpb *= 2;
    return launch_chained(k_sn_update, dim3(blocks, 1, (count + zpb - 1) / zpb), dim3(256), 0, st, P, S, val, stride, b0,
                          atomic, count, zpb);
}

cudaError_t launch_sn_targets(const DevPattern &P, const SnPlanDev &S, uint32_t nsn, uint4 *tgt, cudaStream_t st) {
    if (nsn == 0) return cudaSuccess;
    k_sn_targets<<<148 * 8, 256, 0, st>>>(P, S, nsn, tgt);
    return cudaGetLastError();
}

cudaError_t launch_sn_positions(const DevPattern &P, const SnPlanDev &S, uint32_t nsn, uint32_t *pos,
                                cudaStream_t st) {
    if (nsn == 0) return cudaSuccess;
    k_sn_positions<<<148 * 16, 256, 0, st>>>(P, S, nsn, pos);
    return cudaGetLastError();
}

}  // namespace glu
