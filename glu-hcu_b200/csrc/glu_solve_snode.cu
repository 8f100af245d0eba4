// Supernodal form of the sparse L and U sweeps of the triangular solves.
//
// The reference sweeps column by column (Symbolic_Matrix::solve,
// src/symbolic.cc:226-239).  With the factor's supernodes (runs of columns
// [s, s+w) with a dense diagonal block and a common lower pattern) a sweep
// step is a whole supernode: its w unknowns are solved against the dense
// diagonal block (one warp, the block staged in shared memory) and their
// off-diagonal entries are then scattered into the unknowns they feed:
//   L (forward, unit):  x_S = L11^-1 y_S;  y_r -= L21(r,:) x_S for the m rows
//                       below the block (one thread per row, dot over w);
//   U (backward):       x_S = U11^-1 y_S;  y_i -= U(i,c) x_c for the entries
//                       of the supernode's columns above the block.
// Supernodes are leveled by the sweep's dependencies: L — a supernode waits
// for the supernodes whose L21 rows fall in it; U — for the supernodes that
// hold its update targets.  Finished unknowns go to xo (another block of the
// same supernode may still read y_S) and are copied back after the sweep.
// Every block finds its supernode and part through a precomputed map; small
// supernodes (width <= kSnSmallWidth with at most 32 off-diagonal rows or
// entries) go eight to a block, one warp each.
#include "glu_common.cuh"
#include "glu_kernels.h"

namespace glu {

namespace {
constexpr int kLD = kSnMaxWidth + 1;
constexpr uint32_t kFull = 0xffffffffu;

// L sweep of one small supernode (w <= kSnSmallWidth, m <= 32) by one warp:
// lane k holds unknown s+k and L21 row k; the entries it needs are loaded
// before the dependency chain starts.
__device__ __forceinline__ void sn_sweep_l_small(const DevPattern &P, const SnSweepPlan &W,
                                                 const float *__restrict__ val, float *y, float *xo, uint32_t nrhs,
                                                 uint32_t i, uint32_t lane) {
    constexpr int SW = int(kSnSmallWidth);
    const uint4 md = W.meta[i];
    const uint32_t s = md.x, w = md.y, lbase = md.z, m = md.w, l = s + w - 1, n = P.n;
    const uint32_t dl = lane < w ? P.diag[s + lane] : 0u;
    float lrow[SW], l21[SW];
#pragma unroll
    for (int c = 0; c < SW; ++c) {
        const uint32_t dc = __shfl_sync(kFull, dl, c);
        lrow[c] = (uint32_t(c) < lane && lane < w) ? __ldg(val + dc + (lane - c)) : 0.0f;
        l21[c] = (lane < m && uint32_t(c) < w) ? __ldg(val + dc + (l + 1 - (s + c)) + lane) : 0.0f;
    }
    const uint32_t target = lane < m ? __ldg(P.ridx + lbase + lane) : 0u;
    for (uint32_t q = 0; q < nrhs; ++q) {
        float *yq = y + size_t(q) * n;
        float v = lane < w ? __ldcg(yq + s + lane) : 0.0f;
#pragma unroll
        for (int c = 0; c + 1 < SW; ++c) {
            if (uint32_t(c) + 1 >= w) break;
            const float xc = __shfl_sync(kFull, v, c);
            if (lane > uint32_t(c) && lane < w) v = __fsub_rn(v, __fmul_rn(lrow[c], xc));
        }
        if (lane < w) xo[size_t(q) * n + s + lane] = v;
        float acc = 0.0f;
#pragma unroll
        for (int c = 0; c < SW; ++c) {
            if (uint32_t(c) >= w) break;
            acc = fmaf(l21[c], __shfl_sync(kFull, v, c), acc);
        }
        if (lane < m && acc != 0.0f) atomicAdd(yq + target, -acc);
    }
}

// U sweep of one small supernode (w <= kSnSmallWidth, at most 32 entries above
// the block) by one warp: lane k holds unknown s+k and above-block entry k.
__device__ __forceinline__ void sn_sweep_u_small(const DevPattern &P, const SnSweepPlan &W,
                                                 const float *__restrict__ val, float *y, float *xo, uint32_t nrhs,
                                                 uint32_t i, uint32_t lane) {
    constexpr int SW = int(kSnSmallWidth);
    const uint4 md = W.meta[i];
    const uint32_t s = md.x, w = md.y, n = P.n;
    const uint32_t dl = lane < w ? P.diag[s + lane] : 0u;
    const uint32_t cp = lane < w ? P.cptr[s + lane] : 0u;
    const uint32_t cnt = lane < w ? (dl - lane) - cp : 0u;  // entries of column s+lane above the block
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(kFull, incl, o);
        if (lane >= uint32_t(o)) incl += v;
    }
    const uint32_t pre = incl - cnt, total = __shfl_sync(kFull, incl, 31);
    uint32_t col = 0;  // column of entry `lane`: the last c < w with pre_c <= lane
#pragma unroll
    for (int c = 1; c < SW; ++c) {
        const uint32_t pc = __shfl_sync(kFull, pre, c);
        if (uint32_t(c) < w && pc <= lane) col = c;
    }
    const uint32_t pcol = __shfl_sync(kFull, cp, col) + (lane - __shfl_sync(kFull, pre, col));
    const bool ev = lane < total;
    const uint32_t tg = ev ? __ldg(P.ridx + pcol) : 0u;
    const float ue = ev ? __ldg(val + pcol) : 0.0f;
    float urow[SW];  // U(s+lane, s+cc) for cc > lane, at diag[s+cc] - (cc - lane)
#pragma unroll
    for (int cc = 0; cc < SW; ++cc) {
        const uint32_t dcc = __shfl_sync(kFull, dl, cc);
        urow[cc] = (lane < uint32_t(cc) && uint32_t(cc) < w) ? __ldg(val + dcc - (cc - lane)) : 0.0f;
    }
    const float piv = lane < w ? __ldg(val + dl) : 1.0f;
    for (uint32_t q = 0; q < nrhs; ++q) {
        float *yq = y + size_t(q) * n;
        float v = lane < w ? __ldcg(yq + s + lane) : 0.0f;
#pragma unroll
        for (int cc = SW - 1; cc >= 0; --cc) {
            if (uint32_t(cc) >= w) continue;
            const float xc = __shfl_sync(kFull, v, cc) / __shfl_sync(kFull, piv, cc);
            if (lane == uint32_t(cc)) v = xc;
            if (lane < uint32_t(cc)) v = __fsub_rn(v, __fmul_rn(urow[cc], xc));
        }
        if (lane < w) xo[size_t(q) * n + s + lane] = v;
        const float xe = __shfl_sync(kFull, v, col);
        if (ev && xe != 0.0f) atomicAdd(yq + tg, -__fmul_rn(ue, xe));
    }
}
// Fused sweeps: the block's item and value set from one ticket counter of the
// launch, handed out item-major over the value sets (ticket = item * count +
// set, so every set's sweep advances at once), and a wait (thread 0, bounded)
// until every supernode it solves has received all its releases; a block
// waits only on items of smaller tickets.  Returns {map index, value set},
// the index UINT32_MAX when the ticket is past the end.  Per-level launches
// use {b0 + blockIdx.x, blockIdx.z} instead.
__device__ __forceinline__ uint2 sweep_block(const SnSweepPlan &W, uint32_t b0, const uint32_t *done,
                                             uint32_t *ticket, uint32_t *status, uint32_t spin_limit) {
    if (!done) return make_uint2(b0 + blockIdx.x, blockIdx.z);
    __shared__ uint32_t s_blk, s_z;
    if (threadIdx.x == 0) {
        const uint32_t k = atomicAdd(ticket, 1u);
        const uint32_t blk = k / gridDim.z, z = k % gridDim.z;
        if (blk < W.nblocks) {
            const uint32_t *dz = done + size_t(z) * W.ns;
            for (uint32_t e = W.wait_off[blk]; e < W.wait_off[blk + 1]; ++e) {
                const uint32_t q = W.wait_idx[e];
                wait_count(dz + q, W.indeg[q], status, spin_limit);
            }
        }
        s_blk = blk;
        s_z = z;
    }
    __syncthreads();
    return make_uint2(s_blk < W.nblocks ? s_blk : UINT32_MAX, s_z);
}

// After the block's scatter: one release for every supernode it updated (its
// atomics are made visible first: barrier, then a device-scope fence).
__device__ __forceinline__ void sweep_release(const SnSweepPlan &W, uint32_t blk, uint32_t *done) {
    if (!done) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        for (uint32_t e = W.rel_off[blk]; e < W.rel_off[blk + 1]; ++e) atomicAdd(done + W.rel_idx[e], 1u);
    }
}
}  // namespace

__global__ void __launch_bounds__(256, 2) k_sn_sweep_l(DevPattern P, SnSweepPlan W, const float *__restrict__ val,
                                                    float *y, float *xo, uint32_t nrhs, uint32_t b0,
                                                    uint64_t vstride, uint64_t ystride, uint32_t *done,
                                                    uint32_t *ticket, uint32_t *status, uint32_t spin_limit) {
    pdl_release();
    pdl_wait();  // the previous level's x (per-level launches are chained)
    const uint2 bz = sweep_block(W, b0, done, ticket, status, spin_limit);
    const uint32_t blk = bz.x;
    val += bz.y * vstride;  // value set bz.y, its right-hand sides
    y += bz.y * ystride;
    xo += bz.y * ystride;
    if (done) done += size_t(bz.y) * W.ns;
    if (blk == UINT32_MAX) return;
    __shared__ float sT[kSnMaxWidth * kLD];
    __shared__ float xs[kSnMaxWidth];
    const uint2 bi = W.map[blk];
    if (bi.y & kSnSmallFlag) {  // a group of small supernodes, one per warp
        const uint32_t wi = threadIdx.x >> 5;
        if (wi < (bi.y & ~kSnSmallFlag)) sn_sweep_l_small(P, W, val, y, xo, nrhs, W.small[bi.x + wi], threadIdx.x & 31);
        sweep_release(W, blk, done);
        return;
    }
    const uint4 md = W.meta[bi.x];
    const uint32_t s = md.x, w = md.y, lbase = md.z, m = md.w, t = bi.y;
    const uint32_t l = s + w - 1;
    const uint32_t tid = threadIdx.x, n = P.n;
    __shared__ uint32_t sB[kSnMaxWidth];
    if (tid < w) sB[tid] = P.diag[s + tid];
    __syncthreads();
    // This thread's L21 row and its target: they do not depend on x, so they
    // are loaded before the dependency chain (and serve every right-hand side).
    const uint32_t r = t * blockDim.x + tid;  // L21 row of this thread
    float lr[kSnMaxWidth];
    uint32_t target = 0;
    if (r < m) {
        target = __ldg(P.ridx + lbase + r);
#pragma unroll
        for (int c = 0; c < int(kSnMaxWidth); ++c)
            lr[c] = uint32_t(c) < w ? __ldg(val + sB[c] + (l + 1 - (s + c)) + r) : 0.0f;
    }
    // L11, strictly lower: L(s+k, s+c) at diag[s+c] + (k - c); eight loads in flight per thread
    for (uint32_t e0 = 0; e0 < w * kSnMaxWidth; e0 += 8 * 256) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t e = e0 + u * 256 + tid, c = e >> 6, k = e & 63;
            v[u] = (c < w && k < w && k > c) ? __ldg(val + sB[c] + (k - c)) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t e = e0 + u * 256 + tid, c = e >> 6, k = e & 63;
            if (c < w && k < w && k > c) sT[c * kLD + k] = v[u];
        }
    }
    __syncthreads();
    for (uint32_t q = 0; q < nrhs; ++q) {
        float *yq = y + size_t(q) * n;
        if (tid < 32) {
            const uint32_t k0 = tid, k1 = tid + 32;
            float v0 = k0 < w ? __ldcg(yq + s + k0) : 0.0f;
            float v1 = k1 < w ? __ldcg(yq + s + k1) : 0.0f;
            for (uint32_t c = 0; c + 1 < w; ++c) {
                const float xc = __shfl_sync(0xffffffffu, c < 32 ? v0 : v1, c & 31);
                if (k0 > c && k0 < w) v0 = __fsub_rn(v0, __fmul_rn(sT[c * kLD + k0], xc));
                if (k1 > c && k1 < w) v1 = __fsub_rn(v1, __fmul_rn(sT[c * kLD + k1], xc));
            }
            if (k0 < w) xs[k0] = v0;
            if (k1 < w) xs[k1] = v1;
            if (t == 0) {
                if (k0 < w) xo[size_t(q) * n + s + k0] = v0;
                if (k1 < w) xo[size_t(q) * n + s + k1] = v1;
            }
        }
        __syncthreads();
        if (r < m) {
            float acc = 0.0f;
#pragma unroll
            for (int c = 0; c < int(kSnMaxWidth); ++c)
                if (uint32_t(c) < w) acc = fmaf(lr[c], xs[c], acc);
            if (acc != 0.0f) atomicAdd(yq + target, -acc);
        }
        __syncthreads();
    }
    sweep_release(W, blk, done);
}

__global__ void __launch_bounds__(256, 4) k_sn_sweep_u(DevPattern P, SnSweepPlan W, const float *__restrict__ val,
                                                    float *y, float *xo, uint32_t nrhs, uint32_t b0,
                                                    uint64_t vstride, uint64_t ystride, uint32_t *done,
                                                    uint32_t *ticket, uint32_t *status, uint32_t spin_limit) {
    pdl_release();
    pdl_wait();  // the previous level's x (per-level launches are chained)
    const uint2 bz = sweep_block(W, b0, done, ticket, status, spin_limit);
    const uint32_t blk = bz.x;
    val += bz.y * vstride;  // value set bz.y, its right-hand sides
    y += bz.y * ystride;
    xo += bz.y * ystride;
    if (done) done += size_t(bz.y) * W.ns;
    if (blk == UINT32_MAX) return;
    __shared__ float sT[kSnMaxWidth * kLD];
    __shared__ float xs[kSnMaxWidth];
    __shared__ uint32_t pre[kSnMaxWidth + 1];
    const uint2 bi = W.map[blk];
    if (bi.y & kSnSmallFlag) {  // a group of small supernodes, one per warp
        const uint32_t wi = threadIdx.x >> 5;
        if (wi < (bi.y & ~kSnSmallFlag)) sn_sweep_u_small(P, W, val, y, xo, nrhs, W.small[bi.x + wi], threadIdx.x & 31);
        sweep_release(W, blk, done);
        return;
    }
    const uint32_t s = W.meta[bi.x].x, w = W.meta[bi.x].y, t = bi.y;
    const uint32_t tid = threadIdx.x, n = P.n;
    __shared__ uint32_t sB[kSnMaxWidth], sC[kSnMaxWidth];
    if (tid < 32) {
        // entries of column s+c above the block: positions cptr[s+c] .. diag[s+c]-c-1
        const uint32_t c0 = tid, c1 = tid + 32;
        const uint32_t d0 = c0 < w ? P.diag[s + c0] : 0u, d1 = c1 < w ? P.diag[s + c1] : 0u;
        const uint32_t p0 = c0 < w ? P.cptr[s + c0] : 0u, p1 = c1 < w ? P.cptr[s + c1] : 0u;
        if (c0 < w) {
            sB[c0] = d0;
            sC[c0] = p0;
        }
        if (c1 < w) {
            sB[c1] = d1;
            sC[c1] = p1;
        }
        const uint32_t n0 = c0 < w ? (d0 - c0) - p0 : 0u, n1 = c1 < w ? (d1 - c1) - p1 : 0u;
        uint32_t a0 = n0, a1 = n1;  // inclusive warp scans
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y0 = __shfl_up_sync(0xffffffffu, a0, o), y1 = __shfl_up_sync(0xffffffffu, a1, o);
            if (tid >= uint32_t(o)) {
                a0 += y0;
                a1 += y1;
            }
        }
        const uint32_t tot0 = __shfl_sync(0xffffffffu, a0, 31);
        if (c0 < w) pre[c0] = a0 - n0;
        if (c1 < w) pre[c1] = tot0 + a1 - n1;
        if (c0 == w - 1) pre[w] = a0;
        if (c1 == w - 1) pre[w] = tot0 + a1;
    }
    __syncthreads();
    // U11 with its diagonal: U(s+k, s+c), k <= c, at diag[s+c] - (c - k); eight loads in flight
    for (uint32_t e0 = 0; e0 < w * kSnMaxWidth; e0 += 8 * 256) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t e = e0 + u * 256 + tid, c = e >> 6, k = e & 63;
            v[u] = (c < w && k <= c) ? __ldg(val + sB[c] - (c - k)) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t e = e0 + u * 256 + tid, c = e >> 6, k = e & 63;
            if (c < w && k <= c) sT[c * kLD + k] = v[u];
        }
    }
    __syncthreads();
    const uint32_t e0 = t * kSnSweepAbove, e1 = min(e0 + kSnSweepAbove, pre[w]);
    // kSnSweepAbove / 256 entries above the block per thread: column, target
    // and value do not depend on x, so they are loaded before the chain
    constexpr int kPer = int(kSnSweepAbove / 256);
    uint32_t ecol[kPer], etg[kPer];
    float eval[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const uint32_t e = e0 + tid + u * 256;
        ecol[u] = kSnMaxWidth;  // none
        etg[u] = 0u;
        eval[u] = 0.0f;
        if (e < e1) {
            uint32_t lo = 0, hi = w;  // last c with pre[c] <= e
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (pre[mid] <= e)
                    lo = mid;
                else
                    hi = mid;
            }
            const uint32_t p = sC[lo] + (e - pre[lo]);
            ecol[u] = lo;
            etg[u] = __ldg(P.ridx + p);
            eval[u] = __ldg(val + p);
        }
    }
    for (uint32_t q = 0; q < nrhs; ++q) {
        float *yq = y + size_t(q) * n;
        if (tid < 32) {
            const uint32_t k0 = tid, k1 = tid + 32;
            float v0 = k0 < w ? __ldcg(yq + s + k0) : 0.0f;
            float v1 = k1 < w ? __ldcg(yq + s + k1) : 0.0f;
            for (uint32_t cc = w; cc-- > 0;) {
                const float xc = __shfl_sync(0xffffffffu, cc < 32 ? v0 : v1, cc & 31) / sT[cc * kLD + cc];
                if (k0 == cc) v0 = xc;
                if (k1 == cc) v1 = xc;
                if (k0 < cc) v0 = __fsub_rn(v0, __fmul_rn(sT[cc * kLD + k0], xc));
                if (k1 < cc) v1 = __fsub_rn(v1, __fmul_rn(sT[cc * kLD + k1], xc));
            }
            if (k0 < w) xs[k0] = v0;
            if (k1 < w) xs[k1] = v1;
            if (t == 0) {
                if (k0 < w) xo[size_t(q) * n + s + k0] = v0;
                if (k1 < w) xo[size_t(q) * n + s + k1] = v1;
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            if (ecol[u] >= kSnMaxWidth) continue;
            const float xc = xs[ecol[u]];
            if (xc != 0.0f) atomicAdd(yq + etg[u], -__fmul_rn(eval[u], xc));
        }
        __syncthreads();
    }
    sweep_release(W, blk, done);
}

// Per-level launches of the small-supernode groups alone: blocks
// [b0, b0 + gridDim.x) of the map are all groups, one small supernode per
// warp.  Without the full kernels' 64-wide register rows and shared tiles
// four (L: 64 registers) or five (U: 48) blocks stay resident per SM instead of
// two or four, so the wide first levels of the L sweep (a quarter of a million
// leaf supernodes on the 700 x 700 mesh) take half the waves.  Each warp's
// chain is latency-bound (plan, pattern and factor loads, then w dependent
// steps), so resident warps set the rate.
__global__ void __launch_bounds__(256, 4) k_sn_sweep_l_small(DevPattern P, SnSweepPlan W, const float *__restrict__ val,
                                                          float *y, float *xo, uint32_t nrhs, uint32_t b0,
                                                          uint64_t vstride, uint64_t ystride) {
    pdl_release();
    pdl_wait();  // the previous level's x
    const uint2 bi = W.map[b0 + blockIdx.x];
    const uint32_t wi = threadIdx.x >> 5;
    if (!(bi.y & kSnSmallFlag) || wi >= (bi.y & ~kSnSmallFlag)) return;
    sn_sweep_l_small(P, W, val + blockIdx.z * vstride, y + blockIdx.z * ystride, xo + blockIdx.z * ystride, nrhs,
                     W.small[bi.x + wi], threadIdx.x & 31);
}

__global__ void __launch_bounds__(256, 5) k_sn_sweep_u_small(DevPattern P, SnSweepPlan W, const float *__restrict__ val,
                                                          float *y, float *xo, uint32_t nrhs, uint32_t b0,
                                                          uint64_t vstride, uint64_t ystride) {
    pdl_release();
    pdl_wait();  // the previous level's x
    const uint2 bi = W.map[b0 + blockIdx.x];
    const uint32_t wi = threadIdx.x >> 5;
    if (!(bi.y & kSnSmallFlag) || wi >= (bi.y & ~kSnSmallFlag)) return;
    sn_sweep_u_small(P, W, val + blockIdx.z * vstride, y + blockIdx.z * ystride, xo + blockIdx.z * ystride, nrhs,
                     W.small[bi.x + wi], threadIdx.x & 31);
}

__global__ void k_sn_copy(const float *__restrict__ xo, float *y, uint32_t t, uint32_t n) {
    const size_t off = size_t(blockIdx.y) * n;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < t; j += gridDim.x * blockDim.x) y[off + j] = xo[off + j];
}

cudaError_t run_sn_sweep(const DevPattern &P, const SnSweepPlan &W, bool upper, uint32_t t, const float *val,
                         float *y, float *xo, uint32_t nrhs, const SolveBatch &B, uint32_t *done, uint32_t *ticket,
                         uint32_t *status, uint32_t spin_limit, cudaStream_t st) {
    const uint64_t ystride = uint64_t(nrhs) * P.n;
    if (W.fused && done && W.nblocks) {
        // one launch: blocks in map order by ticket, supernodes wait for their releases
        cudaError_t e = cudaMemsetAsync(done, 0, sizeof(uint32_t) * size_t(W.ns) * B.count, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(ticket, 0, sizeof(uint32_t) * B.count, st);
        if (e != cudaSuccess) return e;
        const dim3 grid(W.nblocks, 1, B.count);
        if (upper)
            k_sn_sweep_u<<<grid, 256, 0, st>>>(P, W, val, y, xo, nrhs, 0, B.vstride, ystride, done, ticket, status,
                                               spin_limit);
        else
            k_sn_sweep_l<<<grid, 256, 0, st>>>(P, W, val, y, xo, nrhs, 0, B.vstride, ystride, done, ticket, status,
                                               spin_limit);
    } else {
        // one launch per level (two where its small-supernode groups get
        // their own), each chained to the one before (its blocks start while
        // the previous launch drains, and wait for its x); the supernodes of
        // one level do not feed each other, so its two launches may run in
        // either order
        for (uint32_t l = 0; l < W.nlev; ++l) {
            const SnSweepLevel &lv = W.levels[l];
            const uint2 k2 = sn_sweep_level_launches(lv, upper);
            cudaError_t e = cudaSuccess;
            if (k2.x) {  // the full kernel: the parts, and the groups unless they launch apart
                const dim3 grid(k2.y ? lv.big : lv.blocks, 1, B.count);
                if (upper)
                    e = launch_chained(k_sn_sweep_u, grid, dim3(256), 0, st, P, W, val, y, xo, nrhs, lv.b0, B.vstride,
                                       ystride, (uint32_t *)nullptr, (uint32_t *)nullptr, status, spin_limit);
                else
                    e = launch_chained(k_sn_sweep_l, grid, dim3(256), 0, st, P, W, val, y, xo, nrhs, lv.b0, B.vstride,
                                       ystride, (uint32_t *)nullptr, (uint32_t *)nullptr, status, spin_limit);
                if (e != cudaSuccess) return e;
            }
            if (k2.y) {  // the small-supernode groups
                const dim3 grid(lv.blocks - lv.big, 1, B.count);
                if (upper)
                    e = launch_chained(k_sn_sweep_u_small, grid, dim3(256), 0, st, P, W, val, y, xo, nrhs,
                                       lv.b0 + lv.big, B.vstride, ystride);
                else
                    e = launch_chained(k_sn_sweep_l_small, grid, dim3(256), 0, st, P, W, val, y, xo, nrhs,
                                       lv.b0 + lv.big, B.vstride, ystride);
                if (e != cudaSuccess) return e;
            }
        }
    }
    if (t > 0) {  // the vectors of all value sets are contiguous: nrhs * count of them
        uint32_t bx = (t + 255) / 256;
        if (bx > 1024) bx = 1024;
        k_sn_copy<<<dim3(bx, nrhs * B.count, 1), 256, 0, st>>>(xo, y, t, P.n);
    }
    return cudaGetLastError();
}

}  // namespace glu
