// Sparse part of the numeric factorization: the level-scheduled right-looking
// column algorithm of the reference (src/numeric.cu:10-345), for the columns
// in front of the dense trailing block.
//
// Per column k of a level (numeric.cu:36-47, 58-89):
//     d = U(k,k)                      (GESP: |d| < pert -> d = pert)
//     L(i,k) /= d                     for i in Lpat(k)
//     A(i,j) -= L(i,k) * A(k,j)       for j in Urow(k), i in Lpat(k)
// Columns of one level are independent except that several may update the
// same A(i,j), so multi-column levels update with atomics (as the reference
// does, numeric.cu:82) and single-column levels with plain read-modify-write.
//
// Differences from the reference's kernels, same arithmetic:
//  * Work is split into items (column k, update target j, chunk of Lpat(k))
//    spread evenly over lane groups, instead of one block per column; the
//    target position of each L row in column j is found in the sorted row list
//    (window search, usually a direct hit) instead of scanning all of column j
//    against an n-long dense scratch column (numeric.cu:58-89), so there is no
//    scratch memory and no atomics on rows outside Lpat(k).
//  * A(k,j) is located through the CSR->CSC position map.
//  * The division L(i,k)/d is recomputed by every reader in the level and the
//    scaled value is written back by the launch that runs the next level
//    (nothing in that launch reads or writes those entries), which removes one
//    grid-wide barrier per level.
//  * Runs of narrow levels execute inside one thread-block cluster that steps
//    through them with hardware cluster barriers (no launch and no host
//    round-trip per level, numeric.cu:615-616).
#include <cooperative_groups.h>

#include "glu_common.cuh"
#include "glu_kernels.h"

namespace cg = cooperative_groups;

namespace glu {

__device__ __forceinline__ float effective_pivot(float d, float pert) {
    // numeric.cu:139-140: a pivot below the threshold is replaced by +pert.
    return (pert > 0.0f && fabsf(d) < pert) ? pert : d;
}

// Scaling of one column's L part (lanes [0,G) of a group).
__device__ __forceinline__ void scale_column(const DevPattern &P, float *__restrict__ val,
                                             uint32_t k, float pert, uint32_t lane, uint32_t G) {
    uint32_t dk = P.diag[k];
    uint32_t l0 = dk + 1, l1 = P.cptr[k + 1];
    float d0 = ld_cg(val + dk);
    float d = effective_pivot(d0, pert);
    for (uint32_t p = l0 + lane; p < l1; p += G) st_cg(val + p, ld_cg(val + p) / d);
    if (lane == 0 && d != d0) st_cg(val + dk, d);
}

// One work item: column k, its jj-th update target, elements [e0, e1) of Lpat(k).
template <bool kAtomic>
__device__ __forceinline__ void update_item(const DevPattern &P, float *__restrict__ val, uint32_t k,
                                            uint32_t jj, uint32_t e0, uint32_t e1, float pert,
                                            uint32_t lane, uint32_t G) {
    uint32_t dk = P.diag[k];
    uint32_t lk0 = dk + 1;
    uint32_t nl = P.cptr[k + 1] - lk0;
    uint32_t e = P.rdiag[k] + 1 + jj;
    uint32_t j = P.cidx[e];
    uint32_t pkj = P.cpos[e];
    float d = effective_pivot(ld_cg(val + dk), pert);
    float s = ld_cg(val + pkj);
    uint32_t t0 = pkj + 1;
    uint32_t nt = P.cptr[j + 1] - t0;
    if (nt < nl) return;  // Lpat(k) must lie inside column j (fill closure); never true for a valid pattern
    uint32_t extra = nt - nl;  // rows of column j below k that are not in Lpat(k)
    for (uint32_t t = e0 + lane; t < e1; t += G) {
        float l = ld_cg(val + lk0 + t) / d;
        uint32_t q = t0 + t;
        if (extra) q = lower_bound_u32(P.ridx, q, q + extra, __ldg(P.ridx + lk0 + t));
        float prod = __fmul_rn(l, s);
        if (kAtomic)
            atomicAdd(val + q, -prod);
        else
            st_cg(val + q, __fsub_rn(ld_cg(val + q), prod));
    }
}

// Items [it0, it1) of one level (sched range [s0, s1)), strided over groups.
__device__ __forceinline__ void level_items(const DevPattern &P, const FactorPlanDev &F,
                                            float *__restrict__ val, uint32_t s0, uint32_t s1,
                                            uint32_t G, bool atomic, float pert, uint32_t group,
                                            uint32_t ngroups, uint32_t lane) {
    const uint32_t CH = G * kItemUnroll;
    uint32_t it0 = F.item_off[s0], it1 = F.item_off[s1];
    for (uint32_t it = it0 + group; it < it1; it += ngroups) {
        uint32_t s = upper_slot(F.item_off, s0, s1, it);
        uint32_t k = F.sched_cols[s];
        uint32_t rem = it - F.item_off[s];
        uint32_t nl = P.cptr[k + 1] - P.diag[k] - 1;
        uint32_t nch = (nl + CH - 1) / CH;
        uint32_t jj = rem / nch, ch = rem - jj * nch;
        uint32_t e0 = ch * CH, e1 = min(e0 + CH, nl);
        if (atomic) {
            update_item<true>(P, val, k, jj, e0, e1, pert, lane, G);
        } else {
            update_item<false>(P, val, k, jj, e0, e1, pert, lane, G);
        }
    }
}

// One level per launch: blocks [0, scale_blocks) scale the L parts of the
// previous level's columns (sched range [q0, q1)), the rest run this level's
// update items.  blockIdx.z selects the value set.
__global__ void __launch_bounds__(256) k_factor_level(DevPattern P, FactorPlanDev F, float *val_base,
                                                      uint64_t val_stride, const float *pert_z,
                                                      uint32_t s0, uint32_t s1, uint32_t G,
                                                      uint32_t atomic, uint32_t q0, uint32_t q1,
                                                      uint32_t scale_blocks) {
    float *val = val_base + blockIdx.z * val_stride;
    float pert = pert_z ? pert_z[blockIdx.z] : 0.0f;
    uint32_t tid = threadIdx.x;
    if (blockIdx.x < scale_blocks) {
        uint32_t w = blockIdx.x * (blockDim.x / 32) + tid / 32;
        uint32_t lane = tid & 31;
        if (q0 + w < q1) scale_column(P, val, F.sched_cols[q0 + w], pert, lane, 32);
        return;
    }
    uint32_t groups_per_block = blockDim.x / G;
    uint32_t group = (blockIdx.x - scale_blocks) * groups_per_block + tid / G;
    uint32_t ngroups = (gridDim.x - scale_blocks) * groups_per_block;
    level_items(P, F, val, s0, s1, G, atomic != 0, pert, group, ngroups, tid % G);
}

// Scaling of the last level's columns (sched range [q0, q1)).
__global__ void __launch_bounds__(256) k_scale_level(DevPattern P, FactorPlanDev F, float *val_base,
                                                     uint64_t val_stride, const float *pert_z,
                                                     uint32_t q0, uint32_t q1) {
    float *val = val_base + blockIdx.z * val_stride;
    float pert = pert_z ? pert_z[blockIdx.z] : 0.0f;
    uint32_t w = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    uint32_t lane = threadIdx.x & 31;
    for (; q0 + w < q1; w += gridDim.x * (blockDim.x / 32))
        scale_column(P, val, F.sched_cols[q0 + w], pert, lane, 32);
}

// A run of narrow levels [l0, l1) inside one cluster (one cluster per value
// set, cluster = the blocks with the same blockIdx.z).  Level l's items run
// together with the scaling of level l-1; a cluster barrier separates levels.
// Values are read through L2 (ld.cg) because other blocks of the cluster wrote
// them since the launch began.
__global__ void __launch_bounds__(kChainThreads) k_factor_chain(DevPattern P, FactorPlanDev F,
                                                                float *val_base, uint64_t val_stride,
                                                                const float *pert_z, uint32_t l0,
                                                                uint32_t l1) {
    cg::cluster_group cluster = cg::this_cluster();
    float *val = val_base + blockIdx.z * val_stride;
    float pert = pert_z ? pert_z[blockIdx.z] : 0.0f;
    const uint32_t nblk = cluster.num_blocks();
    const uint32_t rank = cluster.block_rank();
    const uint32_t tid = threadIdx.x;
    for (uint32_t l = l0; l < l1; ++l) {
        LevelInfo li = F.levels[l];
        uint32_t G = li.G;
        uint32_t groups_per_block = blockDim.x / G;
        level_items(P, F, val, li.s0, li.s1, G, li.atomic != 0, pert,
                    rank * groups_per_block + tid / G, nblk * groups_per_block, tid % G);
        if (l > 0) {  // scale the previous level
            LevelInfo lp = F.levels[l - 1];
            uint32_t w = rank * (blockDim.x / 32) + tid / 32;
            for (uint32_t q = lp.s0 + w; q < lp.s1; q += nblk * (blockDim.x / 32))
                scale_column(P, val, F.sched_cols[q], pert, tid & 31, 32);
        }
        cluster.sync();
    }
}

// ---------------------------------------------------------------- launchers --
const void *chain_kernel_ptr() { return reinterpret_cast<const void *>(k_factor_chain); }

cudaError_t launch_factor_level(const DevPattern &P, const FactorPlanDev &F, float *val,
                                uint64_t stride, uint32_t count, const float *pert_z,
                                const LevelInfo &cur, const LevelInfo *prev, uint32_t items,
                                cudaStream_t st) {
    const uint32_t threads = 256;
    uint32_t q0 = prev ? prev->s0 : 0, q1 = prev ? prev->s1 : 0;
    uint32_t scale_blocks = (q1 - q0 + (threads / 32) - 1) / (threads / 32);
    uint32_t groups_per_block = threads / cur.G;
    uint32_t item_blocks = (items + groups_per_block - 1) / groups_per_block;
    if (item_blocks > kMaxItemBlocks) item_blocks = kMaxItemBlocks;
    dim3 grid(scale_blocks + item_blocks, 1, count);
    k_factor_level<<<grid, threads, 0, st>>>(P, F, val, stride, pert_z, cur.s0, cur.s1, cur.G,
                                             cur.atomic, q0, q1, scale_blocks);
    return cudaGetLastError();
}

cudaError_t launch_scale_level(const DevPattern &P, const FactorPlanDev &F, float *val,
                               uint64_t stride, uint32_t count, const float *pert_z,
                               const LevelInfo &lv, cudaStream_t st) {
    uint32_t cols = lv.s1 - lv.s0;
    if (cols == 0) return cudaSuccess;
    uint32_t blocks = (cols + 7) / 8;
    if (blocks > 4096) blocks = 4096;
    k_scale_level<<<dim3(blocks, 1, count), 256, 0, st>>>(P, F, val, stride, pert_z, lv.s0, lv.s1);
    return cudaGetLastError();
}

cudaError_t launch_factor_chain(const DevPattern &P, const FactorPlanDev &F, float *val,
                                uint64_t stride, uint32_t count, const float *pert_z, uint32_t l0,
                                uint32_t l1, uint32_t cluster, cudaStream_t st) {
    static PerDeviceOnce cluster_attr;
    cudaError_t e = cluster_attr.run([] {
        return cudaFuncSetAttribute(k_factor_chain, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster, 1, count);
    cfg.blockDim = dim3(kChainThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_factor_chain, P, F, val, stride, pert_z, l0, l1);
}

}  // namespace glu
