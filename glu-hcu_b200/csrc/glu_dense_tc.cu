// Trailing update of the dense tail on the 5th-generation tensor cores.
//
// The blocked dense LU of the trailing block (glu_factor_dense.cu) spends
// almost all of its flops in A22 -= L21 U12 with K = 64 .. 256 (one panel or a
// group of up to four), and the deferred coupling of the sparse part adds products of the
// same form.  Here that product runs as tcgen05.mma kind::f16 on BF16
// operands with FP32 accuracy kept by splitting every operand into three BF16
// parts,
//     a = a0 + a1 + a2,  a0 = rna_bf16(a), a1 = rna_bf16(a - a0),
//                        a2 = a - a0 - a1
// (exact: a - a0 has at most 15 significant bits, a - a0 - a1 at most 7, so
// 3 x 8 bits cover FP32's 24), and keeping every product term down to
// 2^-24 relative:
//     a b ~= a0 b0 + (a0 b1 + a1 b0) + (a0 b2 + a1 b1 + a2 b0) + (a1 b2 + a2 b1),
// whose error, about 2^-32 |a b|, is far under FP32 rounding -- 8 BF16 MMAs
// per 16 of K, two thirds of the tensor time of the 6 TF32 products a TF32
// split needs for the same accuracy, and half its operand bytes.  The big
// term a0 b0 (exact in FP32) and the small terms go to separate FP32
// accumulators in tensor memory over the whole K of the update (8 MMAs of K =
// 16 for a panel pair), so the small terms' truncating accumulation stays
// 2^-8 below the big one's; the tile's two sums are then subtracted from the
// entry in FP32 with round to nearest, c := (c - big) - small.  The big sum
// takes one truncation per MMA (K / 16 in all; the FMA kernel rounds once per
// product), and the tile's C is read and written once.

// Data flow per update:
//   1. k_dense_pack, after each panel: the panel's L21 rows and U12 columns
//      split into their three BF16 parts, written K-major as rows of 768
//      BF16 values (slots 0..255 part 0, 256..511 part 1, 512..767 part 2;
//      panel j of a group fills slots 64 j .. 64 j + 63 of each part) -- the
//      operand layout the MMA reads.
//   2. k_dense_update_tc, persistent (one CTA per SM), per 128 x 128 tile of
//      the trailing block:
//        warp 0   TMA producer: cp.async.bulk.tensor loads of 128 x 64 BF16
//                 operand boxes (128-byte swizzle), three parts of A and of B
//                 per 64-wide K chunk (one panel), into a 2-stage ring;
//        warp 1   MMA issuer: 8 tcgen05.mma (M = N = 128, K = 16) per 16
//                 of K into one of two accumulator pairs (big, small), the
//                 pair of the tile before being read meanwhile;
//        warps 2-9 epilogue (two per TMEM lane quarter, 64 columns each):
//                 load the C tile into registers while the MMAs run,
//                 tcgen05.ld the tile's two sums, subtract them, hand the
//                 pair back, store the tile;
//        warp 10  prefetch: each tile's C columns into L2 as soon as the
//                 tile is drawn, so that the epilogue's loads hit L2.
//      C stays where it lies (element (i, j) at val[doff[j] + i]), so in-place
//      tails with irregular column offsets need no copy.
// All waits on mbarriers are bounded (spin_limit polls); a wait that runs out
// sets DEV_TIMEOUT, every role leaves its loop, the CTA waits for its own
// copies and MMAs in flight and frees its tensor memory before returning.
//
// The reference's counterpart is the per-column Schur update
// RL_onecol_updateSubmat (src/numeric.cu:270-319).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "glu_common.cuh"
#include "glu_kernels.h"

namespace glu {
namespace {

constexpr int kTile = 128;                               // M = N of an update tile
constexpr int kChunk = 64;                               // K per stage: one 128-byte row of BF16
constexpr int kStages = 2;
constexpr int kParts = 3;                                // BF16 parts of an operand
constexpr int kSlots = 256;                              // K slots per part: up to four panels
constexpr int kPackRow = kParts * kSlots;                // BF16 values per pack row
constexpr uint32_t kOpBytes = kTile * kChunk * 2;        // one operand part of one stage (16 KB)
constexpr uint32_t kStageBytes = 2 * kParts * kOpBytes;  // A0, A1, A2, B0, B1, B2
constexpr int kEpiWarps = 8;                             // two per TMEM lane quarter, 64 columns each
constexpr int kPrefetchWarp = 2 + kEpiWarps;             // C tiles into L2 ahead of the epilogue
constexpr int kThreads = 32 * (3 + kEpiWarps);           // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue, warp 10 prefetch
constexpr uint32_t kTmemCols = 4 * kTile;                // two pairs (big, small) of FP32 accumulators
constexpr size_t kBarBytes = 256;
constexpr int kRing = 4;  // tile ids in flight between the producer and the other roles
constexpr size_t kOffBytes = sizeof(uint32_t) * kEpiWarps * 64;  // the epilogue warps' column offsets
constexpr size_t kSmemBytes = kStages * kStageBytes + kBarBytes + kOffBytes + 1024;  // + alignment slack

// Instruction descriptor of tcgen05.mma kind::f16: D FP32 (bits 4-5 = 1), A
// and B BF16 (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at
// bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kTile >> 3) << 17) |
                            (uint32_t(kTile >> 4) << 24);

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor of a K-major operand tile in the canonical
// 128-byte-swizzled layout written by a TMA box of 64 BF16 x rows: rows of
// 128 bytes, 8-row groups 1024 bytes apart (stride byte offset), layout type 2
// (128-byte swizzle) at bits 61-63, descriptor version 1 at bits 46-47.  The
// leading byte offset is unused for swizzled K-major layouts.
__device__ __forceinline__ uint64_t kmajor_sw128_desc(uint32_t saddr) {
    uint64_t d = uint64_t((saddr & 0x3FFFFu) >> 4);
    d |= uint64_t(1) << 16;
    d |= uint64_t(1024 >> 4) << 32;
    d |= uint64_t(1) << 46;
    d |= uint64_t(2) << 61;
    return d;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the completion of the phase with the given parity; false when
// `limit` polls pass first.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y,
                                            int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(kIdesc), "r"(accumulate)
        : "memory");
}
// Arrives (once) on the mbarrier when every tcgen05 operation this thread has
// issued so far is complete.
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// 32 consecutive FP32 columns at each of two TMEM addresses of this thread's
// lane, one wait for both.
__device__ __forceinline__ void tc_ld32x2(uint32_t ta, uint32_t tb, float (&va)[32], float (&vb)[32]) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%64];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, "
        "%45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%65];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(ta), "r"(tb)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        va[i] = __uint_as_float(r[i]);
        vb[i] = __uint_as_float(r[32 + i]);
    }
}

struct Tile {
    uint32_t z, rbase, cbase;
};
__device__ __forceinline__ Tile decode_tile(uint32_t t, uint32_t tiles_r, uint32_t tiles_c, const DenseRegion &reg) {
    const uint32_t per = tiles_r * tiles_c;
    Tile o;
    o.z = t / per;
    const uint32_t rem = t - o.z * per;
    const uint32_t tr = rem / tiles_c;
    o.rbase = reg.r_lo + tr * kTile;
    o.cbase = reg.c_lo + (rem - tr * tiles_c) * kTile;
    return o;
}

}  // namespace

// ---------------------------------------------------------------- pack --
// Rows [r_start, m) of the panel's L21 (columns k0 .. k0 + kb - 1) and
// columns [r_start, m) of its U12 (rows k0 .. k0 + kb - 1), split into three
// BF16 parts: pack[z][i][256 * p + slot0 + k] = part p, for k < 64 (zero for
// k >= kb).  Blocks [0, nA) take 128 rows of L21 each, the rest 128 columns of
// U12; blockIdx.z selects the value set.
__global__ void __launch_bounds__(256) k_dense_pack(const float *__restrict__ val_base, uint64_t stride,
                                                    const uint32_t *__restrict__ doff, uint32_t m, uint32_t k0,
                                                    uint32_t kb, uint32_t slot0, uint32_t r_start, uint32_t nA,
                                                    uint16_t *__restrict__ packA, uint16_t *__restrict__ packB) {
    __shared__ float sT[kDenseNB][kTile + 1];
    const float *val = val_base + blockIdx.z * stride;
    const uint32_t tid = threadIdx.x;
    const uint32_t r = tid >> 1, h = tid & 1;  // writer: row (or column) r, K half h
    float x[32];
    uint16_t *dst = nullptr;
    if (blockIdx.x < nA) {
        const uint32_t row0 = r_start + blockIdx.x * kTile;
        for (uint32_t e = tid; e < uint32_t(kDenseNB) * kTile; e += blockDim.x) {
            const uint32_t k = e / kTile, rr = e - k * kTile;
            sT[k][rr] = (k < kb && row0 + rr < m) ? ld_cg(val + doff[k0 + k] + row0 + rr) : 0.0f;
        }
        __syncthreads();
        if (row0 + r >= m) return;
#pragma unroll
        for (int i = 0; i < 32; ++i) x[i] = sT[h * 32 + i][r];
        dst = packA + (size_t(blockIdx.z) * m + row0 + r) * kPackRow + slot0 + h * 32;
    } else {
        const uint32_t j = r_start + (blockIdx.x - nA) * kTile + r;
        if (j >= m) return;
        const float *src = val + doff[j] + k0 + h * 32;
#pragma unroll
        for (int i = 0; i < 32; ++i) x[i] = (h * 32 + i < kb) ? ld_cg(src + i) : 0.0f;
        dst = packB + (size_t(blockIdx.z) * m + j) * kPackRow + slot0 + h * 32;
    }
#pragma unroll
    for (int i = 0; i < 32; i += 4) {
        const float v[4] = {x[i], x[i + 1], x[i + 2], x[i + 3]};
        uint2 p0, p1, p2;
        split_bf16x4(v, p0, p1, p2);
        *reinterpret_cast<uint2 *>(dst + i) = p0;
        *reinterpret_cast<uint2 *>(dst + kSlots + i) = p1;
        *reinterpret_cast<uint2 *>(dst + 2 * kSlots + i) = p2;
    }
}

// ------------------------------------------------------- coupling pack --
// Operands of one group of deferred sparse columns (up to 128, slots slot0 ..
// slot0 + ncols - 1): packA[z][i][256 p + s] = part p of L(t + i, k_s),
// packB[z][j][256 p + s] = part p of U(k_s, t + j), zero where the pattern has
// no entry and for slots past the group.  Block b < nblk takes tail rows
// [128 b, 128 b + 128): four threads of slot s walk column k_s's CSC entries
// [lstart[g][b], lstart[g][b + 1]) (g = slot0 + s), the ones in those rows.
// Block nblk + b takes tail columns [128 b, 128 b + 128): four threads of slot
// s walk row k_s's CSR entries [ustart[g][b], ustart[g][b + 1]), the ones in
// those columns (their CSC positions from cpos).  The start tables (nblk + 1 entries
// per slot) are computed with the plan.  A 128 x 128 tile in shared memory,
// then coalesced writes of the three BF16 parts.
constexpr uint32_t kCoupleLd = kTile + 1;
constexpr size_t kCoupleSmem = sizeof(float) * kTile * kCoupleLd;
constexpr uint32_t kCoupleWalkers = 4;  // threads walking one slot's entries
constexpr uint32_t kCoupleThreads = kTile * kCoupleWalkers;

__global__ void __launch_bounds__(kCoupleThreads) k_couple_pack(const uint32_t *__restrict__ ridx,
                                                       const uint32_t *__restrict__ cidx,
                                                       const uint32_t *__restrict__ cpos,
                                                       const float *__restrict__ val_base, uint64_t stride,
                                                       uint32_t t, uint32_t m, uint32_t ncols, uint32_t slot0,
                                                       const uint32_t *__restrict__ lstart,
                                                       const uint32_t *__restrict__ ustart, uint32_t nblk,
                                                       uint16_t *__restrict__ packA, uint16_t *__restrict__ packB) {
    extern __shared__ float sT[];  // [128][kCoupleLd]: sT[r * kCoupleLd + s]
    const float *val = val_base + blockIdx.z * stride;
    const uint32_t tid = threadIdx.x;
    const bool aside = blockIdx.x < nblk;
    const uint32_t b = aside ? blockIdx.x : blockIdx.x - nblk, b0 = b * kTile;
    for (uint32_t e = tid; e < kTile * kCoupleLd; e += kCoupleThreads) sT[e] = 0.0f;
    __syncthreads();
    // kCoupleWalkers threads per slot, each every kCoupleWalkers-th entry
    const uint32_t sl = tid % kTile, wk = tid / kTile;
    if (sl < ncols) {
        const uint32_t *st = (aside ? lstart : ustart) + size_t(slot0 + sl) * (nblk + 1) + b;
        const uint32_t p0 = __ldg(st) + wk, p1 = __ldg(st + 1);
        if (aside) {
            for (uint32_t p = p0; p < p1; p += kCoupleWalkers)
                sT[(__ldg(ridx + p) - t - b0) * kCoupleLd + sl] = ld_cg(val + p);
        } else {
            for (uint32_t e = p0; e < p1; e += kCoupleWalkers)
                sT[(__ldg(cidx + e) - t - b0) * kCoupleLd + sl] = ld_cg(val + __ldg(cpos + e));
        }
    }
    __syncthreads();
    uint16_t *pack = aside ? packA : packB;
    const uint32_t rows = min(uint32_t(kTile), m - b0);
    for (uint32_t e = tid; e < rows * (kTile / 4); e += kCoupleThreads) {
        const uint32_t r = e / (kTile / 4), q = e - r * (kTile / 4);
        const float *src = sT + r * kCoupleLd + 4 * q;
        const float v[4] = {src[0], src[1], src[2], src[3]};
        uint2 p0, p1, p2;
        split_bf16x4(v, p0, p1, p2);
        uint16_t *dst = pack + (size_t(blockIdx.z) * m + b0 + r) * kPackRow + 4 * q;
        *reinterpret_cast<uint2 *>(dst) = p0;
        *reinterpret_cast<uint2 *>(dst + kSlots) = p1;
        *reinterpret_cast<uint2 *>(dst + 2 * kSlots) = p2;
    }
}

// -------------------------------------------------------------- update --
// Rows [r_lo, r_hi) x columns [c_lo, c_hi) of the trailing block after the
// panels [k0, k0 + K) (relative to r0 = k0 + K), in 128 x 128 tiles; K =
// 32 * nchunks (pack slots beyond the panels' width hold zeros).  Entries of
// a tile outside the region are computed but neither read nor written.
__global__ void __launch_bounds__(kThreads, 1)
    k_dense_update_tc(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                      float *val_base, uint64_t stride, const uint32_t *__restrict__ doff, uint32_t m, uint32_t r0,
                      uint32_t nchunks, DenseRegion reg, uint32_t tiles_r, uint32_t tiles_c, uint32_t count,
                      const float *__restrict__ diag_scratch, uint32_t *status, uint32_t spin_limit,
                      uint32_t *tile_counter) {
    extern __shared__ uint8_t tc_smem_raw[];
    uint8_t *smem = tc_smem_raw + ((1024u - (smem_addr(tc_smem_raw) & 1023u)) & 1023u);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kStages * kStageBytes);
    uint64_t *full = bars;                   // [kStages] stage loaded (TMA bytes)
    uint64_t *empty = bars + kStages;        // [kStages] stage consumed (MMA commit)
    uint64_t *acc_full = bars + 2 * kStages;  // [2] accumulator ready (MMA commit)
    uint64_t *acc_empty = acc_full + 2;       // [2] accumulator read (the epilogue warps)
    uint64_t *done = acc_empty + 2;           // all MMAs of this CTA complete
    uint64_t *tile_full = done + 1;           // [kRing] tile id written (producer)
    uint64_t *tile_empty = tile_full + kRing;  // [kRing] tile id read (MMA issuer, epilogue and prefetch warps)
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tile_empty + kRing);
    uint32_t *tile_id = tmem_slot + 1;        // [kRing]
    uint32_t *epi_off = reinterpret_cast<uint32_t *>(smem + kStages * kStageBytes + kBarBytes);  // [warps][64]
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t total = tiles_r * tiles_c * count;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], kEpiWarps);
        }
        mbar_init(done, 1);
        for (int j = 0; j < kRing; ++j) {
            mbar_init(&tile_full[j], 1);
            mbar_init(&tile_empty[j], 2 + kEpiWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        tc_fence_before();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t g = 0;
            bool ok = true;
            // tiles are drawn from a counter shared by all CTAs (a CTA that
            // starts late takes fewer); each id goes to the other roles through
            // the ring, the id past the last tile ends their loops
            for (uint32_t i = 0; ok; ++i) {
                const uint32_t slot = i % kRing, sph = (i / kRing) & 1;
                if (!mbar_wait(&tile_empty[slot], sph ^ 1, spin_limit)) {
                    ok = false;
                    break;
                }
                const uint32_t t = atomicAdd(tile_counter, 1u);
                tile_id[slot] = t < total ? t : total;
                mbar_arrive(&tile_full[slot]);
                if (t >= total) break;
                const Tile tl = decode_tile(t, tiles_r, tiles_c, reg);
                const int ya = int(r0 + tl.rbase), yb = int(r0 + tl.cbase), zz = int(tl.z);
                for (uint32_t kc = 0; kc < nchunks; ++kc, ++g) {
                    const uint32_t s = g % kStages, ph = (g / kStages) & 1;
                    if (!mbar_wait(&empty[s], ph ^ 1, spin_limit)) {
                        ok = false;
                        break;
                    }
                    uint8_t *st = smem + s * kStageBytes;
                    mbar_arrive_expect_tx(&full[s], kStageBytes);
#pragma unroll
                    for (int p = 0; p < kParts; ++p) {
                        const int x = int(p * kSlots + kc * kChunk);
                        tma_load_3d(st + p * kOpBytes, &mapA, &full[s], x, ya, zz);
                        tma_load_3d(st + (kParts + p) * kOpBytes, &mapB, &full[s], x, yb, zz);
                    }
                }
            }
            if (!ok) atomicOr(status, DEV_TIMEOUT);
            // the last load into every stage lands before the CTA may exit
            for (uint32_t s = 0; s < uint32_t(kStages) && s < g; ++s) {
                const uint32_t f = s + ((g - 1 - s) / kStages) * kStages;
                if (!mbar_wait(&full[s], (f / kStages) & 1, spin_limit)) atomicOr(status, DEV_TIMEOUT);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            uint32_t g = 0;  // stages consumed
            uint32_t u = 0;  // tiles issued (accumulator pair u & 1)
            bool ok = true;
            for (uint32_t i = 0; ok; ++i) {
                const uint32_t slot = i % kRing, sph = (i / kRing) & 1;
                if (!mbar_wait(&tile_full[slot], sph, spin_limit)) {
                    ok = false;
                    break;
                }
                const uint32_t t = tile_id[slot];
                mbar_arrive(&tile_empty[slot]);
                if (t >= total) break;
                // the tile's accumulator pair: free once the epilogue has read
                // the tile two before this one
                const uint32_t a = u & 1, aph = (u >> 1) & 1;
                ++u;
                if (!mbar_wait(&acc_empty[a], aph ^ 1, spin_limit)) {
                    ok = false;
                    break;
                }
                const uint32_t d_big = tmem + a * 2 * kTile, d_small = d_big + kTile;
                for (uint32_t kc = 0; kc < nchunks; ++kc, ++g) {
                    const uint32_t s = g % kStages, ph = (g / kStages) & 1;
                    if (!mbar_wait(&full[s], ph, spin_limit)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t base = smem_addr(smem + s * kStageBytes);
#pragma unroll
                    for (uint32_t k16 = 0; k16 < kChunk / 16; ++k16) {
                        const uint32_t off = k16 * 32;  // 16 BF16 values = 32 bytes along K
                        uint64_t A[kParts], B[kParts];
#pragma unroll
                        for (int p = 0; p < kParts; ++p) {
                            A[p] = kmajor_sw128_desc(base + p * kOpBytes + off);
                            B[p] = kmajor_sw128_desc(base + (kParts + p) * kOpBytes + off);
                        }
                        const uint32_t acc = (kc | k16) != 0;
                        tc_mma_bf16(d_small, A[1], B[2], acc);  // 2^-24 terms first
                        tc_mma_bf16(d_small, A[2], B[1], 1);
                        tc_mma_bf16(d_small, A[0], B[2], 1);  // 2^-16 terms
                        tc_mma_bf16(d_small, A[1], B[1], 1);
                        tc_mma_bf16(d_small, A[2], B[0], 1);
                        tc_mma_bf16(d_small, A[0], B[1], 1);  // 2^-8 terms
                        tc_mma_bf16(d_small, A[1], B[0], 1);
                        tc_mma_bf16(d_big, A[0], B[0], acc);
                    }
                    tc_commit(&empty[s]);
                }
                if (!ok) break;
                tc_commit(&acc_full[a]);
            }
            if (!ok) atomicOr(status, DEV_TIMEOUT);
            tc_commit(done);
            if (!mbar_wait(done, 0, spin_limit)) atomicOr(status, DEV_TIMEOUT);
        }
    } else if (warp == kPrefetchWarp) {
        // ------------------------------------------------ C prefetch
        // Each tile's C columns (128 rows, 512 bytes each) into L2 as soon as
        // the producer has drawn the tile, up to kRing tiles ahead of the
        // epilogue, whose loads then hit L2 instead of waiting on DRAM.
        for (uint32_t i = 0;; ++i) {
            const uint32_t slot = i % kRing, sph = (i / kRing) & 1;
            if (!__all_sync(0xffffffffu, mbar_wait(&tile_full[slot], sph, spin_limit))) {
                if (lane == 0) atomicOr(status, DEV_TIMEOUT);
                break;
            }
            const uint32_t t = tile_id[slot];
            __syncwarp();
            if (lane == 0) mbar_arrive(&tile_empty[slot]);
            if (t >= total) break;
            const Tile tl = decode_tile(t, tiles_r, tiles_c, reg);
            const float *val = val_base + tl.z * stride;
            const uint32_t rows = min(uint32_t(kTile), reg.r_hi - tl.rbase);
            for (uint32_t cc = lane; cc < uint32_t(kTile); cc += 32) {
                const uint32_t col = tl.cbase + cc;
                if (col >= reg.c_hi) break;
                const float *p0 = val + __ldg(doff + r0 + col) + r0 + tl.rbase;
                const uintptr_t a0 = reinterpret_cast<uintptr_t>(p0) & ~uintptr_t(127);
                const uintptr_t a1 = reinterpret_cast<uintptr_t>(p0 + rows - 1);
                for (uintptr_t a = a0; a <= a1; a += 128)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
            }
        }
    } else {
        // ------------------------------------------------ epilogue
        // Warp w takes TMEM lane quarter w % 4 (the quarter a warp may
        // access) and tile columns [64 h, 64 h + 64), h = (w - 2) / 4: two
        // warps per quarter, so two per SM sub-partition hide each other's
        // latencies.  Column offsets go through shared memory once per tile;
        // interior tiles take a path without per-entry bounds.
        const uint32_t ew = warp - 2;
        const uint32_t q = warp & 3;
        const uint32_t half = ew >> 2;
        const uint32_t row = q * 32 + lane;  // tile row of this thread
        uint32_t *soff = epi_off + ew * 64;
        if (reg.writeback) {
            // the factored diagonal block of the panel at wb_k0, kept in
            // scratch while that panel's blocks still read the original
            const uint32_t et = threadIdx.x - 64, wk = reg.wb_k0, wb = min(uint32_t(kDenseNB), m - wk);
            for (uint32_t z = blockIdx.x; z < count; z += gridDim.x) {
                float *val = val_base + z * stride;
                const float *ds = diag_scratch + size_t(z) * kDenseNB * kDenseNB;
                for (uint32_t e = et; e < wb * wb; e += 32 * kEpiWarps) {
                    const uint32_t c = e / wb, rr = e - c * wb;
                    st_cg(val + doff[wk + c] + wk + rr, ds[c * kDenseNB + rr]);
                }
            }
        }
        uint32_t u = 0;  // tiles taken, as the MMA issuer counts them
        for (uint32_t i = 0;; ++i) {
            const uint32_t slot = i % kRing, sph = (i / kRing) & 1;
            if (!__all_sync(0xffffffffu, mbar_wait(&tile_full[slot], sph, spin_limit))) {
                if (lane == 0) atomicOr(status, DEV_TIMEOUT);
                break;
            }
            const uint32_t t = tile_id[slot];
            __syncwarp();
            if (lane == 0) mbar_arrive(&tile_empty[slot]);
            if (t >= total) break;
            const Tile tl = decode_tile(t, tiles_r, tiles_c, reg);
            float *val = val_base + tl.z * stride;
            const uint32_t c0 = tl.cbase + half * 64;  // first tile column of this warp
            const uint32_t ncol = c0 < reg.c_hi ? min(64u, reg.c_hi - c0) : 0u;
            const bool rok = tl.rbase + row < reg.r_hi;
            const bool full_tile = __all_sync(0xffffffffu, rok) && ncol == 64;
            const uint32_t grow = r0 + tl.rbase + row;
            // column offsets of this warp's 64 columns (the previous tile's
            // reads of them are done: the warp reached this point together)
            for (uint32_t e = lane; e < 64; e += 32) soff[e] = e < ncol ? __ldg(doff + r0 + c0 + e) : 0u;
            __syncwarp();
            // C into registers while the MMAs run
            float c[64];
            if (full_tile) {
#pragma unroll
                for (int jj = 0; jj < 64; jj += 4) {
                    const uint4 o = *reinterpret_cast<const uint4 *>(soff + jj);
                    c[jj] = ld_cg(val + o.x + grow);
                    c[jj + 1] = ld_cg(val + o.y + grow);
                    c[jj + 2] = ld_cg(val + o.z + grow);
                    c[jj + 3] = ld_cg(val + o.w + grow);
                }
            } else {
#pragma unroll
                for (int jj = 0; jj < 64; ++jj) c[jj] = (rok && uint32_t(jj) < ncol) ? ld_cg(val + soff[jj] + grow) : 0.0f;
            }
            // the tile's two sums, subtracted in FP32: c := (c - big) - small
            const uint32_t a = u & 1, aph = (u >> 1) & 1;
            ++u;
            // warp-uniform: the tcgen05.ld below needs the whole warp
            if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[a], aph, spin_limit))) {
                if (lane == 0) atomicOr(status, DEV_TIMEOUT);
                break;
            }
            tc_fence_after();
            const uint32_t lane_base = tmem + ((q * 32) << 16) + a * 2 * kTile + half * 64;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                float big[32], sml[32];
                tc_ld32x2(lane_base + cc * 32, lane_base + kTile + cc * 32, big, sml);
#pragma unroll
                for (int jj = 0; jj < 32; ++jj) c[cc * 32 + jj] = (c[cc * 32 + jj] - big[jj]) - sml[jj];
            }
            // the pair takes the tile after next while this one is stored
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[a]);
            if (full_tile) {
#pragma unroll
                for (int jj = 0; jj < 64; jj += 4) {
                    const uint4 o = *reinterpret_cast<const uint4 *>(soff + jj);
                    st_cg(val + o.x + grow, c[jj]);
                    st_cg(val + o.y + grow, c[jj + 1]);
                    st_cg(val + o.z + grow, c[jj + 2]);
                    st_cg(val + o.w + grow, c[jj + 3]);
                }
            } else if (rok) {
#pragma unroll
                for (int jj = 0; jj < 64; ++jj)
                    if (uint32_t(jj) < ncol) st_cg(val + soff[jj] + grow, c[jj]);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// ----------------------------------------------------------------- host --
namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}
}  // namespace

cudaError_t dense_tc_tensor_map(uint16_t *pack, uint32_t m, uint32_t batch, CUtensorMap *map) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t dims[3] = {cuuint64_t(kPackRow), m, batch};
    const cuuint64_t strides[2] = {kPackRow * sizeof(uint16_t), cuuint64_t(m) * kPackRow * sizeof(uint16_t)};
    const cuuint32_t box[3] = {uint32_t(kChunk), uint32_t(kTile), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, pack, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_dense_pack(const float *val, uint64_t stride, uint32_t count, const uint32_t *doff, uint32_t m,
                              uint32_t k0, uint32_t kb, uint32_t slot0, uint16_t *packA, uint16_t *packB,
                              cudaStream_t st) {
    const uint32_t r_start = k0 + kb;
    if (r_start >= m) return cudaSuccess;
    const uint32_t nA = (m - r_start + kTile - 1) / kTile;
    k_dense_pack<<<dim3(2 * nA, 1, count), 256, 0, st>>>(val, stride, doff, m, k0, kb, slot0, r_start, nA, packA,
                                                           packB);
    return cudaGetLastError();
}

namespace {
// Rows [r_lo, r_hi) x columns [c_lo, c_hi) of the block from row and column
// r0 on, K = 32 * nchunks.
cudaError_t launch_tc(const CUtensorMap &mapA, const CUtensorMap &mapB, float *val, uint64_t stride, uint32_t count,
                      const uint32_t *doff, uint32_t m, uint32_t r0, uint32_t nchunks, const float *diag_scratch,
                      DenseRegion reg, uint32_t *status, uint32_t spin_limit, uint32_t num_sms,
                      uint32_t *tile_counter, cudaStream_t st) {
    static PerDeviceOnce attr;
    cudaError_t e = attr.run([] {
        return cudaFuncSetAttribute(k_dense_update_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes));
    });
    if (e != cudaSuccess) return e;
    const uint32_t rows = reg.r_hi > reg.r_lo ? reg.r_hi - reg.r_lo : 0;
    const uint32_t cols = reg.c_hi > reg.c_lo ? reg.c_hi - reg.c_lo : 0;
    const uint32_t tiles_r = (rows + kTile - 1) / kTile, tiles_c = (cols + kTile - 1) / kTile;
    const uint64_t total = uint64_t(tiles_r) * tiles_c * count;
    if (total == 0 && !reg.writeback) return cudaSuccess;
    if (r0 > m || total > 0xFFFFFFFFull || nchunks == 0 || nchunks * kChunk > kSlots) return cudaErrorInvalidValue;
    uint32_t grid = uint32_t(std::min<uint64_t>(std::max<uint64_t>(total, 1), num_sms));
    if (reg.writeback) grid = std::max<uint32_t>(grid, std::min<uint32_t>(count, num_sms));
    e = cudaMemsetAsync(tile_counter, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_dense_update_tc<<<grid, kThreads, kSmemBytes, st>>>(mapA, mapB, val, stride, doff, m, r0, nchunks, reg,
                                                          tiles_r, tiles_c, count, diag_scratch, status, spin_limit,
                                                          tile_counter);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_dense_update_tc(const CUtensorMap &mapA, const CUtensorMap &mapB, float *val, uint64_t stride,
                                   uint32_t count, const uint32_t *doff, uint32_t m, uint32_t k0, uint32_t kb,
                                   const float *diag_scratch, DenseRegion reg, uint32_t *status,
                                   uint32_t spin_limit, uint32_t num_sms, uint32_t *tile_counter, cudaStream_t st) {
    return launch_tc(mapA, mapB, val, stride, count, doff, m, k0 + kb, (kb + kChunk - 1) / kChunk, diag_scratch, reg,
                     status, spin_limit, num_sms, tile_counter, st);
}

cudaError_t launch_couple_pack(const DevPattern &P, const float *val, uint64_t stride, uint32_t count, uint32_t t,
                               uint32_t m, uint32_t ncols, uint32_t slot0, const uint32_t *lstart,
                               const uint32_t *ustart, uint16_t *packA, uint16_t *packB, cudaStream_t st) {
    if (m == 0 || ncols == 0) return cudaSuccess;
    if (ncols > uint32_t(kTile)) return cudaErrorInvalidValue;
    static PerDeviceOnce attr;
    cudaError_t e = attr.run([] {
        return cudaFuncSetAttribute(k_couple_pack, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kCoupleSmem));
    });
    if (e != cudaSuccess) return e;
    const uint32_t nblk = (m + kTile - 1) / kTile;
    k_couple_pack<<<dim3(2 * nblk, 1, count), kCoupleThreads, kCoupleSmem, st>>>(P.ridx, P.cidx, P.cpos, val, stride, t, m,
                                                                      ncols, slot0, lstart, ustart, nblk, packA,
                                                                      packB);
    return cudaGetLastError();
}

cudaError_t launch_couple_update_tc(const CUtensorMap &mapA, const CUtensorMap &mapB, float *val, uint64_t stride,
                                    uint32_t count, const uint32_t *doff, uint32_t m, uint32_t ncols,
                                    uint32_t *status, uint32_t spin_limit, uint32_t num_sms, uint32_t *tile_counter,
                                    cudaStream_t st) {
    const DenseRegion reg{0, m, 0, m, 0, 0};
    return launch_tc(mapA, mapB, val, stride, count, doff, m, 0, (ncols + kChunk - 1) / kChunk, nullptr, reg, status,
                     spin_limit, num_sms, tile_counter, st);
}

}  // namespace glu
