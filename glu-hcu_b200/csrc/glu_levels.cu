// Level sets of the column dependency graph, built on the device.
//
// Symbolic_Matrix::leveling (src/symbolic.cc:106-151) gives column i the level
//     1 + max( level(c) : c in Upat(i) whose column has an L part     (:115-124)
//                         c in CSR row i left of the diagonal )        (:125-130)
// and lists the columns level by level, ascending within a level (a stable
// counting sort, :140-148).  Here:
//   1. longest path: one warp per column, claimed in ascending order through
//      an atomic ticket; it waits (bounded) for the levels of its dependencies,
//      all of which are lower-numbered columns claimed earlier;
//   2. level sizes -> level_ptr by an exclusive scan;
//   3. level_idx by a stable least-significant-digit radix sort of the column
//      indices keyed on their level (8-bit digits, one warp per tile), which
//      keeps ascending order within a level exactly as the counting sort does.
#include "glu_common.cuh"
#include "glu_kernels.h"

namespace glu {

constexpr uint32_t kSortTile = 4096;

__global__ void __launch_bounds__(256) k_longest_path(DevPattern P, int32_t *level_of, uint32_t *count,
                                                      int32_t *num_lev, uint32_t *ticket, uint32_t *status) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(ticket, 1u);
    i = __shfl_sync(0xffffffffu, i, 0);
    if (i >= P.n) return;
    int32_t mx = -1;
    auto dep_level = [&](uint32_t c) -> int32_t {
        uint32_t spins = 0;
        int32_t lv;
        while ((lv = ld_acquire_gpu(level_of + c)) < 0) {
            if (++spins > kSpinLimit) {
                atomicOr(status, DEV_TIMEOUT);
                return 0;
            }
            if ((spins & 1023u) == 0 && (ld_acquire_gpu(status) & DEV_TIMEOUT)) return 0;
            __nanosleep(64);
        }
        return lv;
    };
    // U-part dependencies whose column has an L part
    for (uint32_t p = P.cptr[i] + lane; p < P.diag[i]; p += 32) {
        uint32_t c = P.ridx[p];
        if (P.diag[c] + 1 != P.cptr[c + 1]) mx = max(mx, dep_level(c));
    }
    // L-row dependencies (CSR row i left of the diagonal)
    for (uint32_t e = P.rptr[i] + lane; e < P.rdiag[i]; e += 32) mx = max(mx, dep_level(P.cidx[e]));
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) {
        int32_t lv = mx + 1;
        atomicAdd(count + lv, 1u);
        atomicMax(num_lev, lv + 1);
        __threadfence();
        st_release_gpu(level_of + i, lv);
    }
}

// Exclusive scan of in[0, len) into out[0, len] (out[len] = total), one block.
__global__ void __launch_bounds__(1024) k_scan_single(const uint32_t *in, const int32_t *len_dev,
                                                      uint32_t len_const, int32_t *out) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry;
    const uint32_t len = len_dev ? uint32_t(*len_dev) : len_const;
    const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < len; base += 1024) {
        uint32_t v = (base + tid < len) ? in[base + tid] : 0u;
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= uint32_t(o)) x += y;
        }
        if (lane == 31) warp_sums[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t s = warp_sums[lane];
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= uint32_t(o)) s += y;
            }
            warp_sums[lane] = s;
        }
        __syncthreads();
        uint32_t incl = x + (w > 0 ? warp_sums[w - 1] : 0u);
        if (base + tid < len) out[base + tid] = int32_t(carry + incl - v);
        __syncthreads();
        if (tid == 1023) carry += incl;
        __syncthreads();
    }
    if (tid == 0) out[len] = int32_t(carry);
}

// Per-tile digit histograms, bin-major: hist[d * ntiles + tile].
__global__ void __launch_bounds__(256) k_digit_hist(const int32_t *keys, uint32_t n, uint32_t shift,
                                                    uint32_t ntiles, uint32_t *hist) {
    __shared__ uint32_t h[8][256];
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint32_t d = lane; d < 256; d += 32) h[w][d] = 0;
    __syncwarp();
    const uint32_t tile = blockIdx.x * 8 + w;
    if (tile < ntiles) {
        uint32_t b0 = tile * kSortTile, b1 = min(b0 + kSortTile, n);
        for (uint32_t i = b0 + lane; i < b1; i += 32) atomicAdd(&h[w][(uint32_t(keys[i]) >> shift) & 255u], 1u);
        __syncwarp();
        for (uint32_t d = lane; d < 256; d += 32) hist[d * ntiles + tile] = h[w][d];
    }
}

// Stable scatter of one tile (one warp, elements in order, 32 at a time).
__global__ void __launch_bounds__(256) k_digit_scatter(const int32_t *keys, const int32_t *vals, uint32_t n,
                                                       uint32_t shift, uint32_t ntiles, const int32_t *offs,
                                                       int32_t *okeys, int32_t *ovals) {
    __shared__ uint32_t base[8][256];
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t tile = blockIdx.x * 8 + w;
    if (tile >= ntiles) return;
    for (uint32_t d = lane; d < 256; d += 32) base[w][d] = uint32_t(offs[d * ntiles + tile]);
    __syncwarp();
    uint32_t b0 = tile * kSortTile, b1 = min(b0 + kSortTile, n);
    for (uint32_t i0 = b0; i0 < b1; i0 += 32) {
        uint32_t i = i0 + lane;
        bool ok = i < b1;
        uint32_t mask = __ballot_sync(0xffffffffu, ok);
        if (!ok) break;
        int32_t k = keys[i];
        uint32_t d = (uint32_t(k) >> shift) & 255u;
        uint32_t peers = __match_any_sync(mask, d);
        uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        uint32_t pos = base[w][d] + rank;
        okeys[pos] = k;
        ovals[pos] = vals ? vals[i] : int32_t(i);
        __syncwarp(mask);
        if (rank == 0) base[w][d] += __popc(peers);
        __syncwarp(mask);
    }
}

size_t level_scratch_bytes(uint32_t n) {
    size_t ntiles = (n + kSortTile - 1) / kSortTile;
    // ticket, count[n+1], hist/offs [256*ntiles + 1] x2, keys/vals x2 [n]
    return 256 + sizeof(uint32_t) * (size_t(n) + 1) + 2 * sizeof(uint32_t) * (256 * ntiles + 1) +
           4 * sizeof(int32_t) * size_t(n) + 256;
}

cudaError_t build_levels(const DevPattern &P, void *scratch, int32_t *level_of, int32_t *level_ptr,
                         int32_t *level_idx, int32_t *num_lev_dev, uint32_t *status,
                         cudaStream_t st) {
    const uint32_t n = P.n;
    const uint32_t ntiles = (n + kSortTile - 1) / kSortTile;
    char *s = static_cast<char *>(scratch);
    uint32_t *ticket = reinterpret_cast<uint32_t *>(s);
    s += 256;
    uint32_t *count = reinterpret_cast<uint32_t *>(s);
    s += sizeof(uint32_t) * (size_t(n) + 1);
    uint32_t *hist = reinterpret_cast<uint32_t *>(s);
    s += sizeof(uint32_t) * (256 * size_t(ntiles) + 1);
    int32_t *offs = reinterpret_cast<int32_t *>(s);
    s += sizeof(uint32_t) * (256 * size_t(ntiles) + 1);
    int32_t *kA = reinterpret_cast<int32_t *>(s);
    s += sizeof(int32_t) * n;
    int32_t *vA = reinterpret_cast<int32_t *>(s);
    s += sizeof(int32_t) * n;
    int32_t *kB = reinterpret_cast<int32_t *>(s);
    s += sizeof(int32_t) * n;
    int32_t *vB = reinterpret_cast<int32_t *>(s);

    cudaError_t e;
    if ((e = cudaMemsetAsync(ticket, 0, 4, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(count, 0, sizeof(uint32_t) * (size_t(n) + 1), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(level_of, 0xff, sizeof(int32_t) * n, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(num_lev_dev, 0, sizeof(int32_t), st)) != cudaSuccess) return e;
    k_longest_path<<<(n + 7) / 8, 256, 0, st>>>(P, level_of, count, num_lev_dev, ticket, status);
    k_scan_single<<<1, 1024, 0, st>>>(count, num_lev_dev, 0, level_ptr);
    // stable radix sort of i by level_of[i]; n < 2^31 so at most 4 passes, and
    // levels < n: passes beyond the top significant digit of n are skipped.
    uint32_t passes = 1;
    while (passes < 4 && (uint64_t(n) >> (8 * passes)) > 0) ++passes;
    const int32_t *keys = level_of;
    const int32_t *vals = nullptr;
    for (uint32_t p = 0; p < passes; ++p) {
        int32_t *ok = (p & 1) ? kB : kA;
        int32_t *ov = (p + 1 == passes) ? level_idx : ((p & 1) ? vB : vA);
        k_digit_hist<<<(ntiles + 7) / 8, 256, 0, st>>>(keys, n, 8 * p, ntiles, hist);
        k_scan_single<<<1, 1024, 0, st>>>(hist, nullptr, 256 * ntiles, offs);
        k_digit_scatter<<<(ntiles + 7) / 8, 256, 0, st>>>(keys, vals, n, 8 * p, ntiles, offs, ok, ov);
        keys = ok;
        vals = ov;
    }
    return cudaGetLastError();
}

}  // namespace glu
