// Device-side structures and helpers shared by the GLU kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

namespace glu {

// Device copy of the L+U pattern (Symbolic_Matrix arrays plus csr_pos).
struct DevPattern {
    const uint32_t *cptr;   // sym_c_ptr[n+1]
    const uint32_t *ridx;   // sym_r_idx[nnz]
    const uint32_t *diag;   // l_col_ptr[n]
    const uint32_t *rptr;   // csr_r_ptr[n+1]
    const uint32_t *cidx;   // csr_c_idx[nnz]
    const uint32_t *rdiag;  // csr_diag_ptr[n]
    const uint32_t *cpos;   // CSC position of every CSR entry
    uint32_t n;
    uint32_t nnz;
};

// Device status word bits (set with atomicOr, read back by the host).
enum : uint32_t {
    DEV_ZERO_PIVOT = 1u,
    DEV_NONFINITE_PIVOT = 2u,
    DEV_TIMEOUT = 4u,
    DEV_BAD_INDEX = 8u,
};

// Launch `kern` on st chained to the previous kernel of the stream (see
// pdl_release / pdl_wait).
template <typename... KArgs, typename... Args>
cudaError_t launch_chained(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                           Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// Runs a setup step (a kernel attribute: dynamic shared memory above 48 KB, a
// non-portable cluster size) once per device.  Function attributes belong to
// the device that was current when they were set, and launchers run on the
// device of their handle, from any host thread.
class PerDeviceOnce {
  public:
    template <class F>
    cudaError_t run(F &&setup) {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= 64) return setup();
        const uint64_t bit = uint64_t(1) << dev;
        if (done_.load(std::memory_order_acquire) & bit) return cudaSuccess;
        e = setup();
        if (e == cudaSuccess) done_.fetch_or(bit, std::memory_order_acq_rel);
        return e;
    }

  private:
    std::atomic<uint64_t> done_{0};
};

// Upper bound on spins of any device-side wait before it gives up and
// reports DEV_TIMEOUT (each spin sleeps ~64-256 ns: a few seconds in total).
constexpr uint32_t kSpinLimit = 1u << 24;

#ifdef __CUDACC__
__device__ __forceinline__ float ld_cg(const float *p) { return __ldcg(p); }
__device__ __forceinline__ void st_cg(float *p, float v) { __stcg(p, v); }

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int32_t ld_acquire_gpu(const int32_t *p) {
    int32_t v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release_gpu(int32_t *p, int32_t v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// x rounded to BF16 (1 + 7 explicit significand bits), ties away from zero,
// as the bits of an FP32 value whose 16 low bits are zero: half a BF16 unit
// in the last place added to the magnitude bits, the 16 bits below it cleared
// (a carry into the exponent is the correct rounding up).  Done on the bits so
// that every part of the split is exact; finite inputs.
__device__ __forceinline__ uint32_t bf16_rna_bits(float x) { return (__float_as_uint(x) + 0x8000u) & 0xFFFF0000u; }

// The three BF16 parts of four FP32 values, each part's four as one 8-byte
// word (value u in bits 16 u .. 16 u + 15).
__device__ __forceinline__ void split_bf16x4(const float (&v)[4], uint2 &p0, uint2 &p1, uint2 &p2) {
    uint32_t b[3][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        b[0][u] = bf16_rna_bits(v[u]);
        const float r1 = v[u] - __uint_as_float(b[0][u]);  // exact
        b[1][u] = bf16_rna_bits(r1);
        b[2][u] = __float_as_uint(r1 - __uint_as_float(b[1][u]));  // exact, at most 7 significant bits
    }
    p0 = make_uint2((b[0][0] >> 16) | (b[0][1] & 0xFFFF0000u), (b[0][2] >> 16) | (b[0][3] & 0xFFFF0000u));
    p1 = make_uint2((b[1][0] >> 16) | (b[1][1] & 0xFFFF0000u), (b[1][2] >> 16) | (b[1][3] & 0xFFFF0000u));
    p2 = make_uint2((b[2][0] >> 16) | (b[2][1] & 0xFFFF0000u), (b[2][2] >> 16) | (b[2][3] & 0xFFFF0000u));
}

// Programmatic dependent launch.  A kernel launched with launch_chained may
// start while the previous kernel of its stream is still running:
// pdl_release lets the next chained kernel begin launching, pdl_wait blocks
// until the previous kernel has completed and its writes are visible (a no-op
// when the kernel was not chained).  Plan data may be read before pdl_wait,
// anything a previous kernel writes only after it.
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Bounded wait until *cnt reaches target (at most `limit` polls; a wait that
// sees another wait's timeout in the status word gives up early).  Returns
// false on timeout, with DEV_TIMEOUT set.
__device__ __forceinline__ bool wait_count(const uint32_t *cnt, uint32_t target, uint32_t *status,
                                           uint32_t limit) {
    uint32_t spins = 0;
    while (ld_acquire_gpu(cnt) < target) {
        if (++spins > limit) {
            atomicOr(status, DEV_TIMEOUT);
            return false;
        }
        if ((spins & 1023u) == 0 && (ld_acquire_gpu(status) & DEV_TIMEOUT)) return false;
        __nanosleep(64);
    }
    return true;
}

// First index in [lo, hi] (inclusive, hi is a valid answer) with a[idx] >= key.
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *__restrict__ a, uint32_t lo,
                                                    uint32_t hi, uint32_t key) {
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Last s in [lo, hi) with off[s] <= key (off ascending, off[lo] <= key).
__device__ __forceinline__ uint32_t upper_slot(const uint32_t *__restrict__ off, uint32_t lo,
                                               uint32_t hi, uint32_t key) {
    // invariant: off[lo] <= key, answer in [lo, hi)
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(off + mid) <= key)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}
#endif  // __CUDACC__

}  // namespace glu
