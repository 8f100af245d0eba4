// glu_solve_noalloc: the FP32 solve for callers that cannot allocate device
// memory.
//
// Some hosts of this library may not call cudaMalloc once they are running:
// a simulator whose device memory is owned and pooled by a framework (a second
// allocator would compete with it for the same memory), or a real-time loop
// that must not stall in the allocator.  glu_solve allocates its working
// vectors on first use; this variant takes them from a fixed array in device
// memory that is part of the library itself, so, once the handle exists and
// is factored, a solve needs no allocation at all.
//
// The array below is held by every GPU that loads the library, for the life
// of the process.  Its size bounds what this entry point accepts:
// n * nrhs <= kNoAllocMaxValues and a dense trailing block of order
// m <= 64 * (kNoAllocMaxBlocks - 1).  The environment variable
// GLU_NOALLOC_BLOCK_LIMIT, read once, can lower the second bound (to check
// the rejection path on small matrices); it cannot raise it.
//
// The array keeps the last call's contents.  The sweeps reset the block flags
// and the ticket they wait on at the start of every call; y and xo are fully
// written before they are read.
#include <cuda_runtime.h>

#include <cstdlib>
#include <mutex>

#include "glu_internal.h"

namespace {

constexpr size_t kNoAllocMaxValues = size_t(1) << 20;  // n * nrhs
constexpr uint32_t kNoAllocMaxBlocks = 4096;             // 64-row blocks of the dense tail, plus the ticket
constexpr size_t kNoAllocFloats = 2 * kNoAllocMaxValues + kNoAllocMaxBlocks + 64;

// Working vectors of glu_solve_noalloc: y (permuted right-hand sides), xo
// (finished values of the dividing sweeps), the dense-tail block flags and
// the ticket.  About 8 MiB per GPU.
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float *g_scratch_dev[kMaxDevices] = {};

// Device address of the scratch array on `dev` (which must be current).  The
// host-side name of a __device__ array is not a device address; the runtime
// gives the address for the current device.
glu::Status scratch_address(int dev, float **out) {
    if (dev < 0 || dev >= kMaxDevices) return glu::set_error(GLU_ERR_UNSUPPORTED, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_dev[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return glu::set_error(GLU_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        g_scratch_dev[dev] = static_cast<float *>(p);
    }
    *out = g_scratch_dev[dev];
    return GLU_OK;
}

// Dense-tail block limit: kNoAllocMaxBlocks, or less when the environment asks.
uint32_t block_limit() {
    static const uint32_t lim = [] {
        const char *e = std::getenv("GLU_NOALLOC_BLOCK_LIMIT");
        long v = e ? std::strtol(e, nullptr, 10) : 0;
        return (v > 0 && v < long(kNoAllocMaxBlocks)) ? uint32_t(v) : kNoAllocMaxBlocks;
    }();
    return lim;
}

}  // namespace

extern "C" glu_status glu_solve_noalloc(glu_handle_t h, uint32_t inst, uint32_t nrhs, const float *b, float *x,
                                        glu_stream stream) {
    if (!h) return glu::set_error(GLU_ERR_ARG, "null handle");
    const int dev = glu::handle_device(h);
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return glu::set_error(GLU_ERR_CUDA, "cudaGetDevice failed");
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return glu::set_error(GLU_ERR_CUDA, "cudaSetDevice failed");
    float *base = nullptr;
    glu::Status s = scratch_address(dev, &base);
    if (s == GLU_OK) {
        float *y = base;
        float *xo = base + kNoAllocMaxValues;
        uint32_t *flags = reinterpret_cast<uint32_t *>(base + 2 * kNoAllocMaxValues);
        uint32_t *ticket = flags + kNoAllocMaxBlocks;
        s = glu::solve_f32_scratch(h, inst, nrhs, b, x, y, xo, flags, ticket, kNoAllocMaxValues,
                                   block_limit(), stream);
    }
    if (prev != dev) cudaSetDevice(prev);
    return s;
}
