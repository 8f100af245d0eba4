// FP32 fused multiply-add throughput of the device, for the compute roofline
// of the factorization (the non-tensor FP32 peak is not a published figure).
// Every thread runs eight independent FMA chains; enough blocks for full
// occupancy on every SM.
#include <cuda_runtime.h>

#include "glu_b200.h"

namespace {

__global__ void __launch_bounds__(256) k_ffma(float *out, uint32_t iters, float a, float b) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = float(threadIdx.x + k) * 1e-3f;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains alive
}

}  // namespace

extern "C" glu_status glu_measure_fp32_peak(int device, double *tflops) {
    if (!tflops) return GLU_ERR_ARG;
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return GLU_ERR_ARG;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    glu_status st = GLU_OK;
    const uint32_t blocks = uint32_t(sms) * 8, iters = 1 << 16;
    float ms = 0.0f;
    if (cudaMalloc(&out, sizeof(float) * blocks) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess) {
        st = GLU_ERR_CUDA;
    } else {
        k_ffma<<<blocks, 256>>>(out, iters / 8, 0.999f, 1e-3f);  // warm-up
        cudaEventRecord(e0);
        k_ffma<<<blocks, 256>>>(out, iters, 0.999f, 1e-3f);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0)
            st = GLU_ERR_CUDA;
    }
    if (st == GLU_OK) *tflops = 2.0 * 8.0 * double(iters) * blocks * 256 / (double(ms) * 1e-3) / 1e12;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (out) cudaFree(out);
    if (prev >= 0) cudaSetDevice(prev);
    return st;
}
