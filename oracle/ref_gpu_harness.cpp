// Test / comparison infrastructure only: drives the reference's own GPU numeric
// factorization (src/numeric.cu, LUonDevice) on a Symbolic_Matrix prepared by
// ref_harness.cpp.  Built by oracle/Makefile from the reference tree into
// oracle/_ref/libglu_ref_gpu.so.
//
// LUonDevice (src/numeric.cu:347-639) sizes its dense scratch as
// TMPMEMNUM x n floats from the free memory (numeric.cu:465-488) and indexes
// it with a 32-bit product bid*n (numeric.cu:44,82,99).  When TMPMEMNUM*n
// exceeds 2^32 the scratch columns of different blocks alias and the factors
// are wrong.  ref_gpu_luondevice() can hold a ballast allocation during the
// call so that the free memory, and with it TMPMEMNUM, stays below that bound;
// numeric.cu itself is not modified.
//
// LUonDevice's progress and error text goes to streams in the bad state: this
// library links its C++ runtime statically and formatting numbers through it
// is not possible when the library is loaded into Python.  The call is timed
// here with CUDA events around it (the same span as its own "Total GPU time",
// numeric.cu:431-433,621-625: allocations, copies, factorization); failure is
// detected as the reference's Python binding does, by non-finite factor values
// (src/glu_binding.cpp:119-127).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <ostream>
#include <streambuf>

#include "numeric.h"
#include "symbolic.h"

struct RefCtx;
extern "C" Symbolic_Matrix *ref_symbolic_matrix(RefCtx *c);

namespace {
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};
std::ostream &null_stream() {
    static NullBuf buf;
    static std::ostream os(&buf);
    os.setstate(std::ios::badbit);
    return os;
}
}  // namespace

extern "C" {

// Returns 0 on success, 1 when the factors contain NaN/Inf (the reference's
// own failure signal), 2 when the ballast allocation failed, 3 on a CUDA error
// around the call.  *total_ms: device time of the whole LUonDevice call.
int ref_gpu_luondevice(RefCtx *c, int perturb, size_t keep_free_bytes, float *total_ms, char *err_buf,
                       int err_len) {
    if (err_buf && err_len > 0) err_buf[0] = 0;
    void *ballast = nullptr;
    if (keep_free_bytes > 0) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        if (free_b > keep_free_bytes) {
            if (cudaMalloc(&ballast, free_b - keep_free_bytes) != cudaSuccess) {
                if (err_buf) snprintf(err_buf, err_len, "ballast allocation failed");
                return 2;
            }
        }
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    Symbolic_Matrix *s = ref_symbolic_matrix(c);
    LUonDevice(*s, null_stream(), null_stream(), perturb != 0);
    cudaEventRecord(e1, 0);
    cudaError_t ce = cudaEventSynchronize(e1);
    float ms = -1.0f;
    if (ce == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ballast) cudaFree(ballast);
    *total_ms = ms;
    if (ce != cudaSuccess) {
        if (err_buf) snprintf(err_buf, err_len, "CUDA error: %s", cudaGetErrorString(ce));
        return 3;
    }
    for (float v : s->val)
        if (!std::isfinite(v)) {
            if (err_buf) snprintf(err_buf, err_len, "non-finite factor values");
            return 1;
        }
    return 0;
}

// The part of LUonDevice's "Total GPU time" that is not factorization: the
// same allocations and copies (numeric.cu:435-488: eight pattern and value
// arrays, sixteen streams, the TMPMEMNUM x n scratch sized by the same rule
// from the free memory and cleared, numeric.cu:618-619: the values copied
// back, then the frees), timed the same way with the same ballast.  The
// factorization alone is the total minus this span.  Returns 0, or 2/3 as
// ref_gpu_luondevice.
int ref_gpu_copy_span(RefCtx *c, size_t keep_free_bytes, float *span_ms) {
    void *ballast = nullptr;
    if (keep_free_bytes > 0) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        if (free_b > keep_free_bytes && cudaMalloc(&ballast, free_b - keep_free_bytes) != cudaSuccess) return 2;
    }
    Symbolic_Matrix *s = ref_symbolic_matrix(c);
    const size_t n = s->n, nnz = s->nnz;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    void *d[8] = {};
    const size_t bytes[8] = {(n + 1) * 4, nnz * 4, nnz * 4, n * 4, (n + 1) * 4, nnz * 4, n * 4, n * 4};
    const void *src[8] = {s->sym_c_ptr.data(), s->sym_r_idx.data(), s->val.data(), s->l_col_ptr.data(),
                          s->csr_r_ptr.data(), s->csr_c_idx.data(), s->csr_diag_ptr.data(), s->level_idx.data()};
    cudaError_t ce = cudaSuccess;
    for (int i = 0; i < 8 && ce == cudaSuccess; ++i) ce = cudaMalloc(&d[i], bytes[i]);
    for (int i = 0; i < 8 && ce == cudaSuccess; ++i) ce = cudaMemcpy(d[i], src[i], bytes[i], cudaMemcpyHostToDevice);
    cudaStream_t streams[16] = {};
    for (int j = 0; j < 16 && ce == cudaSuccess; ++j) ce = cudaStreamCreate(&streams[j]);
    void *tmp = nullptr;
    if (ce == cudaSuccess) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t reserve = size_t(4) << 30;
        size_t max_tmp = free_b > reserve ? free_b - reserve : free_b / 2;
        const size_t first = s->level_ptr.size() > 1 ? size_t(s->level_ptr[1] - s->level_ptr[0]) : 1;
        const size_t per_col = 4 * n;
        if (max_tmp < per_col) max_tmp = per_col;
        size_t num = 4 * n * first <= max_tmp ? first : max_tmp / per_col;
        if (num == 0) num = 1;
        ce = cudaMalloc(&tmp, num * per_col);
        if (ce == cudaSuccess) ce = cudaMemset(tmp, 0, num * per_col);
    }
    if (ce == cudaSuccess) ce = cudaMemcpy(s->val.data(), d[2], nnz * 4, cudaMemcpyDeviceToHost);
    cudaEventRecord(e1, 0);
    cudaError_t se = cudaEventSynchronize(e1);
    if (ce == cudaSuccess) ce = se;
    float ms = -1.0f;
    if (ce == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    for (int i = 0; i < 8; ++i)
        if (d[i]) cudaFree(d[i]);
    for (int j = 0; j < 16; ++j)
        if (streams[j]) cudaStreamDestroy(streams[j]);
    if (tmp) cudaFree(tmp);
    if (ballast) cudaFree(ballast);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *span_ms = ms;
    return ce == cudaSuccess ? 0 : 3;
}

}  // extern "C"
