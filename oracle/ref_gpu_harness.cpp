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
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>

#include "numeric.h"
#include "symbolic.h"

struct RefCtx;
extern "C" Symbolic_Matrix *ref_symbolic_matrix(RefCtx *c);

extern "C" {

// Returns 0 on success, 1 when LUonDevice wrote to its error stream, 2 when the
// ballast allocation failed.  *total_ms is LUonDevice's own "Total GPU time"
// (it includes its allocations and copies, numeric.cu:431-433,621-625).
int ref_gpu_luondevice(RefCtx *c, int perturb, size_t keep_free_bytes, float *total_ms,
                       char *err_buf, int err_len) {
    void *ballast = nullptr;
    if (keep_free_bytes > 0) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        if (free_b > keep_free_bytes) {
            if (cudaMalloc(&ballast, free_b - keep_free_bytes) != cudaSuccess) {
                snprintf(err_buf, err_len, "ballast allocation failed");
                return 2;
            }
        }
    }
    std::ostringstream out, err;
    LUonDevice(*ref_symbolic_matrix(c), out, err, perturb != 0);
    if (ballast) cudaFree(ballast);
    *total_ms = -1.0f;
    std::string o = out.str();
    size_t pos = o.find("Total GPU time: ");
    if (pos != std::string::npos) *total_ms = std::stof(o.substr(pos + 16));
    std::string e = err.str();
    if (err_buf && err_len > 0) snprintf(err_buf, err_len, "%s", e.c_str());
    return e.empty() ? 0 : 1;
}

}  // extern "C"
