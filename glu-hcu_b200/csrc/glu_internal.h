// Internal declarations shared by the host and device parts of libglu_b200.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "glu_b200.h"

namespace glu {

using Status = glu_status;

// Records the message for glu_last_error() on this thread and returns s.
Status set_error(Status s, const char *fmt, ...);

// Output of the symbolic phase (the reference's Symbolic_Matrix arrays plus the
// value-placement maps).
struct SymbolicData {
    uint32_t n = 0;
    uint32_t nnz = 0;    // nonzeros of L+U
    uint32_t nnz_a = 0;  // nonzeros of the preprocessed A
    std::vector<uint32_t> sym_c_ptr, sym_r_idx, l_col_ptr;
    std::vector<uint32_t> csr_r_ptr, csr_c_idx, csr_diag_ptr;
    std::vector<uint32_t> csr_pos;  // CSC position of every CSR entry
    std::vector<uint32_t> a_ptr, a_idx, a_slot;  // A's pattern and LU slot per entry
    std::vector<int64_t> lu_src;                 // A entry placed at each LU slot, or -1
};

Status symbolic_analyze(uint32_t n, uint32_t nnz_a, const uint32_t *ap, const uint32_t *ai,
                        SymbolicData &s);
void predict_lu(const SymbolicData &s, const double *ax, float *val);
// CSR transpose with CSC positions, from a CSC pattern alone.
void build_csr(SymbolicData &s);

// Device of a handle.
int handle_device(const glu_handle_s *h);
// FP32 solve of value set inst with device vectors b, x (nrhs x n) whose
// working vectors come from caller-provided device memory: y and xo hold
// max_values floats each, flags holds max_blocks words, ticket one word.
// Allocates nothing.
Status solve_f32_scratch(glu_handle_s *h, uint32_t inst, uint32_t nrhs, const float *b, float *x, float *y,
                         float *xo, uint32_t *flags, uint32_t *ticket, size_t max_values, uint32_t max_blocks,
                         void *stream);

}  // namespace glu
