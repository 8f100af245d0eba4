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

}  // namespace glu
