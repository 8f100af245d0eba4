// glu_luondevice.hpp -- the reference's C++ entry point on top of the C ABI.
//
// Re-provides
//     void LUonDevice(Symbolic_Matrix &A_sym, std::ostream &out, std::ostream &err, bool PERTURB)
// (include/numeric.h:6, src/numeric.cu:347-639) with the same contract:
// factors A_sym.val in place on the host vector (FP32 L+U in the layout of the
// Symbolic_Matrix pattern), uses device 0, is synchronous, writes progress to
// `out` and failures to `err`.  "Total GPU time: ... ms" covers the same span
// as the reference's (numeric.cu:431-433 to 621-625): device set-up and
// upload, the factorization and the copy of the values back; a second line,
// "Factorization time: ... ms", gives the device time of the factorization
// alone.  Unlike the
// reference it also reports a failure through its return value (glu_lu_on_device)
// and never leaves partially factored values behind silently: on failure
// A_sym.val is left unchanged.
//
// Header-only and templated on the matrix type, so it needs nothing from the
// reference but the member names of Symbolic_Matrix (include/symbolic.h:12-23):
// n, nnz, sym_c_ptr, sym_r_idx, l_col_ptr, csr_r_ptr, csr_c_idx, csr_diag_ptr,
// val.  To drop it in for numeric.cu, compile one translation unit with
//     #include "symbolic.h"
//     #define GLU_PROVIDE_LUONDEVICE
//     #include "glu_luondevice.hpp"
// and link libglu_b200.so instead of numeric.o.
#ifndef GLU_LUONDEVICE_HPP
#define GLU_LUONDEVICE_HPP

#include <chrono>
#include <ostream>
#include <vector>

#include "glu_b200.h"

template <class SymbolicMatrix>
inline glu_status glu_lu_on_device(SymbolicMatrix &A, std::ostream &out, std::ostream &err, bool perturb) {
    if (A.n == 0 || A.nnz == 0) {
        err << "Matrix is empty; skipping GPU factorization." << std::endl;
        return GLU_ERR_ARG;
    }
    const auto t0 = std::chrono::steady_clock::now();
    glu_handle_t h = nullptr;
    glu_status s = glu_create_from_pattern(0, A.n, A.nnz, A.sym_c_ptr.data(), A.sym_r_idx.data(),
                                           A.l_col_ptr.data(), A.csr_r_ptr.data(), A.csr_c_idx.data(),
                                           A.csr_diag_ptr.data(), 1, &h);
    if (s == GLU_OK) s = glu_load_lu_values(h, 0, 1, A.val.data(), GLU_HOST, nullptr);
    if (s == GLU_OK) s = glu_factor(h, 0, 1, perturb ? 1 : 0, nullptr);
    if (s == GLU_OK) {
        glu_stats st;
        glu_get_stats(h, &st);
        if (perturb) {
            out << "Gaussian elimination with static pivoting (GESP)..." << std::endl;
            out << "Perturbation value is " << st.pert << std::endl;
        }
        s = glu_store_lu_values(h, 0, 1, A.val.data(), GLU_HOST, nullptr);
        if (s == GLU_OK) {
            const double span = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            out << "Total GPU time: " << span << " ms" << std::endl;
            out << "Factorization time: " << st.last_factor_ms << " ms" << std::endl;
        }
    }
    if (s != GLU_OK) err << "GPU factorization failed: " << glu_last_error() << std::endl;
    glu_destroy(h);
    return s;
}

#ifdef GLU_PROVIDE_LUONDEVICE
// External definition: define GLU_PROVIDE_LUONDEVICE in exactly one
// translation unit (the one that replaces numeric.cu).
void LUonDevice(Symbolic_Matrix &A_sym, std::ostream &out, std::ostream &err, bool PERTURB) {
    (void)glu_lu_on_device(A_sym, out, err, PERTURB);
}
#endif

#endif  // GLU_LUONDEVICE_HPP
