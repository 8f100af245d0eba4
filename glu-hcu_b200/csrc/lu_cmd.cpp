// lu_cmd: command-line driver with the reference's interface (src/lu_cmd.cpp).
//
//   lu_cmd -i matrix.mtx [-p] [-r] [-t tol]
//
// Reads a Matrix Market file (triplets stored column by column), runs NICSLU
// preprocessing, the symbolic phase, the GPU factorization and a solve with
// b = 1, and writes x.dat (one value per line, default stream formatting, as
// src/lu_cmd.cpp:122-130).  -p enables GESP perturbation (lu_cmd.cpp:52-55).
// Additions: -r solves with FP64 iterative refinement (tolerance -t, default
// 1e-10) instead of the plain FP32 solve.  Unlike the reference, a failed GPU
// step is an error: no x.dat is written and the exit status is non-zero.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "glu_b200.h"
#include "glu_preprocess.h"

using namespace std;

static void help_message() {
    cout << endl;
    cout << "GLU program V3.0 (B200)" << endl;
    cout << "Usage: ./lu_cmd -i inputfile" << endl;
    cout << "Additional usage: ./lu_cmd -i inputfile -p" << endl;
    cout << "-p to enable perturbation" << endl;
    cout << "-r to solve with FP64 iterative refinement (-t tolerance, default 1e-10)" << endl;
}

static double ms_since(chrono::steady_clock::time_point t0) {
    return chrono::duration<double, milli>(chrono::steady_clock::now() - t0).count();
}

#define CHECK(call)                                                                  \
    do {                                                                             \
        glu_status s_ = (call);                                                      \
        if (s_ != GLU_OK) {                                                          \
            cerr << #call << " failed (" << int(s_) << "): " << glu_last_error() << endl; \
            return 2;                                                                \
        }                                                                            \
    } while (0)

int main(int argc, char **argv) {
    const char *matrixName = nullptr;
    bool perturb = false, refine = false;
    double tol = 1e-10;
    if (argc < 3) {
        help_message();
        return -1;
    }
    for (int i = 1; i < argc;) {
        if (strcmp(argv[i], "-i") == 0) {
            if (i + 1 >= argc) {
                help_message();
                return -1;
            }
            matrixName = argv[i + 1];
            i += 2;
        } else if (strcmp(argv[i], "-p") == 0) {
            perturb = true;
            i += 1;
        } else if (strcmp(argv[i], "-r") == 0) {
            refine = true;
            i += 1;
        } else if (strcmp(argv[i], "-t") == 0 && i + 1 < argc) {
            tol = atof(argv[i + 1]);
            i += 2;
        } else {
            help_message();
            return -1;
        }
    }
    if (!matrixName) {
        help_message();
        return -1;
    }

    uint32_t n = 0, nnz = 0;
    double *ax = nullptr;
    uint32_t *ai = nullptr, *ap = nullptr;
    printf("Reading matrix...\n");
    int ret = glu_pre_read_mtx(matrixName, &n, &nnz, &ax, &ai, &ap);
    if (ret != 0) {
        cerr << (ret == -4 ? "File cannot open" : "Read invalid matrix") << endl;
        cerr << "Matrix preprocessing failed." << endl;
        return -1;
    }
    printf("Preprocessing matrix...\n");
    auto t0 = chrono::steady_clock::now();
    glu_pre_t pre = nullptr;
    ret = glu_pre_analyze(n, nnz, ax, ai, ap, &pre);
    if (ret != 0) {
        cerr << "Matrix preprocessing failed (NICSLU error " << ret << ")." << endl;
        return -1;
    }
    printf("Preprocessing time: %f ms\n", ms_since(t0));
    cout << "Matrix Row: " << n << endl;
    cout << "Original nonzero: " << nnz << endl;

    vector<double> pax(nnz);
    vector<uint32_t> pai(nnz), pap(n + 1), pos(nnz);
    vector<double> scale(nnz);
    glu_pre_matrix(pre, pax.data(), pai.data(), pap.data());
    glu_pre_source_map(pre, pos.data(), scale.data());

    t0 = chrono::steady_clock::now();
    glu_symbolic_t sym = nullptr;
    CHECK(glu_symbolic_analyze(n, nnz, pap.data(), pai.data(), &sym));
    uint32_t nlu = 0;
    glu_symbolic_sizes(sym, nullptr, &nlu);
    cout << "Symbolic nonzero: " << nlu << endl;
    cout << "Symbolic time: " << ms_since(t0) << " ms" << endl;

    t0 = chrono::steady_clock::now();
    const auto t_gpu = t0;  // the reference's "Total GPU time" span starts at device set-up
    glu_handle_t h = nullptr;
    CHECK(glu_create(sym, 0, 1, &h));
    int32_t nlev = 0;
    glu_levels(h, &nlev, nullptr, nullptr);
    cout << "Number of levels: " << nlev << endl;
    cout << "Leveling time: " << ms_since(t0) << " ms" << endl;

    vector<uint32_t> cp(n), rpi(n), slot(nnz), src_slot(nnz);
    vector<int32_t> piv(n);
    vector<double> csp(n), rs(n);
    int mc64 = 0;
    glu_pre_transform(pre, cp.data(), rpi.data(), piv.data(), csp.data(), rs.data(), &mc64);
    CHECK(glu_set_transform(h, cp.data(), rpi.data(), piv.data(), csp.data(), rs.data(), mc64));
    glu_symbolic_slots(sym, slot.data());
    for (uint32_t q = 0; q < nnz; ++q) src_slot[q] = slot[pos[q]];
    CHECK(glu_set_source(h, nnz, ap, ai, src_slot.data(), scale.data()));

    vector<float> val(nlu);
    glu_predict_lu(sym, pax.data(), val.data());
    CHECK(glu_load_lu_values(h, 0, 1, val.data(), GLU_HOST, nullptr));
    if (refine) CHECK(glu_load_source_values(h, 0, 1, ax, GLU_HOST, nullptr));
    if (perturb) cout << "Gaussian elimination with static pivoting (GESP)..." << endl;
    glu_status fs = glu_factor(h, 0, 1, perturb ? 1 : 0, nullptr);
    glu_stats st{};
    glu_get_stats(h, &st);
    if (perturb) cout << "Perturbation value is " << st.pert << endl;
    if (fs != GLU_OK) {
        cerr << "GPU factorization failed: " << glu_last_error() << endl;
        return 2;
    }
    // Same span as the reference's (numeric.cu:431-433 to 621-625): device
    // set-up, uploads and the factorization; then the factorization alone.
    cout << "Total GPU time: " << ms_since(t_gpu) << " ms" << endl;
    cout << "Factorization time: " << st.last_factor_ms << " ms" << endl;

    vector<double> x(n);
    if (refine) {
        vector<double> b(n, 1.0);
        glu_refine_stats rst{};
        glu_status rs_ = glu_solve_refined(h, 0, 1, 1, b.data(), x.data(), tol, 20, 0, GLU_HOST, &rst, nullptr);
        cout << "Refinement: " << rst.iterations << " steps, relative residual " << rst.residual << endl;
        if (rs_ != GLU_OK && rs_ != GLU_ERR_NOT_CONVERGED) {
            cerr << "Solve failed: " << glu_last_error() << endl;
            return 2;
        }
    } else {
        vector<float> b(n, 1.0f), xf(n);
        CHECK(glu_solve(h, 0, 1, b.data(), xf.data(), GLU_HOST, nullptr));
        for (uint32_t i = 0; i < n; ++i) x[i] = xf[i];
    }
    {
        ofstream x_f("x.dat");
        for (double xx : x) x_f << xx << '\n';
    }
    glu_destroy(h);
    glu_symbolic_destroy(sym);
    glu_pre_destroy(pre);
    glu_pre_free(ax);
    glu_pre_free(ai);
    glu_pre_free(ap);
    return 0;
}
